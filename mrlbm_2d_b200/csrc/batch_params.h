// batch_params.h -- host/device layout of the batched multi-case step (step_batch.cuh).
#pragma once
#include "step_params.h"

namespace mrlbm {

constexpr int ERR_BARRIER_TIMEOUT = 8;     // device flag bit: a grid-barrier wait gave up
constexpr unsigned BAR_SPIN_LIMIT = 1u << 24;   // default grid-barrier polls (~0.1 us each)

// Per-case, per-call values the kernel derives each step's flags from.
struct BatchCase {
    int iter0;               // iteration before the call (the first step runs iter0 + 1)
    int cur0;                // time level holding the current populations (params' src)
    int ring_n0;             // records already in the case's force ring
    int ovr_live;            // first step reads the override list (after a state load)
    int post_process, statsbegin, statsend, iplot, plot_cyl;
    int fs_begin, fs_end;    // field-statistics window (fs_begin > fs_end: off)
    int aux_items, tiles;    // work items of one step
    int pad;
    double* ring;            // force records (REC_WORDS per record)
    double* macro;           // macroscopic output, written on the call's last step if wanted
    double* fstat;           // field-statistics sums or null
};

struct BatchBarrier {
    unsigned count;
    unsigned gen;
    int abort;
    int err;
    unsigned bulk_done;            // bulk blocks of the step launch that have finished (split steps)
};

template <class T>
struct BatchArgs {
    const StepParams<T>* params;   // per case; src/dst as at the start of the call
    const BatchCase* cases;
    const int* aux_off;            // [ncases + 1] prefix sums of aux items
    const int* tile_off;           // [ncases + 1] prefix sums of bulk tiles
    const int* item_case;          // [aux items + bulk tiles] case of each work item (persistent schedule)
    const int* aux_case;           // split steps: case of each auxiliary item
    const int* tile_case;          // split steps: case of each bulk tile
    BatchBarrier* bar;
    int ncases;
    int nsteps;                    // steps this launch advances (persistent schedule)
    int step0;                     // index of this launch's first step within the call
    int call_steps;                // steps of the whole call (macro output on the last)
    int want_macro;
    int full;                      // some case has field statistics, macroscopic output or a body force
    unsigned spin_limit;           // polls a block waits at the grid barrier before it gives up
};

// Host-side launch entry points (step_f64.cu / step_f32.cu).  tile_cfg is a vector shape
// (MRLBM_VEC_LIST); cooperative selects the persistent schedule.  Return 0, -1 on a launch
// error, -2 for a shape that is not a vector shape.
int launch_batch_f64(const BatchArgs<double>& a, int tile_cfg, int grid, bool cooperative, void* stream);
int launch_batch_f32(const BatchArgs<float>& a, int tile_cfg, int grid, bool cooperative, void* stream);
// One step of every case as two launches (graph schedule): the auxiliary items (walked by
// aux_grid blocks of AUX_THREADS), then the bulk tiles of shape tile_cfg (a one-tile-per-block or
// vector shape) over `grid` blocks, each taking a contiguous run of tiles.  Return 0, -1 on a
// launch error, -2 for a shape the split step does not take.
int launch_batch_split_f64(const BatchArgs<double>& a, int tile_cfg, int aux_grid, int grid, void* stream);
int launch_batch_split_f32(const BatchArgs<float>& a, int tile_cfg, int aux_grid, int grid, void* stream);
// Bulk blocks per SM of the split step's bulk kernel for a shape, and its threads per block.
int batch_split_blocks_per_sm(int precision, int tile_cfg);
int batch_split_blocks_per_sm_f64(int tile_cfg);
int batch_split_blocks_per_sm_f32(int tile_cfg);
int batch_split_threads(int tile_cfg);
// Auxiliary block size of the split step (step_common.cuh AUX_THREADS).
constexpr int BATCH_AUX_THREADS = 128;
// Resident blocks per SM of the batch kernel of a vector shape (0: not a vector shape).
int batch_blocks_per_sm(int precision, int tile_cfg);
int batch_blocks_per_sm_f64(int tile_cfg);
int batch_blocks_per_sm_f32(int tile_cfg);
int batch_block_threads(int tile_cfg);

}  // namespace mrlbm
