// statistics.cpp -- the post-processing of 2d_statistics.f90 as library calls: lift-peak
// period and Strouhal number, mean drag coefficient, rms lift coefficient and the surface
// pressure coefficient, averaged over whole shedding cycles.  Same arithmetic order as the
// reference (compiled with -ffp-contract=off).
#include <cmath>

#include "../../include/mrlbm.h"

namespace {

// find_peaks (2d_statistics.f90:183-214): the first two strict local maxima of the signal.
// Indices are 1-based like the reference's.
bool find_peaks(const double* s, int n, int& peak1, int& peak2) {
    peak1 = -1;
    peak2 = -1;
    for (int i = 2; i <= n - 1; ++i) {
        if (s[i - 1] > s[i - 2] && s[i - 1] > s[i]) {
            if (peak1 == -1) {
                peak1 = i;
            } else if (peak2 == -1) {
                peak2 = i;
                break;
            }
        }
    }
    return peak1 != -1 && peak2 != -1;
}

}  // namespace

extern "C" {

int mrlbm_force_statistics(const double* f_drag, const double* f_lift, int32_t nstep, double r_cy, double uo,
                           double rho_infty, double* St, double* Cd_mean, double* Cl_rms, int32_t* cycle_start,
                           int32_t* period, int32_t* n_cycle) {
    if (!f_drag || !f_lift || nstep < 3) return MRLBM_EINVAL;
    const double D_cy = 2.0 * r_cy;                                         // 2d_statistics.f90:30
    const double f_norm = 0.50 * rho_infty * (uo * uo) * D_cy;              // 2d_statistics.f90:32
    int p1, p2;
    if (!find_peaks(f_lift, nstep, p1, p2)) return MRLBM_ESTATE;           // "Could not detect two peaks."
    const int start = p1, per = p2 - p1;
    const int ncyc = (nstep - start) / per;                                 // 2d_statistics.f90:92
    const int end = start + (ncyc * per);                                   // 2d_statistics.f90:96
    double cd_avg = 0.0, cl_avg = 0.0;
    for (int i = start; i <= end; ++i) {                                    // 2d_statistics.f90:114-130
        const int mc = i - start;
        const double cd = f_drag[i - 1] / f_norm;
        const double cl = f_lift[i - 1] / f_norm;
        cd_avg = ((double)mc * cd_avg + cd) / (double)(mc + 1);
        cl_avg = ((double)mc * cl_avg + (cl * cl)) / (double)(mc + 1);
    }
    if (St) *St = D_cy / ((double)per * uo);                                // 2d_statistics.f90:98
    if (Cd_mean) *Cd_mean = cd_avg;
    if (Cl_rms) *Cl_rms = std::sqrt(cl_avg);                                // 2d_statistics.f90:131
    if (cycle_start) *cycle_start = start;
    if (period) *period = per;
    if (n_cycle) *n_cycle = ncyc;
    return MRLBM_OK;
}

int mrlbm_cp_statistics(const double* p_surface, int32_t nstep, int32_t nbct, int32_t cycle_start, int32_t period,
                        int32_t n_cycle, double rho_infty, double uo, double* cp) {
    if (!p_surface || !cp || nbct <= 0 || cycle_start < 1) return MRLBM_EINVAL;
    const int end = cycle_start + n_cycle * period;
    if (end > nstep) return MRLBM_EINVAL;
    const double p_infty = rho_infty / 3.0;                                 // 2d_statistics.f90:29
    const double p_norm = 0.50 * rho_infty * (uo * uo);                     // 2d_statistics.f90:31
    for (int k = 0; k < nbct; ++k) {
        double avg = 0.0;
        for (int i = cycle_start; i <= end; ++i) {                          // 2d_statistics.f90:114-121
            const int mc = i - cycle_start;
            avg = ((double)mc * avg + p_surface[(size_t)(i - 1) * nbct + k]) / (double)(mc + 1);
        }
        cp[k] = (avg - p_infty) / p_norm;
    }
    return MRLBM_OK;
}

}  // extern "C"
