"""Host-side integer arithmetic the kernels rely on, checked on the CPU.

tile_div_magic (mrlbm_2d_b200/csrc/step_params.h) gives the multiplier the step kernels use for
t / tiles_x as a multiply-high: exact for every t with t * d < 2^32, and 0 (plain division) when
a launch's tiles reach that bound.  step_launches gives the launch count per step the handles
report.  The checks compile a small C++ program against the header.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mrlbm_2d_b200", "csrc")
CUDA_INC = "/usr/local/cuda/include"

PROG = r"""
#include <cstdio>
#include <cstdint>
#include "step_params.h"
using namespace mrlbm;
int main() {
    long long bad = 0, checked = 0;
    uint64_t x = 88172645463325252ull;                      // xorshift64 for sample points
    for (int d = 1; d <= 4096; ++d) {
        const long long limit = ((1ll << 32) - 1) / d;       // largest t with t * d < 2^32
        const unsigned long long m = tile_div_magic(d, limit);   // tiles 0..limit-1: tiles * d < 2^32
        if (m == 0) { ++bad; continue; }
        auto check = [&](long long t) {
            const long long q = (long long)(((unsigned long long)t * m) >> 32);
            if (q != t / d) ++bad;
            ++checked;
        };
        for (long long t = 0; t < 2048 && t <= limit; ++t) check(t);
        for (long long t = limit; t > limit - 2048 && t >= 0; --t) check(t);
        for (int r = 0; r < 2048; ++r) {
            x ^= x << 13; x ^= x >> 7; x ^= x << 17;
            check((long long)(x % (unsigned long long)(limit + 1)));
        }
        if (tile_div_magic(d, limit + 1) != 0) ++bad;           // (limit + 1) * d >= 2^32: plain division
    }
    int launches_ok = 1;
    for (int c = 0; c < N_TILE_CFGS; ++c) {
        if (step_launches(true, c) != 1) launches_ok = 0;
        const TileCfg& t = TILE_CFGS[c];
        if (step_launches(false, c) != 2) launches_ok = 0;
        (void)t;
    }
    if (step_launches(true, VEC_CFG0) != 2 || step_launches(false, -1) != 2) launches_ok = 0;
    std::printf("%lld %lld %d\n", checked, bad, launches_ok);
    return 0;
}
"""


@pytest.mark.skipif(not os.path.isdir(CUDA_INC), reason="CUDA headers not installed")
def test_tile_division_magic_and_launch_counts(tmp_path):
    src = tmp_path / "magic.cpp"
    exe = tmp_path / "magic"
    src.write_text(PROG)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-I", CUDA_INC,
                    str(src), "-o", str(exe)], check=True)
    checked, bad, launches_ok = subprocess.run([str(exe)], check=True, capture_output=True,
                                               text=True).stdout.split()
    assert int(checked) > 10_000_000
    assert int(bad) == 0
    assert launches_ok == "1"
