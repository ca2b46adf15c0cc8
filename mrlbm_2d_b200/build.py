"""Build libmrlbm.so in-tree: hand-written sm_100a CUDA kernels plus the C++ host layer.

    python -m mrlbm_2d_b200.build [--force]

Every CUDA translation unit is compiled with
`-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`; the FP64 step additionally with
`-fmad=false` (no contraction, so the FP64 step rounds exactly like the reference).  Host
geometry code is compiled with -ffp-contract=off for the same reason.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "libmrlbm.so")
DRIVER = os.path.join(PKG, "mrlbm_run")
STATS = os.path.join(PKG, "mrlbm_statistics")
BUILD = os.path.join(PKG, "_build")
ROOT = os.path.dirname(PKG)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + ["-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
                      "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills"]
CU_UNITS = {
    "step_f64.cu": ["-fmad=false"],
    "step_f32.cu": [],
    "adjoint.cu": [],
    "noalloc.cu": [],
    "state_io.cu": [],
}
CPP_UNITS = ["geometry.cpp", "capi.cpp", "statistics.cpp"]


def _nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h", ".cpp")):
                out.append(os.path.join(d, f))
    return out


def up_to_date():
    if not os.path.exists(OUT) or not os.path.exists(DRIVER) or not os.path.exists(STATS):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "include")
    # every translation unit is compiled in its own process, all at once
    objs, cmds = [], []
    for src, extra in CU_UNITS.items():
        obj = os.path.join(BUILD, src + ".o")
        cmd = [nvcc] + NVCC_COMMON + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        cmds.append(cmd)
        objs.append(obj)
    for src in CPP_UNITS:
        obj = os.path.join(BUILD, src + ".o")
        cmds.append(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                     "-I" + cuda_inc, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    procs = [subprocess.Popen(c) for c in cmds]
    failed = [c for c, pr in zip(cmds, procs) if pr.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    tmp = OUT + ".tmp"
    subprocess.run([nvcc] + ARCH + ["-shared", "-o", tmp] + objs, check=True)
    os.replace(tmp, OUT)
    # the input.dat-driven host driver (mrlbm_run) over the public C ABI
    drv_obj = os.path.join(BUILD, "driver_main.cpp.o")
    subprocess.run(["g++", "-std=c++17", "-O2", "-c", os.path.join(CSRC, "driver_main.cpp"), "-o", drv_obj],
                   check=True)
    subprocess.run(["g++", "-o", DRIVER, drv_obj, "-L" + PKG, "-lmrlbm", "-Wl,-rpath,$ORIGIN"], check=True)
    # the input_stat.dat-driven post-processing driver (mrlbm_statistics) over the same ABI
    st_obj = os.path.join(BUILD, "stats_main.cpp.o")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-c", os.path.join(CSRC, "stats_main.cpp"), "-o",
                    st_obj], check=True)
    subprocess.run(["g++", "-o", STATS, st_obj, "-L" + PKG, "-lmrlbm", "-Wl,-rpath,$ORIGIN"], check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
