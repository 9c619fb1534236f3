"""Builds pdp3_b200/libpdp3g.so with nvcc for sm_100a (in-tree, no JIT cache).

Translation units of the FP64 plain form are compiled with --fmad=false so
that their arithmetic matches the CPU step's operation by operation; the
FP32 cell-local form keeps fused multiply-add.

    python -m pdp3_b200.build [--force]
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpdp3g.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
# translation unit -> extra flags
UNITS = {
    "capi.cu": [],
    "fields.cu": ["--fmad=false"],
    "particles_f64.cu": ["--fmad=false"],
    # FP32 units: approximate division, square root and flush-to-zero (no
    # quantity of the step is near the subnormal range); the form's error
    # budget is set by FP32 storage, not by these operations
    "particles_f32.cu": ["-use_fast_math"],
    "sort.cu": [],
    "ensemble.cu": ["-use_fast_math"],
    "diag.cu": [],
    "noalloc.cu": [],
    "adjoint.cu": ["-use_fast_math"],
    "probe.cu": [],
    "species_diag.cu": ["--fmad=false"],
    "init.cu": ["--fmad=false"],
    "poisson.cu": ["--fmad=false"],
}
HEADERS = ["pdp3g_internal.cuh", "particles_f32.cuh", "fields_body.cuh", "adjoint_particle.cuh",
           "mj_tables.h"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(src_list, dst):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in src_list)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    nv = nvcc()
    # this file holds the flags: an edit of it rebuilds every unit
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "pdp3g.h"),
                                                       os.path.abspath(__file__)]
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _newer([src] + hdrs, obj):
            cmd = [nv] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _newer(objs, LIB):
        cmd = [nv] + ARCH + ["-shared", "--cudart", "static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    build_host(force, verbose)
    return LIB


HOST = os.path.join(HERE, "host")
HOST_LIB = os.path.join(HERE, "libpdp3_host.so")
LOOP_EXE = os.path.join(HERE, "pdp3g_loop")


def build_host(force=False, verbose=False):
    """The upstream-style C++ class layer (libpdp3_host.so) and the
    pdp3g_loop driver, linked against libpdp3g.so."""
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + HOST]
    rpath = ["-Wl,-rpath,$ORIGIN"]
    srcs = [os.path.join(HOST, "pdp3_classes.cpp"), os.path.join(HOST, "pdp3_classes.h"),
            os.path.join(ROOT, "include", "pdp3g.h")]
    if force or _newer(srcs + [LIB], HOST_LIB):
        cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-o", HOST_LIB,
               os.path.join(HOST, "pdp3_classes.cpp")] + inc + ["-L" + HERE, "-lpdp3g"] + rpath
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    loop_src = os.path.join(HOST, "pdp3g_loop.cpp")
    if force or _newer([loop_src, HOST_LIB], LOOP_EXE):
        cmd = [cxx, "-std=c++17", "-O2", "-o", LOOP_EXE, loop_src] + inc + \
              ["-L" + HERE, "-lpdp3_host", "-lpdp3g"] + rpath
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
