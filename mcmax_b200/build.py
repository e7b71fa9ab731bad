"""Build libmcmax_gpu.so in-tree for sm_100a with nvcc.

The library is plain CUDA C++ behind the C-ABI of include/mcmax_gpu.h.  The
FP64 translation units are compiled with --fmad=false so that every a*b+c is
rounded twice, as in the CPU oracle; that is what makes the opacity tables
and the serial transport replay bit-identical.
"""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmcmax_gpu.so")
BUILD = os.path.join(HERE, "_build")

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off"]
# translation unit -> extra flags
UNITS = {
    "mcg_api.cu": ["--fmad=false"],
    "part_kernels.cu": ["--fmad=false"],
    "transport.cu": ["--fmad=false"],
    "host_tables.cu": ["--fmad=false"],
    "transport_fast.cu": [],
    "mlp_kernels.cu": [],
    "diffuse.cu": ["--fmad=false"],
    "dstruct.cu": ["--fmad=false"],
    "raytrace.cu": ["--fmad=false"],
    "scatfield.cu": ["--fmad=false"],
}
HEADERS = ["detmath.h", "cplx.h", "philox.h", "dhs_core.cuh", "transport_core.cuh", "transport_fast.cuh",
           "mcg_internal.h", "tc_sm100.cuh", "diffuse_core.cuh", "transport_event.cuh",
           "dstruct_core.cuh", "rt_core.cuh", "scat_core.cuh", "scatfield.h", "surrogate_phase.h"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def build(force=False, verbose=False):
    """Compile every CUDA unit and link libmcmax_gpu.so.  Returns the path."""
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "mcmax_gpu.h")]
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= _newest([src] + hdrs):
            continue
        cmd = [nvcc] + NVCC_ARCH + COMMON + extra + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [nvcc] + NVCC_ARCH + ["-shared", "-o", LIB] + objs + ["-lquadmath"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
