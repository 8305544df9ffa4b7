"""Build the CUDA library in-tree: particleclem_b200/_lib/libpcg_hydro.so.

Translation units, all for sm_100a (the kernel units once per species count, 1 and 9,
compiled in parallel):
  pcg_kernels_strict.cu  FP64 kernels, --fmad=false (reference rounding, operation by operation)
  pcg_kernels_fast.cu    FP64 with FMA contraction (and the FP64 step tail of the fast forms)
  pcg_kernels_mixed.cu   the mixed form's FP32 stage kernels (FP32 division and square root
                         approximate)
  pcg_host.cu            host runtime and the C ABI of include/pcg_hydro.h
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libpcg_hydro.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", SRC, "-I", os.path.join(ROOT, "include")]
FAST = ["--fmad=true", "-prec-div=false", "-prec-sqrt=false"]
# (object tag, source, flags): each kernel unit is built once per species count
UNITS = [(f"{name}_ns{ns}", f"pcg_kernels_{name}.cu", [*flags, f"-DPCG_TU_NS={ns}"])
         for name, flags in (("strict", ["--fmad=false"]),
                             # FP32 division and square root as the hardware approximations
                             # (about 2 ulp): the mixed form's tolerance is 1e-6; FP64
                             # arithmetic is not affected by these flags
                             ("fast", FAST), ("mixed", FAST))
         for ns in (1, 9)] + [("host", "pcg_host.cu", [])]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources_mtime() -> float:
    paths = [os.path.join(SRC, f) for f in os.listdir(SRC)] + [os.path.join(ROOT, "include", "pcg_hydro.h")]
    return max(os.path.getmtime(p) for p in paths)


def up_to_date() -> bool:
    return os.path.exists(LIB) and os.path.getmtime(LIB) >= _sources_mtime()


def build(force: bool = False, verbose: bool = False, out: str = LIB, extra=()) -> str:
    """Compile the three translation units and link ``out``. ``extra``: additional nvcc
    flags for the kernel units (e.g. -DPCG_MINB_FLUX2=4 register caps)."""
    if not force and out == LIB and up_to_date():
        return LIB
    os.makedirs(os.path.dirname(out), exist_ok=True)
    cc = nvcc()
    tag = os.path.basename(out).replace(".so", "")

    def compile_unit(item):
        tag_u, src, extra_flags = item
        obj = os.path.join(os.path.dirname(out), tag + "_" + tag_u + ".o")
        flags = list(extra_flags) + (list(extra) if src != "pcg_host.cu" else [])
        cmd = [cc, *COMMON, *ARCH, *flags, "-c", os.path.join(SRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return obj

    with ThreadPoolExecutor(max_workers=min(len(UNITS), max(1, os.cpu_count() or 1))) as ex:
        objs = list(ex.map(compile_unit, UNITS))
    tmp = out + ".tmp"
    cmd = [cc, "-shared", *ARCH, "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, out)
    for o in objs:
        os.remove(o)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
