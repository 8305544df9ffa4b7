"""Build the CUDA library in-tree: particleclem_b200/_lib/libpcg_hydro.so.

Translation units, all for sm_100a (the kernel units once per species count of the
build, compiled in parallel):
  pcg_kernels_strict.cu  FP64 kernels, --fmad=false (reference rounding, operation by operation)
  pcg_kernels_fast.cu    FP64 with FMA contraction (and the FP64 step tail of the fast forms)
  pcg_kernels_mixed.cu   the mixed form's FP32 stage kernels (FP32 division and square root
                         approximate)
  pcg_host.cu            host runtime and the C ABI of include/pcg_hydro.h
  pcg_fluxreg.cu         flux register, reflux and average-down (coarse/fine levels)

Species counts. The reference fixes NUM_SPECIES at compile time from its mechanism
(Source/IndexDefines.H:50-89), and so does this library: PCG_NSPEC (a comma-separated
list, default 1,2,3,9,21: the gamma law, a two-species air, a three-species fuel model,
the 9-species hydrogen mechanism and a 21-species methane mechanism) picks the counts
kernels are compiled for; a PeleC build adds its own mechanism's count. Calls with any
other count return PCG_EUNSUPPORTED.
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
DEFAULT_NSPEC = (1, 2, 3, 9, 21)


def species_counts():
    """The species counts kernels are built for (PCG_NSPEC, e.g. "1,9,53")."""
    env = os.environ.get("PCG_NSPEC", "").strip()
    if not env:
        return DEFAULT_NSPEC
    ns = sorted({int(v) for v in env.replace(" ", "").split(",") if v})
    if not ns or ns[0] < 1:
        raise ValueError(f"PCG_NSPEC={env!r}: species counts must be positive integers")
    return tuple(ns)


def max_species(counts):
    """Bank size of the EOS tables: the largest count, even, at least 16."""
    m = max(16, max(counts))
    return m + (m % 2)


def units(counts):
    """(object tag, source, flags) of every translation unit: each kernel unit once per
    species count, all units with the same EOS bank size."""
    bank = [f"-DPCG_MAXNS={max_species(counts)}"]
    out = [(f"{name}_ns{ns}", f"pcg_kernels_{name}.cu", [*flags, f"-DPCG_TU_NS={ns}", *bank])
           for name, flags in (("strict", ["--fmad=false"]),
                               # FP32 division and square root as the hardware approximations
                               # (about 2 ulp): the mixed form's tolerance is 1e-6; FP64
                               # arithmetic is not affected by these flags
                               ("fast", FAST), ("mixed", FAST))
           for ns in counts]
    # the largest units first, so that they do not start last in the parallel build
    out.sort(key=lambda u: -int(u[0].rsplit("ns", 1)[1]))
    # the coarse/fine calls: FP64 sums in a fixed order without contraction, as the oracle
    return out + [("host", "pcg_host.cu", bank), ("fluxreg", "pcg_fluxreg.cu", ["--fmad=false"])]


UNITS = units(species_counts())
STAMP = os.path.join(LIBDIR, "libpcg_hydro.nspec")  # the species counts of the in-tree build


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources_mtime() -> float:
    paths = [os.path.join(SRC, f) for f in os.listdir(SRC)] + [os.path.join(ROOT, "include", "pcg_hydro.h")]
    return max(os.path.getmtime(p) for p in paths)


def up_to_date() -> bool:
    try:
        stamp = open(STAMP).read().strip()
    except OSError:
        return False
    return (os.path.exists(LIB) and os.path.getmtime(LIB) >= _sources_mtime()
            and stamp == ",".join(map(str, species_counts())))


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
        flags = list(extra_flags) + (list(extra) if src.startswith("pcg_kernels") else [])
        cmd = [cc, *COMMON, *ARCH, *flags, "-c", os.path.join(SRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return obj

    counts = species_counts()
    todo = units(counts)
    with ThreadPoolExecutor(max_workers=min(len(todo), max(1, os.cpu_count() or 1))) as ex:
        objs = list(ex.map(compile_unit, todo))
    tmp = out + ".tmp"
    cmd = [cc, "-shared", *ARCH, "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, out)
    for o in objs:
        os.remove(o)
    if out == LIB:
        with open(STAMP, "w") as f:
            f.write(",".join(map(str, counts)) + "\n")
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
