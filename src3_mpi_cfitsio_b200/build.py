"""Build the engine's C-ABI library for sm_100a with nvcc.

Produces ``src3_mpi_cfitsio_b200/_lib/libmcrt_b200.so`` in-tree.  The FP64
transport translation unit is compiled with ``--fmad=false`` (no FMA
contraction) so that its IEEE operations match the CPU oracle's; the
mixed-precision unit keeps FMA contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libmcrt_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", os.path.join(HERE, "..", "include")]
UNITS = [("mcrt_b200.cu", []), ("mcrt_fp64.cu", ["--fmad=false"]), ("mcrt_mixed.cu", [])]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose: bool = False, ptxas_info: bool = False, out: str = LIB, defines=()) -> str:
    """Compile the library to `out`; `defines` are extra -D macros
    (compile-time tuning knobs of the kernels)."""
    libdir = os.path.dirname(out)
    os.makedirs(libdir, exist_ok=True)
    objs, procs = [], []
    for src, extra in UNITS:          # the translation units compile in parallel
        obj = os.path.join(libdir, src.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, *COMMON, *[f"-D{d}" for d in defines], *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out_s, err_s = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out_s + err_s)
            failed.append(src)
        elif ptxas_info or verbose:
            sys.stderr.write(err_s)
    if failed:
        raise RuntimeError(f"nvcc failed on {', '.join(failed)}")
    cmd = [nvcc(), *ARCH, "-shared", "-o", out, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    for o in objs:
        os.remove(o)
    return out


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
