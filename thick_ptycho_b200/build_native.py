"""Build libtpcuda.so (the sm_100a kernels and their C ABI) in-tree.

Usage: ``python -m thick_ptycho_b200.build_native [--verbose]``.  The library
is written to ``thick_ptycho_b200/_lib/libtpcuda.so``; it links the CUDA
runtime statically and exports only the ``tp_*`` C symbols declared in
``include/tpcuda.h``.

Beside it, ``libtpcuda_c128.so`` is the complex128 check build of the
Crank–Nicolson paths: the same sources compiled with ``-DTP_C128_CHECK``, so
the 2D factorisation and marches (partitioned solve, truncated spikes, PCR
skip, Cayley step, pair-sum store, fused gradient) and the 3D march
(BiCGStab with the four-step or Stockham FFT preconditioner, exact adjoint
and gradient; no learned correction) run with complex128 state, operators
and fields.  It exports the ``tp_cn2d_*`` and ``tp_cn3d_*`` entry points
with every complex buffer complex128.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libtpcuda.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fvisibility=hidden"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; set NVCC or put the CUDA toolkit on PATH")


LIB_C128 = os.path.join(LIBDIR, "libtpcuda_c128.so")
# sources of the complex128 check build (the 2D factorisation and marches)
C128_SOURCES = ("tp_capi.cu", "cn2d.cu", "cn2d_team.cu", "cn3d.cu")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def build(verbose: bool = False, jobs: int = 0) -> str:
    """Compile every .cu under csrc/ for sm_100a and link libtpcuda.so, then
    the complex128 check build libtpcuda_c128.so."""
    lib = _build(sources(), [], LIB, verbose)
    _build([os.path.join(CSRC, f) for f in C128_SOURCES], ["-DTP_C128_CHECK"], LIB_C128, verbose)
    return lib


def _build(srcs, defines, out_lib, verbose):
    os.makedirs(LIBDIR, exist_ok=True)
    cc = nvcc()
    with tempfile.TemporaryDirectory() as tmp:
        objs = []
        procs = []
        for src in srcs:
            obj = os.path.join(tmp, os.path.basename(src) + ".o")
            cmd = [cc, *ARCH, *FLAGS, *defines, "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
            objs.append(obj)
        failed = []
        for src, pr in procs:
            out, _ = pr.communicate()
            if verbose and out:
                sys.stdout.write(out)
            if pr.returncode != 0:
                failed.append((src, out))
        if failed:
            msg = "\n".join(f"--- {s}\n{o}" for s, o in failed)
            raise RuntimeError("nvcc failed:\n" + msg)
        tmp_lib = os.path.join(tmp, os.path.basename(out_lib))
        link = [cc, *ARCH, "-shared", "-cudart", "static", "-o", tmp_lib, *objs]
        r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout)
        shutil.copy2(tmp_lib, out_lib + ".tmp")
        os.replace(out_lib + ".tmp", out_lib)
    return out_lib


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
