"""In-tree build of libofgpu.so (sm_100a) with nvcc.

Each translation unit is compiled to an object next to the sources
(openferric_b200/_build/) and linked into openferric_b200/libofgpu.so with a
static CUDA runtime, so the library carries no dependency on a CUDA install at
load time beyond the driver.  Rebuilds only what changed (mtime of the unit and
of every header in csrc/).

    python -m openferric_b200.build [--verbose] [--force]
"""
import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libofgpu.so")
INCLUDE = os.path.normpath(os.path.join(HERE, "..", "include"))
NVCC = os.environ.get("OF_NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I", CSRC, "-I", INCLUDE]
# Per-unit flags.  The FP64 reference-stream units must not contract a*b+c into
# fma: only explicit fma() calls (the reference's mul_add) may fuse.
UNIT_FLAGS = {
    "mc_reference.cu": ["--fmad=false"],
    "greeks_reference.cu": ["--fmad=false"],
    # FP64 mode: no contraction.  The single-precision flags (flush to zero,
    # approximate sqrt and divide) touch only the FP32 Philox mode.
    "lsm.cu": ["--fmad=false", "-ftz=true", "-prec-sqrt=false", "-prec-div=false"],
    "qmc.cu": ["--fmad=false"],
    "mc_philox.cu": ["-use_fast_math"],
    # explicit fmaf only, so the forward pass and the backward-sweep recompute
    # are bit-identical; MUFU approximations are written as intrinsics
    "adjoint.cu": ["--fmad=false", "-ftz=true"],
    "wgsl_port.cu": [],
}


def _units():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers_mtime():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def build(verbose=False, force=False, ptxas_verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    hdr = _headers_mtime()
    objs = []
    relink = force or not os.path.exists(LIB)
    for src in _units():
        name = os.path.basename(src)
        obj = os.path.join(OBJ, name.replace(".cu", ".o"))
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
            continue
        cmd = [NVCC, *ARCH, *COMMON, *UNIT_FLAGS.get(name, []), "-c", src, "-o", obj]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {name}")
        if verbose or ptxas_verbose:
            sys.stdout.write(r.stderr)
        relink = True
    if relink or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libofgpu.so failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/spill report")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force, ptxas_verbose=a.ptxas))
