"""Build libphieng_sph.so in-tree with nvcc for sm_100a (B200).

    python -m phi_eng_b200.build [--force] [--verbose]

The SPH translation units are compiled with --fmad=false and IEEE division /
square root: the kernels keep the reference's f32 evaluation order, and an
FMA contraction would change results. Nothing here needs a GPU; nvcc
cross-compiles.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libphieng_sph.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", os.path.join(ROOT, "include")]
# exact-f32 units: no FMA contraction, IEEE div/sqrt, no flush-to-zero
EXACT = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]

# (source, extra flags)
UNITS = [
    ("sph_kernels.cu", EXACT),
    ("sph_world.cu", EXACT),
    ("sph_noalloc.cu", EXACT),
    ("sph_mlp.cu", EXACT),
    ("sph3d.cu", EXACT),
    ("sph_slab.cu", EXACT),
]
HEADERS = ["sph_device.cuh", "sph_kernels.h", "sph_mlp.cuh", "sph_mlp_host.h", "sph_warp.cuh", "sph_host.h", "sph_snapshot.h",
           "sph_noise.cuh", "sph_fast.cuh", "sph_tc.cuh", "sph_tc_net.cuh",
           "sph_closure_tc.cuh"]


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def _run(cmd, verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed: {' '.join(cmd)}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr_t = max([_mtime(os.path.join(CSRC, h)) for h in HEADERS] + [_mtime(os.path.join(ROOT, "include", "phieng_sph.h"))])
    objs = []
    relink = force or not os.path.exists(LIB)
    for src, extra in UNITS:
        sp = os.path.join(CSRC, src)
        op = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(op)
        if force or _mtime(op) < max(_mtime(sp), hdr_t, _mtime(__file__)):
            cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", sp, "-o", op]
            if ptxas_v:
                cmd += ["-Xptxas", "-v"]
            _run(cmd, verbose or ptxas_v)
            relink = True
    if relink or any(_mtime(o) > _mtime(LIB) for o in objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs], verbose)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print registers / spills / smem per kernel")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_v=a.ptxas_v))


if __name__ == "__main__":
    main()
