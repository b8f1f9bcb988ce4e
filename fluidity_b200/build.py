"""Builds the CUDA library fluidity_b200/_lib/libfluidity_b200.so for sm_100a.

Every translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` (plus the per-file
flags of EXTRA) and linked into one
shared object with a C-ABI (include/fluidity_b200.h). The library is built in
tree so it travels with the working copy; nothing is installed.

When the FluidiTy sources are present ($FLUIDITY_REFERENCE, or the checkout
beside this repository), the backend-table adapter (adapter/) is compiled
against their headers with g++ into _lib/libfluidity_b200_backend.so, linked
to the CUDA library. It leaves the reference's own symbols (the sparse grid
view's accessors) to the program that loads it, as a plug-in of that tree does.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "csrc"
OUT = HERE / "_lib"
LIB = OUT / "libfluidity_b200.so"
BACKEND = OUT / "libfluidity_b200_backend.so"
SOURCES = ["fl_grid.cu", "fl_p2g.cu", "fl_g2p.cu", "fl_pressure.cu", "fl_quanta.cu", "fl_context.cu", "fl_noalloc.cu",
           "fl_unet.cu", "fl_unet_tc.cu", "fl_snapshot.cu", "fl_mac_pressure.cu", "fl_boundary.cu",
           "fl_unet_train_tc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Per-file flags: the reference-shaped pressure operator keeps every FP64
# product apart from the sum it enters, as the reference's arithmetic does.
EXTRA = {"fl_mac_pressure.cu": ["-fmad=false"], "fl_boundary.cu": ["-fmad=false"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(obj: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    objdir = OUT / "obj"
    objdir.mkdir(exist_ok=True)
    headers = list(SRC.glob("*.h")) + list(SRC.glob("*.cuh")) + [HERE.parent / "include" / "fluidity_b200.h"]
    objs = []
    procs = []
    for src in SOURCES:
        s = SRC / src
        o = objdir / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc(), "-std=c++17", *ARCH, "-O3", "-lineinfo", *EXTRA.get(src, []), "-Xcompiler", "-fPIC", "-c",
                   str(s), "-o", str(o)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out.decode())
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
        if verbose:
            sys.stdout.write(out.decode())
    if force or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", *ARCH, "-o", str(LIB), *map(str, objs), "-lcudart", "-lcublas"]
        subprocess.check_call(cmd)
    build_backend(force)
    return LIB


def reference_root() -> Path:
    return Path(os.environ.get("FLUIDITY_REFERENCE", HERE.parent.parent / "reference"))


def build_backend(force: bool = False) -> Path | None:
    """The LiquidSubstepBackend3D adapter; None where the reference headers are absent."""
    ref = reference_root() / "native" / "include"
    if not ref.is_dir():
        return None
    ad = HERE / "adapter"
    src = ad / "b200_liquid_substep_backend_3d.cc"
    deps = [src, ad / "b200_liquid_substep_backend_3d.h", HERE.parent / "include" / "fluidity_b200.h", LIB]
    deps += list((ad / "absl_shim").rglob("*.h"))
    if force or _stale(BACKEND, deps):
        cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-o", str(BACKEND), str(src),
               f"-I{ad / 'absl_shim'}", f"-I{ref}", f"-I{HERE.parent / 'include'}", f"-L{OUT}", "-lfluidity_b200",
               "-Wl,-rpath,$ORIGIN"]
        subprocess.check_call(cmd)
    return BACKEND


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
