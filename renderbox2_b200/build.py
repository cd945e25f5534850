"""Builds librb2.so in-tree (renderbox2_b200/_lib/librb2.so) for sm_100a.

Run as ``python -m renderbox2_b200.build``.  Host C++ is compiled with
``-ffp-contract=off`` so every float operation rounds once, as written (the
packer's Woop rows and the camera matrices must match the reference bit for
bit).  The CUDA runtime is linked statically so the library does not depend
on which libcudart another extension in the process loaded first.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "librb2.so"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-std=c++17", "-O3", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
            f"-I{INCLUDE}", f"-I{CSRC}", f"-I{CUDA_HOME / 'include'}"]
NVCCFLAGS = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-ffp-contract=off",
             "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]


def _sources():
    return sorted(CSRC.glob("*.cpp")) + sorted(CSRC.glob("*.cu"))


def _headers():
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _digest(extra: str = "") -> str:
    h = hashlib.sha256()
    for p in _sources() + _headers() + [Path(__file__)]:
        h.update(p.name.encode())
        h.update(p.read_bytes())
    h.update(extra.encode())
    return h.hexdigest()


def _compile(src: Path, obj: Path, verbose: bool) -> None:
    if src.suffix == ".cu":
        cmd = [NVCC, *NVCCFLAGS, "-c", str(src), "-o", str(obj)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd = ["g++", *CXXFLAGS, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stderr.strip() or r.stdout.strip()):
        print(r.stdout + r.stderr, file=sys.stderr)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every source under csrc/ and links librb2.so; returns its path."""
    OUT_DIR.mkdir(exist_ok=True)
    obj_dir = OUT_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    stamp = OUT_DIR / "librb2.stamp"
    digest = _digest()
    if not force and LIB.exists() and stamp.exists() and stamp.read_text() == digest:
        return LIB
    srcs = _sources()
    objs = [obj_dir / (s.stem + (".cu.o" if s.suffix == ".cu" else ".o")) for s in srcs]
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        list(ex.map(lambda so: _compile(so[0], so[1], verbose), zip(srcs, objs)))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-cudart", "static", "-lpthread", "-ldl", "-lrt"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    stamp.write_text(digest)
    return LIB


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(p)
