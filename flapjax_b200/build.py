"""Build libfj_uvlm.so (the sm_100a CUDA library) in-tree with nvcc.

``python -m flapjax_b200.build`` compiles every ``csrc/*.cu`` for
``-gencode arch=compute_100a,code=sm_100a`` and links ``flapjax_b200/_lib/libfj_uvlm.so``.
Objects are rebuilt only when a source or header is newer than them.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "libfj_uvlm.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O2,-fvisibility=hidden",
    "-Xptxas",
    "-O3",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: set NVCC or install the CUDA toolkit")


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *_deps()])


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.stem + ".o")
    if not _stale(obj, src):
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(sources))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), sources))
    if LIB.exists() and all(LIB.stat().st_mtime >= o.stat().st_mtime for o in objs):
        return LIB
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def xla_include_dir() -> Path | None:
    """jaxlib's FFI header directory (jax.ffi.include_dir()), or None without JAX."""
    try:
        import jax.ffi
    except ImportError:
        return None
    return Path(jax.ffi.include_dir())


def build_xla(verbose: bool = False) -> Path:
    """libfj_xla.so: the XLA FFI handlers of xla/fj_xla.cc, linked against libfj_uvlm.so."""
    inc = xla_include_dir()
    if inc is None:
        raise RuntimeError("the XLA FFI handlers need jaxlib's headers (jax.ffi.include_dir()); JAX is not installed")
    lib = build(verbose)
    out = LIB_DIR / "libfj_xla.so"
    cmd = [nvcc(), *ARCH, "-shared", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-I", str(inc), "-I", str(INCLUDE),
           str(PKG / "xla" / "fj_xla.cc"), "-o", str(out), "-L", str(LIB_DIR), "-lfj_uvlm", "-lcudart",
           "-Xlinker", "-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"fj_xla.cc failed:\n{r.stdout}\n{r.stderr}")
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
    if "--xla" in sys.argv:
        print(build_xla(verbose="-v" in sys.argv))
