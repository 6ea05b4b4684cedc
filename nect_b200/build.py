"""Build recipe for libnectb.so, the sm_100a CUDA library behind the C ABI.

Compiles every ``csrc/*.cu`` with nvcc for ``sm_100a`` only and links them
into ``nect_b200/_lib/libnectb.so`` (in-tree, so the library travels with the
source tree).  Objects are cached under ``_build/`` and rebuilt when a source
or header is newer.  ``python -m nect_b200.build [-v]`` runs it.
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
OBJ = ROOT / "_build" / "nectb"
LIB = PKG / "_lib" / "libnectb.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC",
    "-I" + str(INCLUDE),
]


def nvcc() -> str:
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda_home) / "bin" / "nvcc"
    if cand.exists():
        return str(cand)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found; set CUDA_HOME")
    return found


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, obj: Path, verbose: bool, ptxas_verbose: bool) -> str:
    cmd = [nvcc(), "-c", str(src), "-o", str(obj)] + NVCC_FLAGS
    if ptxas_verbose:
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    out = res.stdout + res.stderr
    if verbose and out.strip():
        print(out, file=sys.stderr)
    return out


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compile and link libnectb.so; returns its path."""
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    headers = _headers()
    jobs = []
    for src in sources:
        obj = OBJ / (src.stem + ".o")
        if force or ptxas_verbose or _stale(obj, [src] + headers):
            jobs.append((src, obj))
    if jobs:
        workers = min(len(jobs), os.cpu_count() or 4)
        with concurrent.futures.ThreadPoolExecutor(workers) as ex:
            futs = [ex.submit(_compile, s, o, verbose, ptxas_verbose) for s, o in jobs]
            for f in futs:
                f.result()
    objs = [OBJ / (s.stem + ".o") for s in sources]
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-o", str(LIB)] + objs + ARCH + ["-lcudart", "-lcuda"]
        res = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    print(build(verbose=v, force="-f" in sys.argv, ptxas_verbose="--ptxas" in sys.argv))
