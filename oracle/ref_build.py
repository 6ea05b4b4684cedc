"""Compile the reference's own CUDA sampling extension into ``oracle/_ref``.

Test infrastructure only.  This recipe builds ``nect/sampling/ct_sampling.cu``
from the reference checkout named by the ``NECT_REFERENCE`` environment
variable (the ``ref`` target of ``oracle/Makefile`` sets it; with it unset
nothing is built) exactly as its ``setup.py:12-26`` would (same nvcc flags:
``-g -D__USE_GPU -DCUDA_VERSION=12030 -O3``), but for sm_100a only and without
running the reference's build system.  The result, ``oracle/_ref/ct_sampling.so``,
is the GPU-side authority for the sampling kernel: GPU parity tests and the
golden-fixture script import it to compare sample positions and per-ray counts
bit for bit.  Nothing on the product path imports it.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"


def reference_root() -> Path | None:
    root = os.environ.get("NECT_REFERENCE")
    return Path(root) if root else None


def build(verbose: bool = False) -> Path | None:
    root = reference_root()
    if root is None:
        print("[oracle/_ref] NECT_REFERENCE is not set; skipping the reference build", file=sys.stderr)
        return None
    src = root / "nect" / "sampling" / "ct_sampling.cu"
    if not src.exists():
        print(f"[oracle/_ref] reference source {src} not present; skipping", file=sys.stderr)
        return None
    OUT.mkdir(parents=True, exist_ok=True)
    so = OUT / "ct_sampling.so"
    if so.exists() and so.stat().st_mtime >= src.stat().st_mtime:
        return so
    from torch.utils import cpp_extension

    os.environ.setdefault("MAX_JOBS", "4")
    cpp_extension.load(
        name="ct_sampling",
        sources=[str(src)],
        build_directory=str(OUT),
        extra_cflags=["-g", "-D__USE_GPU"],
        extra_cuda_cflags=["-g", "-D__USE_GPU", "-DCUDA_VERSION=12030", "-O3",
                           "-gencode=arch=compute_100a,code=sm_100a"],
        verbose=verbose,
        is_python_module=True,
    )
    return so if so.exists() else None


def load():
    """Import the prebuilt reference extension from ``oracle/_ref``."""
    import importlib.machinery
    import importlib.util

    import torch  # noqa: F401  (the extension links against libtorch)

    so = OUT / "ct_sampling.so"
    if not so.exists():
        raise FileNotFoundError(f"{so} is missing: run `make -C oracle ref` where the reference is checked out")
    loader = importlib.machinery.ExtensionFileLoader("ct_sampling", str(so))
    spec = importlib.util.spec_from_loader("ct_sampling", loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    print(build(verbose=True))
