"""Build recipe for the oracle (test infrastructure only).

- ``oracle/libbh_oracle.so``: the C restatement in ``bh_oracle.c``, compiled
  with gcc, OpenMP and ``-ffp-contract=off`` (every f32 operation rounds as
  written).  Tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
  ``bench.py`` load it; the engine never does.
- ``oracle/_ref/``: a mechanical C++ translation of the reference's own WGSL
  compute shaders, and of the fragment stages of its render shaders, produced
  by ``wgsl_to_cpp.py`` from the shader files where they lie in the
  reference checkout.  Built only where that checkout exists
  (the build container); its outputs stay out of version control.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libbh_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
# Where the reference checkout lies: BH_REFERENCE_CHECKOUT, or the build
# container's mount point.  Absent (e.g. on a GPU host), oracle/_ref is not
# rebuilt and the prebuilt files are used as they are.
REFERENCE_CHECKOUT = os.environ.get("BH_REFERENCE_CHECKOUT") or "/root/reference"

CFLAGS = ["-O3", "-march=x86-64-v2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
          "-fPIC", "-shared", "-std=c11", "-Wall"]


def _newer(target: str, deps: list[str]) -> bool:
    return os.path.exists(target) and all(os.path.getmtime(d) <= os.path.getmtime(target) for d in deps)


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "bh_oracle.c")
    hdr = os.path.join(HERE, "bh_oracle.h")
    if not force and _newer(LIB, [src, hdr, os.path.abspath(__file__)]):
        return LIB
    cc = shutil.which("gcc") or "cc"
    tmp = LIB + ".tmp"
    subprocess.run([cc, *CFLAGS, "-o", tmp, src, "-lm"], check=True)
    os.replace(tmp, LIB)
    return LIB


def build_ref(force: bool = False) -> str | None:
    """Translate and compile the reference WGSL (only where the checkout exists)."""
    shaders = os.path.join(REFERENCE_CHECKOUT, "src", "shaders", "compute")
    if not os.path.isdir(shaders) or not os.path.exists(os.path.join(HERE, "wgsl_to_cpp.py")):
        return None
    sys.path.insert(0, HERE)
    import wgsl_to_cpp  # noqa: E402  (sibling module of this recipe)
    lib = wgsl_to_cpp.build(shaders, REF_DIR, force=force)
    render = os.path.join(REFERENCE_CHECKOUT, "src", "shaders", "render")
    if os.path.isdir(render):
        wgsl_to_cpp.build_render(render, REF_DIR, force=force)
    return lib


def build(force: bool = False) -> None:
    build_oracle(force)
    build_ref(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
