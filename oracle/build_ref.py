"""Builds the reference's own OpenCL C ray cast as a host shared library.

TEST INFRASTRUCTURE ONLY.  Reads ``opencl/treeletRenderer_rgba.cl`` from the
reference checkout named by ``$LIBSVO_REFERENCE`` (or the path given on the
command line: ``python oracle/build_ref.py <reference checkout>``),
rewrites its OpenCL vector literals ``(float3)(...)`` to ``make_float3(...)``
in memory, and pipes ``#include cl_shim.h`` + that text + ``ref_harness.inc``
to g++ over stdin.  No reference source is written to disk; the only output
is ``oracle/_ref/libsvo_ref_cl.so``.

The compile flags match the oracle's (``-O2 -ffp-contract=off``), so both
round every FP32 operation separately in source order.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "_ref"
OUT = OUT_DIR / "libsvo_ref_cl.so"
CL_REL = "opencl/treeletRenderer_rgba.cl"


def reference_root() -> Path | None:
    """The reference checkout named by $LIBSVO_REFERENCE, or None."""
    root = os.environ.get("LIBSVO_REFERENCE")
    return Path(root) if root else None


def transformed_source(cl_text: str) -> str:
    body = re.sub(r"\((float3|float4|int2)\)\s*\(", r"make_\1(", cl_text)
    return (
        f'#include "{HERE / "cl_shim.h"}"\n#line 1 "{CL_REL}"\n'
        + body
        + f'\n#include "{HERE / "ref_harness.inc"}"\n'
    )


def build(force: bool = False, reference: Path | str | None = None) -> Path | None:
    """Compiles the reference kernel for the host from the checkout at
    `reference` (default: $LIBSVO_REFERENCE); returns the .so path, or the
    one built earlier, or None when no checkout is named or present."""
    root = Path(reference) if reference else reference_root()
    cl = root / CL_REL if root else None
    if cl is None or not cl.is_file():
        return OUT if OUT.is_file() else None
    deps = [cl, HERE / "cl_shim.h", HERE / "ref_harness.inc", Path(__file__)]
    if OUT.is_file() and not force:
        if all(OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
            return OUT
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    src = transformed_source(cl.read_text(encoding="utf-8", errors="replace"))
    cmd = [
        "g++", "-x", "c++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math",
        "-fPIC", "-shared", "-pthread", "-w", "-o", str(OUT), "-",
    ]
    subprocess.run(cmd, input=src.encode(), check=True)
    return OUT


if __name__ == "__main__":
    paths = [a for a in sys.argv[1:] if not a.startswith("--")]
    p = build(force="--force" in sys.argv, reference=paths[0] if paths else None)
    print(p if p else "reference not present; nothing built")
