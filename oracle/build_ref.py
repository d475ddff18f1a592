"""Build recipe for oracle/_ref/libref_bitsets.so -- TEST INFRASTRUCTURE ONLY.

The reference compiles its three bitset kernels at run time from a CUDA source
string (``_SOURCE`` in cupami/frequentPattern/_bitsets.py:19-78, NVRTC, cached
per device).  This recipe compiles the same string ahead of time for sm_100a:
it reads the string out of the reference file with ``ast`` (the module is not
imported or executed), writes it to a temporary file under ``oracle/_ref/``
(deleted after the compile) and builds ``oracle/ref_launch.cu`` (host
launchers written here) around it with nvcc.
Outputs go to ``oracle/_ref/`` only; that folder is git-ignored and ships with
the built library.  Without the reference sources (as on a machine that only
has the prebuilt files) it does nothing.

    python oracle/build_ref.py [path/to/cupami]
"""

from __future__ import annotations

import ast
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
LIB = OUT / "libref_bitsets.so"
DEFAULT_ROOT = Path("/root/reference")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def reference_source(root: Path) -> str:
    src = (root / "cupami" / "frequentPattern" / "_bitsets.py").read_text()
    for node in ast.parse(src).body:
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == "_SOURCE" for t in node.targets):
            return ast.literal_eval(node.value)
    raise RuntimeError("_SOURCE not found in the reference's _bitsets.py")


def build(root: Path = DEFAULT_ROOT, force: bool = False) -> Path | None:
    """Compile the reference kernels; returns the library path (None without the sources)."""
    ref_file = root / "cupami" / "frequentPattern" / "_bitsets.py"
    if not ref_file.exists():
        return LIB if LIB.exists() else None
    shim = HERE / "ref_launch.cu"
    if not force and LIB.exists() and LIB.stat().st_mtime >= max(shim.stat().st_mtime, ref_file.stat().st_mtime):
        return LIB
    OUT.mkdir(exist_ok=True)
    cu = OUT / ("ref_bitsets.%d.cu" % os.getpid())  # build intermediate, removed below
    cu.write_text(reference_source(root))
    tmp = LIB.with_suffix(".so.tmp%d" % os.getpid())
    try:
        subprocess.check_call([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                               "-Xcompiler", "-fPIC", "-shared", f'-DREF_KERNELS="{cu}"', "-o", str(tmp), str(shim)])
    finally:
        cu.unlink(missing_ok=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT_ROOT, force=True))
