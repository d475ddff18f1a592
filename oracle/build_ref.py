"""Build recipe for oracle/_ref/libref_bitsets.so -- TEST INFRASTRUCTURE ONLY.

The reference compiles its kernels at run time from CUDA source strings
(``_SOURCE`` in cupami/frequentPattern/_bitsets.py:19-78 -- the three bitset
kernels -- and in cupami/periodicFrequentPattern/_temporal.py:26-53 --
``periodic_counts``; NVRTC, cached per device).  This recipe compiles the same
strings ahead of time for sm_100a: it reads them out of the reference files
with ``ast`` (the modules are not imported or executed), writes them to a
temporary file under ``oracle/_ref/`` (deleted after the compile) and builds
``oracle/ref_launch.cu`` (host launchers written here) around it with nvcc.
Outputs go to ``oracle/_ref/`` only; that folder is git-ignored and ships with
the built library.  Without the reference sources (as on a machine that only
has the prebuilt files) it does nothing.

The cuPAMI checkout is the argument, else ``$CUPAMI_REFERENCE``, else a
directory named ``reference`` beside this repository's own directory.

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
DEFAULT_ROOT = Path(os.environ.get("CUPAMI_REFERENCE", HERE.parent.parent / "reference"))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


SOURCES = (("frequentPattern", "_bitsets.py"), ("periodicFrequentPattern", "_temporal.py"))


def reference_source(root: Path) -> str:
    """The kernel source strings of the reference files in SOURCES, one after the other."""
    out = []
    for package, name in SOURCES:
        src = (root / "cupami" / package / name).read_text()
        for node in ast.parse(src).body:
            if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == "_SOURCE" for t in node.targets):
                out.append(ast.literal_eval(node.value))
                break
        else:
            raise RuntimeError(f"_SOURCE not found in the reference's {name}")
    return "\n".join(out)


def build(root: Path = DEFAULT_ROOT, force: bool = False) -> Path | None:
    """Compile the reference kernels; returns the library path (None without the sources)."""
    ref_files = [root / "cupami" / package / name for package, name in SOURCES]
    if not all(f.exists() for f in ref_files):
        return LIB if LIB.exists() else None
    shim = HERE / "ref_launch.cu"
    newest = max([shim.stat().st_mtime, Path(__file__).stat().st_mtime] + [f.stat().st_mtime for f in ref_files])
    if not force and LIB.exists() and LIB.stat().st_mtime >= newest:
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
