"""In-tree build of ``libcupami_b200.so`` for sm_100a (nvcc cross-compiles; no GPU needed)."""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SOURCES = [PKG / "csrc" / "cpm_runtime.cu"]
HEADERS = (sorted((PKG / "csrc").glob("*.cuh")) + sorted((PKG / "csrc").glob("*.inc"))
           + [ROOT / "include" / "cupami_b200.h"])
OUTPUT = PKG / "libcupami_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3,-fopenmp", "-shared", "-Xptxas", "-O3", "-lgomp",
]


def _nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    return str(path) if path.exists() else "nvcc"


def stale() -> bool:
    if not OUTPUT.exists():
        return True
    built = OUTPUT.stat().st_mtime
    return any(p.stat().st_mtime > built for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if any source is newer than it; returns its path."""
    if not force and not stale():
        return OUTPUT
    tmp = OUTPUT.with_name(OUTPUT.name + f".tmp{os.getpid()}")
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", str(ROOT / "include"), "-o", str(tmp), *map(str, SOURCES)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(tmp, OUTPUT)
    return OUTPUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
