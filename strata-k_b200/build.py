"""Build recipe for the engine's shared library (sm_100a only).

Compiles every ``csrc/*.cu`` with nvcc for ``compute_100a``/``sm_100a`` into
``strata_b200/libstrata_b200.so`` (in-tree, so it travels with the sources).
Objects are rebuilt only when a source or header is newer than the library.

    python strata-k_b200/build.py [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
OUT_DIR = HERE / "strata_b200"
LIB = OUT_DIR / "libstrata_b200.so"
OBJ_DIR = HERE / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    f"-I{INCLUDE}",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA 12.9 toolkit is required to build")
    return cand


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _newest_dep() -> float:
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    deps.append(Path(__file__))
    return max(p.stat().st_mtime for p in deps)


def needs_build() -> bool:
    return not LIB.exists() or LIB.stat().st_mtime < _newest_dep()


def _compile(src: Path, extra: list[str]) -> Path:
    obj = OBJ_DIR / (src.stem + ".o")
    cmd = [nvcc(), *NVFLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None, extra: list[str] | None = None,
          verbose: bool = False) -> Path:
    """Compile the library if it is missing or stale; return its path."""
    if not force and not needs_build():
        return LIB
    OBJ_DIR.mkdir(exist_ok=True)
    extra = list(extra or [])
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), srcs))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    if verbose:
        print(f"built {LIB}")
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true", help="print registers / spills")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_verbose else []
    if a.ptxas_verbose:
        OBJ_DIR.mkdir(exist_ok=True)
        for s in sources():
            cmd = [nvcc(), *NVFLAGS, *extra, "-c", str(s), "-o", str(OBJ_DIR / (s.stem + ".o"))]
            r = subprocess.run(cmd, capture_output=True, text=True)
            sys.stdout.write(r.stderr)
        return 0
    build(force=a.force, jobs=a.jobs, verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
