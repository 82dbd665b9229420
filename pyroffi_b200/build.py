"""Build ``libpyroffi_b200.so`` (sm_100a) in-tree with nvcc.

    python -m pyroffi_b200.build            # build if sources changed
    python -m pyroffi_b200.build --force    # rebuild

Each ``csrc/*.cu`` compiles to an object under ``pyroffi_b200/_build/`` (in
parallel), then the objects link into ``pyroffi_b200/libpyroffi_b200.so``.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libpyroffi_b200.so"
HEADERS = [ROOT / "include" / "pyroffi_b200.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + HEADERS


def _compile(src: Path, verbose_ptxas: bool) -> tuple[Path, str]:
    obj = BUILD / (src.stem + ".o")
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stdout + r.stderr


def build(force: bool = False, verbose_ptxas: bool = False, quiet: bool = True) -> Path:
    srcs = _sources()
    newest_dep = max(p.stat().st_mtime for p in _deps())
    BUILD.mkdir(exist_ok=True)
    todo = []
    for s in srcs:
        obj = BUILD / (s.stem + ".o")
        if force or verbose_ptxas or not obj.exists() or obj.stat().st_mtime < max(s.stat().st_mtime, newest_dep):
            todo.append(s)
    logs = []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 4)) as ex:
            for obj, log in ex.map(lambda s: _compile(s, verbose_ptxas), todo):
                logs.append(log)
    objs = [BUILD / (s.stem + ".o") for s in srcs]
    if todo or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    if not quiet:
        for log in logs:
            if log.strip():
                print(log)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register / spill / smem usage")
    args = ap.parse_args(argv)
    lib = build(force=args.force, verbose_ptxas=args.ptxas_v, quiet=False)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
