"""Builds the native library ``statecraft_b200/_native/libstatecraft_b200.so`` for sm_100a.

    python -m statecraft_b200.build [--verbose] [--ptxas-info]

Every translation unit under ``csrc/`` is compiled by nvcc in parallel into
``csrc/_build/`` and linked into one shared library with the CUDA runtime linked
statically, so the library travels as a single in-tree file.
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
CSRC = PKG / "csrc"
OBJ = CSRC / "_build"
OUT = PKG / "_native" / "libstatecraft_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3,-fvisibility=hidden",
          "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> list[str]:
    # the system g++ is the one CUDA 12.9 supports; some images put another first on PATH
    for cand in ("/usr/bin/g++",):
        if Path(cand).exists():
            return ["-ccbin", cand]
    return []


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _compile(src: Path, verbose: bool, ptxas: bool) -> tuple[Path, str]:
    obj = OBJ / (src.name + ".o")
    deps = [src] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    if obj.exists() and all(obj.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return obj, ""
    cmd = [nvcc(), *host_compiler(), *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
    if ptxas and src.suffix == ".cu":
        cmd += ["-Xptxas", "-v"]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj, res.stderr


def build(verbose: bool = False, ptxas: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    OUT.parent.mkdir(parents=True, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose, ptxas), srcs))
    if ptxas:
        for _, log in results:
            if log:
                print(log)
    objs = [o for o, _ in results]
    newest = max(o.stat().st_mtime for o in objs)
    if OUT.exists() and OUT.stat().st_mtime >= newest:
        return OUT
    cmd = [nvcc(), *host_compiler(), *ARCH, "-shared", "-o", str(OUT), *map(str, objs),
           "-cudart", "static", "-Xcompiler", "-fPIC"]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return OUT


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    args = ap.parse_args(argv)
    out = build(args.verbose, args.ptxas_info)
    print(out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
