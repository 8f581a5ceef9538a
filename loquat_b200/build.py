"""Build the LOQUAT-B200 shared library for sm_100a.

    python -m loquat_b200.build [--verbose-ptxas] [--force]

Compiles every ``csrc/*.cu`` / ``csrc/*.cpp`` with nvcc
(``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``) into objects under
``loquat_b200/_build/`` and links ``loquat_b200/liblqb200.so`` in-tree, with
the CUDA runtime linked statically so the library needs no loader path.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "liblqb200.so"
APP_SRC = PKG / "app" / "loquat_main.cpp"
APP = PKG / "bin" / "loquat"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3,-fvisibility=default",
    f"-I{INCLUDE}", f"-I{CSRC}",
]


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers():
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h")))


def _stale(obj: Path, src: Path, hdr_mtime: float) -> bool:
    if not obj.exists():
        return True
    m = obj.stat().st_mtime
    return m < src.stat().st_mtime or m < hdr_mtime


def _compile(src: Path, ptxas_verbose: bool, extra=(), build_dir: Path = BUILD) -> tuple[Path, str]:
    obj = build_dir / (src.name + ".o")
    cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
    if ptxas_verbose and src.suffix == ".cu":
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = True, defines=(), out: Path | None = None,
          build_dir: Path | None = None) -> Path:
    """Compile and link the library; returns its path.  `defines` adds -D
    options and `out`/`build_dir` place a variant build elsewhere."""
    bdir, lib = BUILD, LIB
    if out is not None:
        bdir, lib = Path(build_dir or Path(out).parent / "_build"), Path(out)
    bdir.mkdir(parents=True, exist_ok=True)
    extra = [f"-D{d}" for d in defines]
    hdr_mtime = max((h.stat().st_mtime for h in _headers()), default=0.0)
    srcs = _sources()
    todo = [s for s in srcs if force or ptxas_verbose or _stale(bdir / (s.name + ".o"), s, hdr_mtime)]
    reports = []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for obj, err in ex.map(lambda s: _compile(s, ptxas_verbose, extra, bdir), todo):
                if err.strip():
                    reports.append((obj.name, err))
    objs = [bdir / (s.name + ".o") for s in srcs]
    if force or todo or not lib.exists() or lib.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if out is None:
        build_app(force=force)
    if not quiet or ptxas_verbose:
        for name, err in reports:
            print(f"== {name}\n{err}", file=sys.stderr)
    return lib


CHECKED_LIB = PKG / "liblqb200_checked.so"


def build_checked(force: bool = False) -> Path:
    """The bounds-checked variant (-D LQ_CHECKED): every index the list and
    grid kernels gather or scatter through is checked before the access and
    a violation is counted (lq_debug_bounds_violations) instead of made.
    It stands in for a device memory checker.  Its Adami walks the lists in
    pairs at every size (LQ_ADAMI_PAIR_TARGETS=0; the product build does so
    from 4 M boundary particles on), so the checked runs cover that path.
    Loaded in place of the product library by setting LOQUAT_B200_LIB to
    its path."""
    return build(force=force, defines=["LQ_CHECKED", "LQ_ADAMI_PAIR_TARGETS=0"], out=CHECKED_LIB,
                 build_dir=PKG / "_build_checked")


def build_app(force: bool = False) -> Path:
    """The `loquat` command-line driver, linked against the library
    (found beside it through an rpath of $ORIGIN/..)."""
    APP.parent.mkdir(exist_ok=True)
    if not force and APP.exists() and APP.stat().st_mtime >= max(APP_SRC.stat().st_mtime, LIB.stat().st_mtime):
        return APP
    cmd = [NVCC, *ARCH, "-O2", "-std=c++17", f"-I{INCLUDE}", str(APP_SRC), f"-L{PKG}", "-llqb200",
           "-Xlinker", "-rpath,$ORIGIN/..", "-o", str(APP)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return APP


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("-D", dest="defines", action="append", default=[], help="preprocessor definition")
    ap.add_argument("--out", type=Path, default=None, help="variant library path (objects beside it)")
    a = ap.parse_args(argv)
    lib = build(force=a.force or bool(a.defines), ptxas_verbose=a.verbose_ptxas, quiet=False, defines=a.defines,
                out=a.out)
    print(lib)


if __name__ == "__main__":
    main()
