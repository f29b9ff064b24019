"""Builds the in-tree shared library ``dg_b200/lib/libdgb.so`` and the ``dgbexec`` driver.

Host setup (C++17) is compiled with g++; the device half with nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``).  Objects are cached under
``dg_b200/_build/`` and rebuilt when a source or header changes.

Usage: python -m dg_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC = PKG / "csrc"
INC = PKG.parent / "include"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libdgb.so"
EXE = LIBDIR / "dgbexec"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-Wall", "-Wno-sign-compare"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-Xptxas", "-warn-spills"] + ARCH
# per-file additions: the sensors take threshold decisions that must see the same separately
# rounded products and sums as the reference's CPU arithmetic, so no multiply-add contraction there
FILE_NVFLAGS = {"dgb_sensor.cu": ["-fmad=false"]}
SHIMS = [(1, "rus"), (1, "hll"), (1, "roe"), (2, "rus"), (2, "roe")]
SHIM_FLUX = {"rus": 0, "hll": 1, "roe": 2}


def _deps_digest(paths: list[Path]) -> str:
    h = hashlib.sha1()
    for p in sorted(paths):
        h.update(p.read_bytes())
    return h.hexdigest()


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    LIBDIR.mkdir(parents=True, exist_ok=True)
    headers = list(SRC.rglob("*.h")) + list(SRC.rglob("*.cuh")) + list(INC.glob("*.h"))
    hdr = _deps_digest(headers)
    objs = []
    jobs = []
    for src in sorted(SRC.rglob("*.cc")) + sorted(SRC.rglob("*.cu")):
        if src.name == "dgbexec.cc" or "shim" in src.parts:
            continue
        key = hashlib.sha1((hdr + src.read_text()).encode()).hexdigest()[:12]
        obj = BUILD / f"{src.stem}.{key}.o"
        objs.append(obj)
        if obj.exists() and not force:
            continue
        if src.suffix == ".cu":
            cmd = [NVCC] + NVFLAGS + FILE_NVFLAGS.get(src.name, []) + [f"-I{INC}", f"-I{SRC}", "-c", str(src), "-o",
                                                                       str(obj)]
        else:
            cmd = ["g++"] + CXXFLAGS + [f"-I{INC}", f"-I{SRC}", "-c", str(src), "-o", str(obj)]
        jobs.append(cmd)
    if jobs:
        import concurrent.futures as cf
        with cf.ThreadPoolExecutor(min(8, len(jobs))) as ex:
            for f in [ex.submit(_run, j, verbose) for j in jobs]:
                f.result()
    for stale in BUILD.glob("*.o"):
        if stale not in objs and not stale.name.startswith("dgb_shim_"):
            stale.unlink()
    stamp = hashlib.sha1("".join(str(o) for o in objs).encode()).hexdigest()
    stamp_file = BUILD / "libdgb.stamp"
    if force or not LIB.exists() or not stamp_file.exists() or stamp_file.read_text() != stamp:
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs], verbose)
        os.replace(tmp, LIB)
        stamp_file.write_text(stamp)
    # link-compatible shims of the reference's kernel launchers, one per (dimension, flux)
    shim_src = SRC / "shim" / "dgb_shim.cu"
    sensor_obj = next(o for o in objs if o.name.startswith("dgb_sensor."))
    shim_objs = []
    for d, flux in SHIMS:
        out = LIBDIR / f"libdgb_shim_{d}d_{flux}.so"
        key = hashlib.sha1((hdr + shim_src.read_text() + str(sensor_obj)).encode()).hexdigest()[:12]
        obj = BUILD / f"dgb_shim_{d}d_{flux}.{key}.o"
        shim_objs.append(obj)
        if force or not obj.exists():
            _run([NVCC] + NVFLAGS + [f"-DDGB_SHIM_D={d}", f"-DDGB_SHIM_FLUX={SHIM_FLUX[flux]}", f"-I{INC}", f"-I{SRC}",
                                     "-c", str(shim_src), "-o", str(obj)], verbose)
            _run([NVCC] + ARCH + ["-shared", "-o", str(out), str(obj), str(sensor_obj)], verbose)
        elif not out.exists():
            _run([NVCC] + ARCH + ["-shared", "-o", str(out), str(obj), str(sensor_obj)], verbose)
    for stale in BUILD.glob("dgb_shim_*.o"):
        if stale not in shim_objs:
            stale.unlink()
    drv = SRC / "dgbexec.cc"
    if drv.exists() and (force or not EXE.exists() or EXE.stat().st_mtime < max(LIB.stat().st_mtime, drv.stat().st_mtime)):
        _run(["g++", "-std=c++17", "-O2", f"-I{INC}", str(drv), "-o", str(EXE), f"-L{LIBDIR}", "-ldgb",
              "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
