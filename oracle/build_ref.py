"""Build recipe for the reference CPU oracle binaries (test infrastructure only).

Compiles the reference's own sources, where they lie under the read-only checkout
(code/src/**/*.cc and *.cu, the latter as C++ exactly as the reference Makefile does for
ARCH=USE_CPU, code/Makefile:187-189), once per compile-time configuration, and links each
set with oracle/ref_harness.cc into ``oracle/_ref/dgref_<variant>``.  Outputs go only to
``oracle/_ref/`` (git-ignored; it travels with the working tree to GPU hosts).

Compile-time configuration follows code/Makefile:147-156 (DEFINES) for the gamma-model
multifluid build: USE_CPU, USE_DOUBLE, MULTIFLUID, GAMNCON, NO_MPI, N_Y=0, and
N_F=4 (1D) / 5 (2D), D=1/2, DF=1, with the flux flag ROE, RUS or HLL; and the same with one
passive mass fraction (N_Y=1, N_F=5 / 6; variants *_y1) and with two or three (*_y2, *_y3); GAMCONS in place of GAMNCON (variants
*_gc); ERROR in place of NOERROR (variant 1d_rus_err); CONS in place of NOCONS (variant
1d_roe_cons).

Out-of-tree additions (none of them touch reference arithmetic):
  * an empty ``gsl/gsl_integration.h`` (code/src/ic/init_cond.cc:10 includes it, never calls it);
  * LP64 OpenBLAS/LAPACK from the image (plain F77 symbol names);
  * ``--wrap`` of blasIdamax, which lacks a return statement (code/src/utils/misc.cc:38-41);
  * ``--wrap`` of RK::RK_integration so the harness can drive single operators;
  * main() renamed to dgref_main.

Usage: python oracle/build_ref.py [--ref <reference checkout>/code/src] [--jobs 8] [variant ...]
(defaults: $DGB_REFERENCE_SRC or /root/reference/code/src; OpenBLAS from $DGB_REF_BLAS or found in
site-packages)
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# the read-only reference checkout; DGB_REFERENCE_SRC overrides it
DEFAULT_REF = Path(os.environ.get("DGB_REFERENCE_SRC", "/root/reference/code/src"))


def find_blas() -> Path:
    """An LP64 OpenBLAS with plain F77 names (dgemm_, dgetrf_, ...): $DGB_REF_BLAS if set, else
    the copy bundled with an installed opencv-python-headless wheel (site-packages/
    opencv_python_headless.libs/libopenblas*.so; its libgfortran sits beside it)."""
    env = os.environ.get("DGB_REF_BLAS")
    if env:
        return Path(env)
    import site
    import sysconfig
    roots = [Path(p) for p in site.getsitepackages() + [sysconfig.get_paths()["purelib"]]]
    for r in roots:
        for cand in sorted((r / "opencv_python_headless.libs").glob("libopenblas*.so*")):
            return cand
    raise FileNotFoundError("no LP64 OpenBLAS found: set DGB_REF_BLAS to a libopenblas*.so with F77 names")

VARIANTS = {
    "1d_roe": dict(dims="ONED", nf=4, d=1, flux="ROE"),
    "1d_rus": dict(dims="ONED", nf=4, d=1, flux="RUS"),
    "1d_hll": dict(dims="ONED", nf=4, d=1, flux="HLL"),
    "2d_roe": dict(dims="TWOD", nf=5, d=2, flux="ROE"),
    "2d_rus": dict(dims="TWOD", nf=5, d=2, flux="RUS"),
    # one passive mass fraction (MASS=1 in code/Makefile: N_Y=1, one more field)
    "1d_roe_y1": dict(dims="ONED", nf=5, d=1, flux="ROE", ny=1),
    "1d_rus_y1": dict(dims="ONED", nf=5, d=1, flux="RUS", ny=1),
    "1d_hll_y1": dict(dims="ONED", nf=5, d=1, flux="HLL", ny=1),
    "2d_roe_y1": dict(dims="TWOD", nf=6, d=2, flux="ROE", ny=1),
    "2d_rus_y1": dict(dims="TWOD", nf=6, d=2, flux="RUS", ny=1),
    # two and three mass fractions (MASS=2, MASS=3)
    "1d_roe_y2": dict(dims="ONED", nf=6, d=1, flux="ROE", ny=2),
    "1d_hll_y3": dict(dims="ONED", nf=7, d=1, flux="HLL", ny=3),
    "2d_rus_y2": dict(dims="TWOD", nf=7, d=2, flux="RUS", ny=2),
    "2d_roe_y3": dict(dims="TWOD", nf=8, d=2, flux="ROE", ny=3),
    # five and ten (MASS=5, MASS=10; the reference's maximum)
    "1d_rus_y5": dict(dims="ONED", nf=9, d=1, flux="RUS", ny=5),
    "1d_roe_y10": dict(dims="ONED", nf=14, d=1, flux="ROE", ny=10),
    "2d_roe_y5": dict(dims="TWOD", nf=10, d=2, flux="ROE", ny=5),
    "2d_rus_y10": dict(dims="TWOD", nf=15, d=2, flux="RUS", ny=10),
    # the ERROR diagnostic compiled in (ERRR=ERROR in code/Makefile): error.dat after the run
    "1d_rus_err": dict(dims="ONED", nf=4, d=1, flux="RUS", err=True),
    # the conservative gamma model (GAMM=GAMCONS in code/Makefile): rho/(gamma-1) as the field
    "1d_roe_gc": dict(dims="ONED", nf=4, d=1, flux="ROE", gc=True),
    "1d_rus_gc": dict(dims="ONED", nf=4, d=1, flux="RUS", gc=True),
    "1d_hll_gc": dict(dims="ONED", nf=4, d=1, flux="HLL", gc=True),
    "2d_roe_gc": dict(dims="TWOD", nf=5, d=2, flux="ROE", gc=True),
    "2d_rus_gc": dict(dims="TWOD", nf=5, d=2, flux="RUS", gc=True),
    # the conservation diagnostic compiled in (CONS=CONS in code/Makefile): conservation.dat
    "1d_roe_cons": dict(dims="ONED", nf=4, d=1, flux="ROE", cons=True),
}

RK_SYM = ("_ZN2RK14RK_integrationEdiiiiiiiPdS0_R8LimitingbR9DG_SOLVERR12COMMUNICATORR7PRINTER"
          "R6SENSORR6TIMERSR11MEM_COUNTERR18LAGRANGE_PARTICLES")


def defines(v: dict) -> list[str]:
    return ["-DHAVE_BLAS", "-DHAVE_LAPACK", "-DUSE_CPU", "-DHOME", "-DUSE_DOUBLE", "-DMULTIFLUID",
            "-DGAMCONS" if v.get("gc") else "-DGAMNCON", f"-D{v['flux']}", f"-D{v['dims']}", "-DNO_MPI", f"-DN_Y={v.get('ny', 0)}", f"-DN_F={v['nf']}",
            "-DERROR" if v.get("err") else "-DNOERROR", "-DCONS" if v.get("cons") else "-DNOCONS", f"-DD={v['d']}", "-DDF=1"]


def sources(ref: Path) -> list[Path]:
    return sorted([p for p in ref.rglob("*") if p.suffix in (".cc", ".cu")])


def includes(ref: Path) -> list[str]:
    dirs = sorted({p.parent for p in ref.rglob("*.h")} | {ref})
    return [f"-I{HERE / 'stub'}"] + [f"-I{d}" for d in dirs]


def compile_one(src: Path, obj: Path, flags: list[str]) -> tuple[Path, int, str]:
    obj.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["g++", "-std=gnu++98", "-O3", "-w", "-x", "c++"] + flags + ["-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return obj, r.returncode, r.stderr[-2000:]


def build_variant(name: str, ref: Path, pool: cf.Executor) -> Path:
    v = VARIANTS[name]
    flags = defines(v) + includes(ref)
    key = hashlib.sha1((" ".join(flags) + str(ref)).encode()).hexdigest()[:8]
    objdir = OUT / f"obj_{name}_{key}"
    jobs = []
    for src in sources(ref):
        rel = src.relative_to(ref)
        obj = objdir / (str(rel).replace("/", "__") + ".o")
        extra = ["-Dmain=dgref_main"] if rel.name == "main.cc" else []
        if obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime:
            continue
        jobs.append(pool.submit(compile_one, src, obj, flags + extra))
    for j in jobs:
        obj, rc, err = j.result()
        if rc != 0:
            raise RuntimeError(f"compile failed for {obj.name}:\n{err}")
    harness_obj = objdir / "ref_harness.o"
    hsrc = HERE / "ref_harness.cc"
    if not harness_obj.exists() or harness_obj.stat().st_mtime < hsrc.stat().st_mtime:
        cmd = ["g++", "-std=gnu++11", "-O3", "-w"] + flags + ["-c", str(hsrc), "-o", str(harness_obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"harness compile failed:\n{r.stderr[-3000:]}")
    exe = OUT / f"dgref_{name}"
    objs = sorted(str(p) for p in objdir.glob("*.o"))
    blas = find_blas()
    link = (["g++", "-o", str(exe)] + objs +
            [f"-Wl,--wrap=_Z10blasIdamaxiPdi", f"-Wl,--wrap={RK_SYM}",
             f"-L{blas.parent}", f"-l:{blas.name}", "-Wl,--disable-new-dtags", f"-Wl,-rpath,{blas.parent}", "-lm"])
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed for {name}:\n{r.stderr[-3000:]}")
    return exe


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", type=Path, default=DEFAULT_REF)
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("variants", nargs="*", default=list(VARIANTS))
    a = ap.parse_args(argv)
    if not a.ref.is_dir():
        print(f"reference sources not found at {a.ref}; nothing built", file=sys.stderr)
        return 1
    OUT.mkdir(parents=True, exist_ok=True)
    with cf.ThreadPoolExecutor(a.jobs) as pool:
        for name in a.variants:
            exe = build_variant(name, a.ref, pool)
            print(f"built {exe}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
