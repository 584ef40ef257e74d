"""Recipe: compile the reference's own CUDA step into oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  The reference (gyf135/EHD-convection-3D) fixes its
grid, geometry and physics as compile-time constants in LBM.h:30-86 and runs
a fixed NSTEPS.  For each named case this script copies the reference sources
from /root/reference into a scratch directory under /tmp (the sources never
enter this repository), rewrites those constants, and compiles

    nvcc -gencode arch=compute_100a,code=sm_100a -O3 --use_fast_math \
         seconds.cpp main.cu -lcufft

(the reference's own build line, README.md:22, retargeted to sm_100a) into
oracle/_ref/<case>/ehd_ref.  Nothing else of the reference's code is changed
except, in every case:

* NSTEPS is read from the environment variable EHD_REF_NSTEPS (LBM.h:82);
* NSAVE = NDMD = printCurrent = 1, so ``i % N == 1`` never fires and the
  time loop runs without in-loop output (main.cu:210-237); a case may keep
  the collector-current print (``Current = %g`` every printCurrent steps,
  main.cu:227-231) at a cadence of its own;
* flag (LBM.h:30) selects the restart path (read data_end.dat) or the
  reference initialisation;
* save_data_end writes %.17g instead of %10.6f (LBM.cu:1551) so the output
  carries full FP64 precision;

and, for the timing-only case "bench", the whole-field text writers outside
the timed loop (main.cu:168,268,273,277) are skipped.

The reference sources are read from $EHD_REFERENCE_SRC, by default
/root/reference.  The GPU machine has no reference sources; the binaries built
here travel with the repository snapshot.
Run:  python oracle/build_ref.py [case ...]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_SRC = Path(os.environ.get("EHD_REFERENCE_SRC", "/root/reference"))
OUT = HERE / "_ref"

# name -> constants.  Geometry: dx = dy = dz = 1/(nz-1), Lx = nx dx, Ly = ny dy.
# "groups" physics is T=200, M=10, C=10, Fe=4000 with magic parameters 1/4.
_GROUPS = dict(nu=0.125, K=2.5e-5, charge0=10.0, diffu=6.25e-5, V=0.25, VC=0.25)
_DEFAULT = dict(nu=0.0251004, K=2.5e-5, charge0=10.0, diffu=6.25e-5, V=1.0 / 12.0,
                VC=1.0e-6)

CASES = {
    # tiny grids, seeded random fields, reference physics defaults
    "tiny_default": dict(nx=16, ny=16, nz=9, threads=16, flag=1, **_DEFAULT),
    # non-square, magic 1/4, moving upper wall and external force switched on
    "tiny_groups": dict(nx=24, ny=16, nz=13, threads=8, flag=1, uw=0.05, exf=100.0,
                        **_GROUPS),
    # the small production-like case: 64 x 64 x 33, hydrostatic + seeded noise
    "config0": dict(nx=64, ny=64, nz=33, threads=64, flag=1, **_GROUPS),
    # 64 x 64 x 33 at T=400 (M=10, C=10, Fe=4000) with the reference's own
    # magic parameters: the developed-convection run to non-finite fields
    "config0_t400": dict(nx=64, ny=64, nz=33, threads=64, flag=1, nu=0.0625, K=2.5e-5,
                         charge0=10.0, diffu=6.25e-5, V=1.0 / 12.0, VC=1.0e-6),
    # the same two starts run on towards non-finite fields, printing the
    # collector current every 1000 steps (main.cu:227-231), no whole-field output
    "config0_long": dict(nx=64, ny=64, nz=33, threads=64, flag=1, no_output=True,
                         print_current=1000, **_GROUPS),
    "config0_t400_long": dict(nx=64, ny=64, nz=33, threads=64, flag=1, no_output=True,
                              print_current=1000, nu=0.0625, K=2.5e-5, charge0=10.0,
                              diffu=6.25e-5, V=1.0 / 12.0, VC=1.0e-6),
    # timing only: 256 x 256 x 129, reference initialisation, no text output
    "bench": dict(nx=256, ny=256, nz=129, threads=128, flag=0, no_output=True, **_GROUPS),
    # the reference's own default case (LBM.h:31-86: 122 x 122 x 101, dx = 1/100,
    # T ~ 996, M = 10, C = 10, Fe = 4000, magic parameters 1/12 and 1e-6),
    # started from data_end.dat, printing the collector current every 1000
    # steps as it does by default (main.cu:227-231); no whole-field output
    "authors": dict(nx=122, ny=122, nz=101, threads=61, flag=1, no_output=True,
                    print_current=1000, **_DEFAULT),
}


def _fmt(x: float) -> str:
    return repr(float(x))


def _sub(text: str, decl: str, value: str) -> str:
    pat = re.compile(r"(" + decl + r"\s*=\s*)[^;]+;")
    new, n = pat.subn(lambda m: m.group(1) + value + ";", text, count=1)
    if n != 1:
        raise RuntimeError(f"pattern not found: {decl}")
    return new


def patch(src_dir: Path, c: dict) -> None:
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    if nx % c["threads"]:
        raise ValueError("NX must be a multiple of nThreads (LBM.h:31)")
    d = 1.0 / (nz - 1)
    h = (src_dir / "LBM.h").read_text()
    h = _sub(h, r"unsigned int flag", str(int(c["flag"])))
    h = _sub(h, r"const int nThreads", str(c["threads"]))
    h = _sub(h, r"const unsigned int NX", str(nx))
    h = _sub(h, r"const unsigned int NY", str(ny))
    h = _sub(h, r"const unsigned int NZ", str(nz))
    h = _sub(h, r"__constant__ double LL", _fmt(nx * d))
    h = _sub(h, r"__constant__ double Lx", _fmt(nx * d))
    h = _sub(h, r"__constant__ double Ly", _fmt(ny * d))
    h = _sub(h, r"__constant__ double dx", _fmt(d))
    h = _sub(h, r"__constant__ double dy", _fmt(d))
    h = _sub(h, r"__constant__ double dz", _fmt(d))
    h = _sub(h, r"__constant__ double dt", _fmt(0.01 * d))
    h = _sub(h, r"double uw_host", _fmt(c.get("uw", 0.0)))
    h = _sub(h, r"double exf_host", _fmt(c.get("exf", 0.0)))
    h = _sub(h, r"__constant__ double charge0", _fmt(c["charge0"]))
    h = _sub(h, r"__constant__ double diffu", _fmt(c["diffu"]))
    h = _sub(h, r"double nu_host", _fmt(c["nu"]))
    h = _sub(h, r"double K_host", _fmt(c["K"]))
    h = _sub(h, r"__constant__ double V ", _fmt(c["V"]))
    h = _sub(h, r"__constant__ double VC", _fmt(c["VC"]))
    h = _sub(h, r"const unsigned int NSTEPS",
             '(unsigned)atoi(getenv("EHD_REF_NSTEPS") ? getenv("EHD_REF_NSTEPS") : "1")')
    h = _sub(h, r"const unsigned int NSAVE ", "1")
    h = _sub(h, r"const unsigned int NDMD  ", "1")
    h = _sub(h, r"const unsigned int printCurrent", str(int(c.get("print_current", 1))))
    (src_dir / "LBM.h").write_text(h)

    cu = (src_dir / "LBM.cu").read_text()
    ten = " ".join(["%10.6f"] * 10)
    if cu.count(ten) != 1:
        raise RuntimeError("save_data_end format not found")
    cu = cu.replace(ten, " ".join(["%.17g"] * 10))
    (src_dir / "LBM.cu").write_text(cu)

    if c.get("no_output"):
        m = (src_dir / "main.cu").read_text()
        for call in ("save_data_tecplot(fout,", "save_data_end(fend,", "record_umax(fumax,"):
            m = m.replace(call, "if (0) " + call)
        (src_dir / "main.cu").write_text(m)


def build_case(name: str, nvcc: str = "nvcc") -> Path:
    c = CASES[name]
    out_dir = OUT / name
    out_dir.mkdir(parents=True, exist_ok=True)
    exe = out_dir / "ehd_ref"
    with tempfile.TemporaryDirectory(prefix=f"ehd_ref_{name}_") as tmp:
        tmp = Path(tmp)
        for f in ("LBM.h", "LBM.cu", "main.cu", "poisson.cu", "seconds.cpp", "seconds.h"):
            shutil.copy(REF_SRC / f, tmp / f)
        patch(tmp, c)
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--use_fast_math",
               "-w", "seconds.cpp", "main.cu", "-lcufft", "-o", str(exe)]
        r = subprocess.run(cmd, cwd=tmp, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {name}:\n{r.stderr[-4000:]}")
    (out_dir / "case.txt").write_text(repr(c) + "\n")
    return exe


def build(names=None) -> None:
    if not REF_SRC.exists():
        print("build_ref: reference sources absent; keeping prebuilt oracle/_ref")
        return
    names = list(names or CASES)
    with cf.ThreadPoolExecutor(max_workers=min(4, len(names))) as ex:
        for name, exe in zip(names, ex.map(build_case, names)):
            print(f"built {name}: {exe}")


if __name__ == "__main__":
    build(sys.argv[1:] or None)
