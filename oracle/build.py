"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/oracle.c into oracle/liboracle.so with OpenMP. The image's
`gcc` wrapper cannot find libgomp's spec file, so the versioned driver is
tried first; if no compiler accepts -fopenmp the oracle is built serial.
"""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle.c")
OUT = os.path.join(HERE, "liboracle.so")
FLAGS = ["-O3", "-march=x86-64-v3", "-fPIC", "-std=c11", "-Wall", "-shared"]


def build(force: bool = False) -> str:
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    compilers = [c for c in ("x86_64-linux-gnu-gcc-13", "gcc-13", "gcc", "cc") if shutil.which(c)]
    errs = []
    for omp in (True, False):
        for cc in compilers:
            cmd = [cc] + FLAGS + (["-fopenmp"] if omp else []) + ["-o", OUT, SRC]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode == 0:
                return OUT
            errs.append(" ".join(cmd) + "\n" + r.stderr[-400:])
    raise RuntimeError("oracle build failed:\n" + "\n".join(errs))


if __name__ == "__main__":
    print(build(force=True))
