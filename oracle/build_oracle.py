"""Build recipe of the CPU oracle (test infrastructure): g++ -> oracle/_build/libvbd_oracle.so.

``-ffp-contract=off`` keeps the FP32 oracle independent of the host compiler's choice to fuse
multiply-adds; OpenMP parallelises the vertices of one color (they are independent within a
color, so the result does not depend on the thread count).
"""

from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "vbd_oracle.cpp"
OUT = HERE / "_build" / "libvbd_oracle.so"


def build(force: bool = False) -> Path:
    stamp = OUT.with_suffix(".sha256")
    fp = hashlib.sha256(SRC.read_bytes()).hexdigest()
    if not force and OUT.exists() and stamp.exists() and stamp.read_text().strip() == fp:
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    compilers = [c for c in (shutil.which("g++"), os.environ.get("CXX"), "/usr/bin/g++") if c]
    tmp = OUT.with_suffix(".so.tmp")
    errors = []
    for cxx in compilers:
        # OpenMP first; a toolchain without libgomp still builds a (serial) oracle
        for omp in (["-fopenmp"], []):
            cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", *omp, "-ffp-contract=off", str(SRC), "-o", str(tmp)]
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode == 0:
                break
            errors.append(f"{' '.join(cmd)}\n{res.stderr}")
        if res.returncode == 0:
            break
    if res.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + "\n".join(errors))
    os.replace(tmp, OUT)
    stamp.write_text(fp)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
