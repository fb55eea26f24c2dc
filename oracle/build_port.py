"""Compile oracle/edlgt_port.c (gcc -O3 -fopenmp) into oracle/_port/.

Test and CPU-baseline infrastructure only (see the header of edlgt_port.c).
"""

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "edlgt_port.c"
OUT = HERE / "_port" / "libedlgt_port.so"


def build_port(force: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    tmp = OUT.with_suffix(".tmp")
    # the system compiler driver ships the OpenMP runtime spec
    cc = shutil.which("x86_64-linux-gnu-gcc-13") or os.environ.get("CC") or "gcc"
    subprocess.run([cc, "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared",
                    str(SRC), "-o", str(tmp)], check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build_port(force=True))
