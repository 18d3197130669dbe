"""Build recipe of the oracle's C restatement: oracle/_lib/liboracle.so (gcc, CPU only).

Test infrastructure: compiled with -ffp-contract=off so the only contractions are the explicit
fma calls of neighbors.c. Run as ``python -m oracle.build``.
"""

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "_lib" / "liboracle.so"
SOURCES = [HERE / "neighbors.c"]


def build() -> Path:
    LIB.parent.mkdir(parents=True, exist_ok=True)
    if LIB.exists() and all(s.stat().st_mtime <= LIB.stat().st_mtime for s in SOURCES):
        return LIB
    command = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off",
               "-fno-fast-math", *map(str, SOURCES), "-o", str(LIB), "-lm"]
    print(" ".join(command), flush=True)
    subprocess.run(command, check=True)
    return LIB


if __name__ == "__main__":
    build()
