"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/nlo_oracle.c`` with gcc into ``oracle/_build/libnlo_oracle.so``.
FMA contraction is disabled so that float32 point maps round exactly like the
device build's explicitly rounded operations.
"""

from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCE = HERE / "nlo_oracle.c"
OUTPUT = HERE / "_build" / "libnlo_oracle.so"


def build(force: bool = False) -> Path:
    if OUTPUT.exists() and not force and OUTPUT.stat().st_mtime >= SOURCE.stat().st_mtime:
        return OUTPUT
    OUTPUT.parent.mkdir(parents=True, exist_ok=True)
    command = [
        "gcc",
        "-O2",
        "-fopenmp",
        "-ffp-contract=off",
        "-fno-fast-math",
        "-fPIC",
        "-shared",
        "-Wall",
        "-o",
        str(OUTPUT),
        str(SOURCE),
        "-lquadmath",
        "-lm",
    ]
    subprocess.run(command, check=True)
    return OUTPUT


if __name__ == "__main__":
    print(build(force=True))
