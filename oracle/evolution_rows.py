"""Amplitude rows of the headline BK workload evolved by the oracle -- test infrastructure.

The reference arm of ``bench.py`` times complete right-hand-side stages of the CPU
restatement at rapidities spread over Y = 0..10.  The cost of a stage depends on the
amplitude there (how many parents are still active, which branches the integrands
take), so each timed stage starts from the amplitude the evolution has reached at that
rapidity.  Those rows come from this script: the oracle's own FP64 evolution
(``oracle.evolve``; RK4, h = 0.1, MV Qs0^2 = 0.2 on 400 r in [1e-7, 1e2]), with K2+Kf on
2^12 Sobol points per stage, which keeps the generation to minutes on a few host cores
and moves the rows by well under a percent against the 2^20-point evolution -- enough to
place every timed stage at the right state.  Nothing here runs on a GPU.

    python -m oracle.evolution_rows      # writes oracle/evolution_rows_400r.npz
"""

from __future__ import annotations

import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUTPUT = HERE / "evolution_rows_400r.npz"
MINR, MAXR, RPOINTS, QS0SQR = 1e-7, 1e2, 399, 0.2
STEP, MAXY, SAMPLES_LOG2 = 0.1, 10.0, 12
EVERY = 5  # keep every 5th row: Y = 0, 0.5, ..., 10


def main() -> None:
    import oracle

    class Config:  # BKConfig's production fields, as oracle.physics reads them
        NC, NF, LambdaQCD, C2, MINR, KSUB = 3.0, 3, 0.241, 1.0, MINR, 0.65
        SYMMETRIZE_Z_Z2_INTEGRATION, FIXED_AS = True, 0.2

    r = oracle.r_grid(MINR, MAXR, RPOINTS)
    N0 = oracle.mv_amplitude(r, QS0SQR)
    state, shift = oracle.sobol_state(4, 0)
    points = oracle.sobol(state, shift, 0, 1 << SAMPLES_LOG2, as_f32=False)
    t0 = time.perf_counter()
    ys, rows = oracle.evolve(N0, r, oracle.physics(Config), points, False, STEP, MAXY, stepper="rk4")
    elapsed = time.perf_counter() - t0
    keep = np.arange(0, ys.size, EVERY)
    np.savez_compressed(OUTPUT, r=r, y=ys[keep], N=rows[keep], samples_log2=np.array([SAMPLES_LOG2]),
                        step=np.array([STEP]))
    print(f"wrote {OUTPUT} ({keep.size} rows, {elapsed:.0f} s)")


if __name__ == "__main__":
    main()
