"""The FP32 tables of csrc/special_tables.cuh for the double-log resummation factor of K1:
G(v) = J1(2 sqrt(-v))/sqrt(-v) (v < 0), I1(2 sqrt(v))/sqrt(v) (v > 0), G(0) = 1.

The device evaluation (dla_factor in csrc/k1.cu) is replayed here in float32 arithmetic with
the tables read from the header, and compared with scipy's Bessel functions at the same
float32 t = 2 sqrt|v|: at most 2e-6 of the envelope of G (1 inside |v| <= 4, the value for
v > 4, 2 sqrt(2 / (pi t)) / t for v < -4).  The header is the output of
gen_special_tables.py, which regenerates it byte for byte."""

from __future__ import annotations

import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import scipy.special as sp

CSRC = Path(__file__).resolve().parents[1] / "nlo_bk_optimized_b200" / "csrc"
f32 = np.float32


def _table(src: str, name: str) -> np.ndarray:
    body = re.search(name + r"\[\d+\] = \{(.*?)\};", src, re.S).group(1)
    return np.array([float(x.strip().rstrip("f")) for x in body.split(",") if x.strip()], dtype=np.float32)


@pytest.fixture(scope="module")
def tables():
    src = (CSRC / "special_tables.cuh").read_text()
    return {k: _table(src, k) for k in ("kDlaPolyF", "kDlaModF", "kDlaPhaseF", "kDlaExpF")}


def _horner(c, x):
    p = f32(0)
    for cj in c[::-1]:
        p = f32(f32(p * x) + cj)
    return p


def _g32(v, T):
    """dla_factor's float32 operation sequence (fused multiply-adds rounded once)."""
    v = f32(v)
    av = abs(v)
    if av <= f32(4):
        return f32(f32(1) + f32(np.float64(v) * np.float64(_horner(T["kDlaPolyF"], v))))
    t = f32(2) * f32(np.sqrt(av))
    s = f32(f32(4) / t)
    srt = f32(s * f32(1 / np.sqrt(np.float64(t))))
    if v < 0:
        m, d = _horner(T["kDlaModF"], s), _horner(T["kDlaPhaseF"], s)
        k = np.rint(f32(np.float64(t) * np.float64(f32(0.15915494309189535)) - 0.375))
        rr = f32(np.float64(t) - k * np.float64(f32(6.28125)))
        rr = f32(np.float64(rr) - k * np.float64(f32(1.9353071795864769e-3)))
        rr = f32(f32(rr - f32(2.3561944901923449)) + d)
        return f32(f32(f32(f32(0.39894228040143268) * m) * srt) * f32(np.cos(rr)))
    h = _horner(T["kDlaExpF"], s)
    half = f32(np.exp(f32(0.5) * t))
    return f32(f32(f32(f32(f32(0.19947114020071634) * h) * srt) * half) * half)


def test_resummation_factor_tables_match_bessel_functions(tables):
    vs = np.concatenate([np.linspace(-1300.0, -4.0, 4001), np.linspace(-4.0, 4.0, 801), np.linspace(4.0, 300.0, 1001)])
    worst = 0.0
    for v in vs:
        v32 = f32(v)
        if v32 == 0:
            continue
        t = float(f32(2) * f32(np.sqrt(abs(v32))))
        if abs(v32) <= 4:
            ref = float(2 * (sp.jv(1, t) if v32 < 0 else sp.iv(1, t)) / t)
            env = max(1.0, abs(ref))
        elif v32 < 0:
            ref = float(2 * sp.jv(1, t) / t)
            env = 2 * np.sqrt(2 / (np.pi * t)) / t
        else:
            ref = float(2 * sp.ive(1, t) / t)  # scaled by e^-t
            env = abs(ref)
            got = float(_g32(v32, tables)) * np.exp(-t)
            worst = max(worst, abs(got - ref) / env)
            continue
        worst = max(worst, abs(float(_g32(v32, tables)) - ref) / env)
    assert worst <= 2e-6, worst
    assert _g32(f32(0), tables) == f32(1)


def test_generator_reproduces_the_header(tmp_path):
    """gen_special_tables.py writes next to itself: run a copy in a scratch folder."""
    copy = tmp_path / "gen_special_tables.py"
    copy.write_text((CSRC / "gen_special_tables.py").read_text())
    subprocess.run([sys.executable, str(copy)], check=True, cwd=tmp_path, timeout=600)
    assert (tmp_path / "special_tables.cuh").read_text() == (CSRC / "special_tables.cuh").read_text()
