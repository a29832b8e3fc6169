"""Generate the golden fixtures in this folder from the reference implementation.

Run in a container that has the reference checkout (read-only) at
``/root/reference``:

    PYTHONPATH=/root/reference/torch_nlo_clean/src python tests/golden/make_golden.py

It imports the reference package ``nlo_torch`` and records, in float64 on the
CPU, the values its own functions return for seeded inputs:

* ``bk_reference.npz``  -- r grid and MV initial condition (bk/evolution.py:584-592,
  bk/initial_conditions.py:29-35), the N and S log-log spline coefficients
  (bk/evolution.py:548-560 with numerics/interpolation.py), the K1 integrand
  ``_lo_integrand`` and the K2+Kf integrand ``_nlo_integrand`` x Jacobian
  (bk/derivatives.py:322-335, 434-612) at seeded points, the pointwise kernels
  ``Kernel_lo``/``Kernel_nlo``/``Kernel_nlo_fermion``, the smooth coupling
  (coupling.py:81-97), the Bessel functions the reference calls
  (numerics/special.py:10-23), the fixed K1 rule summed with the reference
  integrand (custom_kernels/bk/k1/kernel.cu:2040-2092 nodes), one adaptive K1
  derivative (bk/derivatives.py:43-110) and Sobol points of
  ``SobolEngine(4, scramble=True, seed=0)`` (dis/fixed_sobol.py:87-92).
* ``bk_table_mc50w.npz`` -- rows of the C++-evolved NLO BK table shipped with
  the reference (``xb_001_mc50w.dat``), read with the reference's own
  ``load_bk_table`` (dipole/table.py:48-118), and the first rows of its
  two-column initial condition ``xb_001.dat``.
"""

from __future__ import annotations

import math
from dataclasses import replace
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
REFERENCE_ROOT = Path("/root/reference")


def main() -> None:
    from nlo_torch.bk.config import BKConfig
    from nlo_torch.bk.derivatives import (
        _lo_integrand,
        _nlo_integrand,
        rapidity_derivative_lo,
    )
    from nlo_torch.bk.evolution import _evolution_interpolators, _r_grid
    from nlo_torch.bk.initial_conditions import MV
    from nlo_torch.bk_kernels.k1 import Kernel_lo
    from nlo_torch.bk_kernels.k2 import Kernel_nlo
    from nlo_torch.bk_kernels.kf import Kernel_nlo_fermion
    from nlo_torch.coupling import bk_alpha_s
    from nlo_torch.dipole.table import load_bk_table
    from nlo_torch.numerics import special

    torch.set_default_dtype(torch.float64)
    out: dict[str, np.ndarray] = {}

    config = replace(BKConfig(RPOINTS=99, MINR=1e-6, MAXR=1e2), CUDA_FUSION=False)
    r = _r_grid(config, device="cpu", dtype=torch.float64)
    N = MV(qs0sqr=0.2).dipole_amplitude(r)
    out["r"] = r.numpy()
    out["N_mv"] = N.numpy()
    interpolator_N, interpolator_S = _evolution_interpolators(N, r, config)
    for name, spline in (("nspline", interpolator_N._spline), ("sspline", interpolator_S._spline)):
        for field in "xabcd":
            out[f"{name}_{field}"] = getattr(spline, field).numpy()

    generator = torch.Generator().manual_seed(20261203)
    lower = math.log(0.5 * float(r[0]))
    upper = math.log(2 * float(r[-1]))
    u = torch.rand((512, 4), generator=generator, dtype=torch.float64)
    x = torch.stack(
        (
            lower + (upper - lower) * u[:, 0],
            lower + (upper - lower) * u[:, 1],
            2 * math.pi * u[:, 2],
            2 * math.pi * u[:, 3],
        ),
        dim=1,
    )
    out["k2kf_x"] = x.numpy()
    parent_index = np.array([30, 45, 60, 75, 90])
    out["k2kf_parent_index"] = parent_index
    values = []
    for index in parent_index:
        parent = r[int(index)]
        value = _nlo_integrand(
            parent, torch.exp(x[:, 0]), x[:, 2], torch.exp(x[:, 1]), x[:, 3], interpolator_S, r, config
        ) * torch.exp(2 * x[:, 0] + 2 * x[:, 1])
        values.append(value.numpy())
    out["k2kf_value"] = np.stack(values)

    z = torch.exp(math.log(float(r[0])) + (math.log(float(r[-1])) - math.log(float(r[0]))) * u[:, 0])
    theta = math.pi * u[:, 1]
    out["k1_z"] = z.numpy()
    out["k1_theta"] = theta.numpy()
    out["k1_parent_index"] = parent_index
    out["k1_value"] = np.stack(
        [_lo_integrand(r[int(i)], z, theta, interpolator_N, r, config, None, None, None).numpy()
         for i in parent_index]
    )
    out["kernel_lo"] = np.stack([Kernel_lo(r[int(i)], z, theta, config).numpy() for i in parent_index])

    distances = torch.exp(torch.empty((256, 5)).uniform_(math.log(1e-3), math.log(30.0), generator=generator))
    parent = torch.exp(torch.empty(256).uniform_(math.log(1e-2), math.log(10.0), generator=generator))
    out["kernel_nlo_args"] = torch.cat((parent.unsqueeze(1), distances), dim=1).numpy()
    out["kernel_nlo"] = Kernel_nlo(parent, *distances.unbind(1)).numpy()
    out["kernel_nlo_fermion"] = Kernel_nlo_fermion(parent, *distances.unbind(1), config).numpy()

    alpha_r = torch.logspace(-8, 2, 64)
    out["alpha_r"] = alpha_r.numpy()
    out["alpha_s"] = bk_alpha_s(alpha_r, NC=3.0, NF=3, LambdaQCD=0.241, C2=1.0).numpy()
    bessel_x = torch.linspace(0.0, 60.0, 121)
    out["bessel_x"] = bessel_x.numpy()
    out["bessel_j1"] = special.bessel_J1(bessel_x).numpy()
    out["bessel_i1"] = special.bessel_I1(bessel_x).numpy()

    # Fixed K1 rule (8 x 24 nodes per grid interval) summed with the reference integrand.
    x8, w8 = np.polynomial.legendre.leggauss(8)
    x24, w24 = np.polynomial.legendre.leggauss(24)
    log_grid = torch.log(r)
    center = 0.5 * (log_grid[1:] + log_grid[:-1])
    half = 0.5 * (log_grid[1:] - log_grid[:-1])
    log_z = (center.unsqueeze(1) + half.unsqueeze(1) * torch.tensor(x8)).reshape(-1)
    radial_weight = (half.unsqueeze(1) * torch.tensor(w8)).reshape(-1)
    v = 0.5 * (torch.tensor(x24) + 1.0)
    theta_nodes = math.pi * v * v
    angular_weight = torch.tensor(w24) * math.pi * v
    zz = torch.exp(log_z).unsqueeze(1).expand(-1, 24).reshape(-1)
    tt = theta_nodes.unsqueeze(0).expand(log_z.numel(), -1).reshape(-1)
    ww = (radial_weight.unsqueeze(1) * angular_weight.unsqueeze(0)).reshape(-1)
    fixed_index = np.array([20, 40, 60, 80])
    out["k1_fixed_parent_index"] = fixed_index
    out["k1_fixed"] = np.array(
        [
            float(torch.sum(_lo_integrand(r[int(i)], zz, tt, interpolator_N, r, config, None, None, None)
                            * 2 * zz * zz * ww))
            for i in fixed_index
        ]
    )
    adaptive = rapidity_derivative_lo(r[60], interpolator_N, r, config)
    out["k1_adaptive_r60"] = np.array([float(adaptive.value), float(adaptive.error)])

    # SobolEngine computes its first point in the default dtype current at
    # construction; record the draws under torch's normal float32 default.
    torch.set_default_dtype(torch.float32)
    engine = torch.quasirandom.SobolEngine(4, scramble=True, seed=0)
    out["sobol_state"] = engine.sobolstate.numpy().copy()
    out["sobol_shift"] = engine.shift.numpy().copy()
    out["sobol_f32"] = engine.draw(1024, dtype=torch.float32).numpy()
    engine = torch.quasirandom.SobolEngine(4, scramble=True, seed=0)
    out["sobol_f64"] = engine.draw(1024, dtype=torch.float64).numpy()

    np.savez_compressed(HERE / "bk_reference.npz", **out)

    table = load_bk_table(REFERENCE_ROOT / "xb_001_mc50w.dat", dtype=torch.float64)
    rows = [0, 5, 10, 15, 20, 25]
    ic = np.loadtxt(REFERENCE_ROOT / "xb_001.dat", max_rows=20)
    np.savez_compressed(
        HERE / "bk_table_mc50w.npz",
        r=table.r.numpy(),
        y=table.y.numpy()[rows],
        N=table.N.numpy()[rows],
        x0=np.array([table.x0]),
        ic_head=ic,
    )
    print("wrote", HERE / "bk_reference.npz", "and", HERE / "bk_table_mc50w.npz")


if __name__ == "__main__":
    main()
