"""Leading-order photon wave functions and dipole integrand (interface of the reference's
dis/lo.py:12-51), evaluated by the device LO kernel."""

from __future__ import annotations

import math

import torch

from nlo_bk_optimized_b200.dipole.amplitude import GBW, BKDipole
from nlo_bk_optimized_b200.dis.config import DISConfig, Polarization, Quark


def integrand_photon_target_LO(r: torch.Tensor, z: torch.Tensor, xbj: torch.Tensor, Q2: torch.Tensor,
                               polarization: Polarization, quarks: tuple[Quark, ...],
                               dipole: GBW | BKDipole) -> torch.Tensor:
    """sum_q e_q^2 |Psi|^2 N(r, Y) without the radial Jacobian, for scalar Q^2 and x_Bj."""
    from nlo_bk_optimized_b200.dis.observables import TERMS, _integrand, kinematics

    r, z = torch.broadcast_tensors(r, z)
    config = DISConfig(quarks=tuple(quarks), maxr=1.0)
    kin = kinematics(float(Q2), float(xbj), polarization, config)
    x = torch.stack((z.reshape(-1), r.reshape(-1)), dim=1)
    with_jacobian = _integrand(TERMS["LO"], x, kin, dipole, config)
    flat_r = r.reshape(-1)
    safe = torch.where(flat_r > 0, flat_r, torch.ones_like(flat_r))
    value = torch.where(flat_r > 0, with_jacobian / (2 * math.pi * safe), torch.zeros_like(flat_r))
    return value.reshape(r.shape)


__all__ = ["integrand_photon_target_LO"]
