"""Setups of reference regression tests whose gold plotfiles pin the oracle.

TaylorGreenAdvecting / TaylorGreenAdvectingDiffusing: Tests/test_files/
TaylorGreenAdvecting*/ *.i with the initial state of
Exec/RegTests/TaylorGreenVortex/ERF_prob.cpp:26-97 (rho_0 = M_0 = V_0 = 1):
16^3 cells on a (2 pi)^3 box, periodic x/y, slip walls, Upwind_3rd
(the reference default), no gravity, fixed dt 0.16 s.  The inputs' key
`mri_fixed_dt_ratio` is not one ERF reads (ERF.cpp:1429 reads
`fixed_mri_dt_ratio`), so the substep ratio is ERF's CFL estimate
(TimeIntegration/ERF_ComputeTimestep.cpp:54-218): ceil(dt / (0.8 / max((|u|+c)/dx)))
rounded up to even = 2 for this flow.  Without gravity the base state is
uniform (p0 = 1e5 Pa), so it only shifts p' by a constant.
"""
import math

import numpy as np

from erf_b200 import config as C

R_D, P0, GAMMA = 287.0, 1.0e5, 1.4


def _rt_of_p(p):
    return (p * P0 ** (GAMMA - 1)) ** (1 / GAMMA) / R_D


def taylor_green(diffusing: bool):
    n = 16
    c = C.defaults()
    c.nx = c.ny = c.nz = n
    L = 6.283185307179586476925
    c.dx = c.dy = c.dz = L / n
    c.zlo_bc = c.zhi_bc = C.BC_SLIP_WALL
    c.dt, c.mri_ratio = 0.16, 2
    c.ncomp = 5
    c.molec_diff_type = C.MOLEC_CONSTANT if diffusing else C.MOLEC_NONE
    c.dynamic_viscosity = 6.25e-4 if diffusing else 0.0
    c.gravity = 0.0
    x = (np.arange(n) + 0.5) * c.dx
    xf = np.arange(n + 1) * c.dx
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    p = 1.0 * 1.0 * (1.0 / (GAMMA * 1.0 * 1.0) + (1.0 / 16.0) * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2))
    cons = np.zeros((5, n, n, n))
    cons[0] = 1.0
    cons[1] = _rt_of_p(P0) * 1.0 + (_rt_of_p(p) - _rt_of_p(P0))
    cons[4] = 1.0
    Zu, Yu, Xu = np.meshgrid(x, x, xf, indexing="ij")
    u = np.sin(Xu) * np.cos(Yu) * np.cos(Zu)
    Zv, Yv, Xv = np.meshgrid(x, xf, x, indexing="ij")
    v = -np.cos(Xv) * np.sin(Yv) * np.cos(Zv)
    w = np.zeros((n + 1, n, n))
    base = [np.full(n + 2, 1.0), np.full(n + 2, P0), np.full(n + 2, 1.0), np.full(n + 2, _rt_of_p(P0))]
    name = "TaylorGreenAdvectingDiffusing" if diffusing else "TaylorGreenAdvecting"
    return name, c, base, (cons, u, v, w), 10


def plot_variables(state):
    """ERF's plotfile variables (IO/ERF_Plotfile.cpp): density, cell-centred
    velocities, temp, theta, scalar, pressure."""
    cons, u, v, w = state
    rho = cons[0]
    pres = P0 * (R_D * cons[1] / P0) ** GAMMA
    return [rho, 0.5 * (u[:, :, :-1] + u[:, :, 1:]), 0.5 * (v[:, :-1, :] + v[:, 1:, :]), 0.5 * (w[:-1] + w[1:]),
            pres / (R_D * rho), cons[1] / rho, cons[4] / rho, pres]
