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


def _uniform_base(nz, rho0):
    """Base state of the constant-density problems without gravity
    (Prob/ERF_init_constant_density_hse.H, then erf_enforce_hse with g = 0,
    Initialization/ERF_init1d.cpp:152-260): rho0 everywhere, p0 = 1e5 Pa,
    Exner 1, theta0 = rho*theta(p0) / rho0."""
    return [np.full(nz + 2, rho0), np.full(nz + 2, P0), np.full(nz + 2, 1.0), np.full(nz + 2, _rt_of_p(P0) / rho0)]


def ekman_spiral():
    """Tests/test_files/EkmanSpiral/EkmanSpiral.i with the initial state of
    Exec/RegTests/EkmanSpiral/ERF_prob.cpp (init_type uniform:
    ERF_prob_common.H:450-463 sets rho = rho_0 = 1, rho*theta = rho_0 T_0 =
    300; init_custom_pert adds the analytic Ekman profile).  4 x 4 x 400 cells
    over 50 x 50 x 5000 m, periodic x/y, no-slip ground and slip lid, no
    acoustic substepping, fixed dt 0.5 s, no gravity, constant molecular
    viscosity 5 kg/(m s), Coriolis at latitude 90 with a (15, 0) m/s
    geostrophic wind; the reference default schemes (Upwind_3rd)."""
    c = C.defaults()
    c.nx, c.ny, c.nz = 4, 4, 400
    c.dx = c.dy = 50.0 / 4
    c.dz = 5000.0 / 400
    c.zlo_bc, c.zhi_bc = C.BC_NO_SLIP_WALL, C.BC_SLIP_WALL
    c.substepping_type = C.SUBSTEP_NONE
    c.dt = 0.5
    c.ncomp = 5
    c.molec_diff_type = C.MOLEC_CONSTANT
    c.dynamic_viscosity = 5.0
    c.alpha_T = c.alpha_C = 0.0
    c.gravity = 0.0
    T_rot = 86164.0900027328
    C.set_coriolis(c, T_rot, 90.0, geo_wind=(15.0, 0.0, 0.0))
    rho_0, T_0, u_0 = 1.0, 300.0, 15.0
    nx, ny, nz = c.nx, c.ny, c.nz
    cons = np.zeros((5, nz, ny, nx))
    cons[0] = rho_0
    cons[1] = rho_0 * T_0
    f = 4.0 * math.pi / T_rot
    Az = 5.0 / rho_0
    a = 1.0 / math.sqrt(2.0 * Az / f)
    z = (np.arange(nz) + 0.5) * c.dz
    u = np.zeros((nz, ny, nx + 1))
    v = np.zeros((nz, ny + 1, nx))
    u[:] = (u_0 * (1.0 - np.exp(-a * z) * np.cos(-a * z)))[:, None, None]
    v[:] = (-u_0 * np.exp(-a * z) * np.sin(-a * z))[:, None, None]
    w = np.zeros((nz + 1, ny, nx))
    return "EkmanSpiral", c, _uniform_base(nz, rho_0), (cons, u, v, w), 10


def isentropic_vortex_advecting():
    """Tests/test_files/IsentropicVortexAdvecting/IsentropicVortexAdvecting.i
    with Exec/RegTests/IsentropicVortex/ERF_prob.cpp: a Gaussian isentropic
    vortex (beta 1.1088514254079065, R = sigma = 1) in a Mach 1.195 stream
    at 45 degrees on 48 x 48 x 4 cells over [-12, 12]^2 x [-1, 1], periodic
    x/y, slip walls, no acoustic substepping, fixed dt 5e-4 s, no gravity,
    no diffusion, default schemes.  The background is the constant-density
    base state (rho_0 = p_inf / (R_d T_inf)) of init_from_hse
    (Initialization/ERF_init_from_hse.cpp:32-55) plus the problem's
    perturbation."""
    c = C.defaults()
    c.nx, c.ny, c.nz = 48, 48, 4
    c.dx = c.dy = 24.0 / 48
    c.dz = 2.0 / 4
    c.zlo_bc = c.zhi_bc = C.BC_SLIP_WALL
    c.substepping_type = C.SUBSTEP_NONE
    c.dt = 0.0005
    c.ncomp = 5
    c.molec_diff_type = C.MOLEC_NONE
    c.dynamic_viscosity = 0.0
    c.alpha_T = c.alpha_C = 0.0
    c.gravity = 0.0
    p_inf, T_inf, M_inf = 1.0e5, 300.0, 1.1952286093343936
    alpha, beta, R, sigma, gam = 0.7853981633974483, 1.1088514254079065, 1.0, 1.0, GAMMA
    xc = -12.0 + 0.5 * 24.0
    yc = -12.0 + 0.5 * 24.0
    rho_0 = p_inf / (R_D * T_inf)
    a_inf = math.sqrt(gam * R_D * T_inf)
    inv_gm1 = 1.0 / (gam - 1.0)
    rdOcp = R_D / C.CP_D
    nx, ny, nz = c.nx, c.ny, c.nz

    def omg(x, y):
        r2 = ((x - xc) * (x - xc) + (y - yc) * (y - yc)) / (R * R)
        return beta * np.exp(-r2 / (2.0 * sigma * sigma))

    xcc = -12.0 + (np.arange(nx) + 0.5) * c.dx
    ycc = -12.0 + (np.arange(ny) + 0.5) * c.dy
    xf = -12.0 + np.arange(nx + 1) * c.dx
    yf = -12.0 + np.arange(ny + 1) * c.dy
    Y, X = np.meshgrid(ycc, xcc, indexing="ij")
    O = omg(X, Y)
    dT = -(gam - 1.0) / (2.0 * sigma * sigma) * O * O
    rho_norm = (1.0 + dT) ** inv_gm1
    T = (1.0 + dT) * T_inf
    p = rho_norm ** GAMMA / GAMMA * rho_0 * a_inf * a_inf
    rho_theta = rho_0 * rho_norm * (T * (P0 / p) ** rdOcp)
    r_hse, rt_hse = rho_0, _rt_of_p(P0)
    cons = np.zeros((5, nz, ny, nx))
    cons[0] = r_hse + (rho_norm * rho_0 - r_hse)
    cons[1] = rt_hse + (rho_theta - rt_hse)
    r2d = np.sqrt((X - xc) ** 2 + (Y - yc) ** 2)
    cons[4] = 0.25 * (1.0 + np.cos(math.pi * np.minimum(r2d, R) / R))
    Yu, Xu = np.meshgrid(ycc, xf, indexing="ij")
    u2 = (M_inf * math.cos(alpha) - (Yu - yc) / R * omg(Xu, Yu)) * a_inf
    Yv, Xv = np.meshgrid(yf, xcc, indexing="ij")
    v2 = (M_inf * math.sin(alpha) + (Xv - xc) / R * omg(Xv, Yv)) * a_inf
    u = np.repeat(u2[None], nz, axis=0)
    v = np.repeat(v2[None], nz, axis=0)
    w = np.zeros((nz + 1, ny, nx))
    return "IsentropicVortexAdvecting", c, _uniform_base(nz, rho_0), (cons, u, v, w), 10


def plot_fields(state):
    """ERF's plotfile variables by name (IO/ERF_Plotfile.cpp): cell-centred
    velocities, and temp / pressure from the dry equation of state
    (Utils/ERF_EOS.H:42-79)."""
    cons, u, v, w = state
    rho = cons[0]
    pres = P0 * (R_D * cons[1] / P0) ** GAMMA
    return {"density": rho, "x_velocity": 0.5 * (u[:, :, :-1] + u[:, :, 1:]),
            "y_velocity": 0.5 * (v[:, :-1, :] + v[:, 1:, :]), "z_velocity": 0.5 * (w[:-1] + w[1:]),
            "temp": pres / (R_D * rho), "theta": cons[1] / rho, "scalar": cons[4] / rho, "pressure": pres}


def gold_errors(gold, state, rtol=2.0e-10, atol=2.0e-10):
    """Per plot variable (those this path derives; vorticity is skipped):
    (relative L2, max abs error, passed).  A variable passes as in the
    reference's fcompare check (Tests/CMakeLists.txt:3-4, rtol = atol =
    2e-10): relative L2 <= rtol, or max abs error <= atol for variables whose
    values are round-off (z_velocity of the 1-D Ekman column)."""
    f = plot_fields(state)
    out = {}
    for nm, b in zip(gold["names"], gold["data"]):
        nm = str(nm)
        if nm not in f:
            continue
        a = f[nm]
        den = np.linalg.norm(b)
        rel = np.linalg.norm(a - b) / den if den > 0 else np.inf
        ab = float(np.max(np.abs(a - b)))
        out[nm] = (float(rel), ab, bool(rel <= rtol or ab <= atol))
    return out


def abl_most():
    """Tests/test_files/ABL_MOST/ABL_MOST.i with Exec/ABL/ERF_prob.cpp:
    64^3 cells over a 1024 m cube, periodic x/y, a MOST ground (z0 = 0.1 m,
    z_ref = 8 m, Moeng stress, adiabatic) under a slip lid, no gravity,
    Deardorff (Ck = 0.1, Ce = 0.1, sigma_k = 1), uniform rho = 1,
    rho*theta = 300, u = 10 m/s, rho*KE = 0.1, fixed dt 0.1 s.  The substep
    ratio is ERF's acoustic CFL estimate for this state (estTimeStep,
    TimeIntegration/ERF_ComputeTimestep.cpp:55-225): ceil(0.1 / (0.8 /
    ((10 + c) / 16))) = 3, made even: 4."""
    n = 64
    c = C.defaults()
    c.nx = c.ny = c.nz = n
    c.dx = c.dy = c.dz = 1024.0 / n
    c.zlo_bc, c.zhi_bc = C.BC_MOST, C.BC_SLIP_WALL
    c.most_z0, c.most_zref = 0.1, 8.0
    c.dt, c.mri_ratio = 0.1, 4
    c.ncomp = 5
    c.molec_diff_type = C.MOLEC_NONE
    c.alpha_T, c.alpha_C = 0.0, 1.0
    c.les_type = C.LES_DEARDORFF
    c.Ck, c.Ce, c.sigma_k, c.Ce_wall, c.theta_ref = 0.1, 0.1, 1.0, 0.0, 300.0
    c.gravity = 0.0
    cons = np.zeros((5, n, n, n))
    cons[0] = 1.0
    cons[1] = 300.0
    cons[2] = 0.1
    cons[3] = 0.2
    u = np.full((n, n, n + 1), 10.0)
    v = np.zeros((n, n + 1, n))
    w = np.zeros((n + 1, n, n))
    return "ABL_MOST", c, _uniform_base(n, 1.0), (cons, u, v, w), 10
