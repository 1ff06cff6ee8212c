"""Static terrain-following grids and the terrain ABL workload.

Host-side grid construction (done once, FP64, before any step):
  zlevels    -- init_zlevels (Utils/ERF_TerrainMetrics.cpp:10-77): uniform
                levels, or stretched from an initial dz with a constant ratio;
  btf_nodes  -- the basic terrain-following (BTF) grid of
                init_which_terrain_grid (Utils/ERF_TerrainMetrics.cpp:230-335):
                z(i,j,k) = ((z_sfc - z0) z_top + (z_top - z_sfc) z_k) / (z_top - z0);
  hill       -- the synthetic terrain of the terrain ABL case, evaluated on the
                node index modulo the domain so that it is exactly periodic.

The metrics (detJ, face areas, z at cell centres) are derived from z_phys_nd
by the library itself (erf_b200_set_terrain), as make_J / make_areas /
make_zcc do in the reference.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import config as C
from .cases import splitmix64_uniform


def zlevels(nz: int, dz: float, stretch: float = 0.0, dz0: float = 0.0, zsurf: float = 0.0) -> np.ndarray:
    """nz+1 staggered levels: k*dz, or zsurf + sum of dz0*stretch^m."""
    z = np.zeros(nz + 1)
    if stretch == 0.0:
        for k in range(nz + 1):
            z[k] = k * dz
        return z
    z[0] = zsurf
    d = dz0
    for k in range(1, nz + 1):
        z[k] = z[k - 1] + d
        d *= stretch
    return z


def btf_nodes(zlev: np.ndarray, h: np.ndarray) -> np.ndarray:
    """z_phys_nd[nz+1][ny+1][nx+1] from the levels and the surface height
    h[ny+1][nx+1] (the formula is applied at k = 0 as well)."""
    nz = zlev.size - 1
    z_top = zlev[nz]
    z0 = zlev[0]
    out = np.empty((nz + 1,) + h.shape)
    for k in range(nz + 1):
        out[k] = ((h - z0) * z_top + (z_top - h) * zlev[k]) / (z_top - z0)
    return out


def hill(nx: int, ny: int, dx: float, dy: float, h0: float = 300.0, r0: float = 800.0,
         amp: float = 20.0, waves: int = 3) -> np.ndarray:
    """Surface height at the nodes: h0 exp(-r^2/r0^2) about the domain centre
    plus amp sin(2 pi waves x / Lx) sin(2 pi waves y / Ly), where the node
    index is taken modulo the domain (node nx is node 0)."""
    i = np.arange(nx + 1) % nx
    j = np.arange(ny + 1) % ny
    x = i * dx
    y = j * dy
    xc, yc = 0.5 * nx * dx, 0.5 * ny * dy
    X, Y = np.meshgrid(x, y, indexing="xy")
    r2 = (X - xc) ** 2 + (Y - yc) ** 2
    bump = h0 * np.exp(-r2 / (r0 * r0))
    I, J = np.meshgrid(i, j, indexing="xy")
    waves_ = amp * np.sin(2.0 * math.pi * waves * I / nx) * np.sin(2.0 * math.pi * waves * J / ny)
    return bump + waves_


def cell_heights(z_nd: np.ndarray) -> np.ndarray:
    """z at cell centres (mean of the 8 corner nodes), [nz][ny][nx]."""
    return 0.125 * (z_nd[:-1, :-1, :-1] + z_nd[:-1, :-1, 1:] + z_nd[:-1, 1:, :-1] + z_nd[:-1, 1:, 1:]
                    + z_nd[1:, :-1, :-1] + z_nd[1:, :-1, 1:] + z_nd[1:, 1:, :-1] + z_nd[1:, 1:, 1:])


@dataclass
class TerrainCase:
    name: str
    cfg: C.ErfConfig
    z_nd: np.ndarray                # [nz+1][ny+1][nx+1]
    theta3: np.ndarray              # sounding theta at the cell centres [nz][ny][nx]
    qv3: np.ndarray
    theta_sfc: float
    qv_sfc: float
    p_sfc: float
    u0: float
    v0: float
    seed: int
    pert: dict = field(default_factory=dict)
    steps: int = 10

    def build_state(self, base_rho0: np.ndarray):
        """Initial cons, u, v, w from the base density ((nz+2) planes)."""
        cfg = self.cfg
        nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
        rho = base_rho0.reshape(nz + 2, ny, nx)[1:nz + 1].copy()
        theta = self.theta3.copy()
        amp = self.pert.get("noise_amp", 0.0)
        if amp > 0.0:
            zc = cell_heights(self.z_nd)
            agl = zc - cell_heights(np.repeat(self.z_nd[:1], nz + 1, axis=0))
            r = splitmix64_uniform(self.seed, nx * ny * nz).reshape(nz, ny, nx)
            noise = amp * (2.0 * r - 1.0)
            noise[agl > self.pert.get("noise_agl", np.inf)] = 0.0
            theta += noise
        cons = np.zeros((cfg.ncomp, nz, ny, nx))
        cons[0] = rho
        cons[1] = rho * theta
        if "tke0" in self.pert:
            cons[2] = rho * self.pert["tke0"]
        if cfg.moisture != C.MOIST_NONE:
            cons[5] = rho * self.qv3
            if "qr0" in self.pert and cfg.ncomp > 7:
                cons[7] = rho * self.pert["qr0"]
        u = np.full((nz, ny, nx + 1), float(self.u0))
        v = np.full((nz, ny + 1, nx), float(self.v0))
        w = np.zeros((nz + 1, ny, nx))
        return cons, u, v, w


def abl_terrain(nx=256, ny=256, nz=96, dx=25.0, dz0=5.0, stretch=1.04, seed=2, les="deardorff",
                h0=300.0, r0=800.0, amp=20.0, waves=3, dt=0.1, u0=10.0) -> TerrainCase:
    """Terrain-following ABL: dx = dy = 25 m, levels stretched from dz0 = 5 m
    (ratio 1.04), a 300 m Gaussian hill of 800 m radius plus 20 m sinusoids
    (3 wavelengths across the domain), theta 300 K up to 300 m then
    +1 K / 100 m, +-0.2 K seeded perturbations in the lowest 300 m above the
    ground, Deardorff closure (Ck 0.1, Ce 0.93), geostrophic wind (10, 0),
    no-slip ground, slip top."""
    c = C.defaults()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.dx = c.dy = dx
    zl = zlevels(nz, 0.0, stretch, dz0)
    c.dz = zl[nz] / nz                     # computational cell height (prob_hi_z / nz)
    c.zlo_bc, c.zhi_bc = C.BC_NO_SLIP_WALL, C.BC_SLIP_WALL
    c.dt, c.mri_ratio = dt, 6
    c.ncomp, c.moisture = 5, C.MOIST_NONE
    for f in ("dycore_horiz_adv", "dycore_vert_adv", "dryscal_horiz_adv", "dryscal_vert_adv"):
        setattr(c, f, C.UPWIND_5TH)
    c.molec_diff_type = C.MOLEC_NONE
    if les == "deardorff":
        c.les_type = C.LES_DEARDORFF
        c.Ck, c.Ce, c.Ce_wall, c.sigma_k, c.theta_ref = 0.1, 0.93, 0.0, 0.5, 300.0
    else:
        c.les_type, c.Cs = C.LES_SMAGORINSKY, 0.1
    c.gravity = C.CONST_GRAV
    c.buoyancy_type = 1
    C.set_coriolis(c, rotational_time_period=4.0 * math.pi / 1.0e-4, latitude_deg=90.0, geo_wind=(u0, 0.0, 0.0))
    c.use_terrain = 1
    h = hill(nx, ny, dx, dx, h0, r0, amp, waves)
    z_nd = btf_nodes(zl, h)
    zc = cell_heights(z_nd)
    theta3 = np.where(zc < 300.0, 300.0, 300.0 + 0.01 * (zc - 300.0))
    pert = {"noise_amp": 0.2, "noise_agl": 300.0}
    if les == "deardorff":
        pert["tke0"] = 0.1
    return TerrainCase("abl_terrain", c, z_nd, theta3, np.zeros_like(theta3), 300.0, 0.0, 1.0e5,
                       u0, 0.0, seed, pert=pert, steps=100)


def moist_hill(nx=24, ny=20, nz=24, dx=1000.0, dz=250.0, h0=1000.0, r0=4000.0, seed=3, dt=0.5) -> TerrainCase:
    """A moist warm bubble over a Gaussian hill (Kessler with rain, WENO5
    moisture, buoyancy type 1, slip walls, no diffusion): theta 300 K at the
    ground rising as 43 K (z / 12 km)^1.25, relative humidity 0.95 falling to
    0.25 aloft (Tetens saturation over a dry hydrostatic pressure estimate),
    a +2 K bubble of 4 km radius centred 2 km above the hill top in which the
    air is 2 % supersaturated and carries 0.1 g/kg of rain, so that
    condensation, evaporation and sedimentation all act from the first
    step, and a 5 m/s wind across the hill."""
    from . import cases as CS
    c = C.defaults()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.dx = c.dy = dx
    c.dz = dz
    c.zlo_bc = c.zhi_bc = C.BC_SLIP_WALL
    c.dt, c.mri_ratio = dt, 4
    c.ncomp, c.moisture = 8, C.MOIST_KESSLER
    c.dycore_horiz_adv = c.dycore_vert_adv = C.UPWIND_5TH
    c.dryscal_horiz_adv = c.dryscal_vert_adv = C.UPWIND_5TH
    c.moistscal_horiz_adv = c.moistscal_vert_adv = C.WENO_5
    c.molec_diff_type = C.MOLEC_NONE
    c.les_type = C.LES_NONE
    c.gravity = C.CONST_GRAV
    c.buoyancy_type = 1
    c.use_terrain = 1
    zl = zlevels(nz, dz)
    h = hill(nx, ny, dx, dx, h0, r0, 0.0, 1)
    z_nd = btf_nodes(zl, h)
    zc = cell_heights(z_nd)
    theta3 = 300.0 + 43.0 * (zc / 12000.0) ** 1.25
    rh = 0.95 - 0.70 * (zc / 12000.0) ** 1.25
    p = 1.0e5 * (1.0 - C.CONST_GRAV * zc / (C.CP_D * 300.0)) ** (C.CP_D / C.R_D)
    T3 = theta3 * (p / 1.0e5) ** (C.R_D / C.CP_D)
    xc = (np.arange(nx) + 0.5) * dx
    yc = (np.arange(ny) + 0.5) * dx
    X, Y = np.meshgrid(xc, yc)
    zb = h0 + 2000.0
    rr = np.sqrt(((X - 0.5 * nx * dx) / r0)[None] ** 2 + ((Y - 0.5 * ny * dx) / r0)[None] ** 2
                 + ((zc - zb) / 1500.0) ** 2)
    inside = rr < 1.0
    theta3 = theta3 + np.where(inside, 2.0 * np.cos(0.5 * np.pi * np.minimum(rr, 1.0)) ** 2, 0.0)
    qsat = CS._tetens_qsat(T3, p)
    qv3 = np.where(inside, 1.02 * qsat, np.minimum(0.014, rh * qsat))
    return TerrainCase("moist_hill", c, z_nd, theta3, qv3, 300.0, float(qv3[0].mean()), 1.0e5, 5.0, 0.0, seed,
                       pert={"qr0": np.where(inside, 1.0e-4, 0.0)}, steps=10)


# ---------------------------------------------------------------------------
# Moving terrain: the travelling surface wave of the reference's
# Exec/DevTests/MovingTerrain problem on a Sullivan-smoothed grid.
# ---------------------------------------------------------------------------
PI = 3.14159265358979323846264338327950288
P_0, GAMMA = 1.0e5, 1.4


IP_0 = 1.0 / P_0


def _rt_of_p(p):
    """getRhoThetagivenP (Utils/ERF_EOS.H:133-137), dry."""
    return (p * P_0 ** (GAMMA - 1.0)) ** (1.0 / GAMMA) * (1.0 / C.R_D)


def _p_of_rt(rt):
    """getPgivenRTh (Utils/ERF_EOS.H:62-66), dry."""
    return P_0 * (C.R_D * rt * IP_0) ** GAMMA


def wave_surface(nx: int, ny: int, dx: float, ampl: float, wavelength: float, t: float) -> np.ndarray:
    """h[ny+1][nx+1] = ampl sin(kp x - omega t), x = i dx, kp = 2 pi /
    wavelength, omega = sqrt(g kp) (MovingTerrain ERF_prob.cpp:174-197)."""
    kp = 2.0 * PI / wavelength
    om = math.sqrt(C.CONST_GRAV * kp)
    x = np.arange(nx + 1) * dx
    h = np.array([ampl * math.sin(kp * xi - om * t) for xi in x])
    return np.repeat(h[None, :], ny + 1, axis=0)


def sullivan_nodes(zlev: np.ndarray, h: np.ndarray) -> np.ndarray:
    """z_phys_nd[nz+1][ny+1][nx+1] of terrain_smoothing = 2
    (Utils/ERF_TerrainMetrics.cpp:501-536): z_k + (1 - z_k / z_top)^3 h."""
    nz = zlev.size - 1
    z_top = zlev[nz]
    out = np.empty((nz + 1,) + h.shape)
    for k in range(nz + 1):
        out[k] = zlev[k] + math.pow(1.0 - zlev[k] / z_top, 3.0) * h
    out[0] = h
    return out


def isentropic_base_state_terrain(z_nd: np.ndarray, theta: float = 300.0, T_sfc: float = 300.0):
    """Base state of a constant-theta atmosphere over the terrain: per column
    init_isentropic_hse_terrain (Utils/ERF_HSE_utils.H:199-302; Newton on
    rho with MAX_ITER 10, TOL 1e-8) from rho_sfc = p_0 / (R_d T_sfc) at the
    cell centres z_cc, then erf_enforce_hse with terrain
    (Initialization/ERF_init1d.cpp:152-241).  Returns rho0, p0, pi0, th0 in
    (nz+2) planes of ny*nx (plane k+1 = level k)."""
    nzp1, nyp1, nxp1 = z_nd.shape
    nz, ny, nx = nzp1 - 1, nyp1 - 1, nxp1 - 1
    # z_cc for k = 0..nz (k = nz from the extrapolated node level nz+1)
    ztop_x = 2.0 * z_nd[nz] - z_nd[nz - 1]
    zn = np.concatenate([z_nd, ztop_x[None]], axis=0)
    zc = cell_heights(zn)                       # [nz+1][ny][nx]
    g = C.CONST_GRAV
    rho_sfc = P_0 / (C.R_D * T_sfc)
    kgam = GAMMA * P_0 * (C.R_D * theta * IP_0) ** GAMMA
    r = np.empty((nz, ny, nx))
    p = np.empty((nz, ny, nx))
    for j in range(ny):
        for i in range(nx):
            half_dz = zc[0, j, i]
            r0 = rho_sfc
            for _ in range(10):
                p_hse = P_0 - half_dz * r0 * g
                p_eos = _p_of_rt(r0 * theta)
                drho = (p_hse - p_eos) / (kgam * r0 ** (GAMMA - 1.0) + half_dz * g)
                r0 = r0 + drho
                if abs(drho) < 1.0e-8:
                    break
            r[0, j, i] = r0
            p[0, j, i] = _p_of_rt(r0 * theta)
            for k in range(1, nz):
                dz_loc = zc[k, j, i] - zc[k - 1, j, i]
                rk = r[k - 1, j, i]
                for _ in range(10):
                    p_hse = p[k - 1, j, i] - dz_loc * 0.5 * (r[k - 1, j, i] + rk) * g
                    p_eos = _p_of_rt(rk * theta)
                    drho = (p_hse - p_eos) / (kgam * rk ** (GAMMA - 1.0) + dz_loc * g)
                    rk = rk + drho
                    if abs(drho) < 1.0e-8 * r[k - 1, j, i]:
                        break
                r[k, j, i] = rk
                p[k, j, i] = _p_of_rt(rk * theta)
    rho = np.empty((nz + 2, ny, nx))
    rho[1:nz + 1] = r
    rho[0] = r[0]
    rho[nz + 1] = r[nz - 1]
    pres = np.empty((nz + 2, ny, nx))
    hz = zc[0]
    pres[1] = P_0 - hz * rho[1] * g
    pres[0] = P_0 + hz * rho[1] * g
    for k in range(1, nz + 1):
        pres[k + 1] = pres[k] - (zc[k] - zc[k - 1]) * (0.5 * (rho[k + 1] + rho[k])) * g
    rdocp = C.R_D / C.CP_D
    pi0 = (pres * IP_0) ** rdocp
    th0 = _rt_of_p(pres) / rho
    return [a.reshape(-1).copy() for a in (rho, pres, pi0, th0)]


@dataclass
class MovingTerrainCase:
    name: str
    cfg: C.ErfConfig
    z_nd: np.ndarray                # the grid at t = 0
    base: list                      # rho0, p0, pi0, th0, (nz+2) planes
    steps: int

    def build_state(self):
        """init_from_hse plus the problem's init_custom_pert
        (MovingTerrain ERF_prob.cpp:25-112): the pressure and velocity of a
        deep-water gravity wave under the surface, as perturbations."""
        cfg = self.cfg
        nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
        H = nz * cfg.dz
        A, kp = cfg.mt_ampl, 2.0 * PI / cfg.mt_wavelength
        om = math.sqrt(C.CONST_GRAV * kp)
        z_nd = self.z_nd
        zc = cell_heights(z_nd)
        r_hse = self.base[0].reshape(nz + 2, ny, nx)[1:nz + 1]
        p_hse = self.base[1].reshape(nz + 2, ny, nx)[1:nz + 1]
        xc = (np.arange(nx) + 0.5) * cfg.dx
        z = zc - A * np.sin(kp * xc)[None, None, :]
        fac = np.cosh(kp * (z - H)) / math.sinh(kp * H)
        p_prime = -(A * om * om / kp) * fac * np.sin(kp * xc)[None, None, :] * r_hse
        cons = np.zeros((cfg.ncomp, nz, ny, nx))
        cons[0] = r_hse
        rt_hse = _rt_of_p(p_hse)
        cons[1] = rt_hse + (_rt_of_p(p_hse + p_prime) - rt_hse)
        xf = np.arange(nx + 1) * cfg.dx
        zu = 0.25 * (z_nd[:-1, :-1, :] + z_nd[:-1, 1:, :] + z_nd[1:, :-1, :] + z_nd[1:, 1:, :])
        zu = zu - A * np.sin(kp * xf)[None, None, :]
        u = -A * om * (np.cosh(kp * (zu - H)) / math.sinh(kp * H)) * np.sin(kp * xf)[None, None, :]
        v = np.zeros((nz, ny + 1, nx))
        zw = 0.25 * (z_nd[:, :-1, :-1] + z_nd[:, :-1, 1:] + z_nd[:, 1:, :-1] + z_nd[:, 1:, 1:])
        zw = zw - A * np.sin(kp * xc)[None, None, :]
        w = A * om * (np.sinh(kp * (zw - H)) / math.sinh(kp * H)) * np.cos(kp * xc)[None, None, :]
        return cons, u, v, w


def moving_terrain(nx=40, ny=8, nz=79, Lx=200.0, Ly=40.0, H=400.0, ampl=0.16, wavelength=100.0,
                   substeps=False, dt=None, steps=None) -> MovingTerrainCase:
    """Tests/test_files/MovingTerrain_{nosub,sub}/*.i: 40 x 8 x 79 cells over
    200 m x 40 m x 400 m, periodic x / y, slip walls, Centered_2nd everywhere,
    no diffusion, gravity with buoyancy type 1, moving terrain with Sullivan
    smoothing, Ampl 0.16 m.  Without substepping dt = 0.005 s for 20 steps;
    with it dt = 0.1 s, ratio 20, 10 steps, use_lagged_delta_rt = false."""
    c = C.defaults()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.dx, c.dy, c.dz = Lx / nx, Ly / ny, H / nz
    c.zlo_bc = c.zhi_bc = C.BC_SLIP_WALL
    c.ncomp = 5
    for f in ("dycore_horiz_adv", "dycore_vert_adv", "dryscal_horiz_adv", "dryscal_vert_adv"):
        setattr(c, f, C.CENTERED_2ND)
    c.molec_diff_type = C.MOLEC_NONE
    c.les_type = C.LES_NONE
    c.gravity = C.CONST_GRAV
    c.buoyancy_type = 1
    c.use_terrain = 1
    c.terrain_type = C.TERRAIN_MOVING
    c.mt_ampl, c.mt_wavelength = ampl, wavelength
    if substeps:
        c.substepping_type = C.SUBSTEP_IMPLICIT
        c.dt, c.mri_ratio = (0.1 if dt is None else dt), 20
        c.no_lagged_delta_rt = 1       # erf.use_lagged_delta_rt = false
        nsteps = 10 if steps is None else steps
        name = "MovingTerrain_sub"
    else:
        c.substepping_type = C.SUBSTEP_NONE
        c.dt = 0.005 if dt is None else dt
        nsteps = 20 if steps is None else steps
        name = "MovingTerrain_nosub"
    zl = zlevels(nz, c.dz)
    z_nd = sullivan_nodes(zl, wave_surface(nx, ny, c.dx, ampl, wavelength, 0.0))
    base = isentropic_base_state_terrain(z_nd)
    return MovingTerrainCase(name, c, z_nd, base, nsteps)
