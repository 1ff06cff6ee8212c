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
