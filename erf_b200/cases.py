"""Seeded synthetic workloads with the shapes of the reference's benchmark cases.

No dataset is involved: every case is generated here, in FP64, from an analytic
sounding plus seeded perturbations.  The random stream is SplitMix64 (Steele,
Lea & Flood 2014), so that any implementation can regenerate identical inputs.

Cases
  abl_dry      -- dry neutral ABL: periodic, no-slip bottom / slip top,
                  theta 300 K below 500 m then +3 K/km, geostrophic wind (10,0)
                  with f = 1e-4 s^-1, +-0.1 K perturbations below 400 m,
                  Upwind_5th everywhere, Smagorinsky Cs = 0.1, dt 0.5 s, ratio 6.
  moist_bubble -- moist warm bubble: slip walls, analytic tropospheric sounding
                  (theta = 300 + 43 (z/12 km)^1.25 to a 12 km tropopause,
                  isothermal 213 K above), RH 0.95 falling to 0.25 aloft,
                  linear shear 0-12 m/s over 0-5 km, +3 K cosine bubble
                  (10 km horizontal radius, 1.5 km vertical radius, centred at
                  1.5 km), +-0.01 K noise; Kessler; Upwind_5th dycore, WENO5
                  scalars, buoyancy type 2, dt 2 s, ratio 6.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import config as C

_MASK64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64_uniform(seed: int, n: int) -> np.ndarray:
    """n uniform doubles in [0,1) from SplitMix64 (53 high bits)."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


@dataclass
class Case:
    name: str
    cfg: C.ErfConfig
    theta_cc: np.ndarray            # sounding theta at cell centres (nz)
    qv_cc: np.ndarray               # sounding qv at cell centres (nz)
    theta_sfc: float
    qv_sfc: float
    p_sfc: float
    u_cc: np.ndarray                # sounding u at cell centres (nz)
    v_cc: np.ndarray
    seed: int
    pert: dict = field(default_factory=dict)
    steps: int = 10

    def build_state(self, base_rho0: np.ndarray):
        """Initial cons[ncomp][nz][ny][nx], u, v, w (dense, i fastest)."""
        cfg = self.cfg
        nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
        z = (np.arange(nz) + 0.5) * cfg.dz
        x = (np.arange(nx) + 0.5) * cfg.dx
        y = (np.arange(ny) + 0.5) * cfg.dy
        rho = np.broadcast_to(base_rho0[1:nz + 1][:, None, None], (nz, ny, nx)).copy()
        theta = np.broadcast_to(self.theta_cc[:, None, None], (nz, ny, nx)).copy()
        theta += self.theta_perturbation(x, y, z)
        cons = np.zeros((cfg.ncomp, nz, ny, nx))
        cons[0] = rho
        cons[1] = rho * theta
        if cfg.moisture != C.MOIST_NONE:
            cons[5] = rho * self.qv_cc[:, None, None]
        if "tke0" in self.pert:   # initial subgrid TKE (Deardorff)
            e0 = np.where(z <= self.pert.get("tke0_zmax", np.inf), self.pert["tke0"], 1.0e-3)
            cons[2] = rho * e0[:, None, None]
        u = np.broadcast_to(self.u_cc[:, None, None], (nz, ny, nx + 1)).copy()
        v = np.broadcast_to(self.v_cc[:, None, None], (nz, ny + 1, nx)).copy()
        w = np.zeros((nz + 1, ny, nx))
        va = self.pert.get("vel_noise_amp", 0.0)
        if va > 0.0:
            # seeded velocity noise below vel_noise_zmax (periodic faces kept
            # consistent, w = 0 on the walls)
            zmax = self.pert.get("vel_noise_zmax", np.inf)
            zf = np.arange(nz + 1) * cfg.dz
            nu = va * (2.0 * splitmix64_uniform(self.seed + 101, nz * ny * nx).reshape(nz, ny, nx) - 1.0)
            nv = va * (2.0 * splitmix64_uniform(self.seed + 202, nz * ny * nx).reshape(nz, ny, nx) - 1.0)
            nw = va * (2.0 * splitmix64_uniform(self.seed + 303, (nz + 1) * ny * nx).reshape(nz + 1, ny, nx) - 1.0)
            nu[z > zmax] = 0.0
            nv[z > zmax] = 0.0
            nw[zf > zmax] = 0.0
            nw[0] = 0.0
            nw[nz] = 0.0
            u[:, :, :nx] += nu
            u[:, :, nx] = u[:, :, 0]
            v[:, :ny, :] += nv
            v[:, ny, :] = v[:, 0, :]
            w += nw
        return cons, u, v, w

    def theta_perturbation(self, x, y, z):
        cfg = self.cfg
        nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
        p = self.pert
        out = np.zeros((nz, ny, nx))
        amp = p.get("noise_amp", 0.0)
        if amp > 0.0:
            r = splitmix64_uniform(self.seed, nx * ny * nz).reshape(nz, ny, nx)
            noise = amp * (2.0 * r - 1.0)
            zmax = p.get("noise_zmax", np.inf)
            noise[z > zmax, :, :] = 0.0
            out += noise
        if p.get("bubble_amp", 0.0) != 0.0:
            X, Y, Zc = np.meshgrid(x, y, z, indexing="ij")
            xc = p.get("bubble_xc", 0.5 * nx * cfg.dx)
            yc = p.get("bubble_yc", 0.5 * ny * cfg.dy)
            rr = np.sqrt(((X - xc) / p["bubble_rh"]) ** 2 + ((Y - yc) / p["bubble_rh"]) ** 2
                         + ((Zc - p["bubble_zc"]) / p["bubble_rz"]) ** 2)
            bub = np.where(rr < 1.0, p["bubble_amp"] * np.cos(0.5 * math.pi * rr) ** 2, 0.0)
            out += np.transpose(bub, (2, 1, 0))
        return out


def _tetens_qsat(T, p):
    es = 611.2 * np.exp(17.67 * (T - 273.15) / (T - 29.65))
    return 0.622 * es / (p - es)


def abl_dry(nx=64, ny=64, nz=64, seed=0) -> Case:
    c = C.defaults()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.dx = c.dy = c.dz = 50.0
    c.zlo_bc, c.zhi_bc = C.BC_NO_SLIP_WALL, C.BC_SLIP_WALL
    c.dt, c.mri_ratio = 0.5, 6
    c.ncomp, c.moisture = 5, C.MOIST_NONE
    for f in ("dycore_horiz_adv", "dycore_vert_adv", "dryscal_horiz_adv", "dryscal_vert_adv"):
        setattr(c, f, C.UPWIND_5TH)
    c.molec_diff_type = C.MOLEC_NONE
    c.les_type, c.Cs = C.LES_SMAGORINSKY, 0.1
    c.gravity = C.CONST_GRAV
    c.buoyancy_type = 1
    C.set_coriolis(c, rotational_time_period=4.0 * math.pi / 1.0e-4, latitude_deg=90.0, geo_wind=(10.0, 0.0, 0.0))
    z = (np.arange(nz) + 0.5) * c.dz
    theta = np.where(z < 500.0, 300.0, 300.0 + 3.0e-3 * (z - 500.0))
    return Case("abl_dry", c, theta, np.zeros(nz), 300.0, 0.0, 1.0e5,
                np.full(nz, 10.0), np.zeros(nz), seed,
                pert={"noise_amp": 0.1, "noise_zmax": 400.0}, steps=10)


def abl_fine(nx=512, ny=512, nz=128, dx=10.0, dz=10.0, u_g=10.0, dt=0.08, seed=0) -> Case:
    """Fine-grid ABL with the physics of abl_dry (training data of the learned
    closure): geostrophic wind (u_g, 0), Smagorinsky Cs 0.1, theta 300 K below
    500 m then +3 K/km, +-0.1 K theta noise and +-0.5 m/s velocity noise below
    400 m (the velocity noise starts the shear turbulence within the short
    runs used for training)."""
    case = abl_dry(nx=nx, ny=ny, nz=nz, seed=seed)
    c = case.cfg
    c.dx = c.dy = dx
    c.dz = dz
    c.dt = dt
    C.set_coriolis(c, rotational_time_period=4.0 * math.pi / 1.0e-4, latitude_deg=90.0, geo_wind=(u_g, 0.0, 0.0))
    z = (np.arange(nz) + 0.5) * dz
    case.theta_cc = np.where(z < 500.0, 300.0, 300.0 + 3.0e-3 * (z - 500.0))
    case.u_cc = np.full(nz, float(u_g))
    case.name = "abl_fine"
    case.pert.update({"vel_noise_amp": 0.5, "vel_noise_zmax": 400.0})
    return case


def abl_deardorff(nx=64, ny=64, nz=64, seed=0, tke0=0.1) -> Case:
    """abl_dry with the Deardorff TKE closure (Ck 0.1, Ce 0.93, sigma_k 0.5,
    theta_ref 300 K): initial subgrid TKE tke0 m^2/s^2 below 400 m and 1e-3
    above, so that both the neutral and the stably stratified mixing-length
    branches are used."""
    case = abl_dry(nx=nx, ny=ny, nz=nz, seed=seed)
    c = case.cfg
    c.les_type = C.LES_DEARDORFF
    c.Ck, c.Ce, c.Ce_wall, c.sigma_k, c.theta_ref = 0.1, 0.93, 0.0, 0.5, 300.0
    case.name = "abl_deardorff"
    case.pert["tke0"] = tke0
    case.pert["tke0_zmax"] = 400.0
    return case


def abl_most(nx=64, ny=64, nz=64, seed=0, les="smagorinsky", z0=0.1, zref=0.0) -> Case:
    """abl_dry (or abl_deardorff with les="deardorff") over a MOST ground
    (Moeng stress, adiabatic, roughness z0, reference height zref; 0 = the
    first cell centre) with +-0.5 m/s velocity noise below 400 m, so that the
    ground stress varies over the plane."""
    case = abl_deardorff(nx=nx, ny=ny, nz=nz, seed=seed) if les == "deardorff" else abl_dry(nx=nx, ny=ny, nz=nz, seed=seed)
    c = case.cfg
    c.zlo_bc = C.BC_MOST
    c.most_z0, c.most_zref = z0, zref
    case.name = "abl_most_" + les
    case.pert.update({"vel_noise_amp": 0.5, "vel_noise_zmax": 400.0})
    return case


def abl_most_moist(nx=64, ny=64, nz=64, seed=0, les="smagorinsky", z0=0.1, zref=0.0) -> Case:
    """abl_most with Kessler moisture (rain included): water vapour falling
    off from 12 g/kg at the ground with a 1.5 km scale height, moist scalars
    advected with WENO5, buoyancy type 2 (the temperature-perturbation form
    about the moist base state's plane averages).  The adiabatic (Moeng) MOST
    ground applies no moisture flux, as the reference's only computes one for
    its CUSTOM flux type (BoundaryConditions/ERF_ABLMost.cpp:413-433)."""
    case = abl_most(nx=nx, ny=ny, nz=nz, seed=seed, les=les, z0=z0, zref=zref)
    c = case.cfg
    c.ncomp, c.moisture = 8, C.MOIST_KESSLER
    c.moistscal_horiz_adv = c.moistscal_vert_adv = C.WENO_5
    c.buoyancy_type = 2
    z = (np.arange(nz) + 0.5) * c.dz
    case.qv_cc = 0.012 * np.exp(-z / 1500.0)
    case.qv_sfc = 0.012
    case.name = "abl_most_moist_" + les
    return case


def moist_bubble(nx=128, ny=128, nz=80, seed=1) -> Case:
    c = C.defaults()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.dx = c.dy = 1000.0
    c.dz = 250.0
    c.zlo_bc = c.zhi_bc = C.BC_SLIP_WALL
    c.dt, c.mri_ratio = 2.0, 6
    c.ncomp, c.moisture = 8, C.MOIST_KESSLER
    c.dycore_horiz_adv = c.dycore_vert_adv = C.UPWIND_5TH
    c.dryscal_horiz_adv = c.dryscal_vert_adv = C.WENO_5
    c.moistscal_horiz_adv = c.moistscal_vert_adv = C.WENO_5
    c.molec_diff_type = C.MOLEC_NONE
    c.les_type = C.LES_NONE
    c.gravity = C.CONST_GRAV
    c.buoyancy_type = 2
    z = (np.arange(nz) + 0.5) * c.dz
    z_tr, th_tr, T_tr = 12000.0, 343.0, 213.0
    theta = np.where(z <= z_tr, 300.0 + 43.0 * (z / z_tr) ** 1.25,
                     th_tr * np.exp(C.CONST_GRAV / (C.CP_D * T_tr) * (z - z_tr)))
    rh = np.where(z <= z_tr, 0.95 - 0.70 * (z / z_tr) ** 1.25, 0.25)
    # dry hydrostatic pressure estimate for the saturation mixing ratio
    p = np.empty(nz)
    pi_s = 1.0
    for k in range(nz):
        zz = z[k]
        # integrate d(pi)/dz = -g/(cp theta) with the local theta
        if k == 0:
            pi_k = pi_s - C.CONST_GRAV / (C.CP_D * theta[0]) * zz
        else:
            pi_k = pi_prev - C.CONST_GRAV / (C.CP_D * 0.5 * (theta[k] + theta[k - 1])) * c.dz
        p[k] = 1.0e5 * pi_k ** (C.CP_D / C.R_D)
        pi_prev = pi_k
    T = theta * (p / 1.0e5) ** (C.R_D / C.CP_D)
    qv = np.minimum(0.014, rh * _tetens_qsat(T, p))
    u = np.where(z < 5000.0, 12.0 * z / 5000.0, 12.0)
    return Case("moist_bubble", c, theta, qv, 300.0, 0.014, 1.0e5, u, np.zeros(nz), seed,
                pert={"noise_amp": 0.01, "bubble_amp": 3.0, "bubble_rh": 10000.0,
                      "bubble_rz": 1500.0, "bubble_zc": 1500.0}, steps=100)


CASES = {"abl_dry": abl_dry, "moist_bubble": moist_bubble, "abl_deardorff": abl_deardorff}
