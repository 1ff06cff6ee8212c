"""Dycore configuration: a ctypes mirror of ``erf_b200_config`` (include/erf_b200.h).

The fields are the SolverChoice / AdvChoice / DiffChoice / TurbChoice keys the
reference's hot path reads (Source/DataStructs/ERF_DataStruct.H:80-580,
ERF_AdvStruct.H:26-186, ERF_TurbStruct.H:29-210, ERF_DiffStruct.H:26-32), with
the reference's defaults.  ``from_inputs`` accepts the reference's own
``erf.*`` key names so an inputs file can be mapped one to one.
"""
from __future__ import annotations

import ctypes
import math

# AdvType codes (Source/ERF_IndexDefines.H:196-210)
CENTERED_2ND, UPWIND_3RD, CENTERED_4TH, UPWIND_5TH, CENTERED_6TH = 101, 102, 103, 104, 105
WENO_3, WENO_3Z, WENO_5, WENO_5Z, WENO_3MZQ, WENO_7, WENO_7Z = 106, 107, 108, 109, 110, 111, 112
ADV_NAMES = {
    "Centered_2nd": CENTERED_2ND, "Upwind_3rd": UPWIND_3RD, "Centered_4th": CENTERED_4TH,
    "Upwind_5th": UPWIND_5TH, "Centered_6th": CENTERED_6TH, "WENO3": WENO_3, "WENOZ3": WENO_3Z,
    "WENO5": WENO_5, "WENOZ5": WENO_5Z, "WENOMZQ3": WENO_3MZQ, "WENO7": WENO_7, "WENOZ7": WENO_7Z,
}
LES_NONE, LES_SMAGORINSKY, LES_DEARDORFF, LES_MLP = 0, 1, 2, 3
MOLEC_NONE, MOLEC_CONSTANT, MOLEC_CONSTANT_ALPHA = 0, 1, 2
MOIST_NONE, MOIST_KESSLER, MOIST_KESSLER_NORAIN = 0, 1, 2
BC_NO_SLIP_WALL, BC_SLIP_WALL, BC_PERIODIC, BC_MOST = 5, 6, 7, 8
PREC_FP64, PREC_MIXED = 0, 1
SUBSTEP_IMPLICIT, SUBSTEP_NONE = 0, 1
TERRAIN_STATIC, TERRAIN_MOVING = 0, 1
# conserved components (Source/ERF_IndexDefines.H:36-43)
RHO_COMP, RHOTHETA_COMP, RHOKE_COMP, RHOQKE_COMP, RHOSCALAR_COMP, RHOQ1_COMP = 0, 1, 2, 3, 4, 5

R_D = 287.0
CP_D = 1004.5
CONST_GRAV = 9.81


class ErfConfig(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("zlo_bc", ctypes.c_int), ("zhi_bc", ctypes.c_int),
        ("dt", ctypes.c_double), ("mri_ratio", ctypes.c_int), ("force_stage1_single_substep", ctypes.c_int),
        ("ncomp", ctypes.c_int), ("moisture", ctypes.c_int),
        ("dycore_horiz_adv", ctypes.c_int), ("dycore_vert_adv", ctypes.c_int),
        ("dryscal_horiz_adv", ctypes.c_int), ("dryscal_vert_adv", ctypes.c_int),
        ("moistscal_horiz_adv", ctypes.c_int), ("moistscal_vert_adv", ctypes.c_int),
        ("dycore_horiz_upw_frac", ctypes.c_double), ("dycore_vert_upw_frac", ctypes.c_double),
        ("dryscal_horiz_upw_frac", ctypes.c_double), ("dryscal_vert_upw_frac", ctypes.c_double),
        ("moistscal_horiz_upw_frac", ctypes.c_double), ("moistscal_vert_upw_frac", ctypes.c_double),
        ("molec_diff_type", ctypes.c_int),
        ("alpha_T", ctypes.c_double), ("alpha_C", ctypes.c_double),
        ("dynamic_viscosity", ctypes.c_double), ("rho0_trans", ctypes.c_double),
        ("les_type", ctypes.c_int),
        ("Cs", ctypes.c_double), ("Pr_t", ctypes.c_double), ("Sc_t", ctypes.c_double),
        ("Ck", ctypes.c_double), ("Ce", ctypes.c_double), ("Ce_wall", ctypes.c_double),
        ("sigma_k", ctypes.c_double), ("theta_ref", ctypes.c_double),
        ("gravity", ctypes.c_double), ("c_p", ctypes.c_double),
        ("buoyancy_type", ctypes.c_int), ("use_coriolis", ctypes.c_int),
        ("coriolis_factor", ctypes.c_double), ("sinphi", ctypes.c_double), ("cosphi", ctypes.c_double),
        ("abl_geo_forcing", ctypes.c_double * 3),
        ("precision", ctypes.c_int),
        ("use_terrain", ctypes.c_int),
        ("substepping_type", ctypes.c_int),
        ("terrain_type", ctypes.c_int),
        ("no_lagged_delta_rt", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
        ("most_z0", ctypes.c_double), ("most_zref", ctypes.c_double),
        ("mt_ampl", ctypes.c_double), ("mt_wavelength", ctypes.c_double),
    ]

    def copy(self) -> "ErfConfig":
        c = ErfConfig()
        ctypes.pointer(c)[0] = self
        return c

    @property
    def n_cells(self) -> int:
        return self.nx * self.ny * self.nz

    def describe(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if name == "reserved":
                continue
            if hasattr(v, "__len__"):
                v = list(v)
            out[name] = v
        return out


def defaults() -> ErfConfig:
    """Reference defaults (SolverChoice member initialisers)."""
    c = ErfConfig()
    c.nx = c.ny = c.nz = 16
    c.dx = c.dy = c.dz = 1.0
    c.zlo_bc = c.zhi_bc = BC_SLIP_WALL
    c.dt = 1.0
    c.mri_ratio = 6
    c.force_stage1_single_substep = 1
    c.ncomp = 5
    c.moisture = MOIST_NONE
    c.dycore_horiz_adv = c.dycore_vert_adv = UPWIND_3RD
    c.dryscal_horiz_adv = c.dryscal_vert_adv = UPWIND_3RD
    c.moistscal_horiz_adv = c.moistscal_vert_adv = WENO_3
    for f in ("dycore_horiz_upw_frac", "dycore_vert_upw_frac", "dryscal_horiz_upw_frac",
              "dryscal_vert_upw_frac", "moistscal_horiz_upw_frac", "moistscal_vert_upw_frac"):
        setattr(c, f, 1.0)
    c.molec_diff_type = MOLEC_CONSTANT
    c.alpha_T = c.alpha_C = 0.0
    c.dynamic_viscosity = 0.0
    c.rho0_trans = 1.0
    c.les_type = LES_NONE
    c.Cs = 0.0
    c.Pr_t = 1.0 / 3.0
    c.Sc_t = 1.0
    c.Ck = 0.1
    c.Ce = 0.93
    c.Ce_wall = 0.0
    c.sigma_k = 0.5
    c.theta_ref = 300.0
    c.gravity = 0.0
    c.c_p = CP_D
    c.buoyancy_type = 1
    c.use_coriolis = 0
    c.coriolis_factor = c.sinphi = c.cosphi = 0.0
    c.precision = PREC_FP64
    c.most_z0 = 0.1      # ABLMost z0_const
    c.most_zref = 0.0    # 0: half the lowest cell (MOSTAverage's default)
    c.terrain_type = TERRAIN_STATIC
    c.mt_ampl, c.mt_wavelength = 0.0, 100.0
    return c


def set_coriolis(c: ErfConfig, rotational_time_period: float, latitude_deg: float,
                 geo_wind=(0.0, 0.0, 0.0), coriolis_3d: bool = True) -> None:
    """SolverChoice::build_coriolis_forcings (ERF_DataStruct.H:476-510)."""
    c.use_coriolis = 1
    c.coriolis_factor = 2.0 * 2.0 * math.pi / rotational_time_period
    lat = latitude_deg * (math.pi / 180.0)
    c.sinphi = math.sin(lat)
    c.cosphi = math.cos(lat) if coriolis_3d else 0.0
    ug, vg, wg = geo_wind
    c.abl_geo_forcing[0] = -c.coriolis_factor * (vg * c.sinphi - wg * c.cosphi)
    c.abl_geo_forcing[1] = c.coriolis_factor * ug * c.sinphi
    c.abl_geo_forcing[2] = -c.coriolis_factor * ug * c.cosphi


def from_inputs(keys: dict) -> ErfConfig:
    """Map reference ``erf.*`` inputs-file keys onto a config."""
    c = defaults()
    g = lambda k, d=None: keys.get("erf." + k, keys.get(k, d))
    for k in ("dycore_horiz_adv_type", "dycore_vert_adv_type", "dryscal_horiz_adv_type",
              "dryscal_vert_adv_type", "moistscal_horiz_adv_type", "moistscal_vert_adv_type"):
        v = g(k)
        if v is not None:
            setattr(c, k.replace("_type", ""), ADV_NAMES[str(v).strip('"')])
    if g("use_gravity") is not None:
        c.gravity = CONST_GRAV if str(g("use_gravity")).lower() in ("1", "true") else 0.0
    les = g("les_type")
    if les is not None:
        c.les_type = {"None": LES_NONE, "Smagorinsky": LES_SMAGORINSKY, "Deardorff": LES_DEARDORFF}[str(les).strip('"')]
    md = g("molec_diff_type")
    if md is not None:
        c.molec_diff_type = {"None": MOLEC_NONE, "Constant": MOLEC_CONSTANT,
                             "ConstantAlpha": MOLEC_CONSTANT_ALPHA}[str(md).strip('"')]
    for k, f in (("alpha_T", "alpha_T"), ("alpha_C", "alpha_C"), ("dynamicViscosity", "dynamic_viscosity"),
                 ("rho0_trans", "rho0_trans"), ("Cs", "Cs"), ("Pr_t", "Pr_t"), ("Sc_t", "Sc_t"),
                 ("c_p", "c_p"), ("fixed_dt", "dt")):
        if g(k) is not None:
            setattr(c, f, float(g(k)))
    for k in ("fixed_mri_dt_ratio", "mri_fixed_dt_ratio"):
        if g(k) is not None:
            c.mri_ratio = int(g(k))
    if g("buoyancy_type") is not None:
        c.buoyancy_type = int(g("buoyancy_type"))
    if g("use_terrain") is not None:
        c.use_terrain = 1 if str(g("use_terrain")).lower() in ("1", "true") else 0
    tt = g("terrain_type")
    if tt is not None:
        c.terrain_type = {"Static": TERRAIN_STATIC, "Moving": TERRAIN_MOVING}[str(tt).strip('"')]
    if g("use_lagged_delta_rt") is not None:
        c.no_lagged_delta_rt = 0 if str(g("use_lagged_delta_rt")).lower() in ("1", "true") else 1
    if keys.get("prob.Ampl") is not None:
        c.mt_ampl = float(keys["prob.Ampl"])
    st = g("substepping_type")
    if st is not None:
        c.substepping_type = {"None": SUBSTEP_NONE, "Implicit": SUBSTEP_IMPLICIT}[str(st).strip('"')]
    return c
