"""Known-answer tests pinning the CPU oracle (test infrastructure)."""
import numpy as np
import pytest

import oracle
from erf_b200 import cases
from erf_b200 import config as C


def face_stencil(p):
    # the reference's interpolants are finite-volume reconstructions: cell
    # averages over the six unit cells [-3,-2] .. [2,3] around a face at x = 0
    P = p.integ()
    lo = np.arange(6) - 3.0
    return P(lo + 1.0) - P(lo)


@pytest.mark.parametrize("kind,degree", [(C.UPWIND_5TH, 4), (C.CENTERED_6TH, 5), (C.UPWIND_3RD, 2),
                                         (C.CENTERED_4TH, 3), (C.CENTERED_2ND, 1)])
@pytest.mark.parametrize("upw", [1.0, -1.0])
def test_linear_interpolants_exact_on_polynomials(kind, degree, upw):
    rng = np.random.default_rng(kind + degree)
    coef = rng.normal(size=degree + 1)
    p = np.polynomial.Polynomial(coef)
    val = oracle.interp(kind, face_stencil(p), upw, 1.0)
    assert val == pytest.approx(p(0.0), rel=1e-12, abs=1e-12)


def test_upwind5_is_one_order_short_on_quintics():
    p = np.polynomial.Polynomial([0, 0, 0, 0, 0, 1.0])
    s = face_stencil(p)
    assert abs(oracle.interp(C.UPWIND_5TH, s, 1.0, 1.0) - p(0.0)) > 1e-3


def test_weno5_reduces_to_fifth_order_on_smooth_data_and_is_upwind_biased():
    x = np.arange(6) - 3 + 0.5
    s = np.sin(0.01 * x)
    assert oracle.interp(C.WENO_5, s, 1.0) == pytest.approx(0.0, abs=1e-9)
    step = np.array([0, 0, 0, 1, 1, 1.0])
    assert oracle.interp(C.WENO_5, step, 1.0) < 0.05          # takes the upwind (left) side
    assert oracle.interp(C.WENO_5, step, -1.0) > 0.95         # takes the upwind (right) side
    assert oracle.interp(C.WENO_5, step, 0.0) == 0.5          # centred fallback when |u| <= tol


def test_flatau_saturation_polynomial_known_values():
    # esatw(273.16 K) = a0 = 6.11239921 hPa (Flatau et al. 1992, Table 4)
    es = 6.11239921
    assert oracle.qsatw(273.16, 1000.0) == pytest.approx(287.0 / 461.505 * es / (1000.0 - es), rel=1e-14)


def test_base_state_is_discretely_hydrostatic():
    case = cases.moist_bubble(nx=8, ny=8, nz=80)
    r0, p0, pi0, th0 = oracle.make_base_state(case.cfg, case)
    dz, g = case.cfg.dz, 9.81
    for k in range(1, case.cfg.nz + 1):
        lhs = p0[k + 1] - p0[k]
        rhs = -dz * 0.5 * (r0[k + 1] + r0[k]) * g
        assert lhs == pytest.approx(rhs, rel=1e-12)
    # dry density decreases upward
    assert np.all(np.diff(r0[1:-1]) < 0)


def test_oracle_conserves_mass_and_rhotheta_dry():
    case = cases.abl_dry(nx=12, ny=10, nz=12)
    base = oracle.make_base_state(case.cfg, case)
    cons, u, v, w = case.build_state(base[0])
    c2, u2, v2, w2 = oracle.advance(case.cfg, base, cons, u, v, w, 3)
    assert c2[0].sum() == pytest.approx(cons[0].sum(), rel=1e-14)
    assert c2[1].sum() == pytest.approx(cons[1].sum(), rel=1e-14)
    assert np.all(w2[0] == 0.0) and np.all(w2[-1] == 0.0)
    assert np.all(np.isfinite(c2))


def test_oracle_moist_kessler_keeps_water_nonnegative():
    case = cases.moist_bubble(nx=12, ny=12, nz=40)
    case.pert["bubble_rh"] = 3000.0
    base = oracle.make_base_state(case.cfg, case)
    cons, u, v, w = case.build_state(base[0])
    c2, *_ = oracle.advance(case.cfg, base, cons, u, v, w, 3)
    assert c2[0].sum() == pytest.approx(cons[0].sum(), rel=1e-14)
    assert np.all(c2[5:] >= 0.0)


def test_splitmix64_stream_is_fixed():
    r = cases.splitmix64_uniform(0, 3)
    # first outputs of SplitMix64 seeded with 0 (Steele et al. 2014), top 53 bits
    ref = np.array([0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F], dtype=np.uint64)
    assert np.array_equal(r, (ref >> np.uint64(11)).astype(np.float64) / 2.0 ** 53)


def test_oracle_deardorff_stationary_shear():
    """Deardorff known answer (cf. the reference's Deardorff_stationary test):
    in uniform shear u = S z with neutral theta, shear production
    2 K SmnSmn = Ck Delta sqrt(e) S^2 balances dissipation Ce e^1.5 / Delta at
    e = Ck/Ce (S Delta)^2, so interior cells keep that TKE."""
    from erf_b200 import config as C
    case = cases.abl_deardorff(nx=8, ny=8, nz=32)
    cfg = case.cfg
    cfg.use_coriolis = 0
    cfg.abl_geo_forcing[0] = cfg.abl_geo_forcing[1] = 0.0
    cfg.zlo_bc = cfg.zhi_bc = C.BC_SLIP_WALL
    case.theta_cc = np.full(cfg.nz, 300.0)
    case.pert = {}
    base = oracle.make_base_state(cfg, case)
    cons, u, v, w = case.build_state(base[0])
    S = 0.01
    z = (np.arange(cfg.nz) + 0.5) * cfg.dz
    u[:] = (S * z)[:, None, None]
    delta = (cfg.dx * cfg.dy * cfg.dz) ** (1.0 / 3.0)
    e_eq = cfg.Ck / cfg.Ce * (S * delta) ** 2
    cons[2] = cons[0] * e_eq
    c2, *_ = oracle.advance(cfg, base, cons, u, v, w, 1)
    e = c2[2] / c2[0]
    inner = slice(12, 20)
    assert np.max(np.abs(e[inner] / e_eq - 1.0)) < 1e-10
