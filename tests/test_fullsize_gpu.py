"""Full-size GPU checks through properties that do not depend on the grid
size, over runs longer than the field-by-field oracle comparisons of
test_fullsize_parity_gpu.py: the three single-GPU workloads at their full
sizes, advanced on the device.

  * moist bubble 128x128x80 (plain FP64 and the FP32-bulk form): total mass
    is conserved (flux form, no flux through the walls), water stays
    non-negative;
  * dry ABL 64x64x64: total mass and total rho*theta are conserved (no heat
    flux through the walls);
  * terrain ABL 256x256x96: total sum(detJ * rho) is conserved;
and parity cases at prime sizes (partial tiles in every direction) and at
the smallest accepted grid (4 cells across).
"""
import numpy as np
import pytest

import oracle
from erf_b200 import cases
from erf_b200 import config as C
from erf_b200 import terrain as T
from helpers import compare_states

pytestmark = pytest.mark.gpu


def _advance_device(case, nsteps, precision=C.PREC_FP64, z_nd=None):
    import torch
    from erf_b200 import Dycore
    cfg = case.cfg.copy()
    cfg.precision = precision
    dy = Dycore(cfg)
    if z_nd is not None:
        dy.set_terrain(z_nd)
        base = dy.make_base_state_terrain(case)
    else:
        base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons, u, v, w = case.build_state(base[0])
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (cons, u, v, w)]
    torch.cuda.synchronize()   # the context's stream does not order after torch's default stream
    dy.advance(*dev, nsteps)
    torch.cuda.synchronize()
    st = dy.status()
    out = [t.cpu().numpy() for t in dev]
    dy.close()
    return cons, out, st


@pytest.mark.parametrize("precision,tol", [(C.PREC_FP64, 1e-13), (C.PREC_MIXED, 1e-11)])
def test_moist_bubble_full_size_conserves_mass(precision, tol):
    case = cases.moist_bubble()
    cons0, (cons, u, v, w), st = _advance_device(case, 5, precision)
    assert st == 0
    assert all(np.isfinite(a).all() for a in (cons, u, v, w))
    m0, m1 = cons0[0].sum(), cons[0].sum()
    assert abs(m1 - m0) <= tol * m0, (m0, m1)
    for n in range(C.RHOQ1_COMP, case.cfg.ncomp):
        assert cons[n].min() >= 0.0
    assert np.abs(w).max() > 0.01        # the bubble rises


def test_abl_dry_full_size_conserves_mass_and_rhotheta():
    case = cases.abl_dry()
    cons0, (cons, u, v, w), st = _advance_device(case, 5)
    assert st == 0
    for n in (0, 1):
        a0, a1 = cons0[n].sum(), cons[n].sum()
        assert abs(a1 - a0) <= 1e-13 * abs(a0), (n, a0, a1)


def test_terrain_full_size_conserves_detj_mass():
    case = T.abl_terrain()
    cons0, (cons, u, v, w), st = _advance_device(case, 3, z_nd=case.z_nd)
    assert st == 0
    z = case.z_nd
    dz_col = 0.25 * ((z[1:, :-1, :-1] - z[:-1, :-1, :-1]) + (z[1:, :-1, 1:] - z[:-1, :-1, 1:])
                     + (z[1:, 1:, :-1] - z[:-1, 1:, :-1]) + (z[1:, 1:, 1:] - z[:-1, 1:, 1:]))
    detJ = (dz_col / case.cfg.dz).ravel()
    r0 = cons0.reshape(case.cfg.ncomp, -1)[0]
    r1 = cons.reshape(case.cfg.ncomp, -1)[0]
    m0, m1 = (detJ * r0).sum(), (detJ * r1).sum()
    assert abs(m1 - m0) <= 1e-13 * m0, (m0, m1)
    assert all(np.isfinite(a).all() for a in (cons, u, v, w))


def test_prime_sizes_parity():
    """Partial tiles in x, y and the vertical kernels' column tiles."""
    from erf_b200 import Dycore
    case = cases.abl_deardorff(nx=37, ny=29, nz=23)
    dy = Dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    init = case.build_state(base[0])
    got = dy.advance_host(*init, 5)
    assert dy.status() == 0
    dy.close()
    ref = oracle.advance(case.cfg, base, *init, 5)
    errs = compare_states(got, ref)
    bad = {k: v for k, v in errs.items() if not v <= 1e-10}
    assert not bad, errs


@pytest.mark.parametrize("mk", [cases.abl_deardorff, cases.moist_bubble])
def test_minimum_sizes_parity(mk):
    """The smallest grid the library accepts (4 cells, so periodic stencils of
    +-3 wrap once) and odd sizes in y and z."""
    from erf_b200 import Dycore
    case = mk(nx=4, ny=5, nz=7)
    dy = Dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    init = case.build_state(base[0])
    got = dy.advance_host(*init, 3)
    assert dy.status() == 0
    dy.close()
    ref = oracle.advance(case.cfg, base, *init, 3)
    errs = compare_states(got, ref)
    bad = {k: v for k, v in errs.items() if not v <= 1e-10}
    assert not bad, errs


@pytest.mark.parametrize("precision,tol", [(C.PREC_FP64, 1e-12), (C.PREC_MIXED, 5e-11)])
def test_moist_bubble_long_integration(precision, tol):
    """500 steps (1000 s of model time, past the bubble's rise into the
    upper levels and the onset of rain): the state stays finite and valid,
    mass stays conserved and water non-negative.  The mixed form's FP32
    fluxes drift the total mass by about 1.5e-14 per step (7.8e-12 after
    500 steps)."""
    case = cases.moist_bubble()
    cons0, (cons, u, v, w), st = _advance_device(case, 500, precision)
    assert st == 0
    assert all(np.isfinite(a).all() for a in (cons, u, v, w))
    m0, m1 = cons0[0].sum(), cons[0].sum()
    assert abs(m1 - m0) <= tol * m0, (m0, m1)
    for n in range(C.RHOQ1_COMP, case.cfg.ncomp):
        assert cons[n].min() >= 0.0
    assert cons[C.RHOQ1_COMP + 1].max() > 0.0      # cloud water formed
