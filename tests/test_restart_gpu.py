"""Restart equivalence on the GPU: 2 steps, checkpoint, read back into a new
context, 2 more steps == 4 uninterrupted steps, bit for bit (flat and
terrain)."""
import numpy as np
import pytest

from erf_b200 import cases
from erf_b200 import terrain as T
from erf_b200.checkpoint import read_checkpoint

pytestmark = pytest.mark.gpu


def _ctx(case, base, z_nd=None):
    from erf_b200 import Dycore
    dy = Dycore(case.cfg)
    if z_nd is not None:
        dy.set_terrain(z_nd)
    dy.set_base_state(base)
    return dy


@pytest.mark.parametrize("kind", ["moist", "terrain"])
def test_restart_is_bit_identical(tmp_path, kind):
    from erf_b200 import Dycore
    if kind == "moist":
        case = cases.moist_bubble(nx=16, ny=12, nz=16)
        z = None
        dy = Dycore(case.cfg)
        base = dy.make_base_state(case)
    else:
        case = T.abl_terrain(nx=16, ny=12, nz=16, dx=25.0, dz0=20.0, h0=100.0, r0=100.0, amp=5.0)
        z = case.z_nd
        dy = Dycore(case.cfg)
        dy.set_terrain(z)
        base = dy.make_base_state_terrain(case)
    dy.close()
    init = case.build_state(base[0])
    a = _ctx(case, base, z)
    ref = a.advance_host(*init, 4)
    a.close()
    b = _ctx(case, base, z)
    mid = b.advance_host(*init, 2)
    b.close()
    path = str(tmp_path / "chk00002")
    b = _ctx(case, base, z)          # the context's own writer (its base state)
    b.write_checkpoint(path, *mid, z_nd=z, step=2, time=2 * case.cfg.dt)
    b.write_plotfile(str(tmp_path / "plt00002"), *mid, z_nd=z, time=2 * case.cfg.dt, step=2)
    b.close()
    r = read_checkpoint(case.cfg, path)
    assert r["step"] == 2
    c = _ctx(case, r["base"], r["z_nd"])
    got = c.advance_host(r["cons"], r["u"], r["v"], r["w"], 2)
    assert c.status() == 0
    c.close()
    for g, e in zip(got, ref):
        assert np.array_equal(g.reshape(e.shape), e)
