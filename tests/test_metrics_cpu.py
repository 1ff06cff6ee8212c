"""CPU: the per-step JSON metrics lines (erf_b200.metrics.run_logged) over a
stand-in dycore that reports scripted diagnostics: the line layout, the
logging interval, the mass drift against the first line, and a device
status other than OK ending the run with an error."""
import io
import json
import types

import pytest

from erf_b200 import metrics


class FakeDycore:
    def __init__(self, masses, statuses=None):
        self.cfg = types.SimpleNamespace(nx=4, ny=3, nz=2, dt=0.5)
        self.masses = list(masses)
        self.statuses = list(statuses or [])
        self.loaded = None
        self.advanced = []

    def load_state(self, cons, u, v, w):
        self.loaded = (cons, u, v, w)

    def advance_resident(self, n):
        self.advanced.append(n)

    def status(self):
        return self.statuses.pop(0) if self.statuses else 0

    def diagnostics(self):
        m = self.masses.pop(0)
        return {"mass": m, "rhotheta": 300.0 * m, "max_w": 0.25}


def test_lines_interval_and_drift():
    dy = FakeDycore([100.0, 100.0, 100.0 * (1 + 1e-15), 100.0 * (1 - 2e-15)])
    buf = io.StringIO()
    recs = metrics.run_logged(dy, "c", "u", "v", "w", 5, every=2, out=buf, t0=10.0)
    lines = [json.loads(ln) for ln in buf.getvalue().splitlines()]
    assert dy.loaded == ("c", "u", "v", "w")
    assert dy.advanced == [2, 2, 1]
    assert [r["step"] for r in lines] == [0, 2, 4, 5]
    assert [r["time"] for r in lines] == [10.0, 11.0, 12.0, 12.5]
    assert "mass_drift" not in lines[0]
    assert lines[1]["mass_drift"] == 0.0
    assert lines[2]["mass_drift"] == pytest.approx(1e-15, rel=1e-3)
    assert lines[3]["mass_drift"] == pytest.approx(-2e-15, rel=1e-3)
    assert lines[0]["cell_steps_per_s"] is None
    assert all(r["cell_steps_per_s"] > 0 for r in lines[1:])
    assert all(r["rhotheta"] == 300.0 * r["mass"] and r["max_w"] == 0.25 for r in lines)
    assert recs == lines


def test_bad_status_stops_the_run():
    dy = FakeDycore([1.0, 1.0, 1.0], statuses=[0, 4])
    buf = io.StringIO()
    with pytest.raises(RuntimeError, match="status 4 after step 2"):
        metrics.run_logged(dy, 0, 0, 0, 0, 3, out=buf)
    assert len(buf.getvalue().splitlines()) == 2
