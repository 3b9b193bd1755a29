"""Host logic of the continuation driver (IsothermalFullStokesModel.solve_continuation)
on a stand-in model: stage order, parameters per attempt, restart of a diverged stage
from the state it started from, and what stops the driver.  No GPU."""
import numpy as np
import pytest

from helpers import load_fastice

fi = load_fastice()
from fastice_b200 import _lib as L  # noqa: E402
from fastice_b200.models import IsothermalFullStokesModel  # noqa: E402
from fastice_b200.writers import STATE_FIELDS_2D  # noqa: E402


class FakeModel:
    """Records set_params / solve calls; a solve adds 1 to every field, and diverges
    (after scribbling over the state) while its velocity step factor is below
    `needs` for that stage."""

    def __init__(self, needs):
        self.grid = fi.UniformGrid(origin=(0.0, 0.0), extent=(1.0, 1.0), dims=(4, 4))
        self.fields = {f: np.zeros((4, 4)) for f in STATE_FIELDS_2D + ("eta_next",)}
        self.needs, self.calls, self.stage = needs, [], -1
        self.params = None

    def get_field(self, f):
        return self.fields[f].copy()

    def set_field(self, f, a):
        self.fields[f] = np.array(a, dtype=float)

    def copy_field(self, dst, src):
        self.fields[dst] = self.fields[src].copy()

    def apply_bcs(self):
        pass

    def set_params(self, rheology, sp):
        if rheology != getattr(self, "_rheology", None):
            self.stage += 1
        self._rheology, self.params = rheology, sp

    def solve(self, tol, **kw):
        self.calls.append((self.stage, self.params["factor"], tol, kw.get("mode")))
        if self.params["factor"] < self.needs[self.stage]:
            for f in self.fields:
                self.fields[f][...] = np.nan
            raise L.FastIceError(L.FI_ERR_DIVERGED, "simulation failed: non-finite residual")
        for f in self.fields:
            self.fields[f] += 1.0
        return {"iterations": 10, "outer": 0, "seconds": 0.5, "measure": tol / 2, "converged": 1}


def stages(factors, tols=(1e-6, 1e-6, 1e-8)):
    out = []
    for q, (f, t) in enumerate(zip(factors, tols)):
        out.append((f"rheology{q}", (lambda a, f=f: {"factor": f * 2.0 ** a}), t))
    return out


def run(m, st, **kw):
    return IsothermalFullStokesModel.solve_continuation(m, st, **kw)


def test_stages_in_order_without_retries():
    m = FakeModel(needs=[1.0, 1.0, 1.0])
    r = run(m, stages([1.1, 1.1, 4.4]), mode="mixed", ncheck=5)
    assert [c[:3] for c in m.calls] == [(0, 1.1, 1e-6), (1, 1.1, 1e-6), (2, 4.4, 1e-8)]
    assert all(c[3] == "mixed" for c in m.calls)
    assert r["iterations"] == 30 and r["converged"] and len(r["stages"]) == 3
    assert np.all(m.fields["P"] == 3.0)


def test_diverged_stage_restarts_from_its_own_start_with_the_next_attempt():
    m = FakeModel(needs=[1.0, 1.0, 8.8])
    r = run(m, stages([1.1, 1.1, 4.4]), retries=2)
    assert [c[:2] for c in m.calls] == [(0, 1.1), (1, 1.1), (2, 4.4), (2, 8.8)]
    # the retried stage started from the state the first attempt started from
    assert np.all(m.fields["P"] == 3.0) and np.all(m.fields["eta_next"] == m.fields["eta"])
    assert [s.get("diverged", False) for s in r["stages"]] == [False, False, True, False]
    assert r["stages"][-1]["attempt"] == 1 and r["converged"]
    assert r["iterations"] == 30 and r["seconds"] >= 1.5


def test_divergence_past_the_retries_is_raised():
    m = FakeModel(needs=[1.0, 100.0, 1.0])
    with pytest.raises(L.FastIceError) as e:
        run(m, stages([1.1, 1.1, 4.4]), retries=1)
    assert e.value.status == L.FI_ERR_DIVERGED
    assert [c[:2] for c in m.calls] == [(0, 1.1), (1, 1.1), (1, 2.2)]


def test_no_retries_raises_on_the_first_divergence():
    m = FakeModel(needs=[1.0, 2.0, 1.0])
    with pytest.raises(L.FastIceError):
        run(m, stages([1.1, 1.1, 4.4]))
    assert len(m.calls) == 2


def test_plain_dict_parameters_still_accepted():
    m = FakeModel(needs=[1.0, 1.0])
    st = [("a", {"factor": 1.1}, 1e-6), ("b", {"factor": 4.4}, 1e-8)]
    r = run(m, st)
    assert [c[:2] for c in m.calls] == [(0, 1.1), (1, 4.4)] and r["converged"]


def test_glen_stage_parameters_double_the_velocity_factor_per_attempt():
    from fastice_b200 import scenarios
    g = fi.UniformGrid(origin=(0.0, 0.0, 0.0), extent=(1.0, 1.0, 1.0), dims=(32, 32, 32))
    st = scenarios.glacier_glen_stages(g, tol=1e-8)
    assert len(st) == 5 and st[-1][2] == 1e-8 and all(s[2] == 1e-6 for s in st[:-1])
    for (_, sp, _), f in zip(st, (1.1, 1.1, 1.1, 4.4, 4.4)):
        for a in range(3):
            ref = fi.pt_params(g, r=0.9, re_mech=5 * np.pi, vdtau_factor=f * 2.0 ** a)
            assert sp(a) == ref
