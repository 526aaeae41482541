"""Host logic of HydroRun (no GPU): the C-ABI call sequence of one hydro step,
recorded by a stand-in chunk, is the driver's (driver/hydro.cpp:53-108,
driver/timestep.cpp:37-109, driver/advection.cpp:29-105), and with
lagrangian=True one cb_lagrangian call takes the place of exactly the PdV
predictor, accelerate, PdV corrector and flux_calc calls, with the same dt
and halo depth."""
import pytest

from cloverleaf_b200.deck import benchmark_deck, nudged
from cloverleaf_b200.hydro import HydroRun


class RecordingChunk:
    """Records every call HydroRun makes; calc_dt returns a fixed dt."""

    def __init__(self, dt=0.004):
        self.calls = []
        self.dt = dt

    def __getattr__(self, name):
        def call(*args, **kwargs):
            self.calls.append((name, args, tuple(sorted(kwargs.items()))))
            if name == "calc_dt":
                return self.dt, 1, 2, 2, 0
            if name == "field_summary":
                return 1.0, 2.0, 3.0, 4.0, 5.0
            return None
        return call


def step_calls(fold, lagrangian, steps=2):
    dk = nudged(benchmark_deck(32, 10))
    c = RecordingChunk()
    r = HydroRun(c, dk, fold=fold, lagrangian=lagrangian)
    r.start()
    c.calls.clear()
    for _ in range(steps):
        r.hydro_step()
    return c.calls, r


@pytest.mark.parametrize("fold", [True, False])
def test_lagrangian_replaces_exactly_four_calls(fold):
    plain, r1 = step_calls(fold, False)
    fused, r2 = step_calls(fold, True)
    four = ("pdv", "accelerate", "pdv", "flux_calc")
    expect = []
    k = 0
    while k < len(plain):
        if tuple(name for name, _, _ in plain[k:k + 4]) == four:
            dt = plain[k][1][1]
            depth = plain[k + 1][1][1]
            # the predictor's own halo is depth 1; the other three take the driver's depth
            assert plain[k] == ("pdv", (True, dt), (("full", True), ("halo_depth", 1)))
            assert plain[k + 2] == ("pdv", (False, dt), (("halo_depth", depth),))
            assert plain[k + 3][1] == (dt, depth)
            expect.append(("lagrangian", (dt, depth), ()))
            k += 4
        else:
            expect.append(plain[k])
            k += 1
    assert fused == expect
    assert sum(1 for c in fused if c[0] == "lagrangian") == 2
    assert (r1.step, r1.time, r1.dt_trace) == (r2.step, r2.time, r2.dt_trace)


def test_step_sequence_order():
    calls, _ = step_calls(True, False, steps=1)
    names = [c[0] for c in calls if c[0] != "update_halo"]
    assert names == ["ideal_gas", "viscosity", "calc_dt", "pdv", "accelerate", "pdv", "flux_calc", "advec_cell",
                     "advec_mom", "advec_cell", "advec_mom", "reset_field"]
    # x sweep first on the first step, then y first
    adv = [c for c in calls if c[0] == "advec_cell"]
    assert [a[1][:2] for a in adv] == [(1, 1), (2, 2)]
