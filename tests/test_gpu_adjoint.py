"""The adjoint and tangent-linear runs on the GPU.

The map: initial interior density0, energy0 and gamma -> final kinetic
energy, FP64 plain path, dt sequence of the forward run held fixed.  Checks:
* the forward run is the plain path (same kinetic energy as HydroRun);
* the tangent-linear run's values are the plain path's, bit for bit;
* dot-product test: <grad, x'> from the reverse sweep equals the
  tangent-linear derivative in direction x' (both exact up to rounding:
  1e-10 relative);
* central finite differences (h = 1e-6) at seeded cells and for gamma;
* the checkpoint interval changes nothing but memory and recomputation;
* the torch.autograd.Function harness returns the same gradient.
"""
import numpy as np
import pytest

from cloverleaf_b200 import Adjoint, Chunk, HydroRun, benchmark_deck, kinetic_energy_function, nudged

pytestmark = pytest.mark.gpu


def problem(nx, ny, steps, seed=0, scale=0.05, gamma=1.4):
    """The benchmark layout with a seeded +-scale uniform perturbation of the
    initial density and energy of every cell."""
    dk = nudged(benchmark_deck(nx, end_step=steps, ny=ny))
    adj = Adjoint(dk)
    rng = np.random.default_rng(seed)
    rho = adj.read_field("density0")[2:-2, 2:-2] * (1.0 + rng.uniform(-scale, scale, (ny, nx)))
    e = adj.read_field("energy0")[2:-2, 2:-2] * (1.0 + rng.uniform(-scale, scale, (ny, nx)))
    adj.set_initial(rho, e, gamma)
    return adj, rho, e


def test_forward_is_the_plain_path():
    dk = nudged(benchmark_deck(40, end_step=15, ny=32))
    with Adjoint(dk) as adj:
        ke = adj.forward(15)
        c = Chunk(40, 32)
        r = HydroRun(c, dk)
        r.run()
        assert ke == r.summaries[-1].ke
        assert list(adj.dt()) == r.dt_trace
        for f in ("density0", "energy0", "xvel0", "yvel0"):
            assert np.array_equal(adj.read_field(f), c.read(f)), f
        c.close()


@pytest.mark.parametrize("steps", [1, 2, 7])
def test_tangent_values_are_the_plain_path(steps):
    adj, rho, e = problem(24, 16, steps, seed=1)
    adj.forward(steps)
    # (pressure is left out: the forward run's closing field_summary rewrites it)
    final = {f: adj.read_field(f) for f in ("density0", "energy0", "xvel0", "yvel0", "viscosity")}
    rng = np.random.default_rng(2)
    adj.tangent(rng.standard_normal(rho.shape), rng.standard_normal(e.shape), 0.3)
    for f, a in final.items():
        b = adj.read_tangent(f, 0)
        assert np.array_equal(a[2:-2, 2:-2], b[2:-2, 2:-2]), (f, np.abs(a - b).max())
    adj.close()


@pytest.mark.parametrize("nx,ny,steps", [(16, 12, 1), (24, 16, 2), (24, 16, 5), (40, 32, 20)])
def test_dot_product_adjoint_vs_tangent(nx, ny, steps):
    adj, rho, e = problem(nx, ny, steps, seed=3)
    adj.forward(steps)
    gr, ge, gg = adj.gradient()
    rng = np.random.default_rng(4)
    for trial in range(3):
        dr, de, dg = rng.standard_normal(rho.shape), rng.standard_normal(e.shape), float(rng.standard_normal())
        if trial == 1:
            de[:] = 0.0
            dg = 0.0
        if trial == 2:
            dr[:] = 0.0
            de[:] = 0.0
        _, dke = adj.tangent(dr, de, dg)
        lhs = float((gr * dr).sum() + (ge * de).sum() + gg * dg)
        scale = float(np.abs(gr * dr).sum() + np.abs(ge * de).sum() + abs(gg * dg))
        assert abs(lhs - dke) <= 1e-10 * scale, (steps, trial, lhs, dke, scale)
    adj.close()


def test_central_differences():
    nx, ny, steps = 32, 24, 20
    adj, rho, e = problem(nx, ny, steps, seed=5)
    ke0 = adj.forward(steps)
    dts = adj.dt()
    gr, ge, gg = adj.gradient()
    rng = np.random.default_rng(6)
    cells = [(int(rng.integers(ny)), int(rng.integers(nx))) for _ in range(8)]
    h = 1e-6
    worst = 0.0
    for (j, i) in cells:
        for which, g in (("rho", gr), ("e", ge)):
            vals = []
            for s in (1.0, -1.0):
                r2, e2 = rho.copy(), e.copy()
                (r2 if which == "rho" else e2)[j, i] += s * h
                adj.set_initial(r2, e2, 1.4)
                vals.append(adj.forward(steps, dts))
            fd = (vals[0] - vals[1]) / (2 * h)
            err = abs(fd - g[j, i]) / max(abs(g).max(), 1e-300)
            worst = max(worst, err)
            assert err <= 1e-5, (which, i, j, fd, g[j, i])
    # gamma
    vals = []
    for s in (1.0, -1.0):
        adj.set_initial(rho, e, 1.4 + s * h)
        vals.append(adj.forward(steps, dts))
    fd = (vals[0] - vals[1]) / (2 * h)
    assert abs(fd - gg) <= 1e-5 * abs(gg), (fd, gg)
    assert ke0 > 0.0
    adj.close()


def test_checkpoint_interval_changes_only_cost():
    nx, ny, steps = 24, 20, 13
    out = []
    for k in (1, 3, 0, 13):
        adj, rho, e = problem(nx, ny, steps, seed=7)
        adj.set_checkpoint_interval(k)
        adj.forward(steps)
        out.append(adj.gradient())
        st = adj.stats()
        kk = k if k else int(np.ceil(np.sqrt(steps)))
        assert st["checkpoint_interval"] == kk
        assert st["checkpoints"] == -(-steps // kk)
        assert st["recomputed_steps"] >= steps
        adj.close()
    for gr, ge, gg in out[1:]:
        assert np.allclose(gr, out[0][0], rtol=1e-11, atol=1e-13 * np.abs(out[0][0]).max())
        assert np.allclose(ge, out[0][1], rtol=1e-11, atol=1e-13 * np.abs(out[0][1]).max())
        assert abs(gg - out[0][2]) <= 1e-11 * abs(out[0][2])


def test_torch_autograd_harness():
    import torch
    KE = kinetic_energy_function()
    nx, ny, steps = 20, 16, 6
    adj, rho, e = problem(nx, ny, steps, seed=8)
    r = torch.tensor(rho, requires_grad=True)
    en = torch.tensor(e, requires_grad=True)
    g = torch.tensor(1.4, dtype=torch.float64, requires_grad=True)
    ke = KE.apply(r, en, g, adj, steps)
    (2.0 * ke).backward()
    gr, ge, gg = adj.gradient()
    assert np.allclose(r.grad.numpy(), 2.0 * gr, rtol=1e-12, atol=0.0)
    assert np.allclose(en.grad.numpy(), 2.0 * ge, rtol=1e-12, atol=0.0)
    assert abs(g.grad.item() - 2.0 * gg) <= 1e-12 * abs(gg)
    adj.close()


@pytest.mark.parametrize("name,steps", [("sodxy10x10", 75), ("sodbig200", 300)])
def test_dot_product_on_the_reference_sod_decks(name, steps):
    """The dot-product test on the reference's own Sod decks
    (InputDecks/clover_sodxy.in to its end at t = 3, 75 steps;
    clover_sodbig.in, 200^2, over 300 steps), from the decks' own initial
    state: the reverse sweep's gradient against the tangent-linear run, to
    1e-10 relative, through the shocks and their reflections."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from cloverleaf_b200 import deck as D
    from golden_util import deck_text
    dk = D.parse_deck(deck_text(name))
    dk.end_step = steps
    adj = Adjoint(dk)
    ke = adj.forward(steps)
    gr, ge, gg = adj.gradient()
    rng = np.random.default_rng(11)
    dr, de, dg = rng.standard_normal(gr.shape), rng.standard_normal(ge.shape), float(rng.standard_normal())
    _, dke = adj.tangent(dr, de, dg)
    lhs = float((gr * dr).sum() + (ge * de).sum() + gg * dg)
    scale = float(np.abs(gr * dr).sum() + np.abs(ge * de).sum() + abs(gg * dg))
    assert scale > 0.0 and ke > 0.0
    assert abs(lhs - dke) <= 1e-10 * scale, (name, lhs, dke, scale)
    adj.close()
