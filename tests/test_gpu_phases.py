"""Per-phase parity: every C-ABI phase on a seeded random state against the
oracle's restatement of the same reference routine.  FP64 results must be
bit-identical (the FP64 kernels are built without FMA contraction), on every
element the reference writes, halos included.

Meshes: 37x29 (large enough for the library to fold halos into producers)
and 5x3 (too small to fold: every update_halo runs as its own pass, and the
reference's fill reads halo cells).
"""
import itertools

import pytest

from gpu_util import Pair

pytestmark = pytest.mark.gpu

MESHES = [(37, 29), (5, 3)]
ALL = list(range(15))
DT = 0.0123


@pytest.mark.parametrize("nx,ny", MESHES)
@pytest.mark.parametrize("predict", [0, 1])
@pytest.mark.parametrize("depth", [0, 1])
def test_ideal_gas(nx, ny, predict, depth):
    p = Pair(nx, ny, seed=1)
    p.g.ideal_gas(predict, depth)
    p.o.ideal_gas(predict)
    if depth and nx >= 8 and ny >= 8:
        p.o.update_halo([4 == f for f in range(15)], depth)
    p.assert_equal(ALL, "ideal_gas")


@pytest.mark.parametrize("nx,ny", MESHES)
@pytest.mark.parametrize("depth", [0, 1])
def test_viscosity(nx, ny, depth):
    p = Pair(nx, ny, seed=2)
    # make pressure gradients and compression that switch the limiter on
    p.g.viscosity(depth)
    p.o.viscosity()
    if depth and nx >= 8 and ny >= 8:
        p.o.update_halo([f == 5 for f in range(15)], depth)
    p.assert_equal(ALL, "viscosity")


@pytest.mark.parametrize("nx,ny", MESHES)
def test_calc_dt(nx, ny):
    p = Pair(nx, ny, seed=3)
    g = p.g.calc_dt()
    o = p.o.calc_dt()
    assert g == o


@pytest.mark.parametrize("nx,ny", MESHES)
@pytest.mark.parametrize("predict", [1, 0])
@pytest.mark.parametrize("depth", [0, 2])
def test_pdv_kernel(nx, ny, predict, depth):
    p = Pair(nx, ny, seed=4)
    p.g.pdv(predict, DT, full=False, halo_depth=depth)
    p.o.pdv_kernel(predict, DT)
    if depth and nx >= 8 and ny >= 8:
        p.o.update_halo([f in (1, 3) for f in range(15)], depth)
    p.assert_equal(ALL, "pdv")


@pytest.mark.parametrize("nx,ny", MESHES)
def test_pdv_full_predictor(nx, ny):
    """The model's PdV(true): kernel + ideal_gas(predict) + pressure halo + revert."""
    p = Pair(nx, ny, seed=5)
    p.g.pdv(True, DT, full=True, halo_depth=1)
    p.o.pdv(1, DT)
    p.assert_equal(ALL, "pdv full")


@pytest.mark.parametrize("nx,ny", MESHES)
def test_revert(nx, ny):
    p = Pair(nx, ny, seed=6)
    p.g.revert()
    p.o.revert()
    p.assert_equal(ALL, "revert")


@pytest.mark.parametrize("nx,ny", MESHES)
@pytest.mark.parametrize("depth", [0, 2])
def test_accelerate(nx, ny, depth):
    p = Pair(nx, ny, seed=7)
    p.g.accelerate(DT, depth)
    p.o.accelerate(DT)
    if depth and nx >= 8 and ny >= 8:
        p.o.update_halo([f in (8, 10) for f in range(15)], depth)
    p.assert_equal(ALL, "accelerate")


@pytest.mark.parametrize("nx,ny", MESHES)
@pytest.mark.parametrize("depth", [0, 2])
def test_flux_calc(nx, ny, depth):
    p = Pair(nx, ny, seed=8)
    p.g.flux_calc(DT, depth)
    p.o.flux_calc(DT)
    if depth and nx >= 8 and ny >= 8:
        p.o.update_halo([f in (11, 12) for f in range(15)], depth)
    p.assert_equal(ALL, "flux_calc")


@pytest.mark.parametrize("nx,ny", MESHES)
@pytest.mark.parametrize("sweep,direction", list(itertools.product([1, 2], [1, 2])))
@pytest.mark.parametrize("depth", [0, 2])
def test_advec_cell(nx, ny, sweep, direction, depth):
    p = Pair(nx, ny, seed=9 + 2 * sweep + direction)
    p.g.advec_cell(sweep, direction, depth)
    p.o.advec_cell(sweep, direction)
    if depth and nx >= 8 and ny >= 8:
        p.o.update_halo([f in (1, 3, 13 if direction == 1 else 14) for f in range(15)], depth)
    p.assert_equal(ALL, f"advec_cell sweep {sweep} dir {direction}")


@pytest.mark.parametrize("nx,ny", MESHES)
@pytest.mark.parametrize("sweep,direction", list(itertools.product([1, 2], [1, 2])))
@pytest.mark.parametrize("which", [1, 2, 3])
@pytest.mark.parametrize("depth", [0, 2])
def test_advec_mom(nx, ny, sweep, direction, which, depth):
    p = Pair(nx, ny, seed=20 + 4 * sweep + direction)
    p.g.advec_mom(which, sweep, direction, depth)
    if which == 3:
        p.o.advec_mom(1, sweep, direction)
        p.o.advec_mom(2, sweep, direction)
    else:
        if which == 2:
            # which_vel 2 reuses node flux/mass that the which_vel 1 call computes
            saved = p.cpu(8)
            p.o.advec_mom(1, sweep, direction)
            p.o.field(8)[:saved.shape[0], :saved.shape[1]] = saved
        p.o.advec_mom(which, sweep, direction)
    if depth and nx >= 8 and ny >= 8:
        p.o.update_halo([(f == 8 and which & 1) or (f == 10 and which & 2) for f in range(15)], depth)
    p.assert_equal(ALL, f"advec_mom vel {which} sweep {sweep} dir {direction}")


@pytest.mark.parametrize("nx,ny", MESHES)
@pytest.mark.parametrize("depth", [0, 1])
def test_reset_field(nx, ny, depth):
    p = Pair(nx, ny, seed=30)
    p.g.reset_field(depth)
    p.o.reset_field()
    if depth and nx >= 8 and ny >= 8:
        p.o.update_halo([f in (0, 2, 7, 9) for f in range(15)], depth)
    p.assert_equal(ALL, "reset_field")


@pytest.mark.parametrize("nx,ny", MESHES + [(8, 9), (2, 2)])
@pytest.mark.parametrize("depth", [1, 2])
def test_update_halo_every_field(nx, ny, depth):
    p = Pair(nx, ny, seed=31)
    p.g.update_halo(range(15), depth)
    p.o.update_halo([True] * 15, depth)
    p.assert_equal(ALL, f"update_halo depth {depth}")


@pytest.mark.parametrize("nx,ny", MESHES)
def test_field_summary(nx, ny):
    p = Pair(nx, ny, seed=32)
    g = p.g.field_summary()
    ex = p.o.field_summary(exact=True)  # also runs ideal_gas on the oracle
    for a, b in zip(g, ex):
        assert abs(a - b) <= 1e-14 * abs(b), (a, b)
    p.assert_equal([4, 6], "field_summary ideal_gas")


def test_generate_chunk_states():
    """Background + rectangle + circle + point states, velocities included."""
    from cloverleaf_b200 import deck as D
    nx, ny = 33, 21
    p = Pair(nx, ny, seed=33)
    st = [D.State(density=0.2, energy=1.0, xvel=0.1, yvel=-0.05),
          D.State(density=1.0, energy=2.5, xvel=0.3, yvel=0.2, geometry=D.GEOM_RECT, xmin=0.4, xmax=2.1, ymin=0.3, ymax=1.2),
          D.State(density=2.0, energy=3.0, xvel=-0.2, yvel=0.4, geometry=D.GEOM_CIRC, xmin=2.5, ymin=1.0, radius=0.6),
          D.State(density=5.0, energy=4.0, xvel=0.7, yvel=0.7, geometry=D.GEOM_POINT,
                  xmin=p.o.geom("vertexx")[10], ymin=p.o.geom("vertexy")[7])]
    p.g.build_field()
    p.o.build_field()
    p.g.initialise_chunk(0.0, 0.0, 3.7, 1.9)
    p.o.initialise_chunk(0.0, 0.0, 3.7, 1.9)
    p.g.generate_chunk(st)

    class S:  # the oracle wants deck-like state objects
        def __init__(self, s):
            self.__dict__.update(s.__dict__)

    class Dk:
        states = [S(s) for s in st]

    p.o.generate_chunk(Dk)
    p.assert_equal(ALL, "generate_chunk")
    for g in ("cellx", "celly", "celldx", "celldy", "vertexx", "vertexy", "vertexdx", "vertexdy"):
        a = p.g.read_geom(g)
        b = p.o.geom(g)[:a.size]
        assert (a == b).all(), g
