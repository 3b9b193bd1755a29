"""Batched 3D immersed-boundary iterations (fi_ib_batch_*): members of different
sizes advanced by shared launches equal the same models advanced alone, bit for
bit, across calls of odd and even lengths, a member added mid-run, a member whose
state is written between calls and a member removed.  The no-FMA build: the shared
and the single-model kernels run the same source, but where the production build
contracts a product into a fused multiply-add is the compiler's choice per kernel."""
import numpy as np
import pytest

from conftest import load_fastice

pytestmark = pytest.mark.gpu

STATE = ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz", "eta")


def _sphere_psi(n, dx, c, r):
    ax = [(np.arange(n[d] + 3) - 1) * dx[d] for d in range(3)]
    Z, Y, X = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    return np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - r


def _member(fi, n, seed, dtype, rheology=None, library="strict"):
    ext = (1.0, 0.8, 0.9)
    dx = tuple(e / c for e, c in zip(ext, n))
    rng = np.random.default_rng(seed)
    c = (0.5 + 0.1 * rng.standard_normal(), 0.4, 0.45)
    grid = fi.UniformGrid(origin=(0.0, 0.0, 0.0), extent=ext, dims=n)
    trac = fi.TBC(0.0, 0.0, 0.0)
    bcs = {"x": (trac, fi.TBC(0.1, 0.0, 0.0)), "y": (fi.VBC(0.0, 0.05, 0.0), trac), "z": (fi.SBC(0.0, 0.0, 0.0), trac)}
    m = fi.IsothermalImmersedBoundaryFullStokesModel(grid=grid, boundary_conditions=bcs, gravity={"x": 0.1, "y": 0.0, "z": 1.0},
                                                     rheology=rheology or fi.LinearViscousRheology(1.0),
                                                     solver_params=fi.pt_params(grid), dtype=dtype, library=library)
    m.omega_from_psi("ns", -_sphere_psi(n, dx, (c[0], c[1], -0.3), 0.75))
    m.omega_from_psi("na", _sphere_psi(n, dx, c, 0.7))
    for name in STATE:
        shape = m.field_shape(name)
        v = 0.5 + rng.random(shape) if name == "eta" else 0.05 * rng.standard_normal(shape)
        m.set_field(name, v)
    m.set_field("eta_next", m.get_field("eta"))
    m.apply_bcs()
    return m


def _same(a, b):
    bad = []
    for name in STATE:
        x, y = a.get_field(name), b.get_field(name)
        if not np.array_equal(x, y):
            bad.append((name, int(np.sum(x != y))))
    return bad


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_shared_launches_equal_members_alone(dtype):
    fi = load_fastice()
    sizes = [(24, 20, 22), (31, 17, 25), (40, 24, 18)]
    glen = fi.ViscoplasticRegularisation(fi.PowerLawRheology(1.0, 3), 1.0)
    rheos = [None, glen, None]
    batch_m = [_member(fi, n, s, dtype, r) for s, (n, r) in enumerate(zip(sizes, rheos))]
    alone_m = [_member(fi, n, s, dtype, r) for s, (n, r) in enumerate(zip(sizes, rheos))]
    b = fi.BatchedIB3D(batch_m[:2])
    b.advance(3)   # the members' first two full iterations run alone, the third shared
    b.advance(4)
    b.add(batch_m[2])
    b.advance(5)   # odd: the graph pairs plus one single iteration
    # state written from outside: that member runs its first two iterations alone again
    v = batch_m[0].get_field("Vx")
    batch_m[0].set_field("Vx", v * 0.5)
    b.advance(6)
    b.remove(batch_m[1])
    b.advance(3)
    b.synchronize()
    # the same iterations alone: 12, the write, 9; 18; 14
    alone_m[0].advance(12)
    alone_m[0].set_field("Vx", alone_m[0].get_field("Vx") * 0.5)
    alone_m[0].advance(9)
    alone_m[1].advance(18)
    alone_m[2].advance(14)
    bad = {q: _same(batch_m[q], alone_m[q]) for q in range(3)}
    b.close()
    for m in batch_m + alone_m:
        m.close()
    assert not any(bad.values()), bad


def test_batch_rejects_non_immersed_members():
    fi = load_fastice()
    g = fi.UniformGrid(origin=(0, 0, 0), extent=(1, 1, 1), dims=(8, 8, 8))
    s = fi.SBC(0.0, 0.0, 0.0)
    m = fi.IsothermalFullStokesModel(grid=g, boundary_conditions={"x": (s, s), "y": (s, s), "z": (s, s)},
                                     gravity={"x": 0.0, "y": 0.0, "z": 1.0}, rheology=fi.LinearViscousRheology(1.0),
                                     solver_params=fi.pt_params(g))
    with pytest.raises(fi.FastIceError):
        fi.BatchedIB3D([m])  # noqa
    m.close()
