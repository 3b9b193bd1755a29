"""Domain split into slabs (fastice_b200.distributed): slabs of a domain periodic
along the split dimension, advanced with a halo exchange of V and η after every
iteration, reproduce the undivided model bit for bit (no-FMA build).  The ranks
of the ring are emulated in one process: the messages move by device copies,
through the same pack / unpack entry points a multi-GPU run uses."""
import numpy as np
import pytest

from conftest import load_fastice
from helpers import make_bcs

pytestmark = pytest.mark.gpu

STATE = ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz", "eta")
PER = ("periodic", ())
SLIP = ("slip", (0.0, 0.0, 0.0))
TRAC = ("traction", (0.0, 0.0, 0.0))


def _model(fi, n, extent, bcs, path, sp=None):
    grid = fi.UniformGrid(origin=(0.0, 0.0, 0.0), extent=extent, dims=n)
    rheo = fi.ViscoplasticRegularisation(fi.PowerLawRheology(1.0, 3), 50.0)
    # a subdomain iterates with the PT steps of the whole domain (sp)
    return fi.IsothermalFullStokesModel(grid=grid, boundary_conditions=make_bcs(fi, bcs, 3),
                                        gravity={"x": -0.17, "y": 0.05, "z": 0.98}, rheology=rheo,
                                        solver_params=sp or fi.pt_params(grid), dtype="f64", library="strict",
                                        path=path)


def _bits(a):
    return a.view(np.uint64)


@pytest.mark.parametrize("dim,ranks,overlap", [(0, 2, False), (0, 4, False), (1, 2, False), (0, 2, True),
                                                (1, 4, True), (0, 4, True)])
def test_split_run_matches_undivided(dim, ranks, overlap):
    # overlap: each slab iteration in two halves (the tiles of the split faces, then
    # the others on the model's second stream), the halo moved after the first half
    path = "fused"
    fi = load_fastice()
    from fastice_b200 import distributed as D
    # slabs wide enough along the split dimension for several tiles on each side of
    # the tile of position n (the partition of an overlapped iteration)
    nl = [80, 16, 14] if dim == 0 else [24, 40, 14]
    ng = list(nl)
    ng[dim] = nl[dim] * ranks
    ext = [1.0, 0.8, 0.3]
    ext_l = list(ext)
    ext_l[dim] = ext[dim] / ranks
    bcs = ((PER, PER), (PER, PER), (SLIP, TRAC))
    whole = _model(fi, tuple(ng), tuple(ext), bcs, path)
    sp = fi.pt_params(whole.grid)
    slabs = [_model(fi, tuple(nl), tuple(ext_l), bcs, path, sp) for _ in range(ranks)]
    rng = np.random.default_rng(5 + dim + ranks)
    for name in STATE:
        shape = whole.field_shape(name)
        vals = np.exp(0.3 * rng.standard_normal(shape)) if name == "eta" else 0.1 * rng.standard_normal(shape)
        whole.set_field(name, vals)
        loc = fi._lib.FIELD_LOC[name]
        for r, s in enumerate(slabs):
            s.set_field(name, np.ascontiguousarray(D.slab_of(vals, dim, r, ranks, loc[dim] == 1)))
        if name == "eta":
            whole.set_field("eta_next", vals)
            for r, s in enumerate(slabs):
                s.set_field("eta_next", np.ascontiguousarray(D.slab_of(vals, dim, r, ranks, False)))
    whole.apply_bcs()
    for s in slabs:
        s.apply_bcs()
    D.exchange_local(slabs, dim, "state")
    for _ in range(6):
        whole.advance(1)
        D.advance_local(slabs, dim, 1, overlap=overlap)
    bad = []
    for name in STATE:
        g = whole.get_field(name)
        loc = fi._lib.FIELD_LOC[name]
        for r, s in enumerate(slabs):
            a, b = s.get_field(name), np.ascontiguousarray(D.slab_of(g, dim, r, ranks, loc[dim] == 1))
            if not np.array_equal(_bits(a), _bits(b)):
                bad.append((name, r, int(np.sum(a != b))))
    for m in slabs + [whole]:
        m.close()
    assert not bad, bad


@pytest.mark.parametrize("dim,ranks,overlap", [(0, 2, False), (0, 3, True), (1, 3, False), (1, 2, True)])
def test_chain_split_of_a_bounded_domain_matches_undivided(dim, ranks, overlap):
    # a dimension with physical sides split into a chain of slabs: the outer sides keep
    # their boundary conditions (non-zero wall velocities and tractions), the inner
    # sides are halo sides whose ghosts come from the neighbours
    fi = load_fastice()
    from fastice_b200 import distributed as D
    nl = [80, 16, 14] if dim == 0 else [24, 40, 14]
    ng = list(nl)
    ng[dim] *= ranks
    ext = [1.0, 0.8, 0.3]
    ext_l = list(ext)
    ext_l[dim] /= ranks
    lo_bc = ("velocity", (0.1, -0.05, 0.02))
    hi_bc = ("traction", (0.05, 0.0, 0.0))
    sides = [(PER, PER), (PER, PER), (SLIP, TRAC)]
    sides[dim] = (lo_bc, hi_bc)
    whole = _model(fi, tuple(ng), tuple(ext), tuple(sides), "fused")
    sp = fi.pt_params(whole.grid)
    HALO = ("halo", ())
    slabs = []
    for r in range(ranks):
        sl = list(sides)
        sl[dim] = (lo_bc if r == 0 else HALO, hi_bc if r == ranks - 1 else HALO)
        slabs.append(_model(fi, tuple(nl), tuple(ext_l), tuple(sl), "fused", sp))
    rng = np.random.default_rng(17 + dim + ranks)
    for name in STATE:
        shape = whole.field_shape(name)
        vals = np.exp(0.3 * rng.standard_normal(shape)) if name == "eta" else 0.1 * rng.standard_normal(shape)
        whole.set_field(name, vals)
        loc = fi._lib.FIELD_LOC[name]
        for r, s_ in enumerate(slabs):
            s_.set_field(name, np.ascontiguousarray(D.slab_of(vals, dim, r, ranks, loc[dim] == 1)))
        if name == "eta":
            whole.set_field("eta_next", vals)
            for r, s_ in enumerate(slabs):
                s_.set_field("eta_next", np.ascontiguousarray(D.slab_of(vals, dim, r, ranks, False)))
    whole.apply_bcs()
    for s_ in slabs:
        s_.apply_bcs()
    D.exchange_local(slabs, dim, "state", periodic=False)
    for _ in range(6):
        whole.advance(1)
        D.advance_local(slabs, dim, 1, overlap=overlap, periodic=False)
    bad = []
    for name in STATE:
        g = whole.get_field(name)
        loc = fi._lib.FIELD_LOC[name]
        for r, s_ in enumerate(slabs):
            a, b = s_.get_field(name), np.ascontiguousarray(D.slab_of(g, dim, r, ranks, loc[dim] == 1))
            if not np.array_equal(_bits(a), _bits(b)):
                bad.append((name, r, int(np.sum(a != b))))
    for m in slabs + [whole]:
        m.close()
    assert not bad, bad


def test_split_solve_matches_undivided_solve():
    # the driver loop over a split domain (ranks emulated on one device): the same
    # checks, the norms reduced over the slabs, the same decision -- the iteration
    # count and the measure equal the undivided model's own solve (fi_model_solve),
    # and the final state equals it bit for bit (no-FMA build)
    fi = load_fastice()
    from fastice_b200 import distributed as D
    dim, ranks = 0, 2
    nl = [16, 12, 10]
    ng = list(nl)
    ng[dim] *= ranks
    ext = [1.0, 0.75, 0.25]
    ext_l = list(ext)
    ext_l[dim] /= ranks
    noslip = ("velocity", (0.0, 0.0, 0.0))
    bcs = ((PER, PER), (PER, PER), (noslip, TRAC))

    def model(n, e, sp=None):
        grid = fi.UniformGrid(origin=(0.0, 0.0, 0.0), extent=e, dims=n)
        return fi.IsothermalFullStokesModel(grid=grid, boundary_conditions=make_bcs(fi, bcs, 3),
                                            gravity={"x": -0.17, "y": 0.0, "z": 0.98},
                                            rheology=fi.LinearViscousRheology(1.0),
                                            solver_params=sp or fi.pt_params(grid), dtype="f64", library="strict",
                                            path="fused")
    whole = model(tuple(ng), tuple(ext))
    sp = fi.pt_params(whole.grid)
    slabs = [model(tuple(nl), tuple(ext_l), sp) for _ in range(ranks)]
    for m in slabs + [whole]:
        m.set_field("eta", 1.0)
        m.set_field("eta_next", 1.0)
        m.apply_bcs()
    D.exchange_local(slabs, dim, "state")
    kw = dict(max_iter=20000, ncheck=100, tol=1e-9, measure="rel_slab", rho_g_inf=1.0, length_z=0.25)
    ref = whole.solve(**kw)
    rep = D.solve_local(slabs, dim, overlap=True, **kw)
    assert ref["converged"] and rep["converged"], (ref, rep)
    assert rep["iterations"] == ref["iterations"]
    assert rep["measure"] == ref["measure"]
    bad = []
    for name in STATE:
        g = whole.get_field(name)
        loc = fi._lib.FIELD_LOC[name]
        for r, s in enumerate(slabs):
            a, b = s.get_field(name), np.ascontiguousarray(D.slab_of(g, dim, r, ranks, loc[dim] == 1))
            if not np.array_equal(_bits(a), _bits(b)):
                bad.append((name, r, int(np.sum(a != b))))
    for m in slabs + [whole]:
        m.close()
    assert not bad, bad


def test_halo_needs_a_periodic_split_dimension_and_the_fused_sweep():
    fi = load_fastice()
    m = _model(fi, (16, 12, 10), (1.0, 1.0, 0.3), ((SLIP, SLIP), (PER, PER), (SLIP, TRAC)), "auto")
    with pytest.raises(fi.FastIceError):
        m.halo_bytes(0, 0)
    with pytest.raises(fi.FastIceError):
        m.halo_bytes(2, 0)
    # toward the low side a slab sends two node layers of the fields Vertex-located along y
    assert m.halo_bytes(1, 0) > m.halo_bytes(1, 1) > 0
    m.close()
    # the reference-shaped path fills ghost stresses by the boundary copy: no split
    r = _model(fi, (16, 12, 10), (1.0, 1.0, 0.3), ((PER, PER), (PER, PER), (SLIP, TRAC)), "reference")
    with pytest.raises(fi.FastIceError):
        r.halo_bytes(0, 0)
    r.close()
