"""Known answers for the CPU oracle's restatement of the heat-diffusion model (no
GPU).  The reference module (src/Models/Diffusion/Heat/) has no runnable form and
no test, so its restatement is anchored on what one converged implicit step of
(T - T_o)/Δt + ∇·q = 0, q = -λ ∇T must satisfy on the discrete grid:

* insulated sides (Flux 0 everywhere): the total heat is conserved, and the
  cell-centred cosine mode cos(π(i - 1/2)/N) along x is an eigenvector of the
  discrete Laplacian with eigenvalue -(4/Δx²) sin²(π/2N), so the step scales it by
  exactly 1 / (1 + Δt λ (4/Δx²) sin²(π/2N));
* two Value sides and insulated others: the linear profile between the two
  values is steady.
"""
import math

import numpy as np

from conftest import load_fastice, load_oracle

FLUX, VALUE = 1, 0


def _oracle(n, ext, kinds, values, lam, dt):
    fi, O = load_fastice(), load_oracle()
    from fastice_b200 import heat
    grid = fi.UniformGrid(origin=(0.0, 0.0, 0.0), extent=ext, dims=n)
    ip = heat.heat_iter_params(grid, lam, dt)["Δτ"]
    return O.OracleHeat(n, ext, kinds, values, lam, ip["T"], ip["q"], dtype="f64")


def _converge(o, dt, shape, tol=1e-13, chunk=200, max_iter=40000):
    prev = o.interior("T")
    it = 0
    while it < max_iter:
        o.advance(chunk, dt)
        it += chunk
        cur = o.interior("T")
        if np.max(np.abs(cur - prev)) < tol * max(1.0, np.max(np.abs(cur))):
            return it
        prev = cur
    return it


def test_insulated_cosine_mode_decays_by_the_exact_discrete_factor():
    n, ext, lam, dt = (24, 4, 4), (1.0, 0.25, 0.25), 0.7, 0.05
    o = _oracle(n, ext, [[FLUX, FLUX]] * 3, [[0.0, 0.0]] * 3, lam, dt)
    N, dx = n[0], ext[0] / n[0]
    mode = np.cos(math.pi * (np.arange(N) + 0.5) / N)
    T0 = np.broadcast_to(mode[None, None, :], (n[2], n[1], n[0])).copy()
    o.set_interior("T", T0)
    o.set_interior("T_o", T0)
    for q in ("qx", "qy", "qz"):
        o.set_interior(q, np.zeros(o.interior(q).shape))
    o.apply_bcs()
    it = _converge(o, dt, T0.shape)
    factor = 1.0 / (1.0 + dt * lam * 4.0 / dx ** 2 * math.sin(math.pi / (2 * N)) ** 2)
    T = o.interior("T")
    assert it < 40000
    np.testing.assert_allclose(T, factor * T0, rtol=0, atol=1e-10)
    # insulated: the total heat of the step equals that of T_o (zero for this mode)
    assert abs(T.sum()) < 1e-9


def test_insulated_step_conserves_total_heat():
    n, ext, lam, dt = (10, 12, 8), (1.0, 1.2, 0.8), 1.3, 0.2
    o = _oracle(n, ext, [[FLUX, FLUX]] * 3, [[0.0, 0.0]] * 3, lam, dt)
    rng = np.random.default_rng(3)
    To = 1.0 + rng.random((n[2], n[1], n[0]))
    o.set_interior("T", To)
    o.set_interior("T_o", To)
    o.apply_bcs()
    _converge(o, dt, To.shape)
    T = o.interior("T")
    assert abs(T.sum() - To.sum()) < 1e-9 * To.sum()
    assert np.std(T) < np.std(To)  # diffusion smooths


def test_linear_profile_between_two_value_sides_is_steady():
    n, ext, lam, dt = (6, 16, 5), (0.6, 1.0, 0.5), 1.0, 1.0
    kinds = [[FLUX, FLUX], [VALUE, VALUE], [FLUX, FLUX]]
    vals = [[0.0, 0.0], [-0.1, 0.3], [0.0, 0.0]]
    o = _oracle(n, ext, kinds, vals, lam, dt)
    yc = (np.arange(n[1]) + 0.5) / n[1]
    exact = np.broadcast_to((-0.1 + 0.4 * yc)[None, :, None], (n[2], n[1], n[0])).copy()
    o.set_interior("T", np.zeros_like(exact))
    o.set_interior("T_o", exact)
    o.apply_bcs()
    _converge(o, dt, exact.shape)
    np.testing.assert_allclose(o.interior("T"), exact, rtol=0, atol=1e-10)
