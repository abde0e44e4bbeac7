"""The learned preconditioner's CPU oracle (oracle/mpnn.py): its backward pass against finite differences, the
initial network reproducing block-Jacobi exactly, and the preconditioner being SPD whatever the weights."""
import numpy as np
import pytest

import mpnn
from drape_b200 import scenes as S


def sheet_system(oracle_mod, nx=8, steps=3):
    """A small sheet resting on the sphere: the Newton system of its next substep, from the FP64 oracle."""
    scene = S.sheet_on_sphere(n=nx, cg_tolerance=1e-2, max_cg=50)
    scene.garments[0].initial_positions[:, 1] -= 0.147
    o = oracle_mod.OracleSolver()
    o.build(scene)
    for _ in range(steps):
        o.step(1 / 60, 1, 2)
    return o.capture_system(1 / 60)


def graph_of(sysm, pinned=None):
    n = len(sysm["diag_slot"])
    pin = np.zeros(n, bool) if pinned is None else pinned
    return mpnn.Graph(sysm["row_start"], sysm["col_index"], sysm["blocks"], pin, sysm["active"])


@pytest.fixture(scope="module")
def sysm(oracle_mod):
    return sheet_system(oracle_mod)


def _random_params(seed):
    rng = np.random.default_rng(seed)
    flat = mpnn.init_params(seed)
    P = mpnn.unpack(flat)
    P["W_o"] = rng.standard_normal(P["W_o"].shape) * 0.02
    P["b_o"] = rng.standard_normal(P["b_o"].shape) * 0.02
    for name in P:
        if name.startswith("b_") and name != "b_o":
            P[name] = rng.standard_normal(P[name].shape) * 0.05
    return mpnn.pack(P)


def test_param_layout_round_trips():
    flat = mpnn.init_params(3)
    assert len(flat) == mpnn.param_count() == 71312
    assert np.array_equal(mpnn.pack(mpnn.unpack(flat)), flat)


def test_backward_matches_finite_differences(sysm):
    g = graph_of(sysm)
    flat = _random_params(1)
    r = -sysm["grad"]
    value, grad = mpnn.loss_and_grad(g, flat, r, emulate=False)
    assert value > 0
    rng = np.random.default_rng(7)
    for _ in range(4):
        d = rng.standard_normal(flat.shape)
        d /= np.linalg.norm(d)
        h = 1e-6
        lp = mpnn.loss(g, mpnn.forward(g, flat + h * d, emulate=False)[0], r)[0]
        lm = mpnn.loss(g, mpnn.forward(g, flat - h * d, emulate=False)[0], r)[0]
        fd = (lp - lm) / (2 * h)
        an = float(grad @ d)
        assert abs(fd - an) <= 1e-5 * max(abs(fd), 1e-3 * np.linalg.norm(grad)), (fd, an)


def test_per_block_gradients_match_finite_differences(sysm):
    """Individual weight groups, including the encoders and the first layer, which the random directions above mix."""
    g = graph_of(sysm)
    flat = _random_params(2)
    r = -sysm["grad"]
    _, grad = mpnn.loss_and_grad(g, flat, r, emulate=False)
    offsets, k = {}, 0
    for name, shape in mpnn.param_shapes():
        offsets[name] = (k, int(np.prod(shape)))
        k += int(np.prod(shape))
    rng = np.random.default_rng(11)
    for name in ("W_ne", "b_ee", "W_m0", "W_u0", "W_m3", "b_u2", "W_o"):
        k0, size = offsets[name]
        d = np.zeros_like(flat)
        d[k0:k0 + size] = rng.standard_normal(size)
        d /= np.linalg.norm(d)
        h = 1e-6
        lp = mpnn.loss(g, mpnn.forward(g, flat + h * d, emulate=False)[0], r)[0]
        lm = mpnn.loss(g, mpnn.forward(g, flat - h * d, emulate=False)[0], r)[0]
        fd = (lp - lm) / (2 * h)
        an = float(grad @ d)
        assert abs(fd - an) <= 1e-5 * max(abs(fd), 1e-3 * np.linalg.norm(grad[k0:k0 + size])), (name, fd, an)


def test_initial_network_is_block_jacobi(sysm):
    g = graph_of(sysm)
    G, _, _ = mpnn.forward(g, mpnn.init_params(0))
    r = np.random.default_rng(3).standard_normal((g.n, 3))
    z = mpnn.precondition(g, G, r)
    for i in range(g.n):
        Aii = g.A[g.rs[i] + np.searchsorted(g.ci[g.rs[i]:g.rs[i + 1]], i)]
        assert np.allclose(z[i], np.linalg.solve(Aii, r[i]), rtol=1e-9, atol=1e-12)


def test_preconditioner_is_spd_for_any_weights(sysm):
    pinned = np.zeros(len(sysm["diag_slot"]), bool)
    pinned[:5] = True
    g = graph_of(sysm, pinned)
    flat = _random_params(5) * 3.0
    G, _, _ = mpnn.forward(g, flat)
    n = g.n
    free = np.repeat(~pinned, 3)
    M = np.zeros((3 * n, 3 * n))
    for k in range(3 * n):
        x = np.zeros((n, 3))
        x.reshape(-1)[k] = 1.0
        M[:, k] = mpnn.precondition(g, G, x).reshape(-1)
    assert np.allclose(M, M.T, atol=1e-9 * np.abs(M).max())
    assert np.all(M[~free] == 0) and np.all(M[:, ~free] == 0)
    # M = L L^T with L (restricted to the free rows and columns) lower-triangular with a positive diagonal, hence
    # nonsingular: M is positive definite on the free unknowns.
    L = np.zeros((3 * n, 3 * n))
    Ls = mpnn.factor(g, G)
    for s in np.where(g.lower)[0]:
        i, j = g.row[s], g.ci[s]
        L[3 * i:3 * i + 3, 3 * j:3 * j + 3] = Ls[s]
    Lf = L[np.ix_(free, free)]
    assert np.allclose(Lf, np.tril(Lf))
    assert np.all(np.diag(Lf) > 0)
    assert np.allclose(Lf @ Lf.T, M[np.ix_(free, free)], rtol=1e-9, atol=1e-12 * np.abs(M).max())


def test_adam_reduces_the_loss(sysm):
    g = graph_of(sysm)
    flat = mpnn.init_params(0)
    rng = np.random.default_rng(0)
    rs = [-sysm["grad"]] + [rng.standard_normal((g.n, 3)) for _ in range(3)]
    first = np.mean([mpnn.loss(g, mpnn.forward(g, flat)[0], r)[0] for r in rs])
    state = {}
    for it in range(100):
        grad = np.mean([mpnn.loss_and_grad(g, flat, r)[1] for r in rs], axis=0)
        flat = mpnn.adam(flat, grad, state, lr=1e-3)
    last = np.mean([mpnn.loss(g, mpnn.forward(g, flat)[0], r)[0] for r in rs])
    assert last < 0.6 * first, (first, last)


def test_kaporin_gradient_matches_finite_differences(sysm):
    g = graph_of(sysm)
    flat = _random_params(4)
    w = np.random.default_rng(5).standard_normal((g.n, 3))
    value, grad = mpnn.kaporin_and_grad(g, flat, w, emulate=False)
    rng = np.random.default_rng(9)
    for _ in range(4):
        d = rng.standard_normal(flat.shape)
        d /= np.linalg.norm(d)
        h = 1e-6
        fp = mpnn.kaporin(g, *mpnn.forward(g, flat + h * d, emulate=False)[:2], w)[0]
        fm = mpnn.kaporin(g, *mpnn.forward(g, flat - h * d, emulate=False)[:2], w)[0]
        fd = (fp - fm) / (2 * h)
        an = float(grad @ d)
        assert abs(fd - an) <= 1e-5 * max(abs(fd), 1e-3 * np.linalg.norm(grad)), (fd, an)


def test_kaporin_at_identity_is_log_of_normalised_trace(sysm):
    """G = I: the objective is log(w^T Ahat w / N), about log(1) = 0 since Ahat has identity diagonal blocks."""
    g = graph_of(sysm)
    G, o, _ = mpnn.forward(g, mpnn.init_params(0), emulate=False)
    w = np.random.default_rng(1).standard_normal((g.n, 3))
    value, parts = mpnn.kaporin(g, G, o, w)
    ref = float((w.reshape(-1) @ (mpnn.apply_full(g, g.Ahat, w).reshape(-1)))) / mpnn.live_unknowns(g)
    assert abs(value - np.log(ref)) < 1e-12
