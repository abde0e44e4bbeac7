"""The learned preconditioner's device kernels (tcgen05 forward and backward, Adam) against the CPU oracle
(oracle/mpnn.py), through the C ABI.

Bars: BF16 operands are rounded at the same points on both sides, but FP32 accumulation order differs, so a value
near a BF16 rounding boundary can round differently; forward outputs agree to 1e-2 relative (norm), gradients to
3e-2 relative (norm) with a per-group cosine above 0.99. Identity-initialised networks reproduce block-Jacobi to FP32
accuracy.
"""
import numpy as np
import pytest

import mpnn
from drape_b200 import learned
from test_mpnn_oracle import graph_of, sheet_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sysm(oracle_mod):
    return sheet_system(oracle_mod, nx=12)


def _random_params(seed):
    rng = np.random.default_rng(seed)
    P = mpnn.unpack(mpnn.init_params(seed))
    P["W_o"] = rng.standard_normal(P["W_o"].shape) * 0.02
    P["b_o"] = rng.standard_normal(P["b_o"].shape) * 0.02
    for name in P:
        if name.startswith("b_") and name != "b_o":
            P[name] = rng.standard_normal(P[name].shape) * 0.05
    return mpnn.pack(P).astype(np.float32)


def _sample(net, sysm, pinned=None, residuals=None):
    n = len(sysm["diag_slot"])
    pin = np.zeros(n, np.uint8) if pinned is None else pinned.astype(np.uint8)
    res = [-sysm["grad"]] if residuals is None else residuals
    return net.add_sample(sysm["row_start"], sysm["col_index"], sysm["blocks"].astype(np.float32), pin,
                          sysm["active"], np.stack(res).astype(np.float32))


def test_param_count_matches_oracle(gpu):
    assert learned.param_count() == mpnn.param_count()
    assert [s for _, s in learned.param_shapes()] == [s for _, s in mpnn.param_shapes()]


def test_identity_network_is_block_jacobi(gpu, sysm):
    net = learned.LearnedPreconditioner(0)
    sid = _sample(net, sysm)
    r = np.random.default_rng(0).standard_normal((len(sysm["diag_slot"]), 3)).astype(np.float32)
    z = net.apply(sid, r)
    g = graph_of(sysm)
    for i in range(g.n):
        Aii = g.A[g.rs[i] + np.searchsorted(g.ci[g.rs[i]:g.rs[i + 1]], i)]
        ref = np.linalg.solve(Aii, r[i].astype(np.float64))
        assert np.allclose(z[i], ref, rtol=1e-4, atol=1e-6 * np.abs(ref).max())


@pytest.mark.parametrize("pinned_rows", [0, 7])
def test_forward_matches_oracle(gpu, sysm, pinned_rows):
    flat = _random_params(1)
    n = len(sysm["diag_slot"])
    pinned = np.zeros(n, bool)
    pinned[:pinned_rows] = True
    net = learned.LearnedPreconditioner(0, flat)
    sid = _sample(net, sysm, pinned)
    G, L = net.forward(sid)
    g = graph_of(sysm, pinned)
    Gr, _, _ = mpnn.forward(g, flat.astype(np.float64))
    Lr = mpnn.factor(g, Gr)
    assert np.linalg.norm(G - Gr) <= 1e-2 * np.linalg.norm(Gr)
    assert np.linalg.norm(L - Lr) <= 1e-2 * np.linalg.norm(Lr)
    assert np.all(G[~g.lower] == 0) and np.all(L[~g.lower] == 0)


@pytest.mark.parametrize("pinned_rows", [0, 7])
def test_inference_path_matches_oracle_and_training_forward(gpu, sysm, pinned_rows):
    """The solver's inference path (slot and node GEMMs on contiguous tiles, message sums and the output layer as
    row gathers) computes the same L as the training forward and as the oracle, to the forward's bar."""
    flat = _random_params(1)
    n = len(sysm["diag_slot"])
    pinned = np.zeros(n, bool)
    pinned[:pinned_rows] = True
    net = learned.LearnedPreconditioner(0, flat)
    sid = _sample(net, sysm, pinned)
    L_inf = net.forward_inference(sid)
    _, L_train = net.forward(sid)
    g = graph_of(sysm, pinned)
    Gr, _, _ = mpnn.forward(g, flat.astype(np.float64))
    Lr = mpnn.factor(g, Gr)
    assert np.linalg.norm(L_inf - Lr) <= 1e-2 * np.linalg.norm(Lr)
    assert np.linalg.norm(L_inf - L_train) <= 1e-2 * np.linalg.norm(L_train)
    assert np.all(L_inf[~g.lower] == 0)
    assert np.array_equal(net.forward_inference(sid), L_inf)  # deterministic


def _groups_close(grad, grad_ref):
    assert np.linalg.norm(grad - grad_ref) <= 3e-2 * np.linalg.norm(grad_ref)
    k = 0
    for name, shape in mpnn.param_shapes():
        size = int(np.prod(shape))
        a, b = grad[k:k + size].astype(np.float64), grad_ref[k:k + size]
        k += size
        if np.linalg.norm(b) > 1e-6 * np.linalg.norm(grad_ref):
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
            assert cos > 0.99, (name, cos)


def test_kaporin_objective_and_gradient_match_oracle(gpu, sysm):
    flat = _random_params(4)
    net = learned.LearnedPreconditioner(0, flat)
    w = np.random.default_rng(5).standard_normal((len(sysm["diag_slot"]), 3))
    sid = _sample(net, sysm, residuals=[w])
    value, grad = net.loss_grad(sid, 0)
    g = graph_of(sysm)
    ref, grad_ref = mpnn.kaporin_and_grad(g, flat.astype(np.float64), w.astype(np.float32), emulate=True)
    assert abs(value - ref) <= 1e-3 * max(1.0, abs(ref))
    _groups_close(grad, grad_ref)


def test_loss_and_gradient_match_oracle(gpu, sysm):
    flat = _random_params(2)
    net = learned.LearnedPreconditioner(0, flat)
    net.set_objective(learned.DEFECT)
    sid = _sample(net, sysm)
    loss, grad = net.loss_grad(sid, 0)
    g = graph_of(sysm)
    loss_ref, grad_ref = mpnn.loss_and_grad(g, flat.astype(np.float64), -sysm["grad"], emulate=True)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    _groups_close(grad, grad_ref)


def test_gradient_is_deterministic(gpu, sysm):
    net = learned.LearnedPreconditioner(0, _random_params(3))
    sid = _sample(net, sysm)
    l1, g1 = net.loss_grad(sid, 0)
    l2, g2 = net.loss_grad(sid, 0)
    assert l1 == l2 and np.array_equal(g1, g2)


def test_training_on_device_reduces_the_defect(gpu, sysm):
    rng = np.random.default_rng(0)
    n = len(sysm["diag_slot"])
    res = [-sysm["grad"]] + [rng.standard_normal((n, 3)) for _ in range(3)]
    net = learned.LearnedPreconditioner(0)
    net.set_objective(learned.DEFECT)
    sid = _sample(net, sysm, residuals=res)
    before = np.mean([net.loss_grad(sid, k)[0] for k in range(4)])
    losses = net.train(150, lr=1e-3, batch=4, seed=1)
    after = np.mean([net.loss_grad(sid, k)[0] for k in range(4)])
    assert np.isfinite(losses).all()
    assert after < 0.6 * before, (before, after)


def test_kaporin_training_lowers_the_condition_estimate(gpu, sysm):
    """Kaporin training moves toward the factorised sparse approximate inverse: the objective (the log of a condition
    estimate of the preconditioned operator) falls."""
    rng = np.random.default_rng(1)
    n = len(sysm["diag_slot"])
    net = learned.LearnedPreconditioner(0)
    sid = _sample(net, sysm, residuals=[rng.standard_normal((n, 3)) for _ in range(8)])
    before = np.mean([net.loss_grad(sid, k)[0] for k in range(8)])
    net.train(300, lr=1e-3, batch=4, seed=2)
    after = np.mean([net.loss_grad(sid, k)[0] for k in range(8)])
    assert after < before - 0.05, (before, after)
