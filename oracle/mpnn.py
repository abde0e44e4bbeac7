"""CPU oracle (test infrastructure only) for the learned preconditioner: a message-passing network over the block-CSR
graph of a Newton system that emits a block lower-triangular factor L with M^-1 = L L^T.

No counterpart exists in the reference (its PCG is block-Jacobi only, cpu_solver.cpp:169-213); this module states the
network, its loss and its backward pass in numpy so that the device kernels (forward, backward, optimiser) can be
checked against it, and checks itself against finite differences.

Graph and scaling (FP32 system, FP64 here unless `emulate` asks for the device's rounding):
  C_i   = lower Cholesky factor of inv(A_ii) (identity when A_ii is not SPD; zero for a pinned row), so that
          C_i^T A_ii C_i = I;
  Ahat  = S^T A S with S = blockdiag(C_i): Ahat_ij = C_i^T A_ij C_j (zero where i or j is pinned);
  L     = S G, G block lower-triangular on A's pattern, so M^-1 = S G G^T S^T. G = I is block-Jacobi exactly.
Network (hidden 64, 4 layers; BF16 weights and stored activations, FP32 accumulation):
  h_i    = relu(W_ne f_i + b_ne)                      node features f_i (16)
  eps_s  = relu(W_ee e_s + b_ee)                      slot features e_s (16) for every slot s = (i, j)
  layer l: m_s = relu(W_m [h_j; eps_s] + b_m)         off-diagonal slots with i, j unpinned
           a_i = (1/8) sum_{s in row i} m_s
           h_i = h_i + relu(W_u [h_i; a_i] + b_u)
  o_s    = W_o [h_i; h_j; eps_s] + b_o (16)           lower slots (j <= i), i, j unpinned
  G_s    = reshape(o_s[0:9]) for j < i;  G_ii = [[e^o0, 0, 0], [o3, e^o1, 0], [o4, o5, e^o2]] (o0..o2 clamped to
           [-8, 8]).
Loss on a residual r: rhat = S^T r, a = G^T rhat, b = G a, e = Ahat b - rhat, loss = |e|^2 / |rhat|^2
(the preconditioned operator's defect on r: Ahat G G^T = S^T A M^-1 S^-T).
"""
import numpy as np

HIDDEN = 64
LAYERS = 4
NODE_FEATURES = 16
EDGE_FEATURES = 16
OUTPUTS = 16
AGG_SCALE = 1.0 / 8.0
DIAG_CLAMP = 8.0


def param_shapes():
    """Flat parameter layout shared with the device (row-major weights [out, in], then the bias)."""
    shapes = [("W_ne", (HIDDEN, NODE_FEATURES)), ("b_ne", (HIDDEN,)),
              ("W_ee", (HIDDEN, EDGE_FEATURES)), ("b_ee", (HIDDEN,))]
    for l in range(LAYERS):
        shapes += [(f"W_m{l}", (HIDDEN, 2 * HIDDEN)), (f"b_m{l}", (HIDDEN,)),
                   (f"W_u{l}", (HIDDEN, 2 * HIDDEN)), (f"b_u{l}", (HIDDEN,))]
    shapes += [("W_o", (OUTPUTS, 3 * HIDDEN)), ("b_o", (OUTPUTS,))]
    return shapes


def param_count():
    return sum(int(np.prod(s)) for _, s in param_shapes())


def unpack(flat):
    out, k = {}, 0
    for name, shape in param_shapes():
        size = int(np.prod(shape))
        out[name] = np.asarray(flat[k:k + size]).reshape(shape)
        k += size
    return out


def pack(params):
    return np.concatenate([np.asarray(params[name], np.float64).reshape(-1) for name, _ in param_shapes()])


def init_params(seed=0):
    """He-normal hidden weights, zero biases, zero output layer (so the initial preconditioner is block-Jacobi)."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, shape in param_shapes():
        if name.startswith("W_") and name != "W_o":
            p[name] = rng.standard_normal(shape) * np.sqrt(2.0 / shape[1])
        else:
            p[name] = np.zeros(shape)
    return pack(p)


def bf16(x):
    """Round to the nearest BF16 value, ties to even (what __float2bfloat16_rn does), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + np.uint32(0x7FFF)
    return ((u + r) & np.uint32(0xFFFF0000)).view(np.float32)


class Graph:
    """A Newton system's block-CSR graph with the quantities every pass needs."""

    def __init__(self, row_start, col_index, blocks, pinned, active):
        self.rs = np.asarray(row_start, np.int64)
        self.ci = np.asarray(col_index, np.int64)
        self.n = len(self.rs) - 1
        self.A = np.asarray(blocks, np.float64).reshape(-1, 3, 3)
        self.pinned = np.asarray(pinned, bool)
        self.active = np.asarray(active, bool)
        self.row = np.repeat(np.arange(self.n), np.diff(self.rs))
        B = len(self.ci)
        # Transposed slot: slot of (j, i) for slot (i, j).
        key = {(int(i), int(j)): s for s, (i, j) in enumerate(zip(self.row, self.ci))}
        self.tslot = np.array([key[(int(j), int(i))] for i, j in zip(self.row, self.ci)], np.int64)
        live = ~self.pinned[self.row] & ~self.pinned[self.ci]
        self.msg = live & (self.row != self.ci)            # slots that carry messages
        self.lower = live & (self.ci <= self.row)          # slots of G and L
        self.diag = self.row == self.ci
        # Scaling C_i = chol(inv(A_ii)) (lower), identity when A_ii is not SPD, zero when pinned.
        C = np.zeros((self.n, 3, 3))
        for i in range(self.n):
            if self.pinned[i]:
                continue
            Aii = self.A[self.rs[i] + np.searchsorted(self.ci[self.rs[i]:self.rs[i + 1]], i)]
            try:
                np.linalg.cholesky(Aii)
                C[i] = np.linalg.cholesky(np.linalg.inv(Aii))
            except np.linalg.LinAlgError:
                C[i] = np.eye(3)
        self.C = C
        Ahat = np.einsum("sba,sbc,scd->sad", C[self.row], self.A, C[self.ci])
        Ahat[~live] = 0.0
        self.Ahat = Ahat
        self.B = B

    def features(self):
        """Node features f (n, 16) and slot features e (B, 16), FP64."""
        n, Ah = self.n, self.Ahat
        fro = np.sqrt((Ah ** 2).sum(axis=(1, 2)))
        off = self.msg
        deg = np.bincount(self.row[off], minlength=n).astype(np.float64)
        mean = np.bincount(self.row[off], weights=fro[off], minlength=n) / np.maximum(deg, 1.0)
        mx = np.zeros(n)
        np.maximum.at(mx, self.row[off], fro[off])
        rowdiag = np.zeros((n, 3))
        for k in range(3):
            rowdiag[:, k] = np.bincount(self.row[off], weights=Ah[off, k, k], minlength=n)
        f = np.zeros((n, NODE_FEATURES))
        f[:, 0] = 1.0
        f[:, 1] = self.active & ~self.pinned
        f[:, 2] = deg / 16.0
        f[:, 3] = mean
        f[:, 4] = mx
        f[:, 5:8] = rowdiag
        f[:, 8] = self.pinned
        e = np.zeros((self.B, EDGE_FEATURES))
        e[:, 0:9] = Ah.reshape(-1, 9)
        e[:, 9] = fro
        e[:, 10] = self.diag
        e[:, 11] = self.ci < self.row
        return f, e


def _relu(x):
    return np.maximum(x, 0.0)


def forward(g: Graph, flat, emulate=True):
    """Network forward. Returns G (B, 3, 3; zero off the lower live slots), o (B, 16) and the cache for backward.
    With `emulate`, weights, features and stored activations are rounded to BF16 where the device rounds them."""
    P = unpack(flat)
    rnd = bf16 if emulate else (lambda x: np.asarray(x, np.float64))
    W = {k: (rnd(v) if k.startswith("W_") else np.asarray(v, np.float64)) for k, v in P.items()}
    W = {k: np.asarray(v, np.float64) for k, v in W.items()}
    f, e = g.features()
    f, e = np.asarray(rnd(f), np.float64), np.asarray(rnd(e), np.float64)
    cache = {"f": f, "e": e, "W": W, "h": [], "a": []}
    h = np.asarray(rnd(_relu(f @ W["W_ne"].T + W["b_ne"])), np.float64)
    eps = np.asarray(rnd(_relu(e @ W["W_ee"].T + W["b_ee"])), np.float64)
    cache["eps"] = eps
    msg = g.msg
    for l in range(LAYERS):
        cache["h"].append(h)
        X = np.concatenate([h[g.ci], eps], axis=1)
        m = _relu(X @ W[f"W_m{l}"].T + W[f"b_m{l}"])
        m[~msg] = 0.0
        a = np.zeros((g.n, HIDDEN))
        np.add.at(a, g.row, m)
        a = np.asarray(rnd(a * AGG_SCALE), np.float64)
        cache["a"].append(a)
        u = np.concatenate([h, a], axis=1) @ W[f"W_u{l}"].T + W[f"b_u{l}"]
        h = np.asarray(rnd(h + _relu(u)), np.float64)
    cache["h"].append(h)
    X = np.concatenate([h[g.row], h[g.ci], eps], axis=1)
    o = X @ W["W_o"].T + W["b_o"]
    o[~g.lower] = 0.0
    G = np.zeros((g.B, 3, 3))
    off = g.lower & ~g.diag
    G[off] = o[off, :9].reshape(-1, 3, 3)
    d = g.lower & g.diag
    oc = np.clip(o[d, :3], -DIAG_CLAMP, DIAG_CLAMP)
    G[d, 0, 0], G[d, 1, 1], G[d, 2, 2] = np.exp(oc[:, 0]), np.exp(oc[:, 1]), np.exp(oc[:, 2])
    G[d, 1, 0], G[d, 2, 0], G[d, 2, 1] = o[d, 3], o[d, 4], o[d, 5]
    cache["o"] = o
    cache["X_out"] = X
    return G, o, cache


def factor(g: Graph, G):
    """L = S G per lower slot (B, 3, 3)."""
    return np.einsum("sab,sbc->sac", g.C[g.row], G)


def apply_lower_t(g: Graph, M, x):
    """y_j = sum_{i >= j} M_ij^T x_i (M on lower slots)."""
    y = np.zeros((g.n, 3))
    np.add.at(y, g.ci, np.einsum("sba,sb->sa", M, x[g.row]))
    return y


def apply_lower(g: Graph, M, x):
    """y_i = sum_{j <= i} M_ij x_j."""
    y = np.zeros((g.n, 3))
    np.add.at(y, g.row, np.einsum("sab,sb->sa", M, x[g.ci]))
    return y


def apply_full(g: Graph, M, x):
    y = np.zeros((g.n, 3))
    np.add.at(y, g.row, np.einsum("sab,sb->sa", M, x[g.ci]))
    return y


def precondition(g: Graph, G, r):
    """z = L L^T r with L = S G (pinned rows give zero)."""
    L = factor(g, G)
    return apply_lower(g, L, apply_lower_t(g, L, np.asarray(r, np.float64)))


def loss(g: Graph, G, r):
    """|Ahat G G^T rhat - rhat|^2 / |rhat|^2 and the pieces backward needs."""
    rhat = np.einsum("iba,ib->ia", g.C, np.asarray(r, np.float64))
    a = apply_lower_t(g, G, rhat)
    b = apply_lower(g, G, a)
    e = apply_full(g, g.Ahat, b) - rhat
    den = float((rhat ** 2).sum())
    return float((e ** 2).sum()) / den, dict(rhat=rhat, a=a, b=b, e=e, den=den)


def loss_grad_G(g: Graph, G, parts):
    """d loss / d G on the lower live slots (B, 3, 3)."""
    ge = 2.0 * parts["e"] / parts["den"]
    gb = apply_full(g, g.Ahat, ge)
    ga = apply_lower_t(g, G, gb)
    gG = np.einsum("sa,sb->sab", gb[g.row], parts["a"][g.ci]) + np.einsum("sa,sb->sab", parts["rhat"][g.row],
                                                                            ga[g.ci])
    gG[~g.lower] = 0.0
    return gG


def grad_o(g: Graph, o, gG):
    """d loss / d o (B, 16) from d loss / d G."""
    go = np.zeros((g.B, OUTPUTS))
    off = g.lower & ~g.diag
    go[off, :9] = gG[off].reshape(-1, 9)
    d = g.lower & g.diag
    for k in range(3):
        inside = np.abs(o[d, k]) < DIAG_CLAMP
        go[d, k] = gG[d, k, k] * np.exp(np.clip(o[d, k], -DIAG_CLAMP, DIAG_CLAMP)) * inside
    go[d, 3], go[d, 4], go[d, 5] = gG[d, 1, 0], gG[d, 2, 0], gG[d, 2, 1]
    return go


def backward(g: Graph, cache, go, emulate=True):
    """Gradient of the loss with respect to the flat parameters, given d loss / d o. With `emulate`, the gradient
    operands of the tensor-core GEMMs (go, gu, gv, gw) are rounded to BF16 as the device stages them."""
    rnd = bf16 if emulate else (lambda x: np.asarray(x, np.float64))
    W = cache["W"]
    grads = {name: np.zeros(shape) for name, shape in param_shapes()}
    go = np.asarray(rnd(go), np.float64)
    X = cache["X_out"]
    grads["W_o"] = go.T @ X
    grads["b_o"] = go.sum(axis=0)
    gX = go @ W["W_o"]
    gh = np.zeros((g.n, HIDDEN))
    np.add.at(gh, g.row, gX[:, :HIDDEN])
    np.add.at(gh, g.ci, gX[:, HIDDEN:2 * HIDDEN])
    geps = gX[:, 2 * HIDDEN:].copy()
    eps = cache["eps"]
    for l in reversed(range(LAYERS)):
        h, a = cache["h"][l], cache["a"][l]
        Xu = np.concatenate([h, a], axis=1)
        u = Xu @ W[f"W_u{l}"].T + W[f"b_u{l}"]
        gu = np.asarray(rnd(gh * (u > 0)), np.float64)
        grads[f"W_u{l}"] = gu.T @ Xu
        grads[f"b_u{l}"] = gu.sum(axis=0)
        gXu = gu @ W[f"W_u{l}"]
        ga = gXu[:, HIDDEN:]
        gh = gh + gXu[:, :HIDDEN]
        Xm = np.concatenate([h[g.ci], eps], axis=1)
        v = Xm @ W[f"W_m{l}"].T + W[f"b_m{l}"]
        gv = ga[g.row] * AGG_SCALE * (v > 0)
        gv[~g.msg] = 0.0
        gv = np.asarray(rnd(gv), np.float64)
        grads[f"W_m{l}"] = gv.T @ Xm
        grads[f"b_m{l}"] = gv.sum(axis=0)
        gXm = gv @ W[f"W_m{l}"]
        np.add.at(gh, g.ci, gXm[:, :HIDDEN])
        geps += gXm[:, HIDDEN:]
    f, e = cache["f"], cache["e"]
    w = e @ W["W_ee"].T + W["b_ee"]
    gw = np.asarray(rnd(geps * (w > 0)), np.float64)
    grads["W_ee"] = gw.T @ e
    grads["b_ee"] = gw.sum(axis=0)
    q = f @ W["W_ne"].T + W["b_ne"]
    gq = np.asarray(rnd(gh * (q > 0)), np.float64)
    grads["W_ne"] = gq.T @ f
    grads["b_ne"] = gq.sum(axis=0)
    return pack(grads)


def live_unknowns(g: Graph) -> int:
    return 3 * int((~g.pinned).sum())


def kaporin(g: Graph, G, o, w):
    """Stochastic Kaporin objective of B = G^T Ahat G on a probe w (E[w w^T] = I):
    log(w^T G^T Ahat G w / N) - (2 / N) sum over live diagonal slots of the clamped o0..o2 (= log det G),
    N the number of live unknowns. Its minimiser over G on a fixed lower pattern is the factorised sparse approximate
    inverse (Kolotilina and Yeremin 1993), whose condition number bounds PCG's iteration count."""
    w = np.asarray(w, np.float64)
    b = apply_lower(g, G, w)
    c = apply_full(g, g.Ahat, b)
    t = float((b * c).sum())
    N = live_unknowns(g)
    d = g.lower & g.diag
    logdet = float(np.clip(o[d, :3], -DIAG_CLAMP, DIAG_CLAMP).sum())
    return np.log(t / N) - 2.0 * logdet / N, dict(w=w, b=b, c=c, t=t, N=N)


def kaporin_grad_o(g: Graph, o, parts):
    gG = (2.0 / parts["t"]) * np.einsum("sa,sb->sab", parts["c"][g.row], parts["w"][g.ci])
    gG[~g.lower] = 0.0
    go = grad_o(g, o, gG)
    d = g.lower & g.diag
    go[d, :3] -= (2.0 / parts["N"]) * (np.abs(o[d, :3]) < DIAG_CLAMP)
    return go


def kaporin_and_grad(g: Graph, flat, w, emulate=True):
    G, o, cache = forward(g, flat, emulate)
    value, parts = kaporin(g, G, o, w)
    return value, backward(g, cache, kaporin_grad_o(g, o, parts), emulate)


def loss_and_grad(g: Graph, flat, r, emulate=True):
    G, o, cache = forward(g, flat, emulate)
    value, parts = loss(g, G, r)
    gG = loss_grad_G(g, G, parts)
    return value, backward(g, cache, grad_o(g, o, gG), emulate)


def adam(flat, grad, state, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step (Kingma and Ba 2015) on the flat FP32 master parameters; `state` holds m, v and t."""
    state["t"] = state.get("t", 0) + 1
    m = state.setdefault("m", np.zeros_like(flat))
    v = state.setdefault("v", np.zeros_like(flat))
    m[:] = beta1 * m + (1 - beta1) * grad
    v[:] = beta2 * v + (1 - beta2) * grad * grad
    mh = m / (1 - beta1 ** state["t"])
    vh = v / (1 - beta2 ** state["t"])
    return flat - lr * mh / (np.sqrt(vh) + eps)
