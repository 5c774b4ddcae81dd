"""CPU oracle of the learned mesh preconditioner (test infrastructure only).

The reference has no learned preconditioner: the network is this project's
design (a message-passing network over mesh nodes used inside flexible PCG),
so the oracle restates the network as the CUDA path defines it and is pinned
by finite differences of its own FP64 forward pass (parity unpinned against
the reference, which has nothing to compare with).  The CUDA kernels must
match this file: forward within BF16 rounding, gradients within the tolerance
written in the tests.

Network (per node i; N(i) = nodes sharing an element with i, deg_i = |N(i)|):

    d_i    = sqrt(dinv_i)            (3; dinv = 1/diag K_T on free DOFs, 0 on fixed)
    xt_i   = d_i * r_i               (3)
    s      = sqrt(sum_i |xt_i|^2 / Nn)
    f_i    = [xt_i / s, fixed bits (3), c_i, 0 x 9]          (16; c_i = log-modulus feature)
    h_i    = relu(W_e f_i + b_e)                              (64)
    repeat 4x:
      m_i  = (1/deg_i) sum_{j in N(i)} h_j
      h_i  = h_i + relu(W_l [h_i, m_i] + b_l)                 (W_l: 64 x 128)
    o_i    = W_d h_i + b_d                                    (3)
    z_i    = dinv_i * r_i + s * d_i * o_i

With o = 0 the map is the Jacobi preconditioner; z(a r) = a z(r) for a > 0.
BF16 storage (``bf16=True``) rounds f, W_e, W_l, every stored h and m, and
the backward's relu-masked gradient before its tensor-core products, as the
CUDA kernels do; accumulation is FP32 there and FP64 here.
"""
from __future__ import annotations

import numpy as np

HIDDEN = 64
IN_FEATURES = 16
N_LAYERS = 4
OUT = 3


def param_shapes():
    """Flattened parameter order shared with the C ABI (fem_mpnn_* weights)."""
    shapes = [("W_e", (HIDDEN, IN_FEATURES)), ("b_e", (HIDDEN,))]
    for l in range(N_LAYERS):
        shapes += [(f"W_{l}", (HIDDEN, 2 * HIDDEN)), (f"b_{l}", (HIDDEN,))]
    shapes += [("W_d", (OUT, HIDDEN)), ("b_d", (OUT,))]
    return shapes


def n_params():
    return int(sum(np.prod(s) for _, s in param_shapes()))


def unflatten(w):
    out, o = {}, 0
    for name, shp in param_shapes():
        k = int(np.prod(shp))
        out[name] = np.asarray(w[o:o + k], dtype=np.float64).reshape(shp)
        o += k
    return out


def flatten(p):
    return np.concatenate([np.asarray(p[name], dtype=np.float64).reshape(-1) for name, _ in param_shapes()])


def init_params(seed=0, out_scale=0.0):
    """He-style initialisation; the decoder starts at ``out_scale`` (0: Jacobi)."""
    rng = np.random.default_rng(seed)
    p = {"W_e": rng.standard_normal((HIDDEN, IN_FEATURES)) * np.sqrt(2.0 / 7.0),
         "b_e": np.zeros(HIDDEN)}
    for l in range(N_LAYERS):
        p[f"W_{l}"] = rng.standard_normal((HIDDEN, 2 * HIDDEN)) * np.sqrt(2.0 / (2 * HIDDEN)) * 0.5
        p[f"b_{l}"] = np.zeros(HIDDEN)
    p["W_d"] = rng.standard_normal((OUT, HIDDEN)) * out_scale
    p["b_d"] = np.zeros(OUT)
    return flatten(p)


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(np.isfinite(a), out, a.astype(np.float64))


def node_graph(conn, n_nodes):
    """Symmetric node adjacency (nodes sharing an element), CSR sorted by id."""
    conn = np.asarray(conn, dtype=np.int64)
    pairs = []
    for a in range(4):
        for b in range(4):
            if a != b:
                pairs.append(np.stack([conn[:, a], conn[:, b]], 1))
    pr = np.unique(np.concatenate(pairs, 0), axis=0)
    ptr = np.zeros(n_nodes + 1, dtype=np.int64)
    np.add.at(ptr, pr[:, 0] + 1, 1)
    ptr = np.cumsum(ptr)
    return ptr, pr[:, 1].copy()


def log_modulus_feature(conn, n_nodes, elem_modulus):
    """c_i = log(mean modulus of the elements at node i) minus its mean over nodes."""
    conn = np.asarray(conn, dtype=np.int64)
    acc = np.zeros(n_nodes)
    cnt = np.zeros(n_nodes)
    for a in range(4):
        np.add.at(acc, conn[:, a], elem_modulus)
        np.add.at(cnt, conn[:, a], 1.0)
    lm = np.log(acc / np.maximum(cnt, 1.0))
    return lm - lm.mean()


def _aggregate(ptr, idx, h):
    deg = np.diff(ptr)
    s = np.add.reduceat(h[idx], ptr[:-1], axis=0) if idx.size else np.zeros_like(h)
    s[deg == 0] = 0.0
    return s / np.maximum(deg, 1)[:, None]


def _scatter_T(ptr, idx, g):
    """Transpose of the mean aggregation: out_j = sum_{i in N(j)} g_i / deg_i."""
    deg = np.diff(ptr)
    q = g / np.maximum(deg, 1)[:, None]
    return _aggregate(ptr, idx, q) * np.maximum(deg, 1)[:, None]


def forward(w, r, dinv, fixed_bits, c, graph, bf16_storage=True, keep=False):
    """z = M(r).  r, dinv: (Nn, 3); fixed_bits: (Nn,) ints; c: (Nn,)."""
    P = unflatten(w)
    rd = bf16 if bf16_storage else (lambda x: np.asarray(x, dtype=np.float64))
    ptr, idx = graph
    r = np.asarray(r, dtype=np.float64)
    dinv = np.asarray(dinv, dtype=np.float64)
    n = r.shape[0]
    d = np.sqrt(dinv)
    xt = d * r
    s = float(np.sqrt(np.sum(xt * xt) / n))
    if s == 0.0:
        z = np.zeros_like(r)
        return (z, None) if keep else z
    fb = np.asarray(fixed_bits, dtype=np.int64)
    f = np.zeros((n, IN_FEATURES))
    f[:, 0:3] = xt / s
    f[:, 3] = fb & 1
    f[:, 4] = (fb >> 1) & 1
    f[:, 5] = (fb >> 2) & 1
    f[:, 6] = c
    f = rd(f)
    pre0 = f @ rd(P["W_e"]).T + P["b_e"]
    h = rd(np.maximum(pre0, 0.0))
    hs, ms, pres = [h], [], [pre0]
    for l in range(N_LAYERS):
        m = rd(_aggregate(ptr, idx, h))
        a = np.concatenate([h, m], 1)
        pre = a @ rd(P[f"W_{l}"]).T + P[f"b_{l}"]
        h = rd(h + np.maximum(pre, 0.0))
        hs.append(h)
        ms.append(m)
        pres.append(pre)
    o = h @ P["W_d"].T + P["b_d"]
    z = dinv * r + s * d * o
    if keep:
        return z, {"f": f, "hs": hs, "ms": ms, "pres": pres, "s": s, "d": d}
    return z


def backward(w, r, dinv, fixed_bits, c, graph, gz, bf16_storage=True):
    """Gradient of <gz, M(r)> with respect to the flattened parameters."""
    P = unflatten(w)
    rd = bf16 if bf16_storage else (lambda x: np.asarray(x, dtype=np.float64))
    ptr, idx = graph
    z, st = forward(w, r, dinv, fixed_bits, c, graph, bf16_storage, keep=True)
    G = {name: np.zeros(shp) for name, shp in param_shapes()}
    if st is None:
        return flatten(G)
    s, d, hs, ms, pres = st["s"], st["d"], st["hs"], st["ms"], st["pres"]
    go = s * d * np.asarray(gz, dtype=np.float64)
    G["W_d"] = go.T @ hs[-1]
    G["b_d"] = go.sum(0)
    gh = go @ P["W_d"]
    for l in reversed(range(N_LAYERS)):
        h_in, m = hs[l], ms[l]
        a = np.concatenate([h_in, m], 1)
        gpre = gh * (pres[l + 1] > 0.0)
        gpre_r = rd(gpre)
        G[f"W_{l}"] = gpre_r.T @ a
        G[f"b_{l}"] = gpre.sum(0)
        ga = gpre_r @ rd(P[f"W_{l}"])
        gh = gh + ga[:, :HIDDEN] + _scatter_T(ptr, idx, ga[:, HIDDEN:])
    gpre0 = gh * (pres[0] > 0.0)
    G["W_e"] = gpre0.T @ st["f"]
    G["b_e"] = gpre0.sum(0)
    return flatten(G)


def energy_loss(z, r, Az, e_dot_r):
    """||z - e||_A^2 / ||e||_A^2 with A e = r: (z.Az - 2 z.r + e.r) / e.r."""
    return float((np.sum(z * Az) - 2.0 * np.sum(z * r) + e_dot_r) / e_dot_r)


def adam_step(w, g, m, v, t, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update (bias-corrected), as the CUDA optimizer applies it."""
    m = beta1 * m + (1.0 - beta1) * g
    v = beta2 * v + (1.0 - beta2) * g * g
    mh = m / (1.0 - beta1 ** t)
    vh = v / (1.0 - beta2 ** t)
    return w - lr * mh / (np.sqrt(vh) + eps), m, v


def fpcg(apply_A, precond, b, rtol, maxit):
    """Flexible PCG (Polak-Ribiere beta), the outer method around the network."""
    x = np.zeros_like(b)
    r = b.copy()
    rr0 = float(np.sum(r * r))
    if rr0 == 0.0:
        return x, 0
    z = precond(r)
    p = z.copy()
    rz = float(np.sum(r * z))
    for it in range(1, maxit + 1):
        q = apply_A(p)
        alpha = rz / float(np.sum(p * q))
        x += alpha * p
        r -= alpha * q
        if float(np.sum(r * r)) <= rtol * rtol * rr0:
            return x, it
        z = precond(r)
        rz_new = float(np.sum(r * z))
        # Polak-Ribiere: beta = z.(r_new - r_old) / rz_old, and r_new - r_old = -alpha q
        beta = -alpha * float(np.sum(z * q)) / rz
        p = z + beta * p
        rz = rz_new
    return x, maxit
