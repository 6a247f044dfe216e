"""TEST INFRASTRUCTURE ONLY: the FP64 restatement of the learned coarse space's network (an extension with
no counterpart in the reference), with its training objective, backward pass and Adam loop, in numpy.
The oracle's C++ V-cycle evaluates the same network (ora_learned_forward): flat weights W1[20][64],
b1[64], W2[64][64], b2[64], W3[64][24], b3[24], row-major [in][out], tanh after both hidden layers;
output 3 k + c is coordinate c of basis vector k at the node.

Objective. On a logged coarsest operator, whitened by its diagonal blocks (At = L^-1 A L^-T), the
network's outputs form a basis Psi (3n x 8). A logged call brings the whitened residual r and exact
correction d = At^-1 r; the Galerkin correction on the basis captures the share
    q = u^T G^-1 u / (r^T d),  u = Psi^T r,  G = Psi^T At Psi,
of that call's error energy (0 <= q <= 1; 1 when the basis holds the exact correction). The loss is the
mean of 1 - q over calls, with dq/dPsi = 2 (r - At Psi c) c^T / (r^T d), c = G^-1 u.
"""
import numpy as np

IN, HID, K = 20, 64, 8
OUT = 3 * K
SHAPES = ((IN, HID), (HID,), (HID, HID), (HID,), (HID, OUT), (OUT,))
SIZE = sum(int(np.prod(s)) for s in SHAPES)
RIDGE = 1e-8  # G + RIDGE * tr(G) / K * I keeps the small solve defined for dependent columns


def unpack(w):
    out, q = [], 0
    for s in SHAPES:
        k = int(np.prod(s))
        out.append(w[q:q + k].reshape(s))
        q += k
    return out


def init(seed=0):
    """Glorot-scaled weights."""
    rng = np.random.default_rng(seed)
    w = np.zeros(SIZE)
    W1, b1, W2, b2, W3, b3 = unpack(w)
    W1[:] = rng.standard_normal(W1.shape) * np.sqrt(1.0 / IN)
    W2[:] = rng.standard_normal(W2.shape) * np.sqrt(1.0 / HID)
    W3[:] = rng.standard_normal(W3.shape) * np.sqrt(1.0 / HID)
    return w


def forward(w, X, keep=False):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1 = np.tanh(X @ W1 + b1)
    h2 = np.tanh(h1 @ W2 + b2)
    out = h2 @ W3 + b3
    return (out, (X, h1, h2)) if keep else out


def backward(w, cache, dout):
    """dL/dw from dL/dout (rows, 24) through the cached forward pass."""
    X, h1, h2 = cache
    _, _, W2, _, W3, _ = unpack(w)
    g = np.zeros_like(w)
    gW1, gb1, gW2, gb2, gW3, gb3 = unpack(g)
    gW3[:] = h2.T @ dout
    gb3[:] = dout.sum(0)
    dh2 = (dout @ W3.T) * (1 - h2 * h2)
    gW2[:] = h1.T @ dh2
    gb2[:] = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (1 - h1 * h1)
    gW1[:] = X.T @ dh1
    gb1[:] = dh1.sum(0)
    return g


def basis(out):
    """(n, 24) outputs -> (3n, 8) basis, row 3 i + c holding coordinate c of node i."""
    n = len(out)
    return out.reshape(n, K, 3).transpose(0, 2, 1).reshape(3 * n, K)


def unbasis(P):
    n = len(P) // 3
    return P.reshape(n, 3, K).transpose(0, 2, 1).reshape(n, OUT)


def captured(Psi, At, R, D):
    """Shares q (m,) of the calls' error energy captured by the basis, and c (K, m); R, D (3n, m)."""
    G = Psi.T @ At @ Psi
    G = 0.5 * (G + G.T) + RIDGE * np.trace(G) / K * np.eye(K)
    U = Psi.T @ R
    Cc = np.linalg.solve(G, U)
    E = np.sum(R * D, 0)
    return np.sum(U * Cc, 0) / E, Cc, E


def loss_grad(w, ops, calls):
    """(mean of 1 - q over the calls, its gradient) for ops [(At, X)] and calls [(op, r, d)]."""
    g = np.zeros_like(w)
    total, m = 0.0, len(calls)
    by_op = {}
    for op, r, d in calls:
        by_op.setdefault(op, []).append((r, d))
    for op, rd in by_op.items():
        At, X = ops[op]
        out, cache = forward(w, X, keep=True)
        Psi = basis(out)
        R = np.stack([a for a, _ in rd], 1)
        D = np.stack([b for _, b in rd], 1)
        q, Cc, E = captured(Psi, At, R, D)
        total += float(np.sum(1 - q))
        dPsi = -2 * ((R - At @ Psi @ Cc) / E) @ Cc.T / m
        g += backward(w, cache, unbasis(dPsi))
    return total / m, g


def train(ops, calls, steps=600, batch_ops=4, lr=3e-3, seed=0, w=None, op_weights=None):
    """Adam over minibatches of logged operators (all calls of each), drawn uniformly or in proportion to
    op_weights (one per operator); returns (weights, loss every 50 steps)."""
    rng = np.random.default_rng(seed)
    w = init(seed) if w is None else w.copy()
    m, v = np.zeros_like(w), np.zeros_like(w)
    b1, b2, eps = 0.9, 0.999, 1e-8
    by_op = {}
    for c in calls:
        by_op.setdefault(c[0], []).append(c)
    keys = sorted(by_op)
    hist = []
    for t in range(1, steps + 1):
        prob = None
        if op_weights is not None:
            prob = np.array([op_weights[k] for k in keys], np.float64)
            prob /= prob.sum()
        pick = rng.choice(len(keys), min(batch_ops, len(keys)), replace=False, p=prob)
        batch = [c for k in pick for c in by_op[keys[k]]]
        loss, g = loss_grad(w, ops, batch)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        step = lr * (0.1 ** (t / steps))  # decays tenfold over the run
        w -= step * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
        if t % 50 == 0:
            hist.append(loss)
    return w, hist
