"""CPU oracle of the learned start guess -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this module;
the library never does.  The reference (StiffGIPC) has no learned component,
so there is no reference file to follow: this restates the library's own
definition (include/sgmas.h, "learned start guess") in numpy -- features,
forward pass, loss, analytic backward pass, Adam, and the BF16 inference with
its rounding points -- and is itself checked by finite differences
(tests/test_learned_oracle.py).  Parity with the reference is therefore
unpinned for this part; it is measured against plain MAS-PCG.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

N_IN, N_HID, N_OUT = 16, 128, 6
O_W1 = 0
O_B1 = O_W1 + N_IN * N_HID
O_W2 = O_B1 + N_HID
O_B2 = O_W2 + N_HID * N_HID
O_W3 = O_B2 + N_HID
O_B3 = O_W3 + N_HID * N_OUT
N_PARAMS = O_B3 + N_OUT
BANK = 16


def unpack(P):
    P = np.asarray(P, np.float64)
    return (P[O_W1:O_B1].reshape(N_IN, N_HID), P[O_B1:O_W2], P[O_W2:O_B2].reshape(N_HID, N_HID), P[O_B2:O_W3],
            P[O_W3:O_B3].reshape(N_HID, N_OUT), P[O_B3:N_PARAMS])


def pack(W1, b1, W2, b2, W3, b3):
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, W3.ravel(), b3])


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def decode_contacts(pairs):
    """Vertices of each int4 contact (the sign encoding of the reference's
    _buildCollisionConnection_new, SG/MASPreconditioner.cu:1140-1537); -1 = none."""
    P = np.asarray(pairs, np.int64).reshape(-1, 4)
    out = np.full((len(P), 4), -1, np.int64)
    for q, (x, y, z, w) in enumerate(P):
        if x >= 0:
            out[q] = (x, y, z, -w - 1 if w < 0 else w)
        else:
            xx = -x - 1
            if z < 0:
                out[q] = (xx, -y - 1, -z - 1, -w - 1) if y < 0 else (xx, y, -1, -1)
            elif w < 0:
                out[q] = (xx, -y - 1, z, -w - 1) if y < 0 else (xx, y, z, -1)
            else:
                out[q] = (xx, y, z, w)
    return out


def _solve3(M, rhs):
    """Per-vertex 3x3 solves; zero where M is singular."""
    det = np.linalg.det(M)
    out = np.zeros_like(rhs)
    ok = det != 0
    out[ok] = np.linalg.solve(M[ok], rhs[ok][:, :, None])[:, :, 0]
    return out


def row_sums(vals, rows, cols, nrows):
    """3x3 block row sums S_v = sum_j A_vj of the full symmetric matrix stored as upper BCOO."""
    H = np.asarray(vals, np.float64).reshape(-1, 3, 3).transpose(0, 2, 1)   # column-major -> (a, c)
    rows, cols = np.asarray(rows), np.asarray(cols)
    S = np.zeros((nrows, 3, 3))
    np.add.at(S, rows, H)
    off = rows != cols
    np.add.at(S, cols[off], H[off].transpose(0, 2, 1))
    return S


def lumped_step(vals, rows, cols, b, N, fem_offset=0):
    """u_v = S_v^-1 b_v (S = block row sums; D^-1 b_v where S has no positive
    trace and determinant) for the N MAS vertices, and D (diagonal blocks)."""
    vals = np.asarray(vals, np.float64).reshape(-1, 9)
    rows, cols = np.asarray(rows), np.asarray(cols)
    b = np.asarray(b, np.float64).reshape(-1, 3)
    nrows = len(b)
    D = np.tile(np.eye(3), (nrows, 1, 1))
    dk = rows == cols
    D[rows[dk]] = vals[dk].reshape(-1, 3, 3).transpose(0, 2, 1)
    rr = fem_offset + np.arange(N)
    S = row_sums(vals, rows, cols, nrows)[rr]
    usable = (np.trace(S, axis1=1, axis2=2) > 0) & (np.linalg.det(S) > 0)
    u = _solve3(np.where(usable[:, None, None], S, D[rr]), b[rr])
    return u, D[rr]


def features(vals, rows, cols, b, part_map, N, fem_offset=0, prev=None, pairs=None, node_offset=0, dx=None):
    """Slot-ordered features X [Mm,16] (float32), mask [Mm], targets T [Mm,3]
    ((dx - u) / s, when dx is given) and the scales (s, s_b) = RMS of |u|, |b_v|."""
    b = np.asarray(b, np.float64).reshape(-1, 3)
    rr = fem_offset + np.arange(N)
    u, Dv = lumped_step(vals, rows, cols, b, N, fem_offset)
    y = _solve3(Dv, b[rr])
    s = np.sqrt(np.sum(u * u) / max(N, 1))
    sb = np.sqrt(np.sum(b[rr] ** 2) / max(N, 1))
    s = s if s > 0 else 1.0
    sb = sb if sb > 0 else 1.0
    cnt = np.zeros(N, np.int64)
    if pairs is not None and len(pairs):
        v = decode_contacts(pairs) - node_offset
        v = v[(v >= 0) & (v < N)]
        np.add.at(cnt, v, 1)
    t = np.trace(Dv, axis1=1, axis2=2) / 3.0
    t = np.where(t > 0, t, 1.0)
    F = np.zeros((N, 16))
    F[:, 0:3] = u / s
    if prev is not None:
        F[:, 3:6] = np.asarray(prev, np.float64).reshape(-1, 3)[rr] / s
    F[:, 6:9] = y / s
    F[:, 9] = Dv[:, 0, 0] / t - 1.0
    F[:, 10] = Dv[:, 1, 1] / t - 1.0
    F[:, 11] = Dv[:, 2, 2] / t - 1.0
    F[:, 12] = Dv[:, 0, 1] / t
    F[:, 13] = Dv[:, 0, 2] / t
    F[:, 14] = Dv[:, 1, 2] / t
    F[:, 15] = np.minimum(cnt, 32) / 8.0
    pm = np.asarray(part_map)
    Mm = len(pm)
    valid = (pm >= 0) & (pm < N)
    X = np.zeros((Mm, 16), np.float32)
    X[valid] = F[pm[valid]].astype(np.float32)
    mask = valid.astype(np.float32)
    T = None
    if dx is not None:
        T = np.zeros((Mm, 3), np.float32)
        corr = (np.asarray(dx, np.float64).reshape(-1, 3)[rr] - u) / s
        T[valid] = corr[pm[valid]].astype(np.float32)
    return X, mask, T, (s, sb)


def forward(P, X, cache=False):
    W1, b1, W2, b2, W3, b3 = unpack(P)
    X = np.asarray(X, np.float64).reshape(-1, N_IN)
    Z1 = X @ W1 + b1
    H1 = gelu(Z1)
    Z2 = H1 @ W2 + b2
    H2 = gelu(Z2)
    Y = H2 @ W3 + b3
    return (Y, (X, Z1, H1, Z2, H2)) if cache else Y


def prediction(Y, mask):
    """step + mean of the coarse term over each 16-row subdomain (valid rows)."""
    Y = Y.reshape(-1, BANK, N_OUT)
    m = np.asarray(mask, np.float64).reshape(-1, BANK)
    cnt = m.sum(1)
    cm = (m[:, :, None] * Y[:, :, 3:6]).sum(1) / np.where(cnt > 0, cnt, 1.0)[:, None]
    return (Y[:, :, 0:3] + cm[:, None, :]).reshape(-1, 3)


def loss_grad(P, X, T, mask, inv_n):
    """inv_n * sum over valid rows |prediction - T|^2 and its gradient (FP64)."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    Y, (Xd, Z1, H1, Z2, H2) = forward(P, X, cache=True)
    m = np.asarray(mask, np.float64)
    e = (prediction(Y, m) - np.asarray(T, np.float64).reshape(-1, 3)) * m[:, None]
    loss = inv_n * np.sum(e * e)
    dpred = 2.0 * inv_n * e
    dY = np.zeros_like(Y)
    dY[:, 0:3] = dpred
    mb = m.reshape(-1, BANK)
    cnt = mb.sum(1)
    s = dpred.reshape(-1, BANK, 3).sum(1) / np.where(cnt > 0, cnt, 1.0)[:, None]
    dY[:, 3:6] = (mb[:, :, None] * s[:, None, :]).reshape(-1, 3)
    dW3 = H2.T @ dY
    db3 = dY.sum(0)
    dZ2 = (dY @ W3.T) * gelu_d(Z2)
    dW2 = H1.T @ dZ2
    db2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2.T) * gelu_d(Z1)
    dW1 = Xd.T @ dZ1
    db1 = dZ1.sum(0)
    return loss, pack(dW1, db1, dW2, db2, dW3, db3)


def adam(P, M, V, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    M = b1 * M + (1 - b1) * g
    V = b2 * V + (1 - b2) * g * g
    P = P - lr * (M / (1 - b1 ** step)) / (np.sqrt(V / (1 - b2 ** step)) + eps)
    return P, M, V


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


def infer_bf16(P, X):
    """The BF16 inference: inputs, weights and hidden activations rounded to
    BF16, products accumulated in FP32, biases and GELU in FP32."""
    W1, b1, W2, b2, W3, b3 = (np.asarray(a, np.float32) for a in unpack(P))
    X = bf16(np.asarray(X, np.float32).reshape(-1, N_IN))
    g = lambda z: np.asarray(gelu(np.asarray(z, np.float64)), np.float32)
    H1 = bf16(g(X @ bf16(W1) + b1))
    H2 = bf16(g(H1 @ bf16(W2) + b2))
    return H2 @ bf16(W3) + b3


def compose(Y, part_map, N, s, nrows, u, fem_offset=0):
    """x0 [3 nrows]: u + s (step + subdomain mean of the coarse term) at each MAS vertex, 0 elsewhere."""
    pm = np.asarray(part_map)
    mask = ((pm >= 0) & (pm < N)).astype(np.float64)
    pred = prediction(np.asarray(Y, np.float64), mask)
    x0 = np.zeros((nrows, 3))
    v = mask > 0
    x0[fem_offset + pm[v]] = np.asarray(u).reshape(-1, 3)[pm[v]] + s * pred[v]
    return x0.ravel()
