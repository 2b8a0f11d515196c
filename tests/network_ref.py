"""numpy restatement of the preconditioner network (drape_b200/csrc/nn.h, nn.cu) and of its training loss and
gradient through one V-cycle (Context::network_pass): the checker of the CUDA forward, backward and training
kernels. The network has no counterpart in the reference (its direction solver is block-Jacobi PCG only).

bf16=True rounds the dense layers' inputs and weights to bf16 as the tensor-core forward does; the backward pass
is f32/f64 on both sides (the device rebuilds X in f32 and uses the f32 master weights).
"""
import numpy as np

from tests import multilevel_ref as ml

N_IN, H, LAYERS = 16, 64, 4
OFF_WIN, OFF_BIN = 0, N_IN * H
LAYER_SIZE = 2 * H * H + H
OFF_L0 = OFF_BIN + H
OFF_WO = OFF_L0 + LAYERS * LAYER_SIZE
OFF_BO = OFF_WO + H
N_PARAMS = OFF_BO + 1
LOW, SPAN, SHIFT = np.float32(0.8), np.float32(0.2), np.float32(0.0)  # f = LOW + SPAN sigmoid(o + SHIFT) in (0.8, 1); f(0) = 0.9


def bf16(a):
    """Round to nearest-even bf16, returned as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p, np.float64)
    W_in = p[OFF_WIN:OFF_WIN + N_IN * H].reshape(N_IN, H)
    b_in = p[OFF_BIN:OFF_BIN + H]
    Ws, bs = [], []
    for l in range(LAYERS):
        o = OFF_L0 + l * LAYER_SIZE
        Ws.append(p[o:o + 2 * H * H].reshape(2 * H, H))
        bs.append(p[o + 2 * H * H:o + LAYER_SIZE])
    return W_in, b_in, Ws, bs, p[OFF_WO:OFF_WO + H], p[OFF_BO]


def blocks9(blocks):
    return np.asarray(blocks, np.float64).reshape(-1, 9)


def features(row_ptr, col_idx, blocks, omega0):
    """(feat [R][16], w [B]) as features_kernel computes them."""
    Bk = blocks9(blocks)
    R = len(row_ptr) - 1
    feat = np.zeros((R, N_IN))
    w = np.zeros(len(col_idx))
    for i in range(R):
        k0, k1 = row_ptr[i], row_ptr[i + 1]
        ks = np.arange(k0, k1)
        kd = ks[col_idx[k0:k1] == i][0]
        D = Bk[kd].reshape(3, 3)
        tr = np.trace(D)
        dn = np.linalg.norm(D)
        det = np.linalg.det(D)
        Dinv = np.linalg.inv(D) if det != 0 else np.zeros((3, 3))
        off = [k for k in ks if k != kd]
        norms = np.array([np.linalg.norm(Bk[k]) for k in off])
        off_sum = norms.sum()
        local = sum(np.linalg.norm(Dinv @ Bk[k].reshape(3, 3)) for k in off)
        for k, nrm in zip(off, norms):
            w[k] = nrm / off_sum if off_sum > 0 else 0.0
        rt = 1.0 / tr if tr != 0 else 0.0
        rn = 1.0 / dn if dn > 0 else 0.0
        feat[i, :12] = [D[0, 0] * rt, D[1, 1] * rt, D[2, 2] * rt, 0.5 * (D[0, 1] + D[1, 0]) * rt,
                        0.5 * (D[0, 2] + D[2, 0]) * rt, 0.5 * (D[1, 2] + D[2, 1]) * rt, off_sum * rn,
                        (norms.max() if len(norms) else 0.0) * rn, (k1 - k0) / 25.0, omega0, 0.1 * local, 1.0]
    return feat, w


def aggregate(row_ptr, col_idx, w, h):
    R = len(row_ptr) - 1
    rows = np.repeat(np.arange(R), np.diff(row_ptr))
    m = np.zeros_like(h)
    np.add.at(m, rows, w[:, None] * h[col_idx])
    return m


def forward(params, feat, row_ptr, col_idx, w, bf=True):
    """(hs [h0..h4], o, f)."""
    W_in, b_in, Ws, bs, w_o, b_o = unpack(params)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    hs = [np.maximum(r(feat) @ r(W_in) + b_in, 0.0)]
    for l in range(LAYERS):
        X = np.concatenate([hs[-1], aggregate(row_ptr, col_idx, w, hs[-1])], axis=1)
        hs.append(np.maximum(r(X) @ r(Ws[l]) + bs[l], 0.0))
    o = hs[-1] @ w_o + b_o
    return hs, o, LOW + SPAN / (1.0 + np.exp(-(o + SHIFT)))


def backward(params, feat, row_ptr, col_idx, w, hs, o, dfac):
    """Parameter gradient from dL/df (f32/f64 backward, as nn_backward)."""
    W_in, b_in, Ws, bs, w_o, b_o = unpack(params)
    g = np.zeros(N_PARAMS)
    s = 1.0 / (1.0 + np.exp(-(o + SHIFT)))
    do = dfac * SPAN * s * (1 - s)
    g[OFF_WO:OFF_WO + H] = hs[-1].T @ do
    g[OFF_BO] = do.sum()
    dh = do[:, None] * w_o[None, :]
    R = len(row_ptr) - 1
    rows = np.repeat(np.arange(R), np.diff(row_ptr))
    for l in reversed(range(LAYERS)):
        dpre = dh * (hs[l + 1] > 0)
        X = np.concatenate([hs[l], aggregate(row_ptr, col_idx, w, hs[l])], axis=1)
        o_w = OFF_L0 + l * LAYER_SIZE
        g[o_w:o_w + 2 * H * H] = (X.T @ dpre).reshape(-1)
        g[o_w + 2 * H * H:o_w + LAYER_SIZE] = dpre.sum(axis=0)
        dX = dpre @ Ws[l].T
        dm = dX[:, H:]
        dh = dX[:, :H].copy()
        np.add.at(dh, col_idx, w[:, None] * dm[rows])  # dh_j += sum_i w_ij dm_i
    dpre = dh * (hs[0] > 0)
    g[OFF_WIN:OFF_WIN + N_IN * H] = (feat.T @ dpre).reshape(-1)
    g[OFF_BIN:OFF_BIN + H] = dpre.sum(axis=0)
    return g


def coarse_correction(Hh, v):
    """C v = P V_1 P^T v (the cycle below the fine level)."""
    return Hh.P[0] @ Hh.vcycle(Hh.P[0].T @ v, 1)


def loss_and_dfactor(A, Hh, S0, f, b, x):
    """Loss ||x - z||_A^2 / ||x||_A^2 of z = M b with S = f S0 at the fine level, and dL/df."""
    S = f[:, None, None] * S0
    z1 = ml.block_apply(S, b)
    y = z1 + coarse_correction(Hh, b - A @ z1)
    u = b - A @ y
    z = y + ml.block_apply(S, u)
    e = x - z
    N = x @ (A @ x)
    L = e @ (A @ e) / N
    gz = -2.0 * (A @ e) / N
    gy = gz - A @ ml.block_apply(S, gz)
    gz1 = gy - A @ coarse_correction(Hh, gy)
    dfac = (gz.reshape(-1, 3) * ml.block_apply(S0, u).reshape(-1, 3)).sum(1) + \
           (gz1.reshape(-1, 3) * ml.block_apply(S0, b).reshape(-1, 3)).sum(1)
    return L, dfac


def network_loss(params, row_ptr, col_idx, blocks, n, b, x, bf=True, grad=True):
    """(loss, gradient or None, factors) of one tuple, as drape_network_gradient."""
    A = ml.bsr_matrix(row_ptr, col_idx, blocks)
    Hh = ml.Hierarchy(A, n)
    S0 = Hh.S[0]
    feat, w = features(row_ptr, col_idx, blocks, Hh.omega[0])
    hs, o, f = forward(params, feat, row_ptr, col_idx, w, bf)
    L, dfac = loss_and_dfactor(A, Hh, S0, f, b, x)
    g = backward(params, feat, row_ptr, col_idx, w, hs, o, dfac) if grad else None
    return L, g, f


def init_params(seed, scale_out=0.0):
    """Glorot-uniform weights (not the device's generator: tests set parameters explicitly)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS)
    a = np.sqrt(6.0 / (N_IN + H))
    p[OFF_WIN:OFF_WIN + N_IN * H] = rng.uniform(-a, a, N_IN * H)
    for l in range(LAYERS):
        o = OFF_L0 + l * LAYER_SIZE
        a = np.sqrt(6.0 / (3 * H))
        p[o:o + 2 * H * H] = rng.uniform(-a, a, 2 * H * H)
        p[o + 2 * H * H:o + LAYER_SIZE] = rng.uniform(0, 0.05, H)
    p[OFF_WO:OFF_WO + H] = scale_out * rng.standard_normal(H)
    p[OFF_BO] = 0.1 * scale_out
    return p.astype(np.float32)
