"""CPU restatement (numpy) of the learned warm start -- TEST INFRASTRUCTURE.

Only tests/ (and the CPU-baseline leg of bench.py) use this module, as the
checker of libavbd6's avbd_mlp_* entry points and of the solver's
new-contact feature log.  The warm start has no counterpart in the
reference: it replaces the cache-miss defaults of gpu_pool_emit_rows
(src/avbd3d/kernels_6dof.py:2864-2879, lambda 0 and penalties (1e6, 1, 1))
before the prelude consumes them (kernels_6dof.py:1596-1609).  Parity here
is therefore against this restatement of the network, its gradient (checked
against finite differences in the CPU tests) and the feature definition
below, not against reference outputs.

Layouts are those declared with AVBD_MLP_* in include/avbd6.h.
"""

from __future__ import annotations

import numpy as np

MLP_IN, MLP_H, MLP_OUT = 20, 64, 4
N_PARAMS = 5764
N_FLOATS = 3544
P_W1, P_B1, P_W2, P_B2, P_W3, P_B3 = 0, 1280, 1344, 5440, 5504, 5760
O_FMEAN, O_FISTD, O_OMEAN, O_OSTD, O_B1, O_B2, O_B3, O_W1, O_W2, O_W3 = 0, 32, 64, 72, 80, 144, 208, 216, 1240, 3288
PEN_MIN, PEN_MAX = 1.0e6, 1.0e9


def split(theta):
    t = np.asarray(theta, np.float64)
    return (t[P_W1:P_B1].reshape(MLP_H, MLP_IN), t[P_B1:P_W2], t[P_W2:P_B2].reshape(MLP_H, MLP_H), t[P_B2:P_W3],
            t[P_W3:P_B3].reshape(MLP_OUT, MLP_H), t[P_B3:N_PARAMS])


def bf16_round(x):
    """Round float32 values to bfloat16 (round to nearest even), as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def pack(theta, norm):
    """Packed inference block (float32 array with bf16 pairs as raw bits)."""
    W1, b1, W2, b2, W3, b3 = split(theta)
    norm = np.asarray(norm, np.float32)
    pk = np.zeros(N_FLOATS, np.float32)
    pk[O_FMEAN:O_FMEAN + MLP_IN] = norm[:MLP_IN]
    pk[O_FISTD:O_FISTD + MLP_IN] = np.float32(1.0) / norm[MLP_IN:2 * MLP_IN]
    pk[O_OMEAN:O_OMEAN + MLP_OUT] = norm[2 * MLP_IN:2 * MLP_IN + MLP_OUT]
    pk[O_OMEAN + MLP_OUT] = norm[2 * MLP_IN + 2 * MLP_OUT]  # lambda scale
    pk[O_OSTD:O_OSTD + 8] = 1.0
    pk[O_OSTD:O_OSTD + MLP_OUT] = norm[2 * MLP_IN + MLP_OUT:2 * MLP_IN + 2 * MLP_OUT]
    pk[O_B1:O_B1 + MLP_H] = b1
    pk[O_B2:O_B2 + MLP_H] = b2
    pk[O_B3:O_B3 + MLP_OUT] = b3

    def bits(w, rows, cols):
        m = np.zeros((rows, cols), np.float32)
        m[:w.shape[0], :w.shape[1]] = w
        b = bf16_round(m).view(np.uint32) >> 16
        pairs = (b[:, 0::2] | (b[:, 1::2] << 16)).astype(np.uint32)
        return pairs.reshape(-1).view(np.float32)

    pk[O_W1:O_W2] = bits(W1, 64, 32)
    pk[O_W2:O_W3] = bits(W2, 64, 64)
    pk[O_W3:N_FLOATS] = bits(W3, 8, 64)
    return pk


def unpack_weights(pk):
    """bf16 weight matrices of a packed block, as float64 [out][in]."""
    def mat(lo, hi, rows, cols):
        u = np.ascontiguousarray(pk[lo:hi], np.float32).view(np.uint32).reshape(rows, cols // 2)
        m = np.zeros((rows, cols), np.uint32)
        m[:, 0::2] = (u & 0xFFFF) << 16
        m[:, 1::2] = u & 0xFFFF0000
        return m.view(np.float32).astype(np.float64)
    return mat(O_W1, O_W2, 64, 32), mat(O_W2, O_W3, 64, 64), mat(O_W3, N_FLOATS, 8, 64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def infer_bf16(pk, feat):
    """The tensor-core forward pass: BF16 operands (inputs, activations,
    weights), FP32-or-better accumulation, FP32 bias and normalisation."""
    pk = np.asarray(pk, np.float32)
    W1, W2, W3 = unpack_weights(pk)
    f = np.asarray(feat, np.float32)
    xn = (f - pk[O_FMEAN:O_FMEAN + MLP_IN]) * pk[O_FISTD:O_FISTD + MLP_IN]
    x = np.zeros((f.shape[0], 32), np.float64)
    x[:, :MLP_IN] = bf16_round(xn.astype(np.float32))
    h1 = silu(x @ W1.T + pk[O_B1:O_B1 + 64].astype(np.float64))
    h1 = bf16_round(h1.astype(np.float32)).astype(np.float64)
    h2 = silu(h1 @ W2.T + pk[O_B2:O_B2 + 64].astype(np.float64))
    h2 = bf16_round(h2.astype(np.float32)).astype(np.float64)
    o = h2 @ W3.T + pk[O_B3:O_B3 + 8].astype(np.float64)
    return o[:, :MLP_OUT] * pk[O_OSTD:O_OSTD + MLP_OUT] + pk[O_OMEAN:O_OMEAN + MLP_OUT]


def forward(theta, x):
    """FP64 forward of normalised inputs: (z1, h1, z2, h2, out)."""
    W1, b1, W2, b2, W3, b3 = split(theta)
    x = np.asarray(x, np.float64)
    z1 = x @ W1.T + b1
    h1 = silu(z1)
    z2 = h1 @ W2.T + b2
    h2 = silu(z2)
    return z1, h1, z2, h2, h2 @ W3.T + b3


def loss_grad(theta, x, y):
    """loss = mean over samples of the summed squared error; FP64 gradient."""
    W1, b1, W2, b2, W3, b3 = split(theta)
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = x.shape[0]
    z1, h1, z2, h2, out = forward(theta, x)
    e = out - y
    loss = float((e * e).sum() / n)
    d3 = 2.0 * e / n

    def dsilu(z):
        s = 1.0 / (1.0 + np.exp(-z))
        return s * (1.0 + z * (1.0 - s))

    d2 = (d3 @ W3) * dsilu(z2)
    d1 = (d2 @ W2) * dsilu(z1)
    g = np.zeros(N_PARAMS, np.float64)
    g[P_W1:P_B1] = (d1.T @ x).reshape(-1)
    g[P_B1:P_W2] = d1.sum(0)
    g[P_W2:P_B2] = (d2.T @ h1).reshape(-1)
    g[P_B2:P_W3] = d2.sum(0)
    g[P_W3:P_B3] = (d3.T @ h2).reshape(-1)
    g[P_B3:N_PARAMS] = d3.sum(0)
    return loss, g


def adam(theta, g, m, v, t, lr, b1, b2, eps):
    """One bias-corrected Adam step (float32, as the device kernel)."""
    f = np.float32
    g = np.asarray(g, f)
    m = f(b1) * np.asarray(m, f) + f(1.0 - b1) * g
    v = f(b2) * np.asarray(v, f) + f(1.0 - b2) * g * g
    c1, c2 = f(1.0 - b1 ** t), f(1.0 - b2 ** t)
    th = np.asarray(theta, f) - f(lr) * (m / c1) / (np.sqrt(v / c2) + f(eps))
    return th, m, v


def targets(lam, pen):
    """Training targets of contacts from their (lambda, penalty) state."""
    lam = np.asarray(lam, np.float64)
    pen = np.asarray(pen, np.float64)
    ln = lam[:, 0]
    sc = np.abs(ln) + 1.0
    return np.stack([np.log1p(np.maximum(-ln, 0.0)), lam[:, 1] / sc, lam[:, 2] / sc,
                     np.log(np.maximum(pen[:, 0], PEN_MIN))], axis=1)


def decode(y, depth, mus, zeta=1.0):
    """Targets -> (lambda [n,3], k_n [n], accepted [n]) with the fallbacks of
    the device path (separated contact, non-finite, outside the static cone);
    forces are scaled by zeta."""
    y = np.asarray(y, np.float64)
    ln0 = -np.expm1(np.maximum(y[:, 0], 0.0))
    sc = np.abs(ln0) + 1.0
    ln = zeta * ln0
    lt, lb = zeta * y[:, 1] * sc, zeta * y[:, 2] * sc
    kn = np.clip(np.exp(y[:, 3]), PEN_MIN, PEN_MAX)
    ok = (np.asarray(depth) > 0) & np.isfinite(ln) & np.isfinite(lt) & np.isfinite(lb) & \
        (np.sqrt(lt * lt + lb * lb) <= np.asarray(mus) * np.abs(ln))
    return np.stack([ln, lt, lb], axis=1), kn, ok


def _qmat(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _basis(n):
    """First tangent of orthonormal_basis_3d (kernels_6dof.py:2208-2220)."""
    sign = 1.0 if n[2] >= 0.0 else -1.0
    a = -1.0 / (sign + n[2])
    b = n[0] * n[1] * a
    return np.array([1.0 + sign * n[0] * n[0] * a, sign * b, -sign * n[0]])


def contact_features(xa, qa, va, wa, ma, ia, xb, qb, vb, wb, mb, ib, n, offa, offb, depth, mus, mu, sat):
    """The 20 features of one new contact (body a = reference body).  ia, ib
    are the body-frame principal inertias; offa/offb body-frame anchors."""
    n = np.asarray(n, np.float64)
    Ra, Rb = _qmat(np.asarray(qa, np.float64)), _qmat(np.asarray(qb, np.float64))
    na, nb = Ra.T @ n, Rb.T @ n
    ra, rb = Ra @ np.asarray(offa, np.float64), Rb @ np.asarray(offb, np.float64)
    vr = (np.asarray(va) + np.cross(wa, ra)) - (np.asarray(vb) + np.cross(wb, rb))
    t = _basis(n)
    bt = np.cross(n, t)
    nia = sum(na[k] ** 2 / ia[k] for k in range(3) if ia[k] > 0)
    nib = sum(nb[k] ** 2 / ib[k] for k in range(3) if ib[k] > 0)
    onehot = np.zeros(7)
    onehot[min(int(sat), 6)] = 1.0
    return np.concatenate([na, [depth], [vr @ t, vr @ bt, vr @ n], [1 / ma if ma > 0 else 0.0,
                           1 / mb if mb > 0 else 0.0], [nia, nib], [mus, mu], onehot])
