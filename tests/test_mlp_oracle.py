"""CPU checks of the learned-warm-start restatement (oracle/mlp_ref.py) that
the GPU tests use as their checker: its analytic gradient against central
finite differences, the BF16 rounding, the pack layout and the target
transform round trip."""

import numpy as np

from oracle import mlp_ref as M


def _rand_problem(n=37, seed=0):
    rng = np.random.default_rng(seed)
    th = rng.normal(0, 0.3, M.N_PARAMS)
    x = rng.normal(0, 1, (n, M.MLP_IN))
    y = rng.normal(0, 1, (n, M.MLP_OUT))
    return th, x, y


def test_gradient_matches_finite_differences():
    th, x, y = _rand_problem()
    _, g = M.loss_grad(th, x, y)
    rng = np.random.default_rng(1)
    # every bias, and a sample of each weight matrix
    idx = np.concatenate([np.arange(M.P_B1, M.P_W2), np.arange(M.P_B2, M.P_W3), np.arange(M.P_B3, M.N_PARAMS),
                          rng.choice(np.arange(M.P_W1, M.P_B1), 40, replace=False),
                          rng.choice(np.arange(M.P_W2, M.P_B2), 40, replace=False),
                          rng.choice(np.arange(M.P_W3, M.P_B3), 40, replace=False)])
    h = 1e-6
    for k in idx:
        tp, tm = th.copy(), th.copy()
        tp[k] += h
        tm[k] -= h
        fd = (M.loss_grad(tp, x, y)[0] - M.loss_grad(tm, x, y)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


def test_bf16_round_nearest_even():
    v = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.0e38, 1e-40], np.float32)
    r = M.bf16_round(v)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa (1.0) wins;
    # 1 + 3*2^-8 ties between 1+2^-7 and 1+2^-6: 1+2^-6 has the even mantissa
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2.0 ** -6)
    assert r[3] == -2.5
    assert (r.view(np.uint32) & 0xFFFF).max() == 0


def test_pack_layout_round_trip():
    th, _, _ = _rand_problem()
    norm = np.concatenate([np.arange(20) * 0.1, np.arange(1, 21) * 0.5, [1, 2, 3, 4], [5, 6, 7, 8], [0.75]])
    pk = M.pack(th, norm)
    W1, b1, W2, b2, W3, b3 = M.split(th)
    U1, U2, U3 = M.unpack_weights(pk)
    np.testing.assert_array_equal(U1[:, :20], M.bf16_round(W1.astype(np.float32)))
    assert not U1[:, 20:].any()
    np.testing.assert_array_equal(U2, M.bf16_round(W2.astype(np.float32)))
    np.testing.assert_array_equal(U3[:4], M.bf16_round(W3.astype(np.float32)))
    assert not U3[4:].any()
    np.testing.assert_allclose(pk[M.O_FISTD:M.O_FISTD + 20], 1.0 / norm[20:40], rtol=1e-7)
    np.testing.assert_array_equal(pk[M.O_B1:M.O_B1 + 64], b1.astype(np.float32))


def test_bf16_forward_close_to_fp64_forward():
    th, x, _ = _rand_problem(200)
    norm = np.concatenate([np.zeros(20), np.ones(20), np.zeros(4), np.ones(4), [1.0]])
    ref = M.forward(th, x.astype(np.float32))[-1]
    got = M.infer_bf16(M.pack(th, norm), x)
    assert np.abs(got - ref).max() < 0.05 * np.abs(ref).max()


def test_targets_decode_round_trip():
    rng = np.random.default_rng(3)
    ln = -rng.uniform(0, 5e4, 50)
    lt = rng.uniform(-0.3, 0.3, 50) * np.abs(ln)
    lb = rng.uniform(-0.3, 0.3, 50) * np.abs(ln)
    kn = np.exp(rng.uniform(np.log(1e6), np.log(1e9), 50))
    lam = np.stack([ln, lt, lb], 1)
    pen = np.stack([kn, np.ones(50), np.ones(50)], 1)
    y = M.targets(lam, pen)
    lam2, kn2, ok = M.decode(y, depth=np.full(50, 1e-3), mus=np.full(50, 0.5))
    np.testing.assert_allclose(lam2, lam, rtol=1e-9, atol=1e-6)
    np.testing.assert_allclose(kn2, kn, rtol=1e-9)
    assert ok.all()
    _, _, ok = M.decode(y, depth=np.full(50, -1e-3), mus=np.full(50, 0.5))  # separated: zero start
    assert not ok.any()
    _, _, ok = M.decode(y, depth=np.full(50, 1e-3), mus=np.full(50, 0.1))   # outside the cone
    assert (~ok).sum() > 0
