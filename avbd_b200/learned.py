"""Learned warm start for new contacts.

A contact that misses the contact cache starts, in the reference, from
lambda = 0 and penalties (1e6, 1, 1) (gpu_pool_emit_rows,
src/avbd3d/kernels_6dof.py:2864-2879); the dual updates then ramp the
penalty and the force up over the iterations.  The warm start predicts the
cached state the contact would have had -- (lambda_n, lambda_t1, lambda_t2,
k_n) -- from 20 local features, so the prelude (kernels_6dof.py:1596-1609)
starts it near its converged force.  No counterpart exists in the reference.

Everything numeric runs in libavbd6: the BF16 tensor-core inference fused
into the prelude phase of the solve kernel (and avbd_mlp_infer), the FP32
forward/backward (avbd_mlp_loss_grad) and Adam (avbd_mlp_adam).  Python
holds the parameters, normalisation and the training loop.

Targets (per contact): y0 = log1p(-lambda_n), y1 = lambda_t1 / (|lambda_n|+1),
y2 = lambda_t2 / (|lambda_n|+1), y3 = log k_n; features and targets are
z-scored with statistics of the training set, stored with the weights.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

from . import _lib

PEN_MIN = 1.0e6
P_W1, P_B1, P_W2, P_B2, P_W3, P_B3 = 0, 1280, 1344, 5440, 5504, 5760
SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warm_start_pile.npz")


def _ptr(t: torch.Tensor) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform(+-1/sqrt(fan_in)) weights, zero biases."""
    rng = np.random.default_rng(seed)
    th = np.zeros(_lib.MLP_PARAMS, np.float32)
    for lo, rows, cols in ((P_W1, 64, 20), (P_W2, 64, 64), (P_W3, 4, 64)):
        b = 1.0 / np.sqrt(cols)
        th[lo:lo + rows * cols] = rng.uniform(-b, b, rows * cols)
    return th


def targets(lam: np.ndarray, pen: np.ndarray) -> np.ndarray:
    """Training targets from contacts' (lambda, penalty) states [n, >=3]."""
    lam = np.asarray(lam, np.float64)
    ln = lam[:, 0]
    sc = np.abs(ln) + 1.0
    return np.stack([np.log1p(np.maximum(-ln, 0.0)), lam[:, 1] / sc, lam[:, 2] / sc,
                     np.log(np.maximum(np.asarray(pen, np.float64)[:, 0], PEN_MIN))], axis=1).astype(np.float32)


class WarmStartMLP:
    """Parameters + normalisation of the warm-start network.  Pass an
    instance as Solver6DOF(mlp_warm_start=...) or assign solver.warm_start;
    `enabled` switches it off without reallocating the solver."""

    n_floats = _lib.MLP_FLOATS

    def __init__(self, theta=None, norm=None, seed: int = 0):
        self.theta = init_params(seed) if theta is None else np.asarray(theta, np.float32).copy()
        if norm is None:
            norm = np.concatenate([np.zeros(20), np.ones(20), np.zeros(4), np.ones(4)])
        norm = np.asarray(norm, np.float32)
        if norm.shape[0] == 48:
            norm = np.concatenate([norm, [1.0]]).astype(np.float32)
        self.norm = norm.copy()  # feature mean/std, target mean/std, lambda scale zeta
        self.enabled = True

    @property
    def zeta(self) -> float:
        """Scale applied to the predicted forces (a conservative start when < 1)."""
        return float(self.norm[48])

    @zeta.setter
    def zeta(self, z: float) -> None:
        self.norm[48] = float(z)

    # ---- persistence --------------------------------------------------------
    def save(self, path: str, **meta) -> None:
        np.savez(path, theta=self.theta, norm=self.norm, **meta)

    @classmethod
    def load(cls, path: str = SHIPPED) -> "WarmStartMLP":
        z = np.load(path)
        return cls(theta=z["theta"], norm=z["norm"])

    # ---- device views -------------------------------------------------------
    def packed(self, device) -> torch.Tensor:
        """The packed BF16 inference block on `device` (avbd_mlp_pack)."""
        L = _lib.load()
        th = torch.as_tensor(self.theta, device=device)
        nm = torch.as_tensor(self.norm, device=device)
        out = torch.empty(self.n_floats, dtype=torch.float32, device=device)
        st = torch.cuda.current_stream(device)
        _lib.check(L.avbd_mlp_pack(_ptr(th), _ptr(nm), _ptr(out), C.c_void_p(st.cuda_stream)), "mlp_pack")
        st.synchronize()
        return out

    def infer(self, feat, device="cuda") -> np.ndarray:
        """Denormalised targets [n, 4] of raw features [n, 20] on the tensor cores."""
        L = _lib.load()
        f = torch.as_tensor(np.ascontiguousarray(feat, np.float32), device=device)
        n = int(f.shape[0])
        out = torch.empty((max(n, 1), 4), dtype=torch.float32, device=device)
        pk = self.packed(device)
        st = torch.cuda.current_stream(device)
        _lib.check(L.avbd_mlp_infer(_ptr(pk), _ptr(f), n, _ptr(out), C.c_void_p(st.cuda_stream)), "mlp_infer")
        st.synchronize()
        return out[:n].cpu().numpy()

    # ---- training -----------------------------------------------------------
    def fit(self, feat: np.ndarray, targ: np.ndarray, epochs: int = 40, batch: int = 4096, lr: float = 2e-3,
            seed: int = 0, device="cuda", lr_final: float = 1e-4) -> list:
        """Fits normalisation and weights to (raw features, targets); returns
        the mean training loss of each epoch (normalised units)."""
        L = _lib.load()
        feat = np.asarray(feat, np.float64)
        targ = np.asarray(targ, np.float64)
        fm, fs = feat.mean(0), feat.std(0)
        tm, ts = targ.mean(0), targ.std(0)
        fs[fs < 1e-6] = 1.0
        ts[ts < 1e-6] = 1.0
        self.norm = np.concatenate([fm, fs, tm, ts, [self.zeta]]).astype(np.float32)
        X = torch.as_tensor(((feat - fm) / fs).astype(np.float32), device=device)
        Y = torch.as_tensor(((targ - tm) / ts).astype(np.float32), device=device)
        n = int(X.shape[0])
        batch = min(batch, n)
        th = torch.as_tensor(self.theta, device=device).clone()
        m = torch.zeros_like(th)
        v = torch.zeros_like(th)
        g = torch.zeros_like(th)
        loss = torch.zeros(1, dtype=torch.float32, device=device)
        nbytes = int(L.avbd_mlp_scratch_bytes(batch))
        scratch = torch.empty(nbytes // 4 + 1, dtype=torch.float32, device=device)
        gen = torch.Generator(device="cpu").manual_seed(seed)
        st = torch.cuda.current_stream(device)
        sp = C.c_void_p(st.cuda_stream)
        hist, t = [], 0
        steps = epochs * ((n + batch - 1) // batch)
        for ep in range(epochs):
            perm = torch.randperm(n, generator=gen).to(device)
            tot = torch.zeros((), dtype=torch.float32, device=device)
            nb = 0
            for s0 in range(0, n, batch):
                idx = perm[s0:s0 + batch]
                xb, yb = X.index_select(0, idx).contiguous(), Y.index_select(0, idx).contiguous()
                _lib.check(L.avbd_mlp_loss_grad(_ptr(th), _ptr(xb), _ptr(yb), int(xb.shape[0]), _ptr(g), _ptr(loss),
                                                _ptr(scratch), nbytes, sp), "mlp_loss_grad")
                t += 1
                # cosine decay from lr to lr_final
                lr_t = lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * min(1.0, (t - 1) / max(1, steps))))
                _lib.check(L.avbd_mlp_adam(_ptr(th), _ptr(g), _ptr(m), _ptr(v), t, C.c_float(lr_t), C.c_float(0.9),
                                           C.c_float(0.999), C.c_float(1e-8), sp), "mlp_adam")
                tot += loss[0]
                nb += 1
            hist.append(float(tot.item()) / nb)
        self.theta = th.cpu().numpy()
        return hist


# ---- data collection and evaluation ----------------------------------------
def collect_converged(solver, iterations: int = 50):
    """Training samples from the solver's current state: one substep of
    `iterations` iterations is run from the plain zero start with the contact
    cache emptied, so every contact is new and logged with its 20 features
    at emission; each contact is labelled with the state it converged to --
    (lambda n/t1/t2, penalty n) at the end of that substep.  The solver's
    state and iteration count are restored afterwards.  Returns (features
    [n, 20], targets [n, 4])."""
    sd = solver.state_dict()
    log0, it0 = solver.log_new_contacts, solver.iterations
    ws = solver.warm_start
    en0 = ws.enabled if ws is not None else None
    if ws is not None:
        ws.enabled = False
    solver.log_new_contacts = True  # may re-flush (bodies kept): reload the state
    solver.load_state_dict(sd)
    solver.clear_contact_cache()
    solver.iterations = int(iterations)
    try:
        solver.substep()
        feat, gid = solver.new_contact_log()
        lam, pen = solver.group_state(gid)
    finally:
        solver.iterations = it0
        solver.log_new_contacts = log0
        if ws is not None:
            ws.enabled = en0
        solver.load_state_dict(sd)
    return feat, targets(lam[:, 0:3], pen[:, 0:3])


def cold_start_violation(solver, iterations: int = 64, learned: bool = True, clear_cache: bool = True):
    """Max constraint violation over all rows after each iteration of one
    substep from the solver's current state -- with the contact cache emptied
    (every contact new) unless `clear_cache` is False, with or without the
    learned warm start -- and the substep's stats (with the per-iteration max
    violation over the box-box contacts as stats["contact_violation"]).  The
    state is restored afterwards."""
    sd = solver.state_dict()
    it0, rv0 = solver.iterations, solver.record_violation
    ws = solver.warm_start
    en0 = ws.enabled if ws is not None else None
    if ws is not None:
        ws.enabled = bool(learned)
    if clear_cache:
        solver.clear_contact_cache()
    solver.iterations = iterations
    solver.record_violation = True
    solver.substep()
    hist = solver.violation_history()
    stats = solver.stats()
    stats["contact_violation"] = solver.contact_violation_history()
    solver.iterations, solver.record_violation = it0, rv0
    if ws is not None:
        ws.enabled = en0
    solver.load_state_dict(sd)
    return hist, stats


def iterations_to(hist: np.ndarray, tol: float = 1e-4) -> int:
    """First iteration count whose violation is <= tol (len(hist)+1 if none)."""
    ok = np.nonzero(np.asarray(hist) <= tol)[0]
    return int(ok[0]) + 1 if ok.size else len(hist) + 1
