"""Learned boundary correction M = D P0 D of the CG preconditioner.

CPU: the oracle's analytic gradient against its own central finite differences.
GPU: the device loss and gradient (hand-written forward/backward kernels, FP64 transforms)
against the oracle's, and training on plain-CG pairs followed by solves to the 1e-8 FP64
true residual with and without the trained correction."""
import time

import numpy as np
import pytest

import pfb200
from helpers import desc_of, rel

CFG2 = dict(dim=2, cells=(40, 36), covariance="exponential", corr_length=(0.2, 0.05, -0.05, 0.15),
            anisotropy="geometric")
CFG3 = dict(dim=3, cells=(20, 16, 12), covariance="matern32", corr_length=(0.2, 0.1, 0.05),
            anisotropy="axiparallel")


def _theta(H, seed):
    r = np.random.default_rng(seed)
    return np.concatenate([-r.uniform(0.5, 4.0, H), r.uniform(-1, 1, H), 0.3 * r.standard_normal(H),
                           [0.05]])


def _pairs(oracle, d, lam, K, seed):
    g = oracle.resolve(d)
    r = np.random.default_rng(seed)
    B = r.standard_normal((K, g.domain))
    X = np.stack([oracle.matvec(d, lam, 2, b) * (1.0 + 0.1 * r.standard_normal(g.domain)) for b in B])
    return B, X


@pytest.mark.parametrize("residual", [False, True], ids=["solution-norm", "residual-norm"])
@pytest.mark.parametrize("cfg", [CFG2, CFG3], ids=["2d-geo", "3d-axi"])
def test_oracle_gradient_finite_differences(oracle, cfg, residual):
    d = desc_of(cfg)
    lam, st, status = oracle.spectrum(d)
    assert (lam > 0).all()
    H = 4
    th = _theta(H, 1)
    B, X = _pairs(oracle, d, lam, 2, 2)
    L, G = oracle.learned_loss_grad(d, lam, th, H, B, X, residual)
    for p in range(len(th)):
        h = 1e-6 * max(1.0, abs(th[p]))
        tp, tm = th.copy(), th.copy()
        tp[p] += h
        tm[p] -= h
        fd = (oracle.learned_loss_grad(d, lam, tp, H, B, X, residual)[0]
              - oracle.learned_loss_grad(d, lam, tm, H, B, X, residual)[0]) / (2 * h)
        assert abs(fd - G[p]) <= 1e-6 * max(1.0, abs(G).max()), (p, fd, G[p])


@pytest.mark.gpu
@pytest.mark.parametrize("residual", [False, True], ids=["solution-norm", "residual-norm"])
@pytest.mark.parametrize("cfg", [CFG2, CFG3], ids=["2d-geo", "3d-axi"])
def test_device_loss_and_gradient_match_oracle(oracle, cfg, residual):
    d = desc_of(cfg)
    P = pfb200.Plan(d)
    P.spectrum_build()
    lam, _, _ = oracle.spectrum(d)
    H = 6
    Lp = pfb200.Learned(P, hidden=H, seed=3, residual_loss=residual)
    th = _theta(H, 4)
    Lp.params = th
    B, X = _pairs(oracle, d, lam, 3, 5)
    loss, grad = Lp.loss_grad(B, X, fp32=False)
    L0, G0 = oracle.learned_loss_grad(d, lam, th, H, B, X, residual)
    assert abs(loss - L0) <= 1e-10 * abs(L0)
    assert rel(grad, G0) < 1e-9
    # the learned application equals D P0 D on the oracle
    r = np.random.default_rng(6).standard_normal(oracle.resolve(d).domain)
    D = oracle.learned_scale(d, th, H)
    assert rel(Lp.apply(r), D * oracle.matvec(d, lam, 2, D * r)) < 1e-11
    Lp.close()


CG_CFG = dict(dim=3, cells=(48, 48, 48), covariance="exponential",
              corr_length=(0.15, 0.02, 0.0, -0.03, 0.08, 0.01, 0.0, 0.02, 0.04), anisotropy="geometric",
              approximate=True)


def train_and_compare(P, d, K_train=16, K_test=8, epochs=60, H=8, seed=11, inner_fp32=True):
    """Pairs from plain CG, Adam training, then plain vs learned PCG on held-out RHS.
    Returns (loss0, loss1, plain_iters, learned_iters, plain_s, learned_s, residuals)."""
    import torch
    n = P.info.domain_size
    r = np.random.default_rng(seed)
    Bt = torch.tensor(r.standard_normal((K_train, n)), device="cuda")
    Xt = torch.empty_like(Bt)
    for i in range(K_train):
        P.multiply_inverse(Bt[i], x=Xt[i], mode=pfb200.CG_RESIDUAL, tolerance=1e-8, inner_fp32=inner_fp32)
    Lp = pfb200.Learned(P, hidden=H, seed=seed)
    loss0, _ = Lp.loss_grad(Bt, Xt, fp32=True)
    loss1 = Lp.train(Bt, Xt, epochs=epochs, lr=0.05, fp32=True)
    Bs = torch.tensor(r.standard_normal((K_test, n)), device="cuda")
    x = torch.empty(n, dtype=torch.float64, device="cuda")
    out = {}
    for name, attach in (("plain", False), ("learned", True)):
        Lp.attach(attach)
        P.multiply_inverse(Bs[0], x=x, mode=pfb200.CG_RESIDUAL, tolerance=1e-8, inner_fp32=inner_fp32)  # warm
        torch.cuda.synchronize()
        it, res = 0, []
        t0 = time.perf_counter()
        for i in range(K_test):
            _, rep = P.multiply_inverse(Bs[i], x=x, mode=pfb200.CG_RESIDUAL, tolerance=1e-8, inner_fp32=inner_fp32)
            it += rep["iterations"]
            res.append(rep["relative_residual"])
        torch.cuda.synchronize()
        out[name] = (it, time.perf_counter() - t0, max(res))
    Lp.attach(False)
    Lp.close()
    return loss0, loss1, out


@pytest.mark.gpu
def test_trained_correction_reaches_tolerance_and_reports_gain():
    """Trains on 16 plain-CG pairs, solves 8 held-out RHS to the 1e-8 FP64 true residual
    with both preconditioners; the learned run must meet the same residual (plain CG
    judges), must have lowered the training loss, and its iteration count is reported."""
    d = desc_of(CG_CFG)
    P = pfb200.Plan(d)
    P.spectrum_build()
    loss0, loss1, out = train_and_compare(P, d)
    print(f"loss {loss0:.4e} -> {loss1:.4e}; plain {out['plain']}, learned {out['learned']}")
    assert loss1 < loss0
    assert out["plain"][2] <= 1e-8 and out["learned"][2] <= 1e-8
    assert out["learned"][0] <= out["plain"][0]
