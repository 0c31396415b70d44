"""Learned preconditioner: the GPU network kernels against the CPU oracle, the
GPU training loop, and the A/B comparison against the plain Jacobi
preconditioner on held-out problem instances."""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import _lib as L
from hpb import learned as LR
from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu


def test_gradients_match_cpu_oracle():
    import torch
    widths = (17, 16, 16, 1)
    net = LR.MLP(widths, seed=3)
    rng = np.random.default_rng(0)
    X = rng.normal(size=(256, 17)).astype(np.float32)
    T = rng.normal(size=(256, 1)).astype(np.float32)
    net.set_norm(X.mean(0), X.std(0))
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    Md = torch.ones(1, device="cuda")
    g, loss = net.grad(Xd.data_ptr(), Td.data_ptr(), Md.data_ptr(), 256)
    go, lo = MO.grad(net.params().astype(np.float64), widths, X.mean(0), X.std(0), X, T, np.ones(1))
    # BF16 activations: a value within FP32 rounding of a BF16 boundary may round
    # differently on the two sides, so the bound is norm-wise
    assert np.linalg.norm(g - go) / np.linalg.norm(go) < 1e-4
    assert abs(loss - lo) / lo < 1e-5
    # forward pass
    Y = torch.empty((256, 1), device="cuda")
    net.forward(Xd.data_ptr(), Y.data_ptr(), 256)
    torch.cuda.synchronize()
    yo = MO.forward(net.params().astype(np.float64), widths, X.mean(0), X.std(0), X)[-1]
    assert np.max(np.abs(Y.cpu().numpy() - yo)) < 1e-4 * np.max(np.abs(yo))


def test_tensor_core_forward_matches_cpu_oracle():
    """The learned corrections' shape (17 -> 64 -> 64 -> 64 -> 1) runs its forward pass on the
    BF16 tensor cores (k_mlp_forward_mma); against the numpy oracle it agrees up to the order
    of the FP32 sums (an activation within FP32 rounding of a BF16 boundary may round the
    other way, so the bound is norm-wise), for a sample count that is not a multiple of 16."""
    import torch
    widths = (17, 64, 64, 64, 1)
    net = LR.MLP(widths, seed=5)
    rng = np.random.default_rng(2)
    n = 1000 + 7
    X = rng.normal(size=(n, 17)).astype(np.float32)
    net.set_norm(X.mean(0), X.std(0))
    Xd = torch.from_numpy(X).cuda()
    Y = torch.full((n, 1), np.nan, device="cuda")
    net.forward(Xd.data_ptr(), Y.data_ptr(), n)
    torch.cuda.synchronize()
    y = Y.cpu().numpy()
    yo = MO.forward(net.params().astype(np.float64), widths, X.mean(0), X.std(0), X)[-1]
    assert np.all(np.isfinite(y))
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) < 2e-3
    assert np.max(np.abs(y - yo)) < 2e-2 * np.max(np.abs(yo))


def test_training_reduces_loss():
    rng = np.random.default_rng(1)
    X = rng.normal(size=(4096, 17)).astype(np.float32)
    T = np.tanh(X[:, :1] - 0.5 * X[:, 1:2]).astype(np.float32)
    net, hist = LR.train(X, T, widths=(17, 32, 32, 1), steps=300, batch=1024, lr=3e-3)
    assert hist[-20:].mean() < 0.25 * hist[:5].mean()


def _instance(seed, n=32, p=4):
    r = np.random.default_rng(seed)
    ax, ay = r.uniform(-1, 1, 2)
    kc = 10 ** r.uniform(-3, -1.5)
    f = L.Field(L.HP_FIELD_QUADX, (ctypes.c_double * 4)(-1.0, 8.0, 0, 0))
    return lambda: hpb.cd_sinsin(n=n, p=p, ax=ax, ay=ay, kcond=kc, cfl=0.5, field=f, seed=seed)


def test_learned_preconditioner_ab():
    """Trained on solver-generated residual histories of 6 cd instances, the
    network is judged by the FP64 residual on 2 held-out instances: updates to a
    1e-8 drop with the learned correction against the plain Jacobi method."""
    F, T = [], []
    for s in range(6):
        f, t = LR.solver_samples(_instance(100 + s))
        F.append(f)
        T.append(t)
    net, hist = LR.train(np.concatenate(F), np.concatenate(T), steps=400)
    plain_total = learned_total = 0
    for s in (200, 201):
        upd = {}
        for learned in (False, True):
            g = _instance(s)().gpu()
            if learned:
                LR.attach(g, net, 1.0)
            h, sec, u = g.solve(drop=1e-8, max_updates=20000, check_every=10)
            assert h[-1] <= 1e-8
            upd[learned] = u
            g.close()
        plain_total += upd[False]
        learned_total += upd[True]
    print(f"updates to 1e-8: plain {plain_total}, learned {learned_total}")
    assert learned_total <= plain_total
