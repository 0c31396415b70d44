"""Learned correction of the Jacobi preconditioner (include/hp_mlp.h).

Training data come from the solver itself. For each problem instance, the
smoother runs K multistage updates from the same initial state under several
global log-scales c of the element preconditioner tprcn. The per-element
residual measure after the run (hp_gpu_elem_resnorm) is recorded for each c.
The target for an element is the log-scale whose run left it with the smallest
residual; it is 0 when no scale improves on the plain method by more than
`margin`. The network (17 -> 64 -> 64 -> 64 -> 1, BF16, FP32 accumulation) is
trained on the GPU by the library's own kernels (hp_mlp_train_step) and
attached with hp_gpu_set_prcn_net; the plain method is the fallback (detach,
or outputs clamped to 0).
"""
import ctypes

import numpy as np

from . import _lib as L

P = ctypes.c_void_p
_bound = False


def _bind():
    global _bound
    lib = L.lib()
    if _bound:
        return lib
    lib.hp_mlp_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_ulonglong, ctypes.POINTER(P)]
    lib.hp_mlp_destroy.argtypes = [P]
    lib.hp_mlp_nparams.argtypes = [P]
    lib.hp_mlp_dims.argtypes = [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.hp_mlp_set_norm.argtypes = [P, P, P]
    lib.hp_mlp_get_params.argtypes = [P, P]
    lib.hp_mlp_set_params.argtypes = [P, P]
    lib.hp_mlp_forward.argtypes = [P, P, ctypes.c_int, P, P]
    lib.hp_mlp_grad.argtypes = [P, P, P, P, ctypes.c_int, P, ctypes.POINTER(ctypes.c_float)]
    lib.hp_mlp_train_step.argtypes = [P, P, P, P, ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]
    lib.hp_mlp_last_error.restype = ctypes.c_char_p
    lib.hp_gpu_elem_features.argtypes = [P, P]
    lib.hp_gpu_elem_resnorm.argtypes = [P, P]
    lib.hp_gpu_set_prcn_scale.argtypes = [P, P, ctypes.c_int, ctypes.c_float]
    lib.hp_gpu_set_prcn_net.argtypes = [P, P, ctypes.c_float]
    _bound = True
    return lib


def _mcheck(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed ({rc}): {L.lib().hp_mlp_last_error().decode()}")


class MLP:
    """hp_mlp: device-resident network with hand-written BF16 kernels."""

    def __init__(self, widths=(17, 64, 64, 64, 1), seed=1):
        lib = _bind()
        self.widths = tuple(widths)
        w = (ctypes.c_int * len(widths))(*widths)
        h = P()
        _mcheck(lib.hp_mlp_create(len(widths) - 1, w, seed, ctypes.byref(h)), "hp_mlp_create")
        self.h = h
        self.lib = lib
        self.nparams = lib.hp_mlp_nparams(h)
        self.mean = np.zeros(widths[0], np.float32)
        self.std = np.ones(widths[0], np.float32)

    def close(self):
        if self.h:
            self.lib.hp_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_norm(self, mean, std):
        self.mean = np.ascontiguousarray(mean, np.float32)
        self.std = np.ascontiguousarray(std, np.float32)
        _mcheck(self.lib.hp_mlp_set_norm(self.h, L.ptr(self.mean), L.ptr(self.std)), "set_norm")

    def params(self):
        out = np.zeros(self.nparams, np.float32)
        _mcheck(self.lib.hp_mlp_get_params(self.h, L.ptr(out)), "get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _mcheck(self.lib.hp_mlp_set_params(self.h, L.ptr(p)), "set_params")

    def forward(self, x_dev, y_dev, n, stream=None):
        _mcheck(self.lib.hp_mlp_forward(self.h, P(x_dev), n, P(y_dev), stream), "forward")

    def grad(self, x_dev, t_dev, mask_dev, n):
        g = np.zeros(self.nparams, np.float32)
        loss = ctypes.c_float()
        _mcheck(self.lib.hp_mlp_grad(self.h, P(x_dev), P(t_dev), P(mask_dev), n, L.ptr(g), ctypes.byref(loss)),
                "grad")
        return g, loss.value

    def train_step(self, x_dev, t_dev, mask_dev, n, lr):
        loss = ctypes.c_float()
        _mcheck(self.lib.hp_mlp_train_step(self.h, P(x_dev), P(t_dev), P(mask_dev), n, lr, ctypes.byref(loss)),
                "train_step")
        return loss.value


def elem_features(level):
    """[ntri][17] float32 features of a GPULevel's current state (device -> host)."""
    import torch
    lib = _bind()
    m = level.prob.mesh
    d = torch.empty((m.ntri, 17), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()  # the buffer is written on the context's own stream
    L.check(lib.hp_gpu_elem_features(level.h, P(d.data_ptr())), "elem_features")
    L.check(lib.hp_gpu_sync(level.h), "sync")
    return d.cpu().numpy()


def elem_resnorm(level):
    """Per-element residual measure of rsdl(nstage) at the current state."""
    import torch
    lib = _bind()
    m = level.prob.mesh
    level.rsdl(level.prob.phys.nstage)
    d = torch.empty(m.ntri, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # the buffer is written on the context's own stream
    L.check(lib.hp_gpu_elem_resnorm(level.h, P(d.data_ptr())), "elem_resnorm")
    L.check(lib.hp_gpu_sync(level.h), "sync")
    return d.cpu().numpy()


def solver_samples(prob_factory, scales=(-1.0, -0.6, -0.3, 0.0, 0.3), k_updates=8, margin=0.02, snapshots=(0,)):
    """(features, targets) from one problem instance, generated by the solver. With
    `snapshots` (cumulative plain-update counts), the instance is first smoothed by the
    plain method to each snapshot and every snapshot state gives one sample per element,
    so the network also sees the states later in a solve."""
    import torch
    lib = _bind()
    pr = prob_factory()
    g = pr.gpu()
    state = (pr.ugv.copy(), pr.ugs.copy(), pr.ugi.copy())
    ntri = pr.mesh.ntri
    F, Tg = [], []
    done = 0
    for snap in sorted(snapshots):
        if snap > done:
            g.upload(*state)
            assert g.setup_preconditioner() == 0
            g.iterate(snap - done, prcn_interval=0)
            state = g.state()
            done = snap
        g.upload(*state)
        feats = elem_features(g)
        ratios = []
        for c in scales:
            g.upload(*state)
            sc = torch.full((ntri, 1), float(c), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()  # the context reads it on its own stream
            L.check(lib.hp_gpu_set_prcn_scale(g.h, P(sc.data_ptr()), 1, 1.5), "set_prcn_scale")
            assert g.setup_preconditioner() == 0
            r0 = elem_resnorm(g)
            g.iterate(k_updates, prcn_interval=0)
            rk = elem_resnorm(g)
            ratios.append(np.sqrt(rk / np.maximum(r0, 1e-300)))
            L.check(lib.hp_gpu_set_prcn_scale(g.h, None, 1, 0.0), "set_prcn_scale")
            del sc
        R = np.array(ratios)  # [nscales][ntri]
        base = R[list(scales).index(0.0)]
        best = np.argmin(R, axis=0)
        tgt = np.array(scales)[best]
        tgt[(R[best, np.arange(ntri)] > (1.0 - margin) * base) | ~np.isfinite(R).all(axis=0)] = 0.0
        F.append(feats)
        Tg.append(tgt.astype(np.float32))
    g.close()
    return np.concatenate(F), np.concatenate(Tg)


def tet_solver_samples(level_factory, scales=(-1.0, -0.6, -0.3, 0.0, 0.3), k_updates=8, margin=0.02,
                       snapshots=(0,), jacobi=True):
    """(features, targets) of the tet smoother's learned correction from one instance,
    generated by the solver as solver_samples does for tri_hp: level_factory() returns a
    hpb.tet.TetGPU with its boundary set; at each snapshot state (cumulative plain
    updates), every tetrahedron's target is the global log-scale of the smoother's diagonal
    (JACOBI: the Jacobian diagonal; minvrt: its diagonal blocks) whose k_updates left that
    tetrahedron with the smallest residual, 0 where none beats the plain method by margin.
    jacobi=False: the level smooths with minvrt (its factory called set_smoother(1))."""
    import torch
    g = level_factory()
    pr = g.prob
    ntet = pr.mesh.ntet
    state = tuple(a.copy() for a in pr.state)

    def prepare():
        assert g.setup_preconditioner() == 0
        if jacobi:
            g.jacobian_diagonal()

    F, Tg = [], []
    done = 0
    for snap in sorted(snapshots):
        if snap > done:
            g.upload(*state)
            g.set_prcn_scale(None)
            prepare()
            g.iterate(snap - done)
            state = tuple(g.state())
            done = snap
        g.upload(*state)
        feats = g.elem_features()
        ratios = []
        for c in scales:
            g.upload(*state)
            sc = torch.full((ntet,), float(c), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            g.set_prcn_scale(ctypes.c_void_p(sc.data_ptr()), 1.5)
            prepare()
            r0 = g.elem_resnorm()
            g.iterate(k_updates)
            rk = g.elem_resnorm()
            ratios.append(np.sqrt(rk / np.maximum(r0, 1e-300)))
            g.set_prcn_scale(None)
            del sc
        R = np.array(ratios)
        base = R[list(scales).index(0.0)]
        best = np.argmin(R, axis=0)
        tgt = np.array(scales)[best]
        tgt[(R[best, np.arange(ntet)] > (1.0 - margin) * base) | ~np.isfinite(R).all(axis=0)] = 0.0
        ok = np.isfinite(feats).all(axis=1)  # a snapshot state the plain smoother blew up gives no samples
        F.append(feats[ok])
        Tg.append(tgt[ok].astype(np.float32))
    g.close()
    return np.concatenate(F), np.concatenate(Tg)


def train(feats, targets, widths=(17, 64, 64, 64, 1), steps=400, batch=4096, lr=2e-3, seed=1, log=None):
    """Trains an MLP on (features, targets) on the GPU; returns (net, loss history)."""
    import torch
    net = MLP(widths, seed=seed)
    mean = feats.mean(axis=0)
    std = feats.std(axis=0) + 1e-6
    net.set_norm(mean, std)
    X = torch.from_numpy(np.ascontiguousarray(feats, np.float32)).cuda()
    T = torch.from_numpy(np.ascontiguousarray(targets.reshape(len(targets), -1), np.float32)).cuda()
    M = torch.ones(T.shape[1], dtype=torch.float32, device="cuda")
    rng = np.random.default_rng(seed)
    hist = []
    n = X.shape[0]
    for s in range(steps):
        idx = torch.from_numpy(rng.integers(0, n, size=min(batch, n))).cuda()
        xb = X.index_select(0, idx).contiguous()
        tb = T.index_select(0, idx).contiguous()
        torch.cuda.synchronize()
        hist.append(net.train_step(xb.data_ptr(), tb.data_ptr(), M.data_ptr(), xb.shape[0], lr))
        if log and s % 50 == 0:
            log(f"step {s} loss {hist[-1]:.4e}")
    return net, np.array(hist)


def attach(level, net, clampv=1.0):
    _bind()
    L.check(level.lib.hp_gpu_set_prcn_net(level.h, net.h if net is not None else None, clampv), "set_prcn_net")
