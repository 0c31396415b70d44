"""The learned correction of the tet smoother (hp_tet_set_prcn_scale / hp_tet_set_prcn_net):
a per-tetrahedron log-scale multiplies that tetrahedron's contributions to the Jacobian
diagonal (and to minvrt's blocks), so a zero scale changes nothing, a constant scale c
multiplies the diagonal by e^c, and a network trained on the solver's own samples and
attached to the finest level of the FP32 multigrid leaves the converged state the FP64 one."""
import ctypes

import numpy as np
import pytest

from hpb import learned as LR
from hpb.tet import TetGPU, TetHierarchy, TetProblem
from hpb.tetmesh import cube_tets

pytestmark = pytest.mark.gpu


def _level(n=3, p=3, re=100.0):
    pr = TetProblem(cube_tets(n), p, mu=1.0 / re, cfl=0.5).set_beltrami(re=re)
    masks, ff = pr.cube_boundary(re=re)
    g = TetGPU(pr)
    g.set_dirichlet(masks)
    g.set_flux_faces(ff)
    return g


def test_scale_multiplies_the_jacobian_diagonal():
    import torch
    g = _level()
    assert g.setup_preconditioner() == 0
    jd0 = g.jacobian_diagonal()
    for c in (0.0, 0.7):
        sc = torch.full((g.prob.mesh.ntet,), c, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        g.set_prcn_scale(ctypes.c_void_p(sc.data_ptr()), 1.5)
        jd = g.jacobian_diagonal()
        # the diagonal is a finite difference of the scaled contributions, accumulated with
        # FP64 atomics: equal up to the difference's rounding (~1e-16 / dw relative, dw ~ 1e-7)
        for a, b in zip(jd, jd0):
            if b.size == 0:
                continue
            assert np.allclose(a, np.exp(c) * b, rtol=1e-7, atol=1e-9 * np.max(np.abs(b)))
        g.set_prcn_scale(None)
    g.close()


def test_trained_network_keeps_the_fp64_state():
    F, T = [], []
    for k, re in enumerate((60.0, 150.0)):
        f, t = LR.tet_solver_samples(lambda re=re: _level(8, 3, re), snapshots=(0, 50))
        F.append(f)
        T.append(t)
    F, T = np.concatenate(F), np.concatenate(T)
    assert F.shape == (len(T), 17) and np.all(np.isfinite(F))
    net, hist = LR.train(F, T, steps=200)
    assert np.isfinite(hist).all()
    states = {}
    for learned in (False, True):
        H = TetHierarchy(8, 3, hlevels=2, mu=0.01, cfl={1: 2.2, 2: 1.5, 3: 0.5}, minvrt=True)
        if learned:
            H.levels[0].attach_net(net, 1.0)
        h, sec, nc = H.solve(drop=1e-8, max_cycles=400, vw=2, mixed=learned)
        assert h[-1] <= 1e-8
        states[learned] = H.levels[0].state()
        H.close()
    a, b = states[False], [x.copy() for x in states[True]]
    b[0][:, 3] += np.mean(a[0][:, 3]) - np.mean(b[0][:, 3])
    num = np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(a, b)))
    assert num / np.sqrt(sum(np.sum(x * x) for x in a)) < 1e-7
    net.close()
