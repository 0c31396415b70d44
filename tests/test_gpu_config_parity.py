"""GPU parity against the CPU oracle at a configuration's stated size and at convergence.

* C1 as stated: ins Kovasznay, Re 100, 64 x 64 split squares (8,192 triangles), p = 4,
  state = the analytic field projected plus 1e-3 seeded noise; one rsdl, then 100
  multistage updates with the Jacobi preconditioner. The GPU state after 100 updates
  against the oracle's to 1e-10 of max |state|, the maxres history to 1e-9 relative.
* One multigrid W-cycle (block::cycle with vwcycle 2 over p-levels 4 -> 2 -> 1 and one
  h-level) on the GPU against the oracle's restatement of the cycle (tri_hp::mg_restrict,
  mg_prolongate, mg_source): the fine state to 1e-10.
* Converged fields: the oracle converges a small cd and a small ins hierarchy to a 1e-12
  drop of the FP64 residual; the GPU's plain FP64 multigrid, FP32 defect correction and
  learned + FP32 defect correction, each converged to the same drop, must be within 1e-10
  relative L2 of the oracle's converged state.
"""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import learned as LR
from hpb import multigrid as MG
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOLN = 1e-10


def relerr(a, b):
    a = np.concatenate([np.ravel(x) for x in a])
    b = np.concatenate([np.ravel(x) for x in b])
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def rel_l2(a, b):
    num = np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(a, b)))
    return num / np.sqrt(sum(np.sum(y * y) for y in b))


def test_c1_as_stated_rsdl_and_100_updates():
    pr = hpb.kovasznay_ins(n=64, p=4, re=100.0, noise=1e-3)
    assert pr.mesh.ntri == 8192 and pr.ndof == 198147
    g = pr.gpu()
    o = O.Oracle(pr)
    assert g.setup_preconditioner() == 0 and o.setup_preconditioner() == 0
    g.rsdl(pr.phys.nstage)
    o.rsdl(pr.phys.nstage)
    assert relerr(g.residual(), o.residual()) < 1e-12
    hist = g.iterate(100)
    oh = []
    for _ in range(100):
        o.update()
        oh.append(o.maxres()[0])
    oh = np.array(oh)
    assert relerr(g.state(), o.state()) < TOLN
    assert np.max(np.abs(hist - oh) / oh) < 1e-9
    g.close()


def _hier(kind):
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_oracle_multigrid import hierarchy
    return hierarchy(kind)


@pytest.mark.parametrize("kind", ["cd", "ins"])
def test_one_w_cycle_matches_oracle(kind):
    probs, kinds = _hier(kind)
    G = MG.Hierarchy(probs, kinds)
    H = O.OracleHierarchy(probs, kinds)
    lib = G.lib
    for ncyc in (1, 2):
        hp = (ctypes.c_void_p * len(G.levels))(*[lv.h for lv in G.levels])
        assert lib.hp_gpu_vcycle(hp, len(G.levels), 2, 2, 2, 1) == 0
        assert H.cycle(vw=2, itercrsn=2, iterrfne=2, eval_prcn=True) == 0
        assert relerr(G.levels[0].state(), H.levels[0].state()) < TOLN, f"after {ncyc} cycles"
        # the coarsest level's state after its last smoothing
        assert relerr(G.levels[-1].state(), H.levels[-1].state()) < TOLN
    G.close()


@pytest.mark.parametrize("kind", ["cd", "ins"])
def test_converged_states_match_converged_oracle(kind):
    probs, kinds = _hier(kind)
    H = O.OracleHierarchy(probs, kinds)
    oh, onc = H.solve(drop=1e-12, max_cycles=300, vw=2)
    assert oh[-1] <= 1e-12
    uo = H.levels[0].state()
    net = LR.MLP((17, 64, 64, 64, 1), seed=5)  # an untrained network: any correction must keep the fixed point
    errs = {}
    for arm, mixed, learned in (("fp64", False, False), ("fp32_defect_correction", True, False),
                                ("learned_fp32", True, True)):
        G = MG.Hierarchy(probs, kinds)
        if learned:
            LR.attach(G.levels[0], net, 0.5)
        h, sec, nc = G.solve(drop=1e-12, max_cycles=300, vw=2, mixed=mixed)
        assert h[-1] <= 1e-12, (arm, h[-3:])
        errs[arm] = rel_l2(G.levels[0].state(), uo)
        G.close()
    net.close()
    print(kind, errs)
    for arm, e in errs.items():
        assert e < TOLN, (arm, e)
