"""CPU tests of the oracle's multigrid restatement (tri_hp::mg_restrict / mg_prolongate /
mg_source, block::cycle): the transfers keep a state that the coarse level leaves
unchanged, the FAS source makes the restricted state a fixed point of the coarse
residual, and V/W-cycles over p- and h-levels converge to a 1e-10 drop of the FP64
residual (the ins Convergence test's multigrid shape, Testing/tri_hp/ins/Convergence)."""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import _lib as L
from oracle import oracle as O


def quad():
    return L.Field(L.HP_FIELD_QUADX, (ctypes.c_double * 4)(-1.0, 8.0, 0, 0))


def hierarchy(kind, n=8, p=4):
    if kind == "cd":
        mk = lambda n, p, **kw: hpb.cd_sinsin(n=n, p=p, kcond=1e-2, field=quad(), **kw)
        cfl = {4: 0.5, 2: 0.75, 1: 1.0}
    else:
        mk = lambda n, p, **kw: hpb.kovasznay_ins(n=n, p=p, re=100.0, **kw)
        cfl = {4: 1.0, 2: 1.5, 1: 2.5}
    probs = [mk(n=n, p=p, cfl=cfl[p]), mk(n=n, p=2, cfl=cfl[2]), mk(n=n, p=1, cfl=cfl[1]),
             mk(n=n // 2, p=1, cfl=cfl[1])]
    return probs, ["fine", "p", "p", "h"]


@pytest.mark.parametrize("kind", ["cd", "ins"])
def test_restrict_then_prolongate_keeps_the_state(kind):
    probs, kinds = hierarchy(kind)
    H = O.OracleHierarchy(probs, kinds)
    lv = H.levels
    for l in range(1, len(lv)):
        assert lv[l - 1].setup_preconditioner() == 0
        before = lv[l - 1].state()
        lv[l - 1].rsdl(probs[l - 1].phys.nstage)
        O.lib().or_mg_restrict(lv[l].h)
        O.lib().or_mg_prolongate(lv[l].h)
        after = lv[l - 1].state()
        for a, b in zip(before, after):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("kind", ["cd", "ins"])
def test_fas_source_makes_the_restricted_state_a_fixed_point(kind):
    """With fadd = 1 the driving term dres = res0 - R_c(u_c) makes the coarse residual at
    the restricted state equal the restricted fine residual res0 (mg_source,
    nstage.cpp:113-129)."""
    probs, kinds = hierarchy(kind)
    H = O.OracleHierarchy(probs, kinds)
    f, c = H.levels[0], H.levels[1]
    assert f.setup_preconditioner() == 0 and c.setup_preconditioner() == 0
    f.rsdl(probs[0].phys.nstage)
    rf = f.residual()
    O.lib().or_mg_restrict(c.h)
    c.rsdl(probs[1].phys.nstage)
    rc = c.residual()
    sm_c = probs[1].p - 1
    assert np.allclose(rc[0], rf[0], rtol=0, atol=1e-13 * np.max(np.abs(rf[0])))
    assert np.allclose(rc[1], rf[1][:, :sm_c], rtol=0, atol=1e-13 * np.max(np.abs(rf[1])))


@pytest.mark.parametrize("kind,vw,max_cycles", [("cd", 1, 60), ("cd", 2, 40), ("ins", 2, 150)])
def test_oracle_cycles_converge(kind, vw, max_cycles):
    probs, kinds = hierarchy(kind)
    H = O.OracleHierarchy(probs, kinds)
    hist, nc = H.solve(drop=1e-10, max_cycles=max_cycles, vw=vw)
    assert hist[-1] <= 1e-10, (nc, hist[-3:])
    assert np.all(np.diff(np.log(hist[1:])) < 0.5)  # no growth beyond noise
