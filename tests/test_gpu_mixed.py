"""FP32 correction smoothing with FP64 defect correction against plain FP64
smoothing, on the GPU: both reach the 1e-10 drop of the FP64 residual and give
the same converged field (relative difference below 1e-9 in the coefficient
2-norm; both are converged only to the 1e-10 residual drop, so they agree to
that level, not to rounding)."""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import _lib as L

pytestmark = pytest.mark.gpu


def quad_field():
    return L.Field(L.HP_FIELD_QUADX, (ctypes.c_double * 4)(-1.0, 8.0, 0, 0))


@pytest.mark.parametrize("kind", ["cd", "ins"])
def test_mixed_matches_fp64(kind):
    if kind == "cd":
        mk = lambda: hpb.cd_sinsin(n=16, p=4, kcond=1e-2, cfl=0.5, field=quad_field())
    else:
        mk = lambda: hpb.kovasznay_ins(n=6, p=2, re=20.0)
    pa, pb = mk(), mk()
    ga, gb = pa.gpu(), pb.gpu()
    ha, sa, ua = ga.solve(mixed=False, drop=1e-10, max_updates=30000, check_every=20)
    hb, sb, ub = gb.solve(mixed=True, drop=1e-10, max_updates=30000, inner=30)
    assert ha[-1] <= 1e-10, ha[-5:]
    assert hb[-1] <= 1e-10, hb[-5:]
    sa_, sb_ = ga.state(), gb.state()
    num = np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(sa_, sb_)))
    den = np.sqrt(sum(np.sum(x ** 2) for x in sa_))
    assert num / den < 1e-9, num / den
