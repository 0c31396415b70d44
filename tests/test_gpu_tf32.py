"""The FP32 smoother's TF32 tensor-core element kernel (correction form) against the scalar
FP32 kernel: multigrid inside FP64 defect correction reaches the 1e-10 drop of the FP64
residual in about as many cycles, and the converged state is the FP64 one."""
import numpy as np
import pytest

import hpb
from hpb import multigrid as MG

pytestmark = pytest.mark.gpu


def _solve(elem, p, mixed=True):
    mk = lambda n, p, **kw: hpb.kovasznay_ins(n=n, p=p, re=100.0, **kw)
    H = MG.build(mk, n=16, p=p, hlevels=2)
    if elem != "default":
        for lv in H.levels:
            lv.element_kernel(elem)
    h, sec, nc = H.solve(drop=1e-10, max_cycles=400, mixed=mixed, vw=2)
    u = H.levels[0].state()
    H.close()
    return h, nc, u


@pytest.mark.parametrize("p", [2, 4, 6])
def test_tf32_correction_smoother_converges_like_fp32(p):
    h64, c64, u64 = _solve("tensor", p, mixed=False)
    ht, ct, ut = _solve("tensor", p)
    hs, cs, us = _solve("scalar", p)
    assert h64[-1] <= 1e-10 and ht[-1] <= 1e-10 and hs[-1] <= 1e-10, (h64[-2:], ht[-2:], hs[-2:])
    assert ct <= 1.15 * cs + 2, (ct, cs)
    for u in (ut, us):
        num = np.sqrt(sum(np.sum((a - b) ** 2) for a, b in zip(u, u64)))
        den = np.sqrt(sum(np.sum(a * a) for a in u64))
        assert num / den < 1e-9


def test_default_kernels_with_the_point_kernel_converge_like_scalar():
    """The default kernels of a p = 2 hierarchy (scalar at p = 2, the point kernel on the
    p = 1 levels, in the FP64 defect residual and in the FP32 smoother's correction form)
    reach the drop in the cycles of the all-scalar hierarchy, and the FP64 state."""
    h64, c64, u64 = _solve("scalar", 2, mixed=False)
    hd, cd, ud = _solve("default", 2)
    hs, cs, us = _solve("scalar", 2)
    assert hd[-1] <= 1e-10 and hs[-1] <= 1e-10
    assert abs(cd - cs) <= 2, (cd, cs)
    num = np.sqrt(sum(np.sum((a - b) ** 2) for a, b in zip(ud, u64)))
    den = np.sqrt(sum(np.sum(a * a) for a in u64))
    assert num / den < 1e-9
