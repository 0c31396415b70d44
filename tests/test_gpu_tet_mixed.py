"""FP32 smoothing of the 3D tet_hp ins path inside FP64 defect correction
(hp_tet_solve_mg_mixed): the TF32 tensor-core residual in correction form with FP32
relaxation, minvrt and transfers reaches the FP64 residual drop in about as many cycles as
the FP64 multigrid, and to the same state (the pressure level, free with velocity given on
every face, set equal)."""
import numpy as np
import pytest

from hpb.tet import TetHierarchy

pytestmark = pytest.mark.gpu


def _rel_mod_pressure(a, b):
    b = [x.copy() for x in b]
    b[0][:, 3] += np.mean(a[0][:, 3]) - np.mean(b[0][:, 3])
    num = np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(a, b)))
    return num / np.sqrt(sum(np.sum(x * x) for x in a))


@pytest.mark.parametrize("minvrt", [True, False])
def test_tet_mixed_multigrid_converges_like_fp64(minvrt):
    cfl = {1: 2.2, 2: 1.5, 3: 0.5} if minvrt else {1: 0.5, 2: 0.5, 3: 0.5}
    out = {}
    for mixed in (False, True):
        H = TetHierarchy(8, 3, hlevels=2, mu=0.01, cfl=cfl, minvrt=minvrt)
        hist, sec, cyc = H.solve(drop=1e-8, max_cycles=400, vw=2, mixed=mixed)
        out[mixed] = (hist, cyc, H.levels[0].state())
        H.close()
    (h64, c64, u64), (h32, c32, u32) = out[False], out[True]
    assert h64[-1] <= 1e-8 and h32[-1] <= 1e-8, (h64[-2:], h32[-2:])
    assert c32 <= 1.2 * c64 + 3, (c32, c64)
    assert _rel_mod_pressure(u64, u32) < 1e-7


def test_tet_mixed_rejects_outflow_faces():
    H = TetHierarchy(4, 2, hlevels=1, mu=0.01, outflow=True)
    with pytest.raises(RuntimeError, match="inflow"):
        H.solve(drop=1e-8, max_cycles=2, vw=1, mixed=True)
    H.close()
