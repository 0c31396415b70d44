"""Text restart files in the reference's layout (tri_hp/output.cpp:147-181 and
1384-1474): round trip at 8 significant digits, and reading at another p keeps the
shared modes (sides by index, interiors by (row, column)) and zeroes the others."""
import numpy as np

import hpb
from hpb import restart


def test_round_trip(tmp_path):
    pr = hpb.kovasznay_ins(n=4, p=4)
    f = tmp_path / "rstrt1_b0.txt"
    restart.write_text(f, 4, pr.ugv, pr.ugs, pr.ugi)
    lines = open(f).read().splitlines()
    assert lines[0] == "p0 = 4" and lines[2] == "END OF HEADER"
    assert lines[1] == f"npnt = {pr.mesh.npnt}, nseg = {pr.mesh.nseg}, ntri = {pr.mesh.ntri}"
    v, s, i = restart.read_text(f, 4, pr.mesh.npnt, pr.mesh.nseg, pr.mesh.ntri, 3)
    for a, b in ((v, pr.ugv), (s, pr.ugs), (i, pr.ugi)):
        assert np.allclose(a, b, rtol=1e-8, atol=1e-12 * np.max(np.abs(pr.ugv)))


def test_read_at_another_p(tmp_path):
    rng = np.random.default_rng(3)
    npnt, nseg, ntri, NV = 5, 7, 3, 2
    v = rng.uniform(-1, 1, (npnt, NV))
    s6 = rng.uniform(-1, 1, (nseg, 5, NV))
    i6 = rng.uniform(-1, 1, (ntri, 10, NV))
    f = tmp_path / "p6.txt"
    restart.write_text(f, 6, v, s6, i6)
    # down to p = 4: the first 3 side modes; interior rows (m, k) present at both degrees
    _, s4, i4 = restart.read_text(f, 4, npnt, nseg, ntri, NV)
    assert np.allclose(s4, s6[:, :3], rtol=1e-8)
    rows6 = [(m, k) for m in range(1, 5) for k in range(0, 5 - m)]
    rows4 = [(m, k) for m in range(1, 3) for k in range(0, 3 - m)]
    for j, mk in enumerate(rows4):
        assert np.allclose(i4[:, j], i6[:, rows6.index(mk)], rtol=1e-8)
    # back up to p = 8: the p = 6 modes in place, the new ones zero
    restart.write_text(f, 4, v, s4, i4)
    _, s8, i8 = restart.read_text(f, 8, npnt, nseg, ntri, NV)
    assert np.allclose(s8[:, :3], s4, rtol=1e-8) and np.all(s8[:, 3:] == 0)
    rows8 = [(m, k) for m in range(1, 7) for k in range(0, 7 - m)]
    for j, mk in enumerate(rows8):
        if mk in rows4:
            assert np.allclose(i8[:, j], i4[:, rows4.index(mk)], rtol=1e-8)
        else:
            assert np.all(i8[:, j] == 0)
