"""Writes golden fixtures derived from the reference's own test inputs, so that the
CPU tests can pin against them where the reference tree is absent.

Reads (from the reference checkout named by the HP_REFERENCE_DIR environment
variable): Testing/tri_hp/ins/Spatial Accuracy/Inputs/square7.grd, the 64 x 64
split-square mesh of the reference's Kovasznay spatial-accuracy test.
Writes: tests/golden/square7_grd.json with its entity counts and the SHA-256 of
its sorted triangle keys on the integer lattice (each triangle's three vertices
x*64, y*64 rounded, as key x*1000 + y, sorted within the triangle, triangles
sorted), which does not depend on the numbering of points or triangles.

Run: HP_REFERENCE_DIR=<reference checkout> python tests/golden/make_reference_fixtures.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "hp-multiphysics_b200"))


def tri_keys_sha256(pnts, tri_pnt, n):
    q = np.round(pnts[tri_pnt] * n).astype(np.int64)
    keys = np.sort(q[:, :, 0] * 1000 + q[:, :, 1], axis=1)
    keys = keys[np.lexsort(keys.T[::-1])]
    return hashlib.sha256(np.ascontiguousarray(keys).tobytes()).hexdigest()


def main():
    import hpb
    ref = os.environ.get("HP_REFERENCE_DIR")
    if not ref:
        raise SystemExit("set HP_REFERENCE_DIR to the reference checkout")
    g = hpb.read_grd(os.path.join(ref, "Testing/tri_hp/ins/Spatial Accuracy/Inputs/square7.grd"))
    out = {"source": "Testing/tri_hp/ins/Spatial Accuracy/Inputs/square7.grd",
           "npnt": int(g.npnt), "nseg": int(g.nseg), "ntri": int(g.ntri), "lattice": 64,
           "tri_keys_sha256": tri_keys_sha256(g.pnts, g.tri_pnt, 64)}
    with open(os.path.join(HERE, "square7_grd.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


if __name__ == "__main__":
    main()
