"""The algorithmic flop table (profiles/flops_per_element.json) comes from the oracle
built with an operation-counting scalar type (oracle/opcount.cpp): that build computes
the same residual as the plain oracle, bit for bit, and its counts reproduce the table."""
import ctypes
import json
import os

import numpy as np
import pytest

import hpb
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lib():
    import subprocess
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "_build/libhp_oracle_opcount.so"])
    o = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "libhp_oracle_opcount.so"))
    P = ctypes.c_void_p
    o.or_create.restype = P
    o.or_create.argtypes = [P, P, P]
    o.or_destroy.argtypes = [P]
    o.or_set_state.argtypes = [P, P, P, P]
    o.or_get_res.argtypes = [P, P, P, P]
    o.or_setup_preconditioner.argtypes = [P]
    o.or_rsdl.argtypes = [P, ctypes.c_int]
    o.oc_element_flops.argtypes = [P, ctypes.c_int, P]
    return o


@pytest.mark.parametrize("kind,p", [("ins", 2), ("ins", 4), ("cd", 3)])
def test_counting_build_matches_oracle_and_table(kind, p):
    o = _lib()
    pr = hpb.kovasznay_ins(n=4, p=p) if kind == "ins" else hpb.cd_sinsin(n=4, p=p, src=0.5)
    h = o.or_create(ctypes.addressof(pr.desc), ctypes.addressof(pr.tab), ctypes.addressof(pr.phys))
    P = ctypes.c_void_p
    o.or_set_state(h, *[a.ctypes.data_as(P) if a.size else None for a in (pr.ugv, pr.ugs, pr.ugi)])
    o.or_setup_preconditioner(h)
    o.or_rsdl(h, pr.phys.nstage)
    got = [np.zeros_like(a) for a in (pr.ugv, pr.ugs, pr.ugi)]
    o.or_get_res(h, *[a.ctypes.data_as(P) if a.size else None for a in got])
    ref = O.Oracle(pr)
    ref.setup_preconditioner()
    ref.rsdl(pr.phys.nstage)
    for a, b in zip(got, ref.residual()):
        assert np.array_equal(a, b)
    c = (ctypes.c_double * 3)()
    o.oc_element_flops(h, pr.phys.nstage, c)
    o.or_destroy(h)
    table = json.load(open(os.path.join(ROOT, "profiles", "flops_per_element.json")))
    assert c[0] == table[kind][str(p)]["full"] and c[0] > 0
