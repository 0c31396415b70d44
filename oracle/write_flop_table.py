"""Writes profiles/flops_per_element.json: the algorithmic FP64 flops of one element of
tri_hp::rsdl's element loop (ugtouht, element_rsdl, lftog of both parts;
tri_hp/nstage.cpp:52-73), counted by running the oracle built with an
operation-counting scalar type (oracle/opcount.cpp) on straight elements. One
add / sub / mul / div = 1 flop; sqrt and pow are listed apart (not in the flop count).
"full": a stage with beta > 0 (both parts of element_rsdl); "imaginary": beta = 0.
MEASUREMENT INFRASTRUCTURE ONLY (the bench reads the table, never the oracle).

Run: python oracle/write_flop_table.py
"""
import ctypes
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "hp-multiphysics_b200"))


def main():
    import subprocess
    import hpb
    subprocess.check_call(["make", "-s", "-C", HERE, "_build/libhp_oracle_opcount.so"])
    o = ctypes.CDLL(os.path.join(HERE, "_build", "libhp_oracle_opcount.so"))
    P = ctypes.c_void_p
    o.or_create.restype = P
    o.or_create.argtypes = [P, P, P]
    o.or_destroy.argtypes = [P]
    o.or_set_state.argtypes = [P, P, P, P]
    o.or_setup_preconditioner.argtypes = [P]
    o.oc_element_flops.argtypes = [P, ctypes.c_int, P]
    out = {"definition": "FP64 add/sub/mul/div per element of rsdl's element loop (ugtouht, element_rsdl, "
                         "lftog of both parts), straight elements, counted by the oracle's op-counting build",
           "ins": {}, "cd": {}}
    for kind in ("ins", "cd"):
        for p in range(1, 9):
            pr = hpb.kovasznay_ins(n=4, p=p) if kind == "ins" else hpb.cd_sinsin(n=4, p=p, src=0.5)
            h = o.or_create(ctypes.addressof(pr.desc), ctypes.addressof(pr.tab), ctypes.addressof(pr.phys))
            arr = [a.ctypes.data_as(P) if a.size else None for a in (pr.ugv, pr.ugs, pr.ugi)]
            o.or_set_state(h, *arr)
            o.or_setup_preconditioner(h)
            res = {}
            for name, stage in (("full", pr.phys.nstage), ("imaginary", 1)):
                c = (ctypes.c_double * 3)()
                o.oc_element_flops(h, stage, c)
                res[name] = c[0]
                res[name + "_sqrt"] = c[1]
                res[name + "_pow"] = c[2]
            o.or_destroy(h)
            out[kind][str(p)] = res
    path = os.path.join(ROOT, "profiles", "flops_per_element.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps({k: {p: v["full"] for p, v in out[k].items()} for k in ("ins", "cd")}))


if __name__ == "__main__":
    main()
