"""Batched finite-difference element Jacobians (hp_gpu_element_jacobian) against the
oracle's restatement of tri_hp::element_jacobian (tri_hp/nstage.cpp:131-165): ins on the
Kovasznay state and cd with a source, every element. Finite differences with
dw ~ 1e-8 |u| turn rounding differences of the residual into ~1e-8 relative column
differences; compared at 1e-5 of max|K|."""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import _lib as L
from oracle.oracle import Oracle, element_jacobians

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,p", [("ins", 2), ("ins", 4), ("cd", 3)])
def test_element_jacobians_match_oracle(kind, p):
    if kind == "ins":
        pr = hpb.kovasznay_ins(n=4, p=p)
    else:
        pr = hpb.cd_sinsin(n=5, p=p, kcond=1e-2, src=0.7)
    g, o = pr.gpu(), Oracle(pr)
    assert g.setup_preconditioner() == 0 and o.setup_preconditioner() == 0
    Kg, Ko = g.element_jacobians(), element_jacobians(o)
    assert np.all(np.isfinite(Kg))
    assert np.max(np.abs(Kg - Ko)) < 1e-5 * np.max(np.abs(Ko))

