"""CPU: the numpy CPML stepper (oracle/cpml.py) pinned to the C oracle, and the profile formula.

With every position outside the layers the CPML stepper must be the reference's update
(gDiamond/gdiamond.hpp:1193-1221) bit for bit; the C oracle is itself pinned to the compiled
reference (test_oracle_pin.py).  The profile restatement is checked for the properties the
recursion needs: 0 < b <= 1, a <= 0, 1/kappa in (0, 1], layers only within L cells of a face.
"""
import numpy as np

import oracle
from oracle import cpml
from gdiamond_b200 import workloads as W


def test_numpy_stepper_without_layers_is_the_reference_update():
    shape, T = (17, 13, 11), 12
    coefs = W.reference_coefficients(shape, t_pml=3)
    w = W.gaussian_wave(T, delay=4.0, width=2.0, period=5.0)
    src = [oracle.Source("Jz", w, i=8, j=6, k=5), oracle.Source("My", w * np.float32(0.3), i=4, j=9, k=3),
           oracle.Source("Jx", w * np.float32(0.5), k=7, kind=oracle.PLANE_Z)]
    F_c = oracle.run(shape, coefs, T, sources=src)
    F_n = cpml.run(shape, coefs, T, cpml.no_layers(shape), sources=src)
    for c in range(6):
        assert np.array_equal(F_c[c].view(np.uint32), F_n[c].view(np.uint32)), c


def test_profile_properties():
    n, L = 40, 8
    for half in (False, True):
        slot, b, a, ik = cpml.profile(n, L, True, True, 0.1, 0.05, kappa_max=2.0, half=half)
        inside = slot >= 0
        assert inside[:L - 1].all() and inside[n - L:].all()
        assert not inside[L + 1:n - L - 2].any()
        assert (b[inside] > 0).all() and (b <= 1).all()
        assert (a[inside] < 0).all() and (a[~inside] == 0).all()
        assert (ik > 0).all() and (ik <= 1).all()
        # grading deepens towards the faces
        assert b[0] < b[L // 2] and b[n - 1] < b[n - 1 - L // 2]
        assert len(set(slot[inside].tolist())) == inside.sum() and slot.max() < 2 * L + 1
