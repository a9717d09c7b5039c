"""GPU: the allocation-free Fourier pre-solve (gbte_fourier_initial_noalloc).

Callers that must not allocate device memory mid-run (all device memory
handed out from their own pool reserved at start-up, or a fixed
device-memory limit) re-seed a handle with this entry point; its scratch is
a static device array of the library. Its result must match the allocating
entry point gbte_fourier_initial on two calls in a row, also after a call on
a mesh of another size has left other contents in the shared array. This
file is collected last so that a failure here does not stop the other tests.
"""
import numpy as np
import pytest

import make_golden as mg
from giftbte_b200 import GBTE_FP32_MIXED, GBTE_FP64, StaticBTESynthetic

pytestmark = pytest.mark.gpu

TOL = 1e-9  # the FP64 parity tolerance of the other GPU tests


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def allocating_results(deck, precision):
    """Two calls in a row of the allocating entry point on one handle (each
    call starts from the field the previous one left)."""
    s = StaticBTESynthetic.from_deck(deck, precision=precision)
    out = []
    for _ in range(2):
        s.fourier_initial()
        out.append(s.fields())
    s.close()
    return out


@pytest.mark.parametrize("precision", [GBTE_FP64, GBTE_FP32_MIXED])
def test_noalloc_fourier_matches_allocating_entry_point(precision):
    cases = ["gray_square_tri", "quad_heat_specular"]
    expected = {c: allocating_results(mg.load(c)[0], precision) for c in cases}
    for case in cases:  # the second case reuses the array the first one filled
        deck, ref = mg.load(case)
        s = StaticBTESynthetic.from_deck(deck, precision=precision)
        for call in range(2):  # two calls in a row on the same handle
            s.fourier_initial_noalloc()
            f = s.fields()
            assert rel(f["T"], expected[case][call]["T"]) <= TOL
            assert rel(f["q"], expected[case][call]["q"]) <= TOL
            if call == 0:
                assert rel(f["T"], ref["Tf"]) <= TOL
        # the seeded handle still solves to the reference's fixed point
        if precision == GBTE_FP64:
            s.solve(allow_not_converged=False)
            assert rel(s.fields()["T"], ref["T"]) <= TOL
        s.close()
