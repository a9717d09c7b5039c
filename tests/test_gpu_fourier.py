"""GPU: the Fourier pre-solve (gbte_fourier_initial) against the reference's
own Temperature_macro.dat / HeatFlux_macro.dat, and BTE iteration counts
from that start against the reference's."""
import numpy as np
import pytest

import make_golden as mg
from giftbte_b200 import GBTE_FP64, GBTE_FP32_MIXED, GBTEError, StaticBTESynthetic

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("case", mg.ONE_MATERIAL)
def test_fourier_initial_matches_reference(case):
    deck, ref = mg.load(case)
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64)
    s.fourier_initial()
    f = s.fields()
    # T_lattice holds the initial field until the first solve
    assert rel(f["T"], ref["Tf"]) <= 1e-9, rel(f["T"], ref["Tf"])


def iterations_to(margins, tol):
    ok = np.nonzero((margins[:, 0] <= tol) & (margins[:, 1] <= tol))[0]
    return int(ok[0]) + 1 if len(ok) else None


def test_fourier_initial_refuses_several_materials():
    deck, _ = mg.load("interface_2mat")
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64)
    with pytest.raises(GBTEError):
        s.fourier_initial()
    s.close()


@pytest.mark.parametrize("case", [c for c in mg.CONVERGED if c in mg.ONE_MATERIAL])
def test_iterations_from_fourier_start_match_reference(case):
    # from the same (Fourier) start the outer iteration follows the
    # reference's: the number of iterations to margins 1e-8 agrees (near
    # 1e-12 the margins are at rounding level and the counts are noise)
    deck, ref = mg.load(case)
    want = iterations_to(ref["margins"], 1e-8)
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64)
    s.fourier_initial()
    st = s.solve(err_temp=1e-8, err_flux=1e-8, max_iter=3000, allow_not_converged=False)
    assert abs(st["iterations"] - want) <= 1, (st["iterations"], want)
