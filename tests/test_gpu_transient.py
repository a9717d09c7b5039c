"""The explicit transient solver (State=Transient) against the compiled
reference's own run of the thermal-grating strip (tests/golden/
grating_transient.npz): 40 explicit steps of 1e-13 s from
T = cos(2 pi x / ScaleX), the lattice temperature and heat flux after the
last step and the temperature of cell 0 after every step (TTG.dat)."""
import numpy as np
import pytest

import make_golden as mg
from giftbte_b200 import GBTE_FP32_MIXED, GBTE_FP64, GBTEError, StaticBTESynthetic

pytestmark = pytest.mark.gpu
TOL = 1e-9


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def check(s, deck, ref):
    r = s.transient_solve(deck.time_step, deck.total_time, deck.residual_temp, deck.residual_flux, probe_cell=0)
    f = s.fields()
    assert r["steps"] == ref["iters"] == len(ref["ttg"])
    assert rel(r["history"], ref["ttg"][:, 1]) <= TOL, rel(r["history"], ref["ttg"][:, 1])
    assert rel(f["T"], ref["T"]) <= TOL, rel(f["T"], ref["T"])
    assert rel(f["q"], ref["q"]) <= TOL, rel(f["q"], ref["q"])


@pytest.mark.parametrize("cell_order", [0, 1])
def test_grating_matches_reference(cell_order):
    deck, ref = mg.load("grating_transient")
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64, cell_order=cell_order)
    check(s, deck, ref)
    s.close()


def test_grating_from_deck_files(tmp_path):
    deck, ref = mg.load("grating_transient")
    deck.write(str(tmp_path))
    s = StaticBTESynthetic.from_deck_dir(str(tmp_path), precision=GBTE_FP64)
    check(s, deck, ref)
    s.close()


def test_rerun_and_fp32_refused():
    deck, ref = mg.load("grating_transient")
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64)
    a = s.transient_solve(deck.time_step, 10 * deck.time_step)
    b = s.transient_solve(deck.time_step, 10 * deck.time_step)
    assert a["steps"] == b["steps"] == 10 and np.array_equal(a["history"], b["history"])
    s.close()
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP32_MIXED)
    with pytest.raises(GBTEError) as e:
        s.transient_solve(deck.time_step, deck.total_time)
    assert e.value.status == -8
    s.close()
