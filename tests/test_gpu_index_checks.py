"""Index checks on the device path: with GBTE_DEBUG set, gbte_create range-
checks every array it uploads (and the tiles when the solve builds them);
the solve then runs as usual and gives bit-identical fields."""
import numpy as np
import pytest

from giftbte_b200 import GBTE_FP32_MIXED, GBTE_FP64, StaticBTESynthetic, decks

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make,prec", [
    (lambda: decks.config1_deck(16), GBTE_FP64),
    (lambda: decks.interface_deck(8), GBTE_FP64),
    (lambda: decks.config2_deck(h_nm=15.0, n_bands=4, n_phi=4), GBTE_FP32_MIXED),
    (lambda: decks.config3_deck(h_nm=25.0, size_nm=(100.0, 100.0, 100.0), n_bands=4), GBTE_FP32_MIXED),
], ids=["square", "interface", "porous_fp32", "block3d_fp32"])
def test_checked_solve_matches_unchecked(make, prec, monkeypatch):
    d = make()
    out = []
    for flag in ("0", "1"):
        monkeypatch.setenv("GBTE_DEBUG", flag)
        s = StaticBTESynthetic.from_deck(d, precision=prec)
        s.solve(max_iter=3, err_temp=0.0, err_flux=0.0)
        out.append(s.fields())
        s.close()
    for k in ("T", "q"):
        assert np.array_equal(out[0][k], out[1][k]), k
