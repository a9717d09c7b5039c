"""GPU: the transport stage replayed as a CUDA graph (profiling off) gives
bit-identical fields and the same launch count as the kernel-by-kernel
launches (profiling on), for a single cell and for a batch."""
import numpy as np
import pytest

import giftbte_b200 as g
from giftbte_b200 import decks

pytestmark = pytest.mark.gpu


def run(make, profile, iters=25):
    s = make(profile)
    st = s.solve(max_iter=iters, err_temp=0.0, err_flux=0.0)
    f = s.fields()
    s.close()
    return f, st


@pytest.mark.parametrize("prec", [g.GBTE_FP64, g.GBTE_FP32_MIXED])
def test_graph_matches_direct_launches(prec):
    d = decks.config2_deck(h_nm=6.0, n_bands=8, n_phi=8, seed=1)

    def make(profile):
        return g.StaticBTESynthetic.from_deck(d, precision=prec, profile=profile)
    fa, sa = run(make, 0)
    fb, sb = run(make, 1)
    for k in ("T", "E", "q", "Tband"):
        assert np.array_equal(fa[k], fb[k]), k
    assert sa["kernel_launches"] == sb["kernel_launches"]


def test_graph_batch_matches_direct_launches():
    pop = decks.porous_population(3, seed=1, h_nm=(15.0, 22.0), r_nm=(40.0, 80.0), n_bands=4, n_phi=2)

    def make(profile):
        return g.StaticBTESynthetic.from_decks(pop, precision=g.GBTE_FP32_MIXED, profile=profile)
    fa, _ = run(make, 0)
    fb, _ = run(make, 1)
    assert np.array_equal(fa["T"], fb["T"]) and np.array_equal(fa["q"], fb["q"])


def test_profile_toggle():
    d = decks.config2_deck(h_nm=6.0, n_bands=8, n_phi=8, seed=1)
    s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP32_MIXED)
    s.solve(max_iter=3, err_temp=0.0, err_flux=0.0)
    assert not s.stats["kernels"]
    s.set_profile(True)
    st = s.solve(max_iter=3, err_temp=0.0, err_flux=0.0)
    assert st["kernels"]["sweep"]["launches"] == 3
    s.close()
