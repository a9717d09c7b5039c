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


def test_noalloc_fp32_handle_solves_like_allocating_seed():
    # an FP32-mixed handle seeded by the allocation-free call solves to the
    # same fixed point as one seeded by gbte_fourier_initial, within the FP32
    # tolerance of the other tests (the base temperature's gradient is formed
    # on the device in one case, on the host in the other)
    deck, ref = mg.load("gray_square_tri")
    out = []
    for noalloc in (False, True):
        s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP32_MIXED, err_temp=1e-9, err_flux=1e-7)
        s.fourier_initial_noalloc() if noalloc else s.fourier_initial()
        s.solve()
        out.append(s.fields()["T"])
        s.close()
    assert rel(out[1], out[0]) <= 1e-5
    assert rel(out[1], ref["T"]) <= 1e-5


def test_noalloc_grid_wide_cg_branch():
    # 64,800 cells: the Fourier system no longer fits one cluster's shared
    # memory, so both entry points take the grid-wide CG kernel; the
    # allocation-free one then uses the array's four CG vectors and its
    # reduction slots
    from giftbte_b200 import decks

    deck = decks.config1_deck(180)
    assert 58112 < deck.mesh.n_cells <= 131072
    expected = allocating_results(deck, GBTE_FP64)
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64)
    for call in range(2):
        s.fourier_initial_noalloc()
        f = s.fields()
        assert rel(f["T"], expected[call]["T"]) <= TOL
        assert rel(f["q"], expected[call]["q"]) <= TOL
    s.close()


def test_noalloc_allocates_no_device_memory():
    # after the first call has looked up the array's address, a further call
    # changes the device's free memory by less than one 2 MiB allocation
    # granule: it allocates nothing
    import torch

    deck, _ = mg.load("periodic_jitter")
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64)
    s.fourier_initial_noalloc()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        s.fourier_initial_noalloc()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    s.close()
    assert free0 - free1 < 2 * 1024 * 1024, (free0, free1)


def test_noalloc_refuses_batched_and_oversized_handles():
    from giftbte_b200 import GBTE_ERR_ARG, GBTE_ERR_UNSUPPORTED, GBTEError, decks

    d1, _ = mg.load("gray_square_tri")
    d2, _ = mg.load("gray_square_tri")
    b = StaticBTESynthetic.from_decks([d1, d2], precision=GBTE_FP64)
    with pytest.raises(GBTEError) as ei:
        b.fourier_initial_noalloc()
    assert ei.value.status == GBTE_ERR_UNSUPPORTED
    b.close()
    big = decks.config1_deck(260, n_phi=1)  # 135,200 cells > 131,072
    s = StaticBTESynthetic.from_deck(big, precision=GBTE_FP64)
    with pytest.raises(GBTEError) as ei:
        s.fourier_initial_noalloc()
    assert ei.value.status == GBTE_ERR_ARG
    s.close()
