"""GPU: the launch shapes of the upwind sweep. Each thread updates 1, 2 or 4
consecutive bands of a cell with vector accesses (options.sweep_vector), in
the block kernel (a CTA per direction and chunk of bands) or the
warp-independent kernel (a warp per direction and group of bands,
options.sweep_kernel = 2). Every band's arithmetic is the same, in the same
order, so the fields are bit-identical whichever shape runs. A width the
band count does not divide falls back to one band per thread."""
import numpy as np
import pytest

import giftbte_b200 as g
import make_golden as mg
from giftbte_b200 import decks

pytestmark = pytest.mark.gpu


def run(deck, prec, vb, bands=8, iters=15, batch=False, kernel=1):
    kw = dict(precision=prec, sweep_bands=bands, sweep_vector=vb, sweep_kernel=kernel)
    s = g.StaticBTESynthetic.from_decks(deck, **kw) if batch else g.StaticBTESynthetic.from_deck(deck, **kw)
    st = s.solve(max_iter=iters, err_temp=0.0, err_flux=0.0)
    f = s.fields()
    s.close()
    return f, st


@pytest.mark.parametrize("prec,widths", [(g.GBTE_FP32_MIXED, (2, 4)), (g.GBTE_FP64, (2,))])
def test_widths_are_bit_identical(prec, widths):
    d = decks.config2_deck(h_nm=6.0, n_bands=16, n_phi=8, seed=2)
    f1, s1 = run(d, prec, 1)
    assert s1["sweep_vector"] == 1
    for vb in widths:
        for bands in (8, 16):
            fv, sv = run(d, prec, vb, bands=bands)
            assert sv["sweep_vector"] == vb and sv["sweep_bands"] == bands
            for k in ("T", "E", "q", "Tband"):
                assert np.array_equal(f1[k], fv[k]), (vb, bands, k)


def test_batch_widths_are_bit_identical():
    pop = decks.porous_population(3, seed=1, h_nm=(15.0, 22.0), r_nm=(40.0, 80.0), n_bands=8, n_phi=2)
    f1, _ = run(pop, g.GBTE_FP32_MIXED, 1, batch=True)
    f4, s4 = run(pop, g.GBTE_FP32_MIXED, 4, batch=True)
    assert s4["sweep_vector"] == 4
    assert np.array_equal(f1["T"], f4["T"])


def test_width_that_does_not_divide_the_bands_falls_back():
    deck, ref = mg.load("gray_square_tri")  # one band
    s = g.StaticBTESynthetic.from_deck(deck, precision=g.GBTE_FP64, sweep_vector=2)
    s.set_initial(ref["Tf"])
    st = s.solve(allow_not_converged=False)
    assert st["sweep_vector"] == 1
    assert float(np.max(np.abs(s.fields()["T"] - ref["T"])) / np.max(np.abs(ref["T"]))) <= 1e-9
    s.close()


def test_autotuner_reports_its_pick():
    d = decks.config2_deck(h_nm=6.0, n_bands=16, n_phi=8, seed=2)
    s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP32_MIXED)
    st = s.solve(max_iter=3, err_temp=0.0, err_flux=0.0)
    assert st["sweep_vector"] in (1, 2, 4)
    assert 1 <= st["sweep_bands"] <= 16
    assert 1 <= st["sweep_threads"] <= 256
    s.close()


@pytest.mark.parametrize("prec,widths", [(g.GBTE_FP32_MIXED, (1, 2, 4)), (g.GBTE_FP64, (1, 2))])
def test_warp_kernel_is_bit_identical(prec, widths):
    d = decks.config2_deck(h_nm=6.0, n_bands=16, n_phi=8, seed=2)
    f1, _ = run(d, prec, 1)
    for vb in widths:
        fw, sw = run(d, prec, vb, kernel=2)
        assert sw["sweep_kernel"] == 2 and sw["sweep_vector"] == vb
        for k in ("T", "E", "q", "Tband"):
            assert np.array_equal(f1[k], fw[k]), (vb, k)


def test_warp_kernel_batch_and_golden():
    pop = decks.porous_population(3, seed=1, h_nm=(15.0, 22.0), r_nm=(40.0, 80.0), n_bands=8, n_phi=2)
    f1, _ = run(pop, g.GBTE_FP32_MIXED, 1, batch=True)
    fw, sw = run(pop, g.GBTE_FP32_MIXED, 4, batch=True, kernel=2)
    assert sw["sweep_kernel"] == 2
    assert np.array_equal(f1["T"], fw["T"])
    for case in ("quad_heat_specular", "porous_msh"):
        deck, ref = mg.load(case)
        s = g.StaticBTESynthetic.from_deck(deck, precision=g.GBTE_FP64, sweep_kernel=2)
        s.set_initial(ref["Tf"])
        st = s.solve(allow_not_converged=False)
        assert st["sweep_kernel"] == 2
        assert float(np.max(np.abs(s.fields()["T"] - ref["T"])) / np.max(np.abs(ref["T"]))) <= 1e-9
        s.close()


@pytest.mark.parametrize("prec,widths", [(g.GBTE_FP32_MIXED, (1, 2, 4)), (g.GBTE_FP64, (1, 2))])
def test_wide_level_kernel_is_bit_identical(prec, widths):
    # the wide-level kernel (options.sweep_kernel = 3) reads upwind
    # corrections back from device memory instead of a shared ring; it needs
    # records that hold level positions, so both runs plan without far slots
    d = decks.config2_deck(h_nm=6.0, n_bands=16, n_phi=8, seed=2)

    def run_w(vb, kernel, bands):
        s = g.StaticBTESynthetic.from_deck(d, precision=prec, sweep_bands=bands, sweep_vector=vb,
                                           sweep_kernel=kernel, sweep_far_slots=-1)
        st = s.solve(max_iter=15, err_temp=0.0, err_flux=0.0)
        f = s.fields()
        s.close()
        return f, st

    f1, _ = run_w(1, 1, 8)
    for vb in widths:
        for bands in (8, 16):
            fw, sw = run_w(vb, 3, bands)
            assert sw["sweep_kernel"] == 3 and sw["sweep_vector"] == vb
            for k in ("T", "E", "q", "Tband"):
                assert np.array_equal(f1[k], fw[k]), (vb, bands, k)


def test_wide_level_kernel_batch_and_golden():
    pop = decks.porous_population(3, seed=1, h_nm=(15.0, 22.0), r_nm=(40.0, 80.0), n_bands=8, n_phi=2)
    f1, _ = run(pop, g.GBTE_FP32_MIXED, 1, batch=True)
    s = g.StaticBTESynthetic.from_decks(pop, precision=g.GBTE_FP32_MIXED, sweep_bands=8, sweep_vector=4,
                                        sweep_kernel=3, sweep_far_slots=-1)
    sw = s.solve(max_iter=15, err_temp=0.0, err_flux=0.0)
    fw = s.fields()
    s.close()
    assert sw["sweep_kernel"] == 3
    assert np.array_equal(f1["T"], fw["T"])
    for case in ("quad_heat_specular", "porous_msh", "periodic_jitter"):
        deck, ref = mg.load(case)
        s = g.StaticBTESynthetic.from_deck(deck, precision=g.GBTE_FP64, sweep_kernel=3, sweep_far_slots=-1)
        s.set_initial(ref["Tf"])
        st = s.solve(allow_not_converged=False)
        assert st["sweep_kernel"] == 3
        assert float(np.max(np.abs(s.fields()["T"] - ref["T"])) / np.max(np.abs(ref["T"]))) <= 1e-9
        s.close()


@pytest.mark.parametrize("prec", [g.GBTE_FP32_MIXED, g.GBTE_FP64])
@pytest.mark.parametrize("dim", [2, 3])
def test_gradient_and_residual_launch_shapes_are_bit_identical(prec, dim):
    # the LSQ gradient with 1, 2 or 4 directions per thread, a warp per cell
    # with 1 or 2 directions per lane (options.gradient_dirs 5, 6), or
    # shared-memory tiles of two block sizes (7, 8), and the residual as a
    # thread, a warp per cell or a tile (options.residual_form):
    # the arithmetic per band and direction is unchanged. The 3D block runs
    # in direction batches of 5, so direction groups meet a batch whose last
    # group is short
    if dim == 2:
        d = decks.config2_deck(h_nm=6.0, n_bands=16, n_phi=8, seed=2)
        kw = {}
    else:
        d = decks.config3_deck(h_nm=10.0, size_nm=(40.0, 40.0, 100.0), n_bands=8, n_theta=2, n_phi=2)
        kw = {"direction_batch": 5}
    out = {}
    for dg, rf in ((1, 1), (2, 1), (4, 1), (5, 1), (6, 1), (7, 1), (8, 1), (1, 5), (1, 6), (1, 7), (1, 8)):
        s = g.StaticBTESynthetic.from_deck(d, precision=prec, gradient_dirs=dg, residual_form=rf, sweep_bands=8,
                                           sweep_vector=1, sweep_kernel=1, **kw)
        st = s.solve(max_iter=10, err_temp=0.0, err_flux=0.0)
        out[(dg, rf)] = s.fields()
        s.close()
        assert st["gradient_dirs"] == dg and st["residual_form"] == rf
    for key, f in out.items():
        for k in ("T", "E", "q", "Tband"):
            assert np.array_equal(out[(1, 1)][k], f[k]), (key, k)


@pytest.mark.parametrize("dim,nb", [(2, 32), (3, 40), (3, 48)])
def test_eight_lane_gradient_tiles_are_bit_identical(dim, nb):
    # the tiled gradient with eight lanes per cell (options.gradient_dirs 9,
    # 10; FP32-mixed form) against a thread per cell (1) and the four-band
    # tiles (7): the band chunk is 32 + 8 NS bands, each lane taking one
    # 16-byte piece and NS single bands, so 32 bands (NS = 0), 40 (NS = 1)
    # and 48 (NS = 2). The 2D blocks of 128 cells would need 1024 threads:
    # shape 10 falls back to 2 directions per thread there
    shapes = (1, 7, 9, 10)
    if dim == 2:
        d = decks.config2_deck(h_nm=6.0, n_bands=nb, n_phi=4, seed=2)
        kw = {}
    else:
        d = decks.config3_deck(h_nm=10.0, size_nm=(40.0, 40.0, 100.0), n_bands=nb, n_theta=2, n_phi=2)
        kw = {"direction_batch": 5}
    out = {}
    for dg in shapes:
        s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP32_MIXED, gradient_dirs=dg, residual_form=1,
                                           sweep_bands=8, sweep_vector=1, sweep_kernel=1, **kw)
        st = s.solve(max_iter=10, err_temp=0.0, err_flux=0.0)
        out[dg] = s.fields()
        s.close()
        assert st["gradient_dirs"] == (2 if (dim == 2 and dg == 10) else dg)
    for dg, f in out.items():
        for k in ("T", "E", "q", "Tband"):
            assert np.array_equal(out[1][k], f[k]), (dg, k)
