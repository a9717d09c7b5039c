"""GPU parity: the CUDA path through the C ABI against the reference's own
full-precision outputs (golden fixtures) and the CPU oracle restatement."""
import numpy as np
import pytest

import make_golden as mg
from giftbte_b200 import GBTE_FP32_MIXED, GBTE_FP64, GBTEError, StaticBTESynthetic, effective_conductivity

pytestmark = pytest.mark.gpu

# FP64 drop-in form: reference fixed point to <= 1e-9 relative;
# FP32 intensity form: <= 1e-5 relative temperature error.
TOL_FP64 = 1e-9
TOL_FP32 = 1e-5


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def keff_pair(s, q, q_ref, axis=0):
    """Effective conductivity k = <q_axis>_V L / dT (L = dT = 1) of the
    solver's flux and of the reference's on the same cell volumes, the
    post-processing of bin/examples/cross-plane/verify_kappa_crossplane.m:8;
    None when the reference's volume-averaged flux is negligible (a
    symmetric deck) next to its flux scale."""
    _, vol = s.geometry()
    k = effective_conductivity(q, vol, 1.0, 1.0, axis)
    k_ref = effective_conductivity(q_ref, vol, 1.0, 1.0, axis)
    if abs(k_ref) <= 1e-3 * float(np.mean(np.abs(q_ref[:, axis]))):
        return None
    return k, k_ref


@pytest.mark.parametrize("case", mg.CASES)
def test_fp64_matches_reference(case):
    deck, ref = mg.load(case)
    # exact macro solves (the reference's sparse LU solves every Picard step
    # exactly): the outer iterates follow the reference's, so the solve stops
    # where the reference stopped, and a fixed iteration count (the limited
    # scheme) compares the same iterate
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64, macro_exact=1)
    # the reference's start (its Fourier pre-solve): the Sequential scheme
    # without isothermal walls keeps the start's temperature level
    s.set_initial(ref["Tf"], ref["qf"])
    if case in mg.CONVERGED:
        st = s.solve(allow_not_converged=False)
        assert st["err_temp"] <= 1e-12 and st["err_flux"] <= 1e-12
    else:
        # the limited scheme: the reference's state after a fixed number of
        # outer iterations, the same count here
        st = s.solve(max_iter=ref["iters"], err_temp=0.0, err_flux=0.0)
        assert st["iterations"] == ref["iters"]
    f = s.fields()
    assert rel(f["T"], ref["T"]) <= TOL_FP64, rel(f["T"], ref["T"])
    assert rel(f["E"], ref["E"]) <= TOL_FP64
    assert rel(f["Tband"], ref["Tband"]) <= TOL_FP64
    assert rel(f["q"], ref["q"]) <= TOL_FP64, rel(f["q"], ref["q"])
    kk = keff_pair(s, f["q"], ref["q"])
    if kk is not None:
        assert abs(kk[0] - kk[1]) <= TOL_FP64 * abs(kk[1]), kk


@pytest.mark.parametrize("case", mg.CONVERGED)
def test_fp64_default_macro_solves_reach_reference_fixed_point(case):
    # the default warm-started macro solves stop after a 3e-3 residual
    # reduction: the same fixed point along another path. At margins 1e-12
    # temperatures agree to 1e-9; the flux, a difference of band terms three
    # to four orders larger than itself, to a few 1e-9
    deck, ref = mg.load(case)
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64)
    s.set_initial(ref["Tf"], ref["qf"])
    s.solve(allow_not_converged=False)
    f = s.fields()
    s.close()
    assert rel(f["T"], ref["T"]) <= TOL_FP64, rel(f["T"], ref["T"])
    assert rel(f["Tband"], ref["Tband"]) <= TOL_FP64
    assert rel(f["q"], ref["q"]) <= 5e-9, rel(f["q"], ref["q"])


@pytest.mark.parametrize("case", mg.CONVERGED)
def test_fp32_mixed_close_to_reference(case):
    deck, ref = mg.load(case)
    deck.residual_temp = 1e-9
    deck.residual_flux = 1e-7
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP32_MIXED)
    s.set_initial(ref["Tf"], ref["qf"])
    s.solve()
    f = s.fields()
    # relative to the temperature variation, which is what the FP32 deviation form resolves
    span = np.max(ref["T"]) - np.min(ref["T"])
    assert np.max(np.abs(f["T"] - ref["T"])) / max(span, 1e-30) <= 1e-4
    assert rel(f["T"], ref["T"]) <= TOL_FP32


@pytest.mark.parametrize("case", ["porous_firstorder", "periodic_sequential", "quad_firstorder_sequential",
                                  "porous_limiter", "alamode_square", "shengbte_square"])
def test_variant_decks_from_files_match_reference(case, tmp_path):
    # Order=1 / 2limit and IterativeScheme=Sequential read from the CONTROL
    # file of a deck directory select the same variants as the in-memory
    # options; ALAMODE and ShengBTE mode lists named in PHONON reduce to the
    # reference's band tables
    deck, ref = mg.load(case)
    deck.write(str(tmp_path))
    s = StaticBTESynthetic.from_deck_dir(str(tmp_path), precision=GBTE_FP64,
                                         macro_exact=int(case not in mg.CONVERGED))
    s.set_initial(ref["Tf"], ref["qf"])
    if case in mg.CONVERGED:
        s.solve(allow_not_converged=False)
    else:
        s.solve(max_iter=ref["iters"], err_temp=0.0, err_flux=0.0)
    f = s.fields()
    s.close()
    assert rel(f["T"], ref["T"]) <= TOL_FP64, rel(f["T"], ref["T"])
    assert rel(f["q"], ref["q"]) <= TOL_FP64, rel(f["q"], ref["q"])


def test_limiter_needs_the_fp64_form():
    deck, _ = mg.load("porous_limiter")
    with pytest.raises(GBTEError):
        StaticBTESynthetic.from_deck(deck, precision=GBTE_FP32_MIXED)


@pytest.mark.parametrize("case", ["porous_msh", "porous_firstorder", "periodic_sequential", "porous_limiter"])
def test_iterates_follow_reference_step_by_step(case):
    # with exact macro solves (options.macro_exact) the outer iterates
    # themselves follow the reference's: five iterations from the same start
    # against the CPU restatement, which repeats the reference's arithmetic
    import oracle

    deck, ref = mg.load(case)
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64, macro_exact=1)
    s.set_initial(ref["Tf"])
    s.solve(max_iter=5, err_temp=0.0, err_flux=0.0)
    f = s.fields()
    s.close()
    o = oracle.solve(deck, T0=ref["Tf"], max_iter=5, err_T=0.0, err_q=0.0)
    assert rel(f["T"], o["T"]) <= 1e-10, rel(f["T"], o["T"])
    assert rel(f["q"], o["q"]) <= 1e-9, rel(f["q"], o["q"])


@pytest.mark.parametrize("precision", [GBTE_FP64, GBTE_FP32_MIXED])
def test_benchmark_cell_full_size_follows_reference(precision):
    # the benchmarked 2D workload itself (17,939 triangles, 40 bands, 64
    # directions): three outer iterations from the reference's Fourier
    # start, with exact macro solves, against the compiled reference's state
    # after the same three iterations
    deck, ref = mg.load("config2_iter3")
    s = StaticBTESynthetic.from_deck(deck, precision=precision, macro_exact=1)
    s.set_initial(ref["Tf"], ref["qf"])
    st = s.solve(max_iter=mg.CONFIG2_ITERS, err_temp=0.0, err_flux=0.0)
    assert st["iterations"] == mg.CONFIG2_ITERS
    f = s.fields()
    kk = keff_pair(s, f["q"], ref["q"])
    s.close()
    tb = f["Tband"][ref["bands_kept"]]
    if precision == GBTE_FP64:
        assert rel(f["T"], ref["T"]) <= 1e-10, rel(f["T"], ref["T"])
        assert rel(f["E"], ref["E"]) <= 1e-10, rel(f["E"], ref["E"])
        assert rel(tb, ref["Tband"]) <= 1e-10, rel(tb, ref["Tband"])
        assert rel(f["q"], ref["q"]) <= TOL_FP64, rel(f["q"], ref["q"])
        assert abs(kk[0] - kk[1]) <= TOL_FP64 * abs(kk[1]), kk
    else:
        assert rel(f["T"], ref["T"]) <= TOL_FP32, rel(f["T"], ref["T"])
        assert rel(f["q"], ref["q"]) <= 1e-4, rel(f["q"], ref["q"])
        assert abs(kk[0] - kk[1]) <= 1e-4 * abs(kk[1]), kk


@pytest.mark.skipif(not mg.have("config2_converged"), reason="converged full-size fixture not generated")
def test_benchmark_cell_converged_matches_reference():
    # the same cell converged: with exact macro solves the outer iterates
    # follow the reference's, so stopping at the reference's margins (1e-9)
    # stops at its iteration; the fields and the effective conductivity
    # k_x = <q_x>_V L / dT then agree to 1e-9
    deck, ref = mg.load("config2_converged")
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64, macro_exact=1)
    s.set_initial(ref["Tf"], ref["qf"])
    st = s.solve(max_iter=4000, err_temp=1e-9, err_flux=1e-9)  # the reference run's margins
    f = s.fields()
    kk = keff_pair(s, f["q"], ref["q"])
    s.close()
    assert abs(st["iterations"] - ref["iters"]) <= 1, (st["iterations"], ref["iters"])
    assert rel(f["T"], ref["T"]) <= TOL_FP64, rel(f["T"], ref["T"])
    assert rel(f["q"], ref["q"]) <= TOL_FP64, rel(f["q"], ref["q"])
    assert abs(kk[0] - kk[1]) <= TOL_FP64 * abs(kk[1]), kk


@pytest.mark.skipif(not mg.have("config2_converged"), reason="converged full-size fixture not generated")
def test_benchmark_cell_fp32_form_converged_close_to_reference():
    deck, ref = mg.load("config2_converged")
    deck.residual_temp = deck.residual_flux = 1e-9
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP32_MIXED)
    s.set_initial(ref["Tf"], ref["qf"])
    s.solve(max_iter=4000)
    f = s.fields()
    kk = keff_pair(s, f["q"], ref["q"])
    s.close()
    assert rel(f["T"], ref["T"]) <= TOL_FP32, rel(f["T"], ref["T"])
    assert abs(kk[0] - kk[1]) <= 1e-4 * abs(kk[1]), kk
