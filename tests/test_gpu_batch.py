"""Batched solve of independent geometries (gbte_batch_create) against
individual solves of the same decks: one handle over the disjoint union
reaches, geometry by geometry, the fixed point each single solve reaches."""
import functools

import numpy as np
import pytest

import giftbte_b200 as g
from giftbte_b200 import decks

pytestmark = pytest.mark.gpu


@functools.lru_cache(maxsize=None)
def population():
    return decks.porous_population(3, seed=1, h_nm=(15.0, 22.0), r_nm=(40.0, 80.0), n_bands=4, n_phi=2,
                                   residual_temp=1e-11, residual_flux=1e-11, max_iter=4000)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("prec", [g.GBTE_FP64, g.GBTE_FP32_MIXED])
def test_batch_matches_individual_solves(prec):
    pop = population()
    tol = 1e-9 if prec == g.GBTE_FP64 else 1e-5
    b = g.StaticBTESynthetic.from_decks(pop, precision=prec)
    off = b.geometry_offsets()
    assert list(np.diff(off)) == [d.mesh.n_cells for d in pop]
    if prec == g.GBTE_FP64:
        st = b.solve(allow_not_converged=False)
        assert st["err_temp"] <= 1e-11 and st["err_flux"] <= 1e-11
    else:  # FP32 intensities: the margins the FP32 parity tests use
        b.solve(err_temp=1e-9, err_flux=1e-7, max_iter=4000)
    fb = b.fields()
    b.close()
    for k, d in enumerate(pop):
        s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64)
        s.solve(allow_not_converged=False)
        f = s.fields()
        s.close()
        sl = slice(off[k], off[k + 1])
        assert rel(fb["T"][sl], f["T"]) <= tol, (k, rel(fb["T"][sl], f["T"]))
        assert rel(fb["q"][sl], f["q"]) <= (1e-8 if prec == g.GBTE_FP64 else 1e-4)
        assert rel(fb["Tband"][:, sl], f["Tband"]) <= tol


def test_batch_fourier_start_and_split():
    pop = population()
    # iterates (not the fixed point) are compared: exact macro solves, whose
    # accuracy does not depend on what else shares the batch's CG
    b = g.StaticBTESynthetic.from_decks(pop, precision=g.GBTE_FP64, macro_exact=1)
    b.fourier_initial()
    b.solve(max_iter=5, err_temp=0.0, err_flux=0.0)
    parts = b.split(b.fields()["T"])
    b.close()
    assert [len(p) for p in parts] == [d.mesh.n_cells for d in pop]
    for k, d in enumerate(pop):
        s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64, macro_exact=1)
        s.fourier_initial()
        s.solve(max_iter=5, err_temp=0.0, err_flux=0.0)
        T = s.fields()["T"]
        s.close()
        # 5 outer iterations from the same Fourier start: the batch's Picard
        # loop runs until every geometry settles, so the early iterates can
        # differ slightly; the fixed point is checked above
        assert rel(parts[k], T) <= 1e-4
