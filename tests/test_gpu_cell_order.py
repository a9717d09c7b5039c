"""GPU: the library's internal cell order (Morton order of cell centres,
options.cell_order = 0) against the caller's order (cell_order = 1). Every
cell array of the ABI is in the caller's order either way, so the two runs
agree to rounding: fields, geometry, a heat source, a non-uniform initial
field, the batched form and the written output files."""
import os

import numpy as np
import pytest

import giftbte_b200 as g
import make_golden as mg
from giftbte_b200 import decks

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def solve_pair(deck, prec, T0=None, heat=None, iters=None):
    out = []
    for order in (0, 1):
        s = g.StaticBTESynthetic.from_deck(deck, precision=prec, cell_order=order, cell_heat=heat)
        if T0 is not None:
            s.set_initial(T0)
        if iters:
            s.solve(max_iter=iters, err_temp=0.0, err_flux=0.0, allow_not_converged=True)
        else:
            s.solve(allow_not_converged=False)
        out.append((s.fields(), s.geometry()))
        s.close()
    return out


@pytest.mark.parametrize("case", mg.CONVERGED)
def test_orders_agree_on_golden_decks(case):
    deck, ref = mg.load(case)
    (fa, ga), (fb, gb) = solve_pair(deck, g.GBTE_FP64, T0=ref["Tf"])
    assert np.array_equal(ga[0], gb[0]) and np.array_equal(ga[1], gb[1])
    for k in ("T", "E", "q", "Tband"):
        assert rel(fa[k], fb[k]) <= 1e-10, (k, rel(fa[k], fb[k]))
    assert rel(fa["T"], ref["T"]) <= 1e-9


def test_geometry_is_in_callers_order():
    deck = decks.config2_deck(h_nm=3.0, n_bands=4, n_phi=16, seed=0)
    s = g.StaticBTESynthetic.from_deck(deck, precision=g.GBTE_FP64)
    c, v = s.geometry()
    s.close()
    # triangles: the centre is the mean of the vertices, in metres
    cen = np.asarray(deck.mesh.nodes)[np.asarray(deck.mesh.cells)].mean(axis=1) * deck.scale[0]
    assert np.max(np.abs(c[:, :2] - cen)) <= 1e-9 * np.max(np.abs(cen))
    assert np.all(v > 0)


@pytest.mark.parametrize("prec", [g.GBTE_FP64, g.GBTE_FP32_MIXED])
def test_orders_agree_with_source_and_field_start(prec):
    # a cell heat source and a non-uniform initial field given in the
    # caller's order; ten outer iterations (no convergence cut-off)
    deck = decks.config2_deck(h_nm=3.0, n_bands=4, n_phi=16, seed=0)
    nc = deck.mesh.n_cells
    rng = np.random.default_rng(3)
    heat = rng.uniform(0.0, 1e15, nc)
    T0 = deck.tref + rng.uniform(-0.5, 0.5, nc)
    (fa, _), (fb, _) = solve_pair(deck, prec, T0=T0, heat=heat, iters=10)
    tol = 1e-10 if prec == g.GBTE_FP64 else 1e-5
    for k in ("T", "E", "q", "Tband"):
        assert rel(fa[k], fb[k]) <= tol, (k, rel(fa[k], fb[k]))


def test_orders_agree_3d():
    # jittered tetrahedra (40 x 40 x 100 nm, h = 10 nm), 4 bands, 32
    # directions, solved to 1e-11 margins: faces that close an upwind cycle
    # are lagged by cell index, so the two orders may take different paths
    # to the same fixed point
    deck = decks.config3_deck(h_nm=10.0, size_nm=(40.0, 40.0, 100.0), n_bands=4, n_theta=2, n_phi=2,
                              residual_temp=1e-11, residual_flux=1e-11, max_iter=4000)
    (fa, _), (fb, _) = solve_pair(deck, g.GBTE_FP64)
    assert rel(fa["T"], fb["T"]) <= 1e-9, rel(fa["T"], fb["T"])
    assert rel(fa["q"], fb["q"]) <= 1e-8, rel(fa["q"], fb["q"])


def test_batch_orders_agree():
    pop = decks.porous_population(3, seed=1, h_nm=(15.0, 22.0), r_nm=(40.0, 80.0), n_bands=4, n_phi=2)
    out = []
    for order in (0, 1):
        s = g.StaticBTESynthetic.from_decks(pop, precision=g.GBTE_FP64, cell_order=order)
        off = s.geometry_offsets()
        s.solve(max_iter=12, err_temp=0.0, err_flux=0.0, allow_not_converged=True)
        out.append((off, s.fields()))
        s.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert rel(out[0][1]["T"], out[1][1]["T"]) <= 1e-10


def test_written_files_follow_callers_order(tmp_path):
    deck, _ = mg.load(mg.CASES[0])
    rows = []
    for order in (0, 1):
        d = tmp_path / str(order)
        os.makedirs(d)
        s = g.StaticBTESynthetic.from_deck(deck, precision=g.GBTE_FP64, cell_order=order)
        s.solve(allow_not_converged=False)
        s.write_outputs(str(d))
        s.close()
        rows.append({n: np.loadtxt(d / n) for n in ("Temperature.dat", "HeatFlux.dat", "Tempband.dat")})
        with open(d / "Result.vtk") as f:
            vtk = f.read()
        rows[-1]["cells"] = vtk[vtk.index("CELLS"):vtk.index("CELL_DATA")]
    for n in ("Temperature.dat", "HeatFlux.dat", "Tempband.dat"):
        assert rows[0][n].shape == rows[1][n].shape
        # per column, relative to the column's largest magnitude
        scale = np.maximum(np.max(np.abs(rows[1][n]), axis=0), 1e-300)
        assert np.max(np.abs(rows[0][n] - rows[1][n]) / scale) <= 1e-10
    assert rows[0]["cells"] == rows[1]["cells"]
