"""GPU: the drop-in boundary end to end, and the output files.

oracle/_ref/BTE_B200 is the reference's own program (BTEMain.cpp,
Solution.cpp and the rest of its sources, unmodified) compiled against the
B200 drop-in classes of giftbte_b200/shim/ in place of its own
StaticBTESynthetic and Transient (make -C oracle dropin). Run on a deck directory, it
reads the deck with the reference's readers, runs the reference's Fourier
pre-solve on the CPU, hands its fields to the drop-in class exactly as
SolutionAll::_BTE_Solver does (src/Solution/Solution.cpp:262-414), solves
on the GPU, and writes the reference's result files. Its fields must match
the compiled reference's (golden fixtures) to 1e-9, and its files, like
those of gbte_write_outputs, must have the reference's layout.
"""
import os
import subprocess

import numpy as np
import pytest

import make_golden as mg
import oracle
from giftbte_b200 import GBTE_FP64, StaticBTESynthetic

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(oracle.DROPIN_BIN), reason="drop-in program not built")]

TOL = 1e-9


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("case", ["gray_square_tri", "quad_heat_specular", "periodic_jitter", "porous_msh",
                                  "porous_firstorder", "periodic_sequential", "quad_firstorder_sequential",
                                  "porous_limiter", "interface_2mat", "alamode_square", "shengbte_square"])
def test_reference_program_with_b200_solver_matches_reference(case, tmp_path):
    # every variant the CONTROL file selects (Order 1/2/2limit, Synthetic or
    # Sequential) goes through its own solve* method of the drop-in class
    deck, ref = mg.load(case)
    deck.write(str(tmp_path))
    out = oracle.run_reference(str(tmp_path), timeout=1200, binary=oracle.DROPIN_BIN)
    assert out["iters"] > 0
    if case not in mg.CONVERGED:
        assert out["iters"] == ref["iters"]
    assert rel(out["T"], ref["T"]) <= TOL, rel(out["T"], ref["T"])
    assert rel(out["E"], ref["E"]) <= TOL, rel(out["E"], ref["E"])
    assert rel(out["q"], ref["q"]) <= TOL, rel(out["q"], ref["q"])
    assert rel(out["Tband"], ref["Tband"]) <= TOL, rel(out["Tband"], ref["Tband"])
    # the same Fourier start (the reference's own pre-solve ran on the CPU)
    assert rel(out["Tf"], ref["Tf"]) <= 1e-12


def tokens(path):
    with open(path) as f:
        return [line.split() for line in f if line.strip()]


# columns compared on one scale: coordinates together, the three flux
# components together (as the field parity tests take the flux's max norm)
COLUMN_GROUPS = {"Temperature.dat": [(0, 1, 2), (3,)], "TempLattice.dat": [(0, 1, 2), (3,)],
                 "HeatFlux.dat": [(0, 1, 2), (3, 4, 5)], "Tempband.dat": [(0,), (1, 2, 3), (4,)]}


def assert_same_file(ours, theirs, tol=TOL):
    """Line by line and column by column: the same words where the
    reference writes words (headers, VTK keywords), and numbers within tol
    relative to the largest magnitude of their column group: the groups of
    COLUMN_GROUPS for the .dat files; in Result.vtk all columns of a
    section (a section starts at each line that begins with a word), so
    points, cells, temperatures and flux vectors each have their own scale."""
    a, b = tokens(ours), tokens(theirs)
    assert len(a) == len(b), (ours, len(a), len(b))
    groups_of = COLUMN_GROUPS.get(os.path.basename(ours))
    groups = {}
    section = 0
    for la, lb in zip(a, b):
        assert len(la) == len(lb), (ours, la, lb)
        try:
            float(lb[0])
        except ValueError:
            section += 1
        for col, (x, y) in enumerate(zip(la, lb)):
            try:
                fy = float(y)
            except ValueError:
                assert x == y, (ours, x, y)
                continue
            if groups_of:
                key = (section, [i for i, gcols in enumerate(groups_of) if col in gcols][0])
            else:
                key = (section,)
            groups.setdefault(key, []).append((float(x), fy))
    for key, pairs in groups.items():
        v = np.asarray(pairs)
        scale = max(float(np.max(np.abs(v[:, 1]))), 1e-300)
        err = float(np.max(np.abs(v[:, 0] - v[:, 1]))) / scale
        assert err <= tol, (ours, key, err)


@pytest.mark.parametrize("case", ["quad_heat_specular", "periodic_jitter"])
def test_output_files_match_reference_files(case, tmp_path):
    # the compiled reference's own files on the CPU, the drop-in program's,
    # and gbte_write_outputs' from the library's API, on the same deck
    deck, _ = mg.load(case)
    ref_dir, drop_dir, api_dir = (tmp_path / n for n in ("ref", "dropin", "api"))
    for d in (ref_dir, drop_dir, api_dir):
        d.mkdir()
    deck.write(str(ref_dir))
    deck.write(str(drop_dir))
    oracle.run_reference(str(ref_dir), timeout=1200)
    oracle.run_reference(str(drop_dir), timeout=1200, binary=oracle.DROPIN_BIN)
    files = ["Temperature.dat", "TempLattice.dat", "HeatFlux.dat", "Tempband.dat", "Result.vtk"]
    for f in files:
        assert_same_file(str(drop_dir / f), str(ref_dir / f))
    # the library's writer: the reference's fixed point from its Fourier start
    ref = oracle.read_reference_outputs(str(ref_dir))
    s = StaticBTESynthetic.from_deck(deck, precision=GBTE_FP64, macro_exact=1)
    s.set_initial(ref["Tf"], ref["qf"])
    s.solve(allow_not_converged=False)
    s.write_outputs(str(api_dir))
    s.close()
    for f in files:
        assert_same_file(str(api_dir / f), str(ref_dir / f))


def test_reference_program_transient_with_b200_solver(tmp_path):
    # State=Transient: SolutionAll::_Transient_BTE_Solver (Solution.cpp:500-520)
    # hands the drop-in Transient class its objects; the GPU run's TTG.dat,
    # Tempcell.dat and HeatFlux.dat match the compiled reference's
    deck, ref = mg.load("grating_transient")
    deck.write(str(tmp_path))
    out = oracle.run_reference(str(tmp_path), timeout=600, binary=oracle.DROPIN_BIN)
    assert len(out["ttg"]) == len(ref["ttg"])
    assert np.array_equal(out["ttg"][:, 0], ref["ttg"][:, 0])
    assert rel(out["ttg"][:, 1], ref["ttg"][:, 1]) <= TOL, rel(out["ttg"][:, 1], ref["ttg"][:, 1])
    assert np.array_equal(out["xyz"], ref["xyz"])
    assert rel(out["T"], ref["T"]) <= TOL, rel(out["T"], ref["T"])
    assert rel(out["q"], ref["q"]) <= TOL, rel(out["q"], ref["q"])
