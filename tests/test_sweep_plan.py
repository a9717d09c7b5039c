"""Host checks of the sweep plan (no GPU).

The device sweep keeps the corrections of the last `ring` level-order
positions and, for the few upwind reads older than that, on-chip far slots
allocated per direction by the host plan (mesh.cpp build_sweep_plan). These
tests compile tests/cpp/sweep_plan_check.cpp against the library's host
sources and run, on several decks and ring sizes, a sweep that uses only the
ring and the far slots (level-parallel order, as on the device) against a
direct sweep: they must agree bit for bit. A planted wrong slot must be
caught.
"""
import functools
import os
import subprocess

import pytest

from giftbte_b200 import decks
from tests.golden import make_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "giftbte_b200", "csrc")
EXE = os.path.join(ROOT, "giftbte_b200", "_build", "tests", "sweep_plan_check")


@pytest.fixture(scope="module")
def checker():
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    srcs = [os.path.join(ROOT, "tests", "cpp", "sweep_plan_check.cpp")] + [
        os.path.join(CSRC, f) for f in ("mesh.cpp", "angles.cpp", "deck.cpp")]
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-pthread", "-I", CSRC, *srcs, "-o", EXE])
    return EXE


@functools.lru_cache(maxsize=None)
def _decks():
    out = {"config2_4bands": decks.config2_deck(h_nm=3.0, n_bands=4, n_phi=16, seed=0),
           "config1_gray": decks.config1_deck(20)}
    for name in ("periodic_jitter", "porous_msh", "quad_heat_specular"):
        out[name] = make_golden.load(name)[0]
    return out


@pytest.mark.parametrize("name", ["config2_4bands", "config1_gray", "periodic_jitter", "porous_msh",
                                  "quad_heat_specular"])
@pytest.mark.parametrize("min_ring", [1, 512])
def test_ring_and_far_slots_match_direct_sweep(checker, tmp_path, name, min_ring):
    d = _decks()[name]
    d.write(str(tmp_path))
    r = subprocess.run([checker, str(tmp_path), str(min_ring)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    f = dict(zip(r.stdout.split()[0::2], r.stdout.split()[1::2]))
    assert float(f["max_abs_diff"]) == 0.0
    ring = int(f["ring"])
    assert ring & (ring - 1) == 0


@pytest.mark.parametrize("name", ["config2_4bands", "periodic_jitter"])
def test_batch_of_copies_matches_direct_sweep(checker, tmp_path, name):
    # three copies as one batched problem: per-copy levels, ring and far
    # slots, tags remapped per copy (periodic partners stay in their copy)
    _decks()[name].write(str(tmp_path))
    r = subprocess.run([checker, str(tmp_path), "1", "plain", "3"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    f = dict(zip(r.stdout.split()[0::2], r.stdout.split()[1::2]))
    assert float(f["max_abs_diff"]) == 0.0


@pytest.mark.parametrize("name,copies", [("config2_4bands", 1), ("periodic_jitter", 1), ("porous_msh", 2),
                                         ("quad_heat_specular", 1)])
def test_locality_order_keeps_the_mesh(checker, tmp_path, name, copies):
    # cells renumbered along a Morton curve of their centres (inside each
    # copy of a batch): same cells, faces and boundary sides, neighbours
    # closer in memory, and the ring/far-slot sweep still exact
    _decks()[name].write(str(tmp_path))
    r = subprocess.run([checker, str(tmp_path), "1", "plain", str(copies), "morton"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    f = dict(zip(r.stdout.split()[0::2], r.stdout.split()[1::2]))
    assert float(f["max_abs_diff"]) == 0.0
    assert int(f["gap_after"]) <= max(8, int(f["gap_before"]))


def test_planted_wrong_slot_is_caught(checker, tmp_path):
    d = decks.config2_deck(h_nm=3.0, n_bands=4, n_phi=16, seed=0)
    d.write(str(tmp_path))
    r = subprocess.run([checker, str(tmp_path), "1", "perturb"], capture_output=True, text=True)
    f = dict(zip(r.stdout.split()[0::2], r.stdout.split()[1::2]))
    assert int(f["far_refs"]) > 0 and int(f["far_slots"]) > 1
    assert r.returncode == 1


def test_inspect_reports_the_plan():
    import giftbte_b200 as g

    info = g.inspect(decks.config2_deck(h_nm=3.0, n_bands=4, n_phi=16, seed=0))
    assert info["sweep_ring"] >= max(512, info["max_level_width"])
    assert info["sweep_ring"] & (info["sweep_ring"] - 1) == 0
    assert 0 < info["far_slots"] <= 2048
    assert info["far_refs"] > 0
