"""The C ABI: symbols, host-only inspection and error behaviour (no GPU)."""
import os
import re

import numpy as np
import pytest

import giftbte_b200 as g
from giftbte_b200 import decks

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "giftbte.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(gbte_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = g.library()
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(g.EXPORTS) == names


def test_status_strings():
    lib = g.library()
    for code in (0, -1, -2, -3, -4, -5, -6, -7, -8, 1):
        assert lib.gbte_status_string(code).decode() != "unknown status"


def test_inspect_gray_square():
    info = g.inspect(decks.config1_deck(40))
    assert info["num_cells"] == 3200 and info["num_nodes"] == 1681
    assert info["num_faces"] == 3 * 3200 // 2 + 160 // 2
    assert info["num_boundaries"] == 160 and info["num_boundary_sides"] == 320
    assert info["num_directions"] == 32 and info["num_bands"] == 1
    assert info["lagged_faces"] == 0 and info["max_levels"] > 40
    assert info["kappa_bulk"] == pytest.approx(1.66e6 * 6400.0 ** 2 * (1e-7 / 6400.0) / 2, rel=1e-14)
    assert info["total_volume"] == pytest.approx(1e-12, rel=1e-12)


@pytest.mark.parametrize("fmt", ["COMSOL", "MSH"])
def test_deck_files_round_trip(tmp_path, fmt):
    d = decks.config2_deck(h_nm=15.0, n_bands=5, n_phi=4, mesh_format=fmt)
    d.write(str(tmp_path))
    a = g.inspect(d)
    b = g.inspect_deck(str(tmp_path))
    for k in ("num_cells", "num_nodes", "num_faces", "num_boundaries", "num_bands", "num_directions", "max_levels"):
        assert a[k] == b[k], k
    assert b["kappa_bulk"] == pytest.approx(a["kappa_bulk"], rel=1e-15)
    assert b["total_volume"] == pytest.approx(a["total_volume"], rel=1e-12)
    # annulus area: 300 nm square minus a polygonal r = 100 nm pore
    assert b["total_volume"] == pytest.approx((300e-9) ** 2 - np.pi * (100e-9) ** 2, rel=2e-3)
    assert b["err_temp"] == d.residual_temp


@pytest.mark.parametrize("method,dim,nt,nphi,nd", [(1, 2, 4, 8, 32), (2, 2, 4, 16, 64), (1, 3, 2, 2, 32),
                                                   (2, 3, 4, 4, 128)])
def test_quadrature_sizes(method, dim, nt, nphi, nd):
    d = decks.config1_deck(4, angle_method=method, material_dim=dim, n_theta=nt, n_phi=nphi)
    assert g.inspect(d)["num_directions"] == nd


def test_missing_deck_is_io_error(tmp_path):
    with pytest.raises(g.GBTEError) as e:
        g.inspect_deck(str(tmp_path / "nope"))
    assert e.value.status == -2


def test_periodic_without_partner_is_mesh_error():
    d = decks.config1_deck(6)
    d.bcs = [decks.BC(1, -7, 1.0), decks.BC(2, 1, 0.0), decks.BC(3, 2, 0.0), decks.BC(4, 2, 0.0)]
    with pytest.raises(g.GBTEError) as e:
        g.inspect(d)
    assert e.value.status == -7


def test_bad_lattice_ratio_is_argument_error():
    d = decks.config1_deck(6)
    d.bands.lattice_ratio = d.bands.lattice_ratio * 0.5
    with pytest.raises(g.GBTEError) as e:
        g.inspect(d)
    assert e.value.status == -1


def test_interface_deck_reads_on_the_host(tmp_path):
    # two materials and an interface wall (BC type 5, transmissivity file)
    # written in the reference's formats read back on the host; the same
    # deck from memory gives the same sizes
    d = decks.interface_deck(8)
    d.write(str(tmp_path))
    a = g.inspect_deck(str(tmp_path))
    b = g.inspect(d)
    assert a["num_materials"] == 2 and b["num_materials"] == 2
    assert a["num_cells"] == b["num_cells"] == d.mesh.n_cells
    assert a["num_boundaries"] == b["num_boundaries"]


def test_interface_file_missing_and_type4_refused(tmp_path):
    d = decks.config1_deck(6)
    d.write(str(tmp_path))
    with open(tmp_path / "input" / "bc.dat", "w") as f:
        f.write("1 #n\n\nheader\n1 5 0 input/trans.dat\n")
    with pytest.raises(g.GBTEError) as e:
        g.inspect_deck(str(tmp_path))
    assert e.value.status == -2
    with open(tmp_path / "input" / "bc.dat", "w") as f:
        f.write("1 #n\n\nheader\n1 4 0 input/trans.dat\n")
    with pytest.raises(g.GBTEError) as e:
        g.inspect_deck(str(tmp_path))
    assert e.value.status == -8


def test_create_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(g.GBTEError) as e:
        g.StaticBTESynthetic.from_deck(decks.config1_deck(4))
    assert e.value.status == -3


@pytest.mark.parametrize("make", [lambda: decks.config1_deck(12), lambda: decks.config2_deck(h_nm=15.0, n_bands=4, n_phi=4),
                                  lambda: decks.interface_deck(8),
                                  lambda: decks.config3_deck(h_nm=25.0, size_nm=(100.0, 100.0, 100.0), n_bands=4)],
                         ids=["square", "porous", "interface", "block3d"])
def test_index_checks_pass_on_built_meshes(make, monkeypatch):
    # GBTE_DEBUG turns on the range checks of every CSR and index array the
    # solver would upload (mesh, schedule, sweep records, gradient and
    # residual tiles); they are off by default
    d = make()
    monkeypatch.delenv("GBTE_DEBUG", raising=False)
    assert g.inspect(d)["index_entries_checked"] == 0
    monkeypatch.setenv("GBTE_DEBUG", "1")
    info = g.inspect(d)
    assert info["index_entries_checked"] > 10 * info["num_cells"]


def test_index_checks_catch_planted_entries(tmp_path):
    # the checker itself, host only: tests/cpp/index_check_main.cpp builds the
    # arrays the solver uploads for a porous-cell deck, expects them to pass,
    # then plants one bad entry per array kind (a neighbour past the cells,
    # decreasing offsets, a negative stencil index, a wall side past the
    # range, a cell visited twice by a level order, a sweep record reading a
    # later position, tile indices past or beside their unions) and expects
    # each to be caught as a mesh error
    import shutil
    import subprocess

    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    csrc = os.path.join(ROOT, "giftbte_b200", "csrc")
    exe = str(tmp_path / "index_check")
    subprocess.check_call([gxx, "-std=c++17", "-O1", "-I", csrc, os.path.join(ROOT, "tests", "cpp", "index_check_main.cpp")] +
                          [os.path.join(csrc, f) for f in ("deck.cpp", "mesh.cpp", "angles.cpp")] +
                          ["-lpthread", "-o", exe])
    decks.config2_deck(h_nm=15.0, n_bands=4, n_phi=4).write(str(tmp_path / "deck"))
    r = subprocess.run([exe, str(tmp_path / "deck")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    assert lines[0].startswith("built: pass") and lines[1].startswith("tiles: pass")
    assert sum(": caught" in l for l in lines) == 8 and lines[-1] == "OK"


@pytest.mark.parametrize("kind", ["ALAMODE", "ShengBTE"])
def test_mode_list_band_files_read_on_the_host(kind, tmp_path):
    # a PHONON that names an ALAMODE lifetime file or a ShengBTE output
    # directory: the library's reader and the Python restatement of the
    # reference's reduction give the same band table to the last bit (through
    # kappa_bulk = sum C v^2 tau / dim and C_bulk = sum C)
    d = decks.mode_list_deck(kind)
    d.write(str(tmp_path))
    a = g.inspect_deck(str(tmp_path))
    b = g.inspect(d)
    assert a["num_bands"] == 12
    assert a["kappa_bulk"] == b["kappa_bulk"] and a["capacity_bulk"] == b["capacity_bulk"]
    t = d.bands
    assert b["kappa_bulk"] == pytest.approx(float(np.sum(t.C * t.v ** 2 * t.tau)) / 2, rel=1e-13)
    assert np.sum(t.lattice_ratio) == pytest.approx(1.0, abs=1e-12)
    assert np.sum(t.heat_ratio) == pytest.approx(1.0, abs=1e-12)


def test_mode_list_reductions_follow_the_reference_rules():
    # equal mode counts in file order, the last band taking the remainder;
    # ALAMODE: Gamma's zero modes count as modes of zero capacity; ShengBTE:
    # NaN and negative-rate modes are dropped before binning
    a = decks.synthetic_alamode(nk=7, nbr=6, seed=3)
    t = a.band_table(4)  # 42 modes: 10, 10, 10, 12
    kap = (a.kappa[..., 0] + a.kappa[..., 4] + a.kappa[..., 8]) * a.mult[:, None]
    tau = a.tau_ps * 1e-12
    with np.errstate(divide="ignore", invalid="ignore"):
        C = np.where((tau == 0) | (a.vel == 0), 0.0, kap / a.vel ** 2 / tau).ravel()
    assert t.C[0] == pytest.approx(C[:10].sum(), rel=1e-14)
    assert t.C[3] == pytest.approx(C[30:].sum(), rel=1e-14)
    s = decks.synthetic_shengbte(nirr=6, nq=20, nbr=3, seed=2)
    ts = s.band_table(2)
    assert np.all(np.isfinite(ts.v)) and np.all(ts.C > 0)


def test_mode_list_missing_files_are_io_errors(tmp_path):
    for kind, victim in (("ALAMODE", "input/alamode_1.dat"), ("ShengBTE", "input/shengbte_1/BTE.w_final")):
        d = decks.mode_list_deck(kind)
        root = tmp_path / kind
        d.write(str(root))
        os.remove(str(root / victim))
        with pytest.raises(g.GBTEError) as e:
            g.inspect_deck(str(root))
        assert e.value.status == -2


def test_transient_deck_reads_on_the_host(tmp_path):
    # CONTROL State=Transient with TimeStep and TotalTime; without them the
    # deck is refused as the reference refuses it (src/BTEMain.cpp:197-200)
    d = decks.grating_deck(steps=12)
    d.write(str(tmp_path / "a"))
    info = g.inspect_deck(str(tmp_path / "a"))
    assert info["transient"] == 1 and info["time_step"] == 1e-13
    assert info["total_time"] == pytest.approx(12e-13, rel=1e-15)
    d.write(str(tmp_path / "b"))
    ctl = tmp_path / "b" / "input" / "CONTROL"
    ctl.write_text(ctl.read_text().split("TimeStep=")[0])
    with pytest.raises(g.GBTEError) as e:
        g.inspect_deck(str(tmp_path / "b"))
    assert e.value.status == -2


def test_field_scatter_to_caller_order(tmp_path):
    # host only: gbte_get_fields moves each field from the library's cell
    # order to the caller's with gbte::scatter_rows, on the host's threads
    # (whole columns per thread, or ranges of rows for few columns);
    # tests/cpp/scatter_rows_main.cpp checks it against the serial scatter
    # on random permutations
    import shutil
    import subprocess

    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    csrc = os.path.join(ROOT, "giftbte_b200", "csrc")
    exe = str(tmp_path / "scatter_rows")
    subprocess.check_call([gxx, "-std=c++17", "-O1", "-I", csrc, os.path.join(ROOT, "tests", "cpp", "scatter_rows_main.cpp")] +
                          [os.path.join(csrc, f) for f in ("deck.cpp", "mesh.cpp", "angles.cpp")] +
                          ["-lpthread", "-o", exe])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.splitlines()[-1] == "OK", r.stdout + r.stderr


def test_fields_fill_caller_arrays(monkeypatch):
    # StaticBTESynthetic.fields(out=...) passes the caller's arrays to
    # gbte_get_fields (here a stand-in that writes through the pointers it
    # gets) and refuses arrays of the wrong shape, type or layout
    nc, nb = 7, 3

    class FakeLib:
        def gbte_get_fields(self, h, TE, TL, q, TB):
            for p, n, base in ((TE, nc, 1.0), (TL, nc, 2.0), (q, 3 * nc, 3.0), (TB, nb * nc, 4.0)):
                for i in range(n):
                    p[i] = base + i
            return g.GBTE_OK

    monkeypatch.setattr(g, "library", lambda: FakeLib())
    s = g.StaticBTESynthetic.__new__(g.StaticBTESynthetic)
    s._h, s.num_cells, s.num_bands = None, nc, nb
    out = {"T": np.zeros(nc), "Tband": np.zeros((nb, nc))}
    f = s.fields(out=out)
    assert f["T"] is out["T"] and f["Tband"] is out["Tband"]
    assert np.array_equal(f["T"], 2.0 + np.arange(nc)) and np.array_equal(f["E"], 1.0 + np.arange(nc))
    assert np.array_equal(f["q"], (3.0 + np.arange(3 * nc)).reshape(nc, 3))
    assert np.array_equal(f["Tband"], (4.0 + np.arange(nb * nc)).reshape(nb, nc))
    assert np.array_equal(s.fields()["q"], f["q"])
    for bad in (np.zeros(nc + 1), np.zeros(nc, dtype=np.float32), np.zeros((2, nc))[:, 0]):
        with pytest.raises(ValueError):
            s.fields(out={"E": bad})
