"""3D (tetrahedral) path: the config-3 hotspot-block decks.

The reference's public release has no 3D mesh code, so 3D parity is pinned
to the CPU oracle restatement (FP64, dimension-generic formulas), not to
reference outputs. Host-only tests check the deck tooling; the GPU tests
compare the CUDA path with the oracle.
"""
import dataclasses
import functools

import numpy as np
import pytest

import giftbte_b200 as g
import oracle
from giftbte_b200 import decks

TOL_FP64 = 1e-9
TOL_FP32 = 1e-5


@functools.lru_cache(maxsize=None)
def small_block(specular_sides: bool = False):
    """40 x 40 x 100 nm block, h = 10 nm (960 tets), 4 bands, 32 Gauss
    directions, heat in the top 20 nm; optionally specular x/y sides."""
    d = decks.config3_deck(h_nm=10.0, size_nm=(40.0, 40.0, 100.0), n_bands=4, n_theta=2, n_phi=2,
                           residual_temp=1e-11, residual_flux=1e-11, max_iter=4000)
    if specular_sides:
        d.bcs = [decks.BC(1, 1, 300.0), decks.BC(2, 2, 0.0)] + [decks.BC(t, 3, 0.0) for t in (3, 4, 5, 6)]
    return d


@functools.lru_cache(maxsize=None)
def oracle_fields(specular_sides: bool):
    return oracle.solve(small_block(specular_sides))


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_block_mesh_is_valid():
    m = decks.hex_tet_block_mesh(4, 4, 8, 2.5, jitter=0.2, seed=1, region_z=15.0)
    p = m.nodes[m.cells]
    vol = np.abs(np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])) / 6
    assert vol.min() > 0
    assert abs(vol.sum() - 10.0 * 10.0 * 20.0) < 1e-9
    assert m.n_cells == 4 * 4 * 8 * 6
    # every boundary triangle lies on one outer face, 2 per boundary square
    counts = {t: int(np.sum(m.edge_tags == t)) for t in range(1, 7)}
    assert counts == {1: 32, 2: 32, 3: 64, 4: 64, 5: 64, 6: 64}
    assert set(np.unique(m.cell_region)) == {0, 1}


def test_config3_sizes():
    info = g.inspect(small_block())
    assert info["dimension"] == 3 and info["num_cells"] == 960
    assert info["num_directions"] == 32
    full = decks.config3_deck.__defaults__  # h 2.5 nm, 40 bands, Ntheta 4, Nphi 4
    assert full[0] == 2.5 and full[1] == 40 and 8 * full[2] * full[3] == 128


def test_deck_files_round_trip_3d(tmp_path):
    d = small_block()
    d.write(str(tmp_path))
    a = g.inspect(d)
    b = g.inspect_deck(str(tmp_path))
    for k in ("dimension", "num_cells", "num_nodes", "num_faces", "num_boundaries", "num_directions",
              "max_levels", "lagged_faces"):
        assert a[k] == b[k], k
    assert abs(a["total_volume"] - b["total_volume"]) <= 1e-12 * a["total_volume"]


@pytest.mark.gpu
@pytest.mark.parametrize("specular", [False, True])
def test_fp64_matches_oracle_3d(specular):
    d = small_block(specular)
    o = oracle_fields(specular)
    s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64)
    st = s.solve(allow_not_converged=False)
    f = s.fields()
    s.close()
    assert st["err_temp"] <= 1e-11
    assert rel(f["T"], o["T"]) <= TOL_FP64, rel(f["T"], o["T"])
    assert rel(f["E"], o["E"]) <= TOL_FP64
    assert rel(f["Tband"], o["Tband"]) <= TOL_FP64
    assert rel(f["q"], o["q"]) <= 1e-9, rel(f["q"], o["q"])


@pytest.mark.gpu
def test_fp32_mixed_close_to_oracle_3d():
    d = small_block()
    o = oracle_fields(False)
    s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP32_MIXED, err_temp=1e-9, err_flux=1e-7)
    s.solve()
    f = s.fields()
    s.close()
    assert rel(f["T"], o["T"]) <= TOL_FP32, rel(f["T"], o["T"])


@pytest.mark.gpu
def test_deck_dir_and_memory_decks_agree_3d(tmp_path):
    d = small_block()
    d.write(str(tmp_path))
    a = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64)
    a.solve(max_iter=20, err_temp=0.0, err_flux=0.0, allow_not_converged=True)
    b = g.StaticBTESynthetic.from_deck_dir(str(tmp_path), precision=g.GBTE_FP64)
    b.set_initial(np.full(d.mesh.n_cells, d.tref))
    b.solve(max_iter=20, err_temp=0.0, err_flux=0.0, allow_not_converged=True)
    fa, fb = a.fields(), b.fields()
    a.close()
    b.close()
    assert rel(fa["T"], fb["T"]) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("opts", [{"sweep_far_slots": -1}, {"sweep_bands": 3}, {"sweep_bands": 1, "sweep_far_slots": 4},
                                  {"sweep_far_slots": -1, "sweep_kernel": 3},
                                  {"sweep_far_slots": -1, "sweep_kernel": 3, "sweep_bands": 3, "sweep_vector": 1}])
def test_sweep_variants_match_oracle_3d(opts):
    # far slots off (upwind reads older than the ring go to memory), an odd
    # band chunk (element-wise residual staging) and a far-slot cap below
    # what the plan needs (falls back to memory): same fixed point
    d = small_block()
    o = oracle_fields(False)
    s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64, **opts)
    s.solve(allow_not_converged=False)
    f = s.fields()
    s.close()
    assert rel(f["T"], o["T"]) <= TOL_FP64, rel(f["T"], o["T"])
    assert rel(f["q"], o["q"]) <= 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [g.GBTE_FP64, g.GBTE_FP32_MIXED])
def test_direction_batches_match_oracle_3d(prec):
    # the transport stage in uneven batches of 5 directions (32 = 6 x 5 + 2):
    # batch-sized gradient/residual/correction buffers, moments accumulated
    # over batches; same fixed point
    d = small_block()
    o = oracle_fields(False)
    kw = {} if prec == g.GBTE_FP64 else {"err_temp": 1e-9, "err_flux": 1e-7}
    s = g.StaticBTESynthetic.from_deck(d, precision=prec, direction_batch=5, **kw)
    st = s.solve(allow_not_converged=prec != g.GBTE_FP64)
    f = s.fields()
    s.close()
    assert st["direction_batch"] == 5
    tol = TOL_FP64 if prec == g.GBTE_FP64 else TOL_FP32
    assert rel(f["T"], o["T"]) <= tol, rel(f["T"], o["T"])


@pytest.mark.gpu
def test_extensions_match_oracle_3d():
    # partially specular side walls (p = 0.4) and per-cell scattering
    # multipliers on tetrahedra: the CUDA forward against the oracle
    d = dataclasses.replace(small_block(), bcs=[decks.BC(1, 1, 300.0), decks.BC(2, 2, 0.0)] +
                            [decks.BC(t, 6, 0.4) for t in (3, 4, 5, 6)])
    sc = decks.lognormal_scatter(d.mesh.n_cells, sigma=0.2, seed=7)
    o = oracle.solve(d, cell_scatter=sc)
    s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64, cell_scatter=sc)
    s.solve(allow_not_converged=False)
    f = s.fields()
    s.close()
    assert rel(f["T"], o["T"]) <= TOL_FP64, rel(f["T"], o["T"])
    assert rel(f["q"], o["q"]) <= 1e-9
