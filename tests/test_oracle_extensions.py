"""CPU: the oracle's two extensions reduce to the reference at their neutral
values. The extensions are a per-cell scattering multiplier s_c and the
partially specular wall (type 6, value p). Unit multipliers give the plain
solve bit for bit. p = 0 and p = 1 are the diffuse and specular walls. Values
in between give a field that differs from both ends."""
import dataclasses

import numpy as np

import oracle
from giftbte_b200 import decks


def small(p=None):
    d = decks.config4_deck(h_nm=20.0, n_bands=4, n_phi=4, seed=2, residual_temp=1e-10, residual_flux=1e-10,
                           max_iter=4000, specularity=0.3 if p is None else p)
    return d


def with_type(d, t):
    return dataclasses.replace(d, bcs=[b if b.tag != 5 else decks.BC(5, t, 0.0) for b in d.bcs])


def test_unit_multipliers_are_the_reference():
    d = small()
    a = oracle.solve(d)
    b = oracle.solve(d, cell_scatter=np.ones(d.mesh.n_cells))
    assert np.array_equal(a["T"], b["T"]) and np.array_equal(a["q"], b["q"])


def test_specularity_ends_are_the_reference_walls():
    for p, t in ((0.0, 2), (1.0, 3)):
        a = oracle.solve(small(p))
        b = oracle.solve(with_type(small(p), t))
        assert np.array_equal(a["T"], b["T"]) and np.array_equal(a["q"], b["q"])
    mid = oracle.solve(small(0.3))["q"]
    for t in (2, 3):
        end = oracle.solve(with_type(small(), t))["q"]
        assert np.max(np.abs(mid - end)) > 1e-6 * np.max(np.abs(end))


def test_scatter_field_changes_the_solution():
    d = small()
    s = decks.lognormal_scatter(d.mesh.n_cells, sigma=0.2, seed=2)
    a = oracle.solve(d)["q"]
    b = oracle.solve(d, cell_scatter=s)["q"]
    assert np.max(np.abs(a - b)) > 1e-4 * np.max(np.abs(a))
