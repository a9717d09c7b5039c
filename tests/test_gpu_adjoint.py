"""GPU: the adjoint (gbte_vjp) of the converged FP64 solve.

The parameters are those of the adjoint workload:
- a multiplier on each band's relaxation time;
- a per-cell scattering multiplier field, log-normal with sigma 0.2 and seed 2;
- the specularity p = 0.3 of a partially specular pore wall.
The objective is k_x, the effective conductivity along the 1 K periodic jump.

The adjoint gradient is checked against central finite differences (relative
step 1e-6) of the forward solve run on the GPU, and against central
differences of the CPU oracle's solve (the FP64 reference gradient). Both
sides are converged to 1e-12 margins. The agreement asked for is 1e-4.
First, the two forward extensions (per-cell multiplier, partial specularity)
are checked against the oracle.
"""
import dataclasses
import functools

import numpy as np
import pytest

import giftbte_b200 as g
import oracle
from giftbte_b200 import decks

pytestmark = pytest.mark.gpu

L = 300e-9      # cell side: k_x = <q_x>_V L / dT with dT = 1 K
TOL = 1e-4      # adjoint vs finite differences
H = 1e-6        # relative central-difference step


@functools.lru_cache(maxsize=None)
def base_deck():
    """Config-4 cell at h = 20 nm (405 cells), 4 bands, 16 directions."""
    return decks.config4_deck(h_nm=20.0, n_bands=4, n_phi=4, seed=2, residual_temp=1e-12, residual_flux=1e-12,
                              max_iter=8000)


@functools.lru_cache(maxsize=None)
def scatter():
    return decks.lognormal_scatter(base_deck().mesh.n_cells, sigma=0.2, seed=2)


def variant(tau_mult=None, p=None):
    d = base_deck()
    bands = d.bands
    if tau_mult is not None:
        bands = dataclasses.replace(bands, tau=bands.tau * tau_mult)
    bcs = [b if (b.tag != 5 or p is None) else decks.BC(5, 6, p) for b in d.bcs]
    return dataclasses.replace(d, bands=bands, bcs=bcs)


def keff_from(q, vol):
    return float(np.sum(q[:, 0] * vol) / vol.sum() * L / 1.0)


def solve_gpu(d, s_c):
    s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64, cell_scatter=s_c)
    s.solve(allow_not_converged=False)
    return s


def keff_gpu(d, s_c):
    s = solve_gpu(d, s_c)
    _, vol = s.geometry()
    k = keff_from(s.fields()["q"], vol)
    s.close()
    return k


@functools.lru_cache(maxsize=None)
def volumes():
    s = g.StaticBTESynthetic.from_deck(base_deck(), precision=g.GBTE_FP64)
    _, vol = s.geometry()
    s.close()
    return vol


def keff_oracle(d, s_c):
    o = oracle.solve(d, cell_scatter=s_c)
    return keff_from(o["q"], volumes())


@functools.lru_cache(maxsize=None)
def adjoint():
    s = solve_gpu(base_deck(), scatter())
    qb = s.keff_cotangent(axis=0, length=L, delta_T=1.0)
    out = s.vjp(q_bar=qb)
    out["J"] = float(np.sum(qb * s.fields()["q"]))
    s.close()
    return out


def components(n_cells=5):
    """(name, perturbed deck and multipliers) pairs for the checked
    components: every band multiplier, the pore wall's specularity, the
    cells with the largest adjoint sensitivity, and a seeded random
    direction over all cell multipliers."""
    a = adjoint()
    nb = base_deck().bands.n_bands
    out = []
    for b in range(nb):
        def f(h, b=b):
            m = np.ones(nb)
            m[b] += h
            return variant(tau_mult=m), scatter()
        out.append((f"tau[{b}]", a["tau"][b], f))

    def fp(h):
        return variant(p=0.3 + h), scatter()
    spec_row = [i for i, b in enumerate(base_deck().bcs) if b.tag == 5][0]
    out.append(("p", a["specularity"][spec_row], fp))
    top = np.argsort(-np.abs(a["scatter"]))[:n_cells]
    for c in top:
        def fc(h, c=int(c)):
            s = scatter().copy()
            s[c] *= 1 + h
            return base_deck(), s
        # d/d(ln s_c) = s_c dJ/ds_c
        out.append((f"s[{c}]", a["scatter"][c] * scatter()[c], fc))
    v = np.random.default_rng(20).standard_normal(base_deck().mesh.n_cells)

    def fv(h):
        return base_deck(), scatter() * (1 + h * v)
    out.append(("s.v", float(np.dot(a["scatter"] * scatter(), v)), fv))
    return out


def check(keff, label):
    rows = []
    scale = max(abs(x) for _, x, _ in components())
    for name, g_adj, make in components():
        kp = keff(*make(H))
        km = keff(*make(-H))
        fd = (kp - km) / (2 * H)
        err = abs(g_adj - fd) / max(abs(fd), 1e-2 * scale)
        rows.append((name, g_adj, fd, err))
    text = "\n".join(f"{label} {n:8s} adjoint {a: .10e} fd {f: .10e} rel {e:.2e}" for n, a, f, e in rows)
    print(text)
    assert max(r[3] for r in rows) <= TOL, text


def test_extensions_match_oracle():
    # per-cell scattering multipliers and a partially specular wall: the
    # CUDA forward against the oracle
    d = base_deck()
    s = solve_gpu(d, scatter())
    f = s.fields()
    s.close()
    o = oracle.solve(d, cell_scatter=scatter())
    assert np.max(np.abs(f["T"] - o["T"])) / np.max(np.abs(o["T"])) <= 1e-9
    assert np.max(np.abs(f["q"] - o["q"])) / np.max(np.abs(o["q"])) <= 1e-8


def test_adjoint_converged():
    st = adjoint()["stats"]
    assert st["change"] <= 1e-10 and st["picard_steps"] >= 1 and st["iterations"] > 1


def test_adjoint_matches_gpu_finite_differences():
    check(keff_gpu, "gpu-fd")


def test_adjoint_matches_oracle_finite_differences():
    check(keff_oracle, "oracle-fd")


def test_temperature_objective():
    # mean macro temperature of the cells with x < L/4: the temperature
    # cotangent enters through the transposed synthetic correction
    s = solve_gpu(base_deck(), scatter())
    cen, vol = s.geometry()
    sel = cen[:, 0] < 0.25 * L
    Tb = np.where(sel, vol, 0.0) / vol[sel].sum()
    a = s.vjp(T_bar=Tb)
    s.close()

    def J(d, s_c):
        t = solve_gpu(d, s_c)
        v = float(np.dot(Tb, t.fields()["T"]))
        t.close()
        return v
    nb = base_deck().bands.n_bands
    for b in (0, nb - 1):
        m = np.ones(nb)
        m[b] += H
        jp = J(variant(tau_mult=m), scatter())
        m[b] -= 2 * H
        jm = J(variant(tau_mult=m), scatter())
        fd = (jp - jm) / (2 * H)
        scale = np.max(np.abs(a["tau"]))
        assert abs(a["tau"][b] - fd) <= TOL * max(abs(fd), 1e-2 * scale), (b, a["tau"][b], fd)
    jp = J(variant(p=0.3 + H), scatter())
    jm = J(variant(p=0.3 - H), scatter())
    fd = (jp - jm) / (2 * H)
    row = [i for i, b in enumerate(base_deck().bcs) if b.tag == 5][0]
    assert abs(a["specularity"][row] - fd) <= TOL * max(abs(fd), 1e-12), (a["specularity"][row], fd)


def test_adjoint_rejects_unsupported():
    d = base_deck()
    s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP32_MIXED)
    s.solve(max_iter=3, err_temp=0.0, err_flux=0.0)
    with pytest.raises(g.GBTEError):
        s.vjp(q_bar=np.zeros((d.mesh.n_cells, 3)))
    s.close()
    s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64)
    with pytest.raises(g.GBTEError):
        s.vjp(q_bar=np.zeros((d.mesh.n_cells, 3)))
    s.close()


def fd_check(make_deck, s_c, objective, components):
    """Adjoint of `objective` (a function of a solved handle returning
    (J, T_bar, q_bar)) against central differences for the listed
    (name, adjoint-gradient getter, perturbed-deck maker) components."""
    s = solve_gpu(make_deck(0.0, None), s_c)
    _, Tb, qb = objective(s)
    a = s.vjp(T_bar=Tb, q_bar=qb)
    s.close()
    out = []
    for name, get, make in components:
        vals = []
        for h in (H, -H):
            t = solve_gpu(*make(h))
            vals.append(objective(t)[0])
            t.close()
        fd = (vals[0] - vals[1]) / (2 * H)
        out.append((name, get(a), fd))
    return out


def test_scalar_band_kernels():
    # 3 bands (not a multiple of 4): the one-band-per-thread adjoint kernels
    def deck(p=0.3):
        return decks.config4_deck(h_nm=25.0, n_bands=3, n_phi=4, seed=3, specularity=p, residual_temp=1e-12,
                                  residual_flux=1e-12, max_iter=8000)
    d0 = deck()
    sc = decks.lognormal_scatter(d0.mesh.n_cells, sigma=0.2, seed=4)

    def objective(s):
        qb = s.keff_cotangent(axis=0, length=L, delta_T=1.0)
        return float(np.sum(qb * s.fields()["q"])), None, qb

    def tau_mult(b, h):
        m = np.ones(3)
        m[b] += h
        return dataclasses.replace(d0, bands=dataclasses.replace(d0.bands, tau=d0.bands.tau * m))
    row = [i for i, b in enumerate(d0.bcs) if b.tag == 5][0]
    rows = fd_check(lambda h, _: d0, sc, objective, [
        ("tau[1]", lambda a: a["tau"][1], lambda h: (tau_mult(1, h), sc)),
        ("p", lambda a: a["specularity"][row], lambda h: (deck(0.3 + h), sc)),
        ("s[0]", lambda a: a["scatter"][0] * sc[0], lambda h: (d0, sc * np.where(np.arange(len(sc)) == 0, 1 + h, 1.0))),
    ])
    for name, ga, fd in rows:
        assert abs(ga - fd) <= TOL * max(abs(fd), 1e-3 * max(abs(r[2]) for r in rows)), (name, ga, fd)


def test_3d_hotspot_temperature():
    # 3D tetrahedra (40 x 40 x 100 nm, h = 10 nm), 4 bands, 32 Gauss
    # directions, heat in the top 20 nm, partially specular side walls
    # (p = 0.4); objective: the mean temperature of the heated region
    def deck(p=0.4, m=None):
        d = decks.config3_deck(h_nm=10.0, size_nm=(40.0, 40.0, 100.0), n_bands=4, n_theta=2, n_phi=2,
                               residual_temp=1e-12, residual_flux=1e-12, max_iter=8000)
        d = dataclasses.replace(d, bcs=[decks.BC(1, 1, 300.0), decks.BC(2, 2, 0.0)] +
                                [decks.BC(t, 6, p) for t in (3, 4, 5, 6)])
        if m is not None:
            d = dataclasses.replace(d, bands=dataclasses.replace(d.bands, tau=d.bands.tau * m))
        return d
    d0 = deck()
    heat = d0.cell_heat()
    hot = heat > 0

    def objective(s):
        _, vol = s.geometry()
        Tb = np.where(hot, vol, 0.0) / vol[hot].sum()
        return float(np.dot(Tb, s.fields()["T"])), Tb, None

    def mult(b, h):
        m = np.ones(4)
        m[b] += h
        return m
    rows_bc = [i for i, b in enumerate(d0.bcs) if b.type == 6]
    rows = fd_check(lambda h, _: d0, None, objective, [
        ("tau[0]", lambda a: a["tau"][0], lambda h: (deck(m=mult(0, h)), None)),
        ("tau[3]", lambda a: a["tau"][3], lambda h: (deck(m=mult(3, h)), None)),
        ("p", lambda a: sum(a["specularity"][i] for i in rows_bc), lambda h: (deck(p=0.4 + h), None)),
    ])
    for name, ga, fd in rows:
        assert abs(ga - fd) <= TOL * max(abs(fd), 1e-3 * max(abs(r[2]) for r in rows)), (name, ga, fd)


def test_forward_state_survives_vjp():
    # the adjoint reuses only the transport scratch: a solve continued after
    # gbte_vjp matches one that was never interrupted, bit for bit
    d = base_deck()
    qb = None
    out = []
    for with_vjp in (True, False):
        s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64, cell_scatter=scatter())
        s.solve(max_iter=40, err_temp=0.0, err_flux=0.0)
        if with_vjp:
            qb = s.keff_cotangent(axis=0, length=L, delta_T=1.0)
            s.vjp(q_bar=qb, max_iter=20)
        s.solve(max_iter=15, err_temp=0.0, err_flux=0.0)
        out.append(s.fields())
        s.close()
    for k in ("T", "E", "q", "Tband"):
        assert np.array_equal(out[0][k], out[1][k]), k


def test_adjoint_rejects_solver_variants():
    # the adjoint transposes the second-order Synthetic scheme only
    import make_golden as mg

    for case in ("porous_firstorder", "periodic_sequential"):
        d, _ = mg.load(case)
        s = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64)
        s.solve(max_iter=3, err_temp=0.0, err_flux=0.0)
        with pytest.raises(g.GBTEError):
            s.vjp(q_bar=np.zeros((d.mesh.n_cells, 3)))
        s.close()


def test_config4_full_size_against_finite_differences():
    # the adjoint workload at full size: the 300 nm porous cell (3 nm mesh,
    # 17,939 triangles), 40 bands, 64 directions, pore wall p = 0.3,
    # log-normal cell multipliers (sigma 0.2, seed 2); objective k_x. The
    # partially specular wall gives this cell a slow mode (about 0.9977 per
    # outer iteration: 13,000 iterations from margins 1e-8 to 1e-12), so each
    # central difference (relative step 1e-6) compares two forward runs of
    # the same fixed number of iterations from the same Fourier start: their
    # remaining slow-mode parts nearly cancel in the difference. Twenty
    # seeded components: eight band tau multipliers (seeded draw), the
    # specularity, and eleven seeded random directions over the cell
    # multiplier field with positive weights U(0, 1) (one cell alone moves
    # k_x by ~1e-10 relative, below what differences resolve, and signed
    # weights cancel to the same level). The adjoint stops on its residual
    # bound.
    n_fd = 1200
    d0 = decks.config4_deck(h_nm=3.0, n_bands=40, n_phi=16, seed=0, specularity=0.3, max_iter=20000)
    nc = d0.mesh.n_cells
    sc = decks.lognormal_scatter(nc, sigma=0.2, seed=2)
    s = g.StaticBTESynthetic.from_deck(d0, precision=g.GBTE_FP64, cell_scatter=sc)
    s.fourier_initial()
    s.solve(err_temp=1e-10, err_flux=1e-10, max_iter=20000)
    qb = s.keff_cotangent(axis=0, length=L, delta_T=1.0)
    a = s.vjp(q_bar=qb, tol=1e-8, max_iter=20000)
    s.close()
    assert a["stats"]["residual"] <= 1e-8
    rng = np.random.default_rng(20)
    nb = d0.bands.n_bands
    spec_row = [i for i, b in enumerate(d0.bcs) if b.tag == 5][0]

    def keff(d, s_c):
        h = g.StaticBTESynthetic.from_deck(d, precision=g.GBTE_FP64, cell_scatter=s_c)
        h.fourier_initial()
        h.solve(max_iter=n_fd, err_temp=0.0, err_flux=0.0)
        _, vol = h.geometry()
        k = keff_from(h.fields()["q"], vol)
        h.close()
        return k

    checks = []
    for b in rng.choice(nb, size=8, replace=False):
        def f(hh, b=int(b)):
            m = np.ones(nb)
            m[b] += hh
            return dataclasses.replace(d0, bands=dataclasses.replace(d0.bands, tau=d0.bands.tau * m)), sc
        checks.append((f"tau[{b}]", a["tau"][b], f))

    def fp(hh):
        return dataclasses.replace(d0, bcs=[b if b.tag != 5 else decks.BC(5, 6, 0.3 + hh) for b in d0.bcs]), sc
    checks.append(("p", a["specularity"][spec_row], fp))
    for i in range(11):
        v = rng.uniform(0.0, 1.0, nc)

        def fv(hh, v=v):
            return d0, sc * (1 + hh * v)
        # d/dh J(s (1 + h v)) = sum_c v_c s_c dJ/ds_c
        checks.append((f"cells.v{i}", float(np.sum(v * sc * a["scatter"])), fv))
    for name, adj, make in checks:
        kp = keff(*make(H))
        km = keff(*make(-H))
        fd = (kp - km) / (2 * H)
        assert abs(adj - fd) <= TOL * max(abs(fd), 1e-30), (name, adj, fd)


def test_anderson_and_plain_adjoint_agree():
    # the Anderson-accelerated transposed iteration (default) and the plain
    # one (adjoint_history = -1) solve the same adjoint equations: the same
    # gradient, both at the residual bound, the accelerated one in fewer
    # iterations
    out = {}
    for hist in (-1, 0):
        s = g.StaticBTESynthetic.from_deck(base_deck(), precision=g.GBTE_FP64, cell_scatter=scatter(),
                                           adjoint_history=hist)
        s.solve(allow_not_converged=False)
        qb = s.keff_cotangent(axis=0, length=L, delta_T=1.0)
        out[hist] = s.vjp(q_bar=qb, tol=1e-10, max_iter=20000)
        s.close()
        assert out[hist]["stats"]["residual"] <= 1e-10
    a, p = out[0], out[-1]
    for k in ("tau", "scatter"):
        assert np.max(np.abs(a[k] - p[k])) <= 1e-7 * np.max(np.abs(p[k])), k
    assert a["stats"]["iterations"] <= p["stats"]["iterations"]
