"""Input-deck tooling: seeded synthetic meshes and reference-format deck files.

A GiftBTE run reads three keyword files from ``./input`` (CONTROL, GEOMETRY,
PHONON), a boundary-condition table, a mesh file and a material band table.
This module builds the meshes used by the parity tests and the benchmark and
writes them in exactly those formats, so the same deck can be handed to the
reference binary and to this library.

File formats follow the readers of the reference:
  * CONTROL / GEOMETRY / PHONON: keyword line, value on the next line
    (``src/BTEMain.cpp:87-315``).
  * BC table: count line, two header lines, then ``index type value``
    (``src/BTEBoundaryCondition/BTEBoundaryCondition.cpp:8-31``).
  * COMSOL ``.mphtxt`` 2D mesh (``src/BTEMesh/ReadinMesh.cpp:228-400``):
    vertex block, then ``vtx``/``edg``/``tri``/``quad`` element types each
    followed by their geometric-entity indices (0-based in the file; the
    reader adds 1 to edge tags and subtracts 1 from domain indices).
  * gmsh MSH 4.1 2D mesh (``src/BTEMesh/ReadinMesh.cpp:407-534``).
  * DATABASE band table: one line per band, ``|v| tau C lattice_ratio
    heat_ratio`` (``src/BTEBand/BTEBand.cpp:64-79``).
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


# ----------------------------------------------------------------------------
# meshes
# ----------------------------------------------------------------------------
@dataclasses.dataclass
class Mesh2D:
    """A 2D mesh in unit coordinates (multiplied by ScaleX/ScaleY on read).

    nodes:      (Nn, 2) float64
    cells:      list of vertex tuples (3 = triangle, 4 = quad in COMSOL
                "Z" order v0 v1 v2 v3 with faces v0-v1, v1-v3, v3-v2, v2-v0)
    edges:      (Ne, 2) int boundary edges
    edge_tags:  (Ne,) int boundary tags (1-based, as the BC file names them)
    cell_region:(Nc,) int region index (0-based, GeometryMaterialType row - 1)
    """

    nodes: np.ndarray
    cells: np.ndarray
    edges: np.ndarray
    edge_tags: np.ndarray
    cell_region: np.ndarray

    @property
    def n_cells(self) -> int:
        return int(self.cells.shape[0])


@dataclasses.dataclass
class Mesh3D:
    """A 3D tetrahedral mesh in unit coordinates (multiplied by ScaleX/Y/Z on
    read). Same field names as :class:`Mesh2D`, with triangles as boundary
    elements:

    nodes:      (Nn, 3) float64
    cells:      (Nc, 4) int tetrahedra
    edges:      (Nb, 3) int boundary triangles
    edge_tags:  (Nb,) int boundary tags (1-based, as the BC file names them)
    cell_region:(Nc,) int region index (0-based, GeometryMaterialType row - 1)
    """

    nodes: np.ndarray
    cells: np.ndarray
    edges: np.ndarray
    edge_tags: np.ndarray
    cell_region: np.ndarray

    @property
    def n_cells(self) -> int:
        return int(self.cells.shape[0])


def hex_tet_block_mesh(nx: int, ny: int, nz: int, h: float, jitter: float = 0.0, seed: int = 0,
                       region_z: Optional[float] = None) -> Mesh3D:
    """Structured nx x ny x nz grid of cubes of edge h on [0, nx h] x [0, ny h]
    x [0, nz h], each cube split into the 6 tetrahedra around its
    (0,0,0)-(1,1,1) diagonal (the same split in every cube, so faces match).
    Vertices are moved by a uniform random offset of up to jitter * h per
    coordinate (seeded), except along the coordinates in which they lie on
    the outer boundary. Boundary tags: 1 bottom (z = 0), 2 top, 3 x = 0,
    4 x = max, 5 y = 0, 6 y = max. Cells whose centre has z >= region_z are
    region 1, the rest region 0."""
    ix, iy, iz = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    grid = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1)  # node id = (i * (ny+1) + j) * (nz+1) + k

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    nodes = grid.astype(np.float64) * h
    if jitter > 0:
        rng = np.random.default_rng(seed)
        off = rng.uniform(-jitter * h, jitter * h, size=nodes.shape)
        lim = np.array([nx, ny, nz])
        off[(grid == 0) | (grid == lim)] = 0.0
        nodes += off
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    e = np.eye(3, dtype=int)
    tets = []
    for perm in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
        a = np.zeros(3, dtype=int)
        b = e[perm[0]]
        c = b + e[perm[1]]
        d = np.ones(3, dtype=int)
        tets.append(np.stack([nid(ci + p[0], cj + p[1], ck + p[2]) for p in (a, b, c, d)], axis=1))
    cells = np.stack(tets, axis=1).reshape(-1, 4)
    # boundary triangles: tet faces that occur once
    faces = np.concatenate([cells[:, [0, 1, 2]], cells[:, [0, 1, 3]], cells[:, [0, 2, 3]], cells[:, [1, 2, 3]]])
    key = np.sort(faces, axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    bfaces = faces[cnt[inv.ravel()] == 1]
    g = grid[bfaces]  # integer coordinates of the three vertices
    tags = np.zeros(len(bfaces), dtype=np.int64)
    for t, (axis, val) in enumerate(((2, 0), (2, nz), (0, 0), (0, nx), (1, 0), (1, ny)), start=1):
        on = np.all(g[:, :, axis] == val, axis=1)
        tags[(tags == 0) & on] = t
    assert np.all(tags > 0)
    cz = nodes[cells][:, :, 2].mean(axis=1)
    region = np.zeros(len(cells), dtype=np.int64)
    if region_z is not None:
        region[cz >= region_z] = 1
    # cells grouped by region, the order in which the MSH file lists them
    order = np.argsort(region, kind="stable")
    return Mesh3D(nodes=nodes, cells=cells[order], edges=bfaces, edge_tags=tags, cell_region=region[order])


def square_tri_mesh(nx: int, ny: int) -> Mesh2D:
    """Structured nx x ny grid on [0,1]^2, each square split into 2 triangles
    along its (0,0)-(1,1) diagonal. Boundary tags: 1 left, 2 right,
    3 bottom, 4 top."""
    xs = np.linspace(0.0, 1.0, nx + 1)
    ys = np.linspace(0.0, 1.0, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel()], axis=1)

    def nid(i, j):
        return i * (ny + 1) + j

    tris = []
    for i in range(nx):
        for j in range(ny):
            n00, n10, n01, n11 = nid(i, j), nid(i + 1, j), nid(i, j + 1), nid(i + 1, j + 1)
            tris.append((n00, n10, n11))
            tris.append((n00, n11, n01))
    edges, tags = [], []
    for j in range(ny):
        edges.append((nid(0, j), nid(0, j + 1))); tags.append(1)
        edges.append((nid(nx, j), nid(nx, j + 1))); tags.append(2)
    for i in range(nx):
        edges.append((nid(i, 0), nid(i + 1, 0))); tags.append(3)
        edges.append((nid(i, ny), nid(i + 1, ny))); tags.append(4)
    return Mesh2D(nodes=nodes, cells=np.asarray(tris, dtype=np.int64),
                  edges=np.asarray(edges, dtype=np.int64),
                  edge_tags=np.asarray(tags, dtype=np.int64),
                  cell_region=np.zeros(len(tris), dtype=np.int64))


def square_quad_mesh(nx: int, ny: int) -> Mesh2D:
    """Structured quad grid on [0,1]^2 (COMSOL vertex order), tags as in
    :func:`square_tri_mesh`."""
    xs = np.linspace(0.0, 1.0, nx + 1)
    ys = np.linspace(0.0, 1.0, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel()], axis=1)

    def nid(i, j):
        return i * (ny + 1) + j

    quads = []
    for i in range(nx):
        for j in range(ny):
            quads.append((nid(i, j), nid(i + 1, j), nid(i, j + 1), nid(i + 1, j + 1)))
    m = square_tri_mesh(nx, ny)
    return Mesh2D(nodes=nodes, cells=np.asarray(quads, dtype=np.int64), edges=m.edges,
                  edge_tags=m.edge_tags, cell_region=np.zeros(len(quads), dtype=np.int64))


def jitter_interior(mesh: Mesh2D, amount: float, seed: int) -> Mesh2D:
    """Move interior nodes by a uniform random offset in [-amount, amount]^2
    (unit coordinates); boundary nodes stay on the boundary."""
    rng = np.random.default_rng(seed)
    nodes = mesh.nodes.copy()
    bnd = np.zeros(len(nodes), dtype=bool)
    bnd[mesh.edges.ravel()] = True
    d = rng.uniform(-amount, amount, size=nodes.shape)
    nodes[~bnd] += d[~bnd]
    return dataclasses.replace(mesh, nodes=nodes)


def _poisson_disk(rng, h, inside, bbox, k=20):
    """Bridson-style Poisson-disk sample with spacing h inside bbox."""
    (x0, y0), (x1, y1) = bbox
    cell = h / np.sqrt(2.0)
    gw, gh = int(np.ceil((x1 - x0) / cell)) + 1, int(np.ceil((y1 - y0) / cell)) + 1
    grid = -np.ones((gw, gh), dtype=np.int64)
    pts: List[Tuple[float, float]] = []
    active: List[int] = []

    def fits(p):
        gi, gj = int((p[0] - x0) / cell), int((p[1] - y0) / cell)
        for a in range(max(gi - 2, 0), min(gi + 3, gw)):
            for b in range(max(gj - 2, 0), min(gj + 3, gh)):
                q = grid[a, b]
                if q >= 0 and (pts[q][0] - p[0]) ** 2 + (pts[q][1] - p[1]) ** 2 < h * h:
                    return False
        return True

    def add(p):
        pts.append(p)
        grid[int((p[0] - x0) / cell), int((p[1] - y0) / cell)] = len(pts) - 1
        active.append(len(pts) - 1)

    while True:
        p = (rng.uniform(x0, x1), rng.uniform(y0, y1))
        if inside(p):
            add(p)
            break
    while active:
        idx = active[rng.integers(len(active))]
        base = pts[idx]
        placed = False
        for _ in range(k):
            r = rng.uniform(h, 2 * h)
            t = rng.uniform(0, 2 * np.pi)
            p = (base[0] + r * np.cos(t), base[1] + r * np.sin(t))
            if x0 <= p[0] < x1 and y0 <= p[1] < y1 and inside(p) and fits(p):
                add(p)
                placed = True
                break
        if not placed:
            active.remove(idx)
    return np.asarray(pts, dtype=np.float64)


def porous_cell_mesh(h: float, pores: Sequence[Tuple[float, float, float]], seed: int,
                     side: float = 1.0) -> Mesh2D:
    """Periodic square cell [0,side]^2 with circular pores (cx, cy, r), all
    in unit coordinates, meshed as a Delaunay triangulation of Poisson-disk
    interior points plus evenly spaced boundary points. ``h`` is the target
    mean edge length: boundary points are h apart and the Poisson-disk
    minimum distance is h / 1.5 (the mean Delaunay edge of a maximal
    Poisson-disk sample is about 1.5 times its minimum distance).

    The x- and y-faces carry identical node positions (translation-matched),
    which the reference's nearest-face-centre periodic pairing needs
    (``src/BTEMesh/BTEMesh.cpp:905-924``). Tags: 1 left, 2 right, 3 bottom,
    4 top, 5 + k for the wall of pore k.
    """
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    n_side = max(int(round(side / h)), 2)
    s = np.linspace(0.0, side, n_side + 1)
    bpts = []
    for v in s[:-1]:
        bpts += [(v, 0.0), (side, v), (side - v, side), (0.0, side - v)]
    pore_pts = []
    for (cx, cy, r) in pores:
        m = max(int(round(2 * np.pi * r / h)), 8)
        t = np.arange(m) * 2 * np.pi / m
        pore_pts.append(np.stack([cx + r * np.cos(t), cy + r * np.sin(t)], axis=1))

    margin = 0.5 * h

    def inside(p):
        if p[0] < margin or p[0] > side - margin or p[1] < margin or p[1] > side - margin:
            return False
        for (cx, cy, r) in pores:
            if (p[0] - cx) ** 2 + (p[1] - cy) ** 2 < (r + margin) ** 2:
                return False
        return True

    ipts = _poisson_disk(rng, h / 1.5, inside, ((0.0, 0.0), (side, side)))
    pts = np.concatenate([np.asarray(bpts)] + pore_pts + [ipts], axis=0)
    tri = Delaunay(pts)
    simp = tri.simplices
    cent = pts[simp].mean(axis=1)
    keep = np.ones(len(simp), dtype=bool)
    for (cx, cy, r) in pores:
        keep &= (cent[:, 0] - cx) ** 2 + (cent[:, 1] - cy) ** 2 > r * r
    simp = simp[keep]
    # drop unused nodes (none expected) and renumber
    used = np.unique(simp)
    remap = -np.ones(len(pts), dtype=np.int64)
    remap[used] = np.arange(len(used))
    pts = pts[used]
    simp = remap[simp]
    # boundary edges = edges used by exactly one triangle
    e = np.concatenate([simp[:, [1, 2]], simp[:, [2, 0]], simp[:, [0, 1]]], axis=0)
    es = np.sort(e, axis=1)
    uniq, cnt = np.unique(es, axis=0, return_counts=True)
    bedges = uniq[cnt == 1]
    tags = np.zeros(len(bedges), dtype=np.int64)
    mid = pts[bedges].mean(axis=1)
    tol = 1e-9 * side
    tags[np.abs(mid[:, 0]) < tol] = 1
    tags[np.abs(mid[:, 0] - side) < tol] = 2
    tags[np.abs(mid[:, 1]) < tol] = 3
    tags[np.abs(mid[:, 1] - side) < tol] = 4
    for k, (cx, cy, r) in enumerate(pores):
        d = np.hypot(mid[:, 0] - cx, mid[:, 1] - cy)
        tags[(tags == 0) & (d < r + 0.5 * h)] = 5 + k
    if np.any(tags == 0):
        raise RuntimeError("porous_cell_mesh: unclassified boundary edge")
    return Mesh2D(nodes=pts, cells=simp.astype(np.int64), edges=bedges.astype(np.int64),
                  edge_tags=tags, cell_region=np.zeros(len(simp), dtype=np.int64))


# ----------------------------------------------------------------------------
# bands
# ----------------------------------------------------------------------------
@dataclasses.dataclass
class BandTable:
    """Per-band properties of one material (DATABASE columns)."""

    v: np.ndarray          # |group velocity| m/s
    tau: np.ndarray        # relaxation time s
    C: np.ndarray          # heat capacity J/m^3K
    lattice_ratio: np.ndarray
    heat_ratio: np.ndarray

    @property
    def n_bands(self) -> int:
        return int(len(self.v))


def gray_band(v: float, mfp: float, C: float) -> BandTable:
    one = np.ones(1)
    return BandTable(v=one * v, tau=one * (mfp / v), C=one * C, lattice_ratio=one.copy(),
                     heat_ratio=one.copy())


HBAR = 1.054571817e-34
KB = 1.380649e-23


def sine_dispersion_bands(n_bands: int, T: float = 300.0, kmax: float = 1.1e10,
                          wmax_la: float = 7.0e13, wmax_ta: float = 2.8e13,
                          n_k: int = 4000) -> BandTable:
    """Isotropic sine dispersion (1 LA + 2 TA branches, w = wmax sin(pi k /
    2 kmax)), binned into n_bands equal-frequency bands.

    Per mode: v = dw/dk, C = Bose-Einstein mode heat capacity at T with a
    spherical-shell density of states k^2 dk / (2 pi^2), and
    tau^-1 = 1.3e-45 w^4 + 1.7e-19 w^2 T exp(-137/T).
    Band aggregation: C_b = sum C, v_b = sum C v / C_b,
    tau_b = sum C v^2 tau / (C_b v_b^2), lattice_ratio = heat_ratio = C_b / C.
    """
    k = (np.arange(n_k) + 0.5) * kmax / n_k
    dk = kmax / n_k
    wmax_all = max(wmax_la, wmax_ta)
    edges = np.linspace(0.0, wmax_all, n_bands + 1)
    Cb = np.zeros(n_bands); Cv = np.zeros(n_bands); Cv2t = np.zeros(n_bands)
    for wmax, mult in ((wmax_la, 1), (wmax_ta, 2)):
        w = wmax * np.sin(0.5 * np.pi * k / kmax)
        v = wmax * 0.5 * np.pi / kmax * np.cos(0.5 * np.pi * k / kmax)
        x = HBAR * w / (KB * T)
        cm = KB * x * x * np.exp(x) / np.expm1(x) ** 2 * k * k * dk / (2 * np.pi ** 2) * mult
        tau = 1.0 / (1.3e-45 * w ** 4 + 1.7e-19 * w ** 2 * T * np.exp(-137.0 / T))
        idx = np.clip(np.searchsorted(edges, w, side="right") - 1, 0, n_bands - 1)
        np.add.at(Cb, idx, cm)
        np.add.at(Cv, idx, cm * v)
        np.add.at(Cv2t, idx, cm * v * v * tau)
    vb = Cv / Cb
    taub = Cv2t / (Cb * vb * vb)
    ratio = Cb / Cb.sum()
    # renormalise so the ratios sum to one at 17 significant digits
    ratio = ratio / ratio.sum()
    return BandTable(v=vb, tau=taub, C=Cb, lattice_ratio=ratio, heat_ratio=ratio.copy())


# ----------------------------------------------------------------------------
# first-principles mode lists (ALAMODE lifetime files, ShengBTE outputs)
# ----------------------------------------------------------------------------
def _div(a: float, b: float) -> float:
    """a / b with IEEE semantics where Python raises (b == 0)."""
    if b != 0.0:
        return a / b
    if a != a or a == 0.0:
        return math.nan
    return math.copysign(math.inf, a) * math.copysign(1.0, b)


def bin_modes(C: Sequence[float], v: Sequence[float], k: Sequence[float], n_bands: int) -> BandTable:
    """A mode list (capacity C, |v|, conductivity contribution k, in file
    order) reduced to n_bands bands of equal mode count, the last taking the
    remainder, as the reference's readers do (src/BTEBand/BTEBand.cpp:568-613,
    :691-724): v = sum C v / sum C, C = sum C, tau = sum k / C / v / v,
    lattice_ratio = (C / tau) / sum (C / tau), heat_ratio = C / sum C. The
    sums run mode by mode in file order (plain float arithmetic, so the table
    is the C++ reader's to the last bit)."""
    n = len(C)
    per = n // n_bands
    sC = [0.0] * n_bands
    sCv = [0.0] * n_bands
    sk = [0.0] * n_bands
    for j in range(n):
        b = min(j // per, n_bands - 1) if per > 0 else n_bands - 1
        sC[b] += float(C[j])
        sCv[b] += float(C[j]) * float(v[j])
        sk[b] += float(k[j])
    vb, tb, cb = [], [], []
    sumL = sumheat = 0.0
    for b in range(n_bands):
        vv = _div(sCv[b], sC[b])
        cc = sC[b]
        tt = _div(_div(_div(sk[b], cc), vv), vv)
        vb.append(vv)
        cb.append(cc)
        tb.append(tt)
        sumL += _div(cc, tt)
        sumheat += cc
    lat = [_div(_div(cb[b], tb[b]), sumL) for b in range(n_bands)]
    hr = [_div(cb[b], sumheat) for b in range(n_bands)]
    return BandTable(v=np.array(vb), tau=np.array(tb), C=np.array(cb), lattice_ratio=np.array(lat),
                     heat_ratio=np.array(hr))


@dataclasses.dataclass
class AlamodeModes:
    """An ALAMODE lifetime file (`anphon` result analyser output): per
    (k-point, branch) the frequency [cm^-1], lifetime [ps], |v| [m/s], MFP
    [nm], multiplicity and the per-mode conductivity tensor xx .. zz
    [W/mK]."""

    freq: np.ndarray     # (nk, nbr)
    tau_ps: np.ndarray   # (nk, nbr)
    vel: np.ndarray      # (nk, nbr)
    mfp: np.ndarray      # (nk, nbr)
    mult: np.ndarray     # (nk,) integers
    kappa: np.ndarray    # (nk, nbr, 9)
    seed: Optional[int] = None  # synthetic_alamode's seed, when it made them

    def write(self, path: str) -> None:
        nk, nbr = self.freq.shape
        with open(path, "w") as f:
            f.write("# Result analyzer ver. 1.0.5\n# Input file : synthetic.result\n")
            f.write("# Phonon lifetime at temperature 300 K.\n")
            f.write(f"# kpoint range 1 {nk}\n# mode   range 1 {nbr}\n")
            f.write("#  ik,  is, Frequency [cm^{-1}], Lifetime [ps], |Velocity| [m/s], MFP [nm], Multiplicity, "
                    "Thermal conductivity par mode (xx, xy, ...) [W/mK]\n")
            for i in range(nk):
                for b in range(nbr):
                    f.write("%5d %4d %.17g %.17g %.17g %.17g %d %s\n" % (
                        i + 1, b + 1, self.freq[i, b], self.tau_ps[i, b], self.vel[i, b], self.mfp[i, b],
                        int(self.mult[i]), " ".join("%.17g" % x for x in self.kappa[i, b])))

    def band_table(self, n_bands: int) -> BandTable:
        """The reference's reduction (BTEBand.cpp:629-731): kappa = (xx + yy
        + zz) multiplicity, C = kappa / v / v / tau (0 where tau or v is 0)."""
        nk, nbr = self.freq.shape
        C, v, k = [], [], []
        for i in range(nk):
            for b in range(nbr):
                t = float(self.tau_ps[i, b]) * 1e-12
                vel = float(self.vel[i, b])
                kap = (float(self.kappa[i, b, 0]) + float(self.kappa[i, b, 4]) + float(self.kappa[i, b, 8])) \
                    * float(self.mult[i])
                C.append(0.0 if (t == 0.0 or vel == 0.0) else kap / vel / vel / t)
                v.append(vel)
                k.append(kap)
        return bin_modes(C, v, k, n_bands)


def synthetic_alamode(nk: int = 203, nbr: int = 6, seed: int = 0) -> AlamodeModes:
    """Seeded synthetic modes in the ALAMODE layout: three acoustic and
    nbr - 3 optical branches, the first k-point's acoustic modes at zero
    frequency, lifetime and velocity (as at Gamma), the conductivity tensor
    nearly isotropic with small off-diagonal terms."""
    rng = np.random.default_rng(seed)
    kk = (np.arange(nk) + 0.5) / nk
    freq = np.zeros((nk, nbr))
    for b in range(nbr):
        top = 150.0 + 70.0 * b if b < 3 else 400.0 + 15.0 * b
        freq[:, b] = top * (np.sin(0.5 * np.pi * kk) if b < 3 else 1.0 - 0.1 * kk) * rng.uniform(0.97, 1.03, nk)
    tau_ps = np.exp(rng.uniform(np.log(0.5), np.log(300.0), (nk, nbr)))
    vel = rng.uniform(300.0, 9000.0, (nk, nbr))
    mult = rng.choice([1, 2, 4, 6, 8, 12, 24, 48], nk)
    cmode = rng.uniform(20.0, 400.0, (nk, nbr))
    kappa = np.zeros((nk, nbr, 9))
    for i in range(9):
        kappa[:, :, i] = cmode * vel ** 2 * tau_ps * 1e-12 / 3.0 / mult[:, None] * (
            rng.uniform(0.9, 1.1, (nk, nbr)) if i in (0, 4, 8) else rng.uniform(-1e-3, 1e-3, (nk, nbr)))
    freq[0, :3] = 1e-10
    tau_ps[0, :3] = 0.0
    vel[0, :3] = 0.0
    kappa[0, :3, :] = 0.0
    mfp = vel * tau_ps * 1e-3
    return AlamodeModes(freq=freq, tau_ps=tau_ps, vel=vel, mfp=mfp, mult=mult, kappa=kappa, seed=seed)


# the constants of the reference's ShengBTE reader (BTEBand.cpp:521-523)
SHENGBTE_KB = 1.38062e-23
SHENGBTE_HBAR = 1.05459e-34


@dataclasses.dataclass
class ShengBTEData:
    """A ShengBTE output directory: CONTROL (lfactor [nm], lattice vectors,
    T), BTE.omega (irreducible q-points x branches, rad/ps),
    BTE.qpoints_full (full grid: index, irreducible index, coordinates),
    BTE.w_final and BTE.v (one row per branch and irreducible q-point,
    branch-major: frequency and scattering rate [1/ps]; velocity [km/s])."""

    lfactor: float
    lattvec: np.ndarray   # (3, 3), row r = lattvec(:, r + 1)
    T: float
    omega: np.ndarray     # (nirr, nbr)
    q_irr: np.ndarray     # (nq,) 1-based irreducible index of each full-grid point
    q_xyz: np.ndarray     # (nq, 3)
    w: np.ndarray         # (nbr * nirr,) scattering rates
    v: np.ndarray         # (nbr * nirr, 3)
    seed: Optional[int] = None  # synthetic_shengbte's seed, when it made them

    def write(self, directory: str) -> None:
        os.makedirs(directory, exist_ok=True)
        a = self.lattvec
        with open(os.path.join(directory, "CONTROL"), "w") as f:
            f.write("&allocations\n        nelements=1,\n        natoms=2,\n        ngrid(:)=5 5 5\n&end\n")
            f.write("&crystal\n        lfactor=%.17g,\n" % self.lfactor)
            for r in range(3):
                f.write("        lattvec(:,%d)= %.17g %.17g %.17g\n" % (r + 1, a[r, 0], a[r, 1], a[r, 2]))
            f.write('        elements="Xx"\n        types=1 1,\n&end\n')
            f.write("&parameters\n        T=%.17g\n        scalebroad=1\n&end\n" % self.T)
            f.write("&flags\n        convergence=.TRUE.\n        isotopes=.true.\n&end\n")
        nirr, nbr = self.omega.shape
        with open(os.path.join(directory, "BTE.omega"), "w") as f:
            for i in range(nirr):
                f.write(" ".join("%.17g" % x for x in self.omega[i]) + "\n")
        with open(os.path.join(directory, "BTE.qpoints_full"), "w") as f:
            for q in range(len(self.q_irr)):
                f.write("%d %d %.17g %.17g %.17g\n" % (q + 1, int(self.q_irr[q]), *self.q_xyz[q]))
        with open(os.path.join(directory, "BTE.w_final"), "w") as f:
            for r in range(nbr * nirr):
                f.write("%.17g %s\n" % (self.omega[r % nirr, r // nirr],
                                         "NaN" if self.w[r] != self.w[r] else "%.17g" % self.w[r]))
        with open(os.path.join(directory, "BTE.v"), "w") as f:
            for r in range(nbr * nirr):
                f.write("%.17g %.17g %.17g\n" % tuple(self.v[r]))

    def cell_volume(self) -> float:
        """The reference's cell volume (BTEBand.cpp:296), lattvec(1,2) in
        place of lattvec(2,1) in one term, times lfactor^3 and 1e-27."""
        a = [[float(x) for x in row] for row in self.lattvec]
        lf = float(self.lfactor)
        vol = (a[0][0] * a[1][1] * a[2][2] + a[1][0] * a[2][1] * a[0][2] + a[0][1] * a[1][2] * a[2][0]
               - a[0][2] * a[1][1] * a[2][0] - a[0][1] * a[0][1] * a[2][2] - a[0][0] * a[1][2] * a[2][1]) \
            * lf * lf * lf
        return abs(vol) * 1e-27

    def band_table(self, n_bands: int) -> BandTable:
        """The reference's reduction (BTEBand.cpp:506-613): per full-grid mode,
        branch by branch, C = (1/V) kB x^2 e^x / (e^x - 1)^2 / Nq with
        x = hbar omega / (kB T), tau = 1 / w, k = C v^2 tau; modes whose k is
        NaN or negative are dropped."""
        nirr, nbr = self.omega.shape
        nq = len(self.q_irr)
        V = self.cell_volume()
        T = float(self.T)
        C, v, k = [], [], []
        for b in range(nbr):
            for q in range(nq):
                irr = int(self.q_irr[q]) - 1
                row = b * nirr + irr
                om = float(self.omega[irr, b]) * 1e12
                t = _div(1.0, float(self.w[row])) * 1e-12
                vx, vy, vz = (float(x) * 1000 for x in self.v[row])
                vel = math.pow(math.pow(vx, 2) + math.pow(vy, 2) + math.pow(vz, 2), 0.5)
                x = SHENGBTE_HBAR * om / SHENGBTE_KB / T
                ex = math.exp(x)
                cap = _div(1 / V * SHENGBTE_KB * x * x * ex, math.pow(ex - 1, 2))
                kk = cap / nq * vel * vel * t
                if kk != kk or not kk >= 0:
                    continue
                C.append(cap / nq)
                v.append(vel)
                k.append(kk)
        return bin_modes(C, v, k, n_bands)


def synthetic_shengbte(nirr: int = 40, nq: int = 150, nbr: int = 6, seed: int = 1) -> ShengBTEData:
    """Seeded synthetic ShengBTE outputs: a skewed cell (so the reference's
    volume quirk matters), the first irreducible point at zero frequency with
    a NaN rate (Gamma), one negative rate (its modes drop out), and every
    full-grid point mapped to an irreducible one."""
    rng = np.random.default_rng(seed)
    lattvec = np.array([[0.0, 0.30, 0.28], [0.26, 0.0, 0.29], [0.27, 0.31, 0.0]]) * 10.0
    kk = (np.arange(nirr) + 0.5) / nirr
    omega = np.zeros((nirr, nbr))
    for b in range(nbr):
        top = 15.0 + 8.0 * b if b < 3 else 50.0 + 2.0 * b
        omega[:, b] = top * (np.sin(0.5 * np.pi * kk) if b < 3 else 1.0 - 0.1 * kk) * rng.uniform(0.97, 1.03, nirr)
    omega[0, :] = 0.0
    w = np.exp(rng.uniform(np.log(1e-3), np.log(2.0), nbr * nirr))
    w[[b * nirr for b in range(nbr)]] = np.nan
    w[nirr + 7] = -w[nirr + 7]
    v = rng.uniform(-8.0, 8.0, (nbr * nirr, 3))
    q_irr = np.concatenate([[1], rng.integers(1, nirr + 1, nq - 1)])
    q_xyz = rng.uniform(-0.5, 0.5, (nq, 3))
    return ShengBTEData(lfactor=0.1, lattvec=lattvec, T=300.0, omega=omega, q_irr=q_irr, q_xyz=q_xyz, w=w, v=v,
                        seed=seed)


# ----------------------------------------------------------------------------
# writers
# ----------------------------------------------------------------------------
def write_mphtxt(path: str, mesh: Mesh2D) -> None:
    """COMSOL text mesh, 2D, in the layout the reference parser expects."""
    nn = len(mesh.nodes)
    out = ["# Created by COMSOL Multiphysics.", "", "# Major & minor version", "0 1 ",
           "1 # number of tags", "# Tags", "5 mesh1 ", "1 # number of types", "# Types",
           "3 obj ", "", "# --------- Object 0 ----------", "", "0 0 1 ", "4 Mesh # class",
           "4 # version", "2 # sdim", f"{nn} # number of mesh vertices",
           "0 # lowest mesh vertex index", "", "# Mesh vertex coordinates"]
    out += [f"{x:.17g} {y:.17g} " for x, y in mesh.nodes]
    by_nv: Dict[int, List[int]] = {}
    for i, c in enumerate(mesh.cells):
        by_nv.setdefault(len(c), []).append(i)
    types = [("edg", 2, mesh.edges, mesh.edge_tags - 1)]
    for nv, name in ((3, "tri"), (4, "quad")):
        if nv in by_nv:
            ids = by_nv[nv]
            types.append((name, nv, np.asarray(mesh.cells)[ids], np.asarray(mesh.cell_region)[ids] + 1))
    out += ["", f"{len(types)} # number of element types"]
    for t, (name, nv, elems, ent) in enumerate(types):
        out += ["", f"# Type #{t}", "", f"3 {name} # type name", "", "",
                f"{nv} # number of vertices per element", f"{len(elems)} # number of elements",
                "# Elements"]
        out += [" ".join(str(int(v)) for v in e) + " " for e in elems]
        out += ["", f"{len(elems)} # number of geometric entity indices",
                "# Geometric entity indices"]
        out += [f"{int(v)} " for v in ent]
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def write_msh41(path: str, mesh: Mesh2D) -> None:
    """gmsh MSH 4.1 ASCII, 2D: one node block, line elements tagged by their
    boundary tag (entity tag), triangle/quad elements in entity (region+1)."""
    nn = len(mesh.nodes)
    lines = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$Nodes",
             f"1 {nn} 1 {nn}", f"2 1 0 {nn}"]
    lines += [str(i + 1) for i in range(nn)]
    lines += [f"{x:.17g} {y:.17g} 0" for x, y in mesh.nodes]
    lines += ["$EndNodes", "$Elements"]
    blocks = []
    tags = np.unique(mesh.edge_tags)
    for t in tags:
        sel = mesh.edges[mesh.edge_tags == t]
        blocks.append((1, int(t), 1, sel))
    for reg in np.unique(mesh.cell_region):
        cs = np.asarray(mesh.cells)[np.asarray(mesh.cell_region) == reg]
        tri = [c for c in cs if len(c) == 3]
        quad = [c for c in cs if len(c) == 4]
        if tri:
            blocks.append((2, int(reg) + 1, 2, np.asarray(tri)))
        if quad:
            # gmsh quads are counter-clockwise; the reader maps a0 a1 a3 a2
            q = np.asarray(quad)[:, [0, 1, 3, 2]]
            blocks.append((2, int(reg) + 1, 3, q))
    total = sum(len(b[3]) for b in blocks)
    lines.append(f"{len(blocks)} {total} 1 {total}")
    eid = 1
    for dim, tag, typ, els in blocks:
        lines.append(f"{dim} {tag} {typ} {len(els)}")
        for e in els:
            lines.append(f"{eid} " + " ".join(str(int(v) + 1) for v in e))
            eid += 1
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_msh41_3d(path: str, mesh: Mesh3D) -> None:
    """gmsh MSH 4.1 ASCII, 3D: one node block, boundary triangles tagged by
    their boundary tag (entity tag), tetrahedra in entity (region + 1)."""
    nn = len(mesh.nodes)
    lines = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$Nodes",
             f"1 {nn} 1 {nn}", f"3 1 0 {nn}"]
    lines += [str(i + 1) for i in range(nn)]
    lines += [f"{x:.17g} {y:.17g} {z:.17g}" for x, y, z in mesh.nodes]
    lines += ["$EndNodes", "$Elements"]
    blocks = []
    for t in np.unique(mesh.edge_tags):
        blocks.append((2, int(t), 2, mesh.edges[mesh.edge_tags == t]))
    for reg in np.unique(mesh.cell_region):
        blocks.append((3, int(reg) + 1, 4, mesh.cells[mesh.cell_region == reg]))
    total = sum(len(b[3]) for b in blocks)
    lines.append(f"{len(blocks)} {total} 1 {total}")
    eid = 1
    for dim, tag, typ, els in blocks:
        lines.append(f"{dim} {tag} {typ} {len(els)}")
        for el in els:
            lines.append(f"{eid} " + " ".join(str(int(v) + 1) for v in el))
            eid += 1
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_band_database(path: str, bands: BandTable) -> None:
    with open(path, "w") as f:
        for i in range(bands.n_bands):
            f.write(f"{bands.v[i]:.17g} {bands.tau[i]:.17g} {bands.C[i]:.17g} "
                    f"{bands.lattice_ratio[i]:.17g} {bands.heat_ratio[i]:.17g}\n")


def write_interface_file(path: str, trans) -> None:
    """The reference's interface file: per material a line "<m> # matter
    index" (0-based) and one transmissivity per band, blocks separated by
    an empty line."""
    t = np.asarray(trans, dtype=np.float64)
    with open(path, "w") as f:
        for m in range(t.shape[0]):
            f.write(f"{m} # matter index\n")
            for v in t[m]:
                f.write(f"{v:.17g}\n")
            f.write("\n")


@dataclasses.dataclass
class BC:
    tag: int
    type: int      # 1 isothermal, 2 diffuse, 3 specular, 5 interface, <0 periodic (partner = -type),
                   # 6 partially specular
    value: float   # wall temperature / periodic temperature jump / specularity (type 6)
    # type 5: transmissivity of every band from each material's side,
    # (n_materials, n_bands); written as the reference's interface file
    trans: Optional[np.ndarray] = None


@dataclasses.dataclass
class Deck:
    """A complete steady synthetic-BTE input deck."""

    mesh: Mesh2D
    bands: BandTable
    bcs: List[BC]
    scale: Tuple[float, float] = (1e-6, 1e-6)
    material_dim: int = 2
    angle_method: int = 1
    n_theta: int = 4
    n_phi: int = 8
    tref: float = 300.0
    residual_temp: float = 1e-8
    residual_flux: float = 1e-8
    max_iter: int = 10000
    order: str = "2"                      # CONTROL Order: "1" or "2"
    scheme: str = "Synthetic"             # CONTROL IterativeScheme: "Synthetic" or "Sequential"
    heat_source: Optional[float] = None   # uniform volumetric heat (W/m^3)
    mesh_format: str = "COMSOL"           # COMSOL or MSH (3D meshes: MSH)
    region_heat: Optional[List[float]] = None  # heat per region (W/m^3), HeatType REGION
    # more materials: extra_materials[k] is material k + 1 (material 0 is
    # `bands`, same band count); region_material[r] is region r's material
    # (0-based; None: every region is material 0)
    extra_materials: List[BandTable] = dataclasses.field(default_factory=list)
    region_material: Optional[List[int]] = None
    # where each material's bands come from in the written deck: None (or a
    # None entry) writes the band table as a DATABASE file; an AlamodeModes
    # or ShengBTEData entry writes that mode list instead (MaterialFile
    # ALAMODE / ShengBTE), whose reduction the material's BandTable must be
    material_sources: Optional[List[object]] = None
    # CONTROL State: "Steady", or "Transient" with TimeStep and TotalTime (s)
    state: str = "Steady"
    time_step: float = -1.0
    total_time: float = -1.0

    @property
    def materials(self) -> List[BandTable]:
        return [self.bands] + list(self.extra_materials)

    def region_materials(self) -> List[int]:
        if self.region_material is not None:
            return list(self.region_material)
        return [0] * self.n_regions

    @property
    def dimension(self) -> int:
        return int(self.mesh.nodes.shape[1])

    @property
    def n_regions(self) -> int:
        return int(np.max(self.mesh.cell_region)) + 1

    def cell_heat(self) -> Optional[np.ndarray]:
        """Volumetric heat per cell, or None when there is none."""
        if self.region_heat is not None:
            return np.asarray(self.region_heat, dtype=np.float64)[np.asarray(self.mesh.cell_region)]
        if self.heat_source is not None:
            return np.full(self.mesh.n_cells, float(self.heat_source))
        return None

    def write(self, root: str) -> str:
        """Write ``root/input/*``; returns the input directory."""
        d = os.path.join(root, "input")
        os.makedirs(d, exist_ok=True)
        mesh_name = "mesh.mphtxt" if self.mesh_format == "COMSOL" else "mesh.msh"
        if self.dimension == 3:
            if self.mesh_format != "MSH":
                raise ValueError("3D meshes are written as MSH")
            write_msh41_3d(os.path.join(d, mesh_name), self.mesh)
        elif self.mesh_format == "COMSOL":
            write_mphtxt(os.path.join(d, mesh_name), self.mesh)
        else:
            write_msh41(os.path.join(d, mesh_name), self.mesh)
        band_files = []  # (PHONON source keyword, path under input/)
        for k, bt in enumerate(self.materials):
            src = self.material_sources[k] if self.material_sources and k < len(self.material_sources) else None
            if isinstance(src, AlamodeModes):
                name = f"alamode_{k + 1}.dat"
                src.write(os.path.join(d, name))
                band_files.append(("ALAMODE", name))
            elif isinstance(src, ShengBTEData):
                name = f"shengbte_{k + 1}"
                src.write(os.path.join(d, name))
                band_files.append(("ShengBTE", name))
            else:
                name = "bands.dat" if k == 0 else f"bands_{k + 1}.dat"
                write_band_database(os.path.join(d, name), bt)
                band_files.append(("DATABASE", name))
        with open(os.path.join(d, "bc.dat"), "w") as f:
            f.write(f"{len(self.bcs)} #Number of boundaries\n\n")
            f.write("BoundaryIndex BoundaryType BoundaryValue\n")
            for b in self.bcs:
                if b.type == 5:
                    tname = f"interface_{b.tag}.dat"
                    write_interface_file(os.path.join(d, tname), b.trans)
                    f.write(f"{b.tag} {b.type} {b.value:.17g} input/{tname}\n")
                else:
                    f.write(f"{b.tag} {b.type} {b.value:.17g}\n")
        with open(os.path.join(d, "CONTROL"), "w") as f:
            f.write("State=\n%s\nOrder=\n%s\nIterativeScheme=\n%s\nMatrixSolver=\nLU\n"
                    "Tref=\n%.17g\nMaxNumIter=\n%d\nResidualTemp=\n%.17g\nResidualFlux=\n%.17g\n"
                    % (self.state, self.order, self.scheme, self.tref, self.max_iter, self.residual_temp,
                       self.residual_flux))
            if self.state == "Transient":
                f.write("TimeStep=\n%.17g\nTotalTime=\n%.17g\n" % (self.time_step, self.total_time))
        with open(os.path.join(d, "GEOMETRY"), "w") as f:
            f.write("GeometryDimension=\n%d\nScaleX=\n%.17g\nScaleY=\n%.17g\n"
                    % (self.dimension, self.scale[0], self.scale[1]))
            if self.dimension == 3:
                f.write("ScaleZ=\n%.17g\n" % self.scale[2])
            f.write("BCFile=\ninput/bc.dat\nMeshType=\n%s\nMeshFile=\ninput/%s\n"
                    % (self.mesh_format, mesh_name))
            if self.heat_source is not None:
                f.write("UniformHeat=\n%.17g\n" % self.heat_source)
            if self.region_heat is not None:
                f.write("HeatType=\nREGION\nHeatFile=\ninput/heat.dat\n")
        if self.region_heat is not None:
            with open(os.path.join(d, "heat.dat"), "w") as f:
                f.write(f"{len(self.region_heat)}\n")
                for i, q in enumerate(self.region_heat):
                    f.write(f"{i + 1} {q:.17g}\n")
        rm = self.region_materials()
        with open(os.path.join(d, "PHONON"), "w") as f:
            f.write("MaterialNumber=\n%d\nBandNumber=\n%d\n\n" % (len(band_files), self.bands.n_bands))
            for k, (kind, name) in enumerate(band_files):
                f.write("MaterialFile %d:  %s\ninput/%s\n\n" % (k + 1, kind, name))
            f.write("GeometryMaterialType=\n%s\n\nMaterialDimension=\n%d\nAngle_method=\n%d\n"
                    "Ntheta=\n%d\nNphi=\n%d\n"
                    % ("\n".join(f"{r + 1} {rm[r] + 1}" for r in range(self.n_regions)),
                       self.material_dim, self.angle_method, self.n_theta, self.n_phi))
        return d


# ----------------------------------------------------------------------------
# the named workloads
# ----------------------------------------------------------------------------
def two_region_tri_mesh(nx: int, ny: int) -> Mesh2D:
    """square_tri_mesh with the cells right of x = 1/2 in region 1 and the
    edges on x = 1/2 as boundary elements of tag 5 (nx even): two materials
    meeting at an interface wall."""
    if nx % 2:
        raise ValueError("nx must be even")
    m = square_tri_mesh(nx, ny)
    cen = m.nodes[np.asarray(m.cells)].mean(axis=1)
    region = (cen[:, 0] > 0.5).astype(np.int64)

    def nid(i, j):
        return i * (ny + 1) + j
    i = nx // 2
    extra = [(nid(i, j), nid(i, j + 1)) for j in range(ny)]
    edges = np.concatenate([np.asarray(m.edges), np.asarray(extra, dtype=np.int64)])
    tags = np.concatenate([np.asarray(m.edge_tags), np.full(len(extra), 5, dtype=np.int64)])
    return Mesh2D(nodes=m.nodes, cells=m.cells, edges=edges, edge_tags=tags, cell_region=region)


def interface_deck(n: int = 16, n_bands: int = 4, n_phi: int = 4, **kw) -> Deck:
    """Two materials in a 100 nm square, meeting at x = 50 nm across an
    interface wall (BC type 5): left material the sine-dispersion bands,
    right material the same bands with group velocities x0.6 and relaxation
    times x1.5; band transmissivities from the left side 0.2 .. 0.8, from
    the right side 0.7 .. 0.1. Left wall 301 K, right wall 299 K, top and
    bottom specular."""
    left = sine_dispersion_bands(n_bands)
    right = dataclasses.replace(left, v=left.v * 0.6, tau=left.tau * 1.5)
    t = np.stack([np.linspace(0.2, 0.8, n_bands), np.linspace(0.7, 0.1, n_bands)])
    bcs = [BC(1, 1, 301.0), BC(2, 1, 299.0), BC(3, 3, 0.0), BC(4, 3, 0.0), BC(5, 5, 0.0, trans=t)]
    kw.setdefault("n_phi", n_phi)
    kw.setdefault("angle_method", 1)
    kw.setdefault("tref", 300.0)
    return Deck(mesh=two_region_tri_mesh(n, n), bands=left, bcs=bcs, scale=(1e-7, 1e-7),
                extra_materials=[right], region_material=[0, 1], **kw)


def mode_list_deck(kind: str, n: int = 12, n_bands: int = 12, seed: int = 0, **kw) -> Deck:
    """A 100 nm square (n x n squares split into triangles) whose one
    material's bands come from a seeded synthetic mode list in the
    ALAMODE or ShengBTE layout (kind), reduced to n_bands bands; left 301 K,
    right 299 K isothermal, top and bottom diffuse."""
    if kind == "ALAMODE":
        src = synthetic_alamode(seed=seed)
    elif kind == "ShengBTE":
        src = synthetic_shengbte(seed=seed)
    else:
        raise ValueError("kind must be ALAMODE or ShengBTE")
    bcs = [BC(1, 1, 301.0), BC(2, 1, 299.0), BC(3, 2, 0.0), BC(4, 2, 0.0)]
    kw.setdefault("n_phi", 4)
    kw.setdefault("angle_method", 1)
    kw.setdefault("tref", 300.0)
    return Deck(mesh=square_tri_mesh(n, n), bands=src.band_table(n_bands), bcs=bcs, scale=(1e-7, 1e-7),
                material_sources=[src], **kw)


def grating_deck(nx: int = 24, ny: int = 6, n_bands: int = 3, steps: int = 40, **kw) -> Deck:
    """A transient thermal-grating strip for the explicit solver: 300 x 75 nm
    of triangles, x-periodic (no jump), specular top and bottom, sine-
    dispersion bands; the reference's transient solver starts from
    T = cos(2 pi x / ScaleX) and takes `steps` explicit steps of 1e-13 s."""
    m = square_tri_mesh(nx, ny)
    m = Mesh2D(nodes=m.nodes * np.array([1.0, 0.25]), cells=m.cells, edges=m.edges, edge_tags=m.edge_tags,
               cell_region=m.cell_region)
    bcs = [BC(1, -2, 0.0), BC(2, -1, 0.0), BC(3, 3, 0.0), BC(4, 3, 0.0)]
    kw.setdefault("n_phi", 4)
    kw.setdefault("angle_method", 1)
    return Deck(mesh=m, bands=sine_dispersion_bands(n_bands), bcs=bcs, scale=(3e-7, 3e-7), tref=0.0,
                state="Transient", time_step=1e-13, total_time=steps * 1e-13, residual_temp=1e-14,
                residual_flux=1e-14, **kw)


def config1_deck(n: int = 40, **kw) -> Deck:
    """Gray 2D square, 1 um x 1 um, n x n squares split into 2 triangles,
    |v| = 6400 m/s, MFP 100 nm, C = 1.66e6 J/m^3K, 32 CADOM directions,
    left 301 K / right 299 K isothermal, top/bottom diffuse."""
    mesh = square_tri_mesh(n, n)
    bands = gray_band(6400.0, 1e-7, 1.66e6)
    bcs = [BC(1, 1, 301.0), BC(2, 1, 299.0), BC(3, 2, 0.0), BC(4, 2, 0.0)]
    kw.setdefault("n_phi", 8)
    kw.setdefault("angle_method", 1)
    return Deck(mesh=mesh, bands=bands, bcs=bcs, scale=(1e-6, 1e-6), **kw)


def config2_deck(h_nm: float = 3.0, n_bands: int = 40, n_phi: int = 16, seed: int = 0,
                 **kw) -> Deck:
    """Non-gray 2D nanoporous periodic cell: 300 nm square with a centred
    r = 100 nm pore (diffuse wall), Poisson-disk Delaunay mesh with spacing
    h, sine-dispersion bands binned to n_bands, 4*n_phi directions,
    x-periodic with a 1 K jump, y-periodic."""
    L = 300e-9
    mesh = porous_cell_mesh(h_nm * 1e-9 / L, [(0.5, 0.5, 100e-9 / L)], seed)
    bands = sine_dispersion_bands(n_bands)
    bcs = [BC(1, -2, 1.0), BC(2, -1, 0.0), BC(3, -4, 0.0), BC(4, -3, 0.0), BC(5, 2, 0.0)]
    kw.setdefault("n_phi", n_phi)
    kw.setdefault("angle_method", 1)
    kw.setdefault("tref", 0.0)
    return Deck(mesh=mesh, bands=bands, bcs=bcs, scale=(L, L), **kw)


def config4_deck(h_nm: float = 3.0, n_bands: int = 40, n_phi: int = 16, seed: int = 0, specularity: float = 0.3,
                 **kw) -> Deck:
    """The config-2 cell with a partially specular pore wall (BC type 6,
    value = specularity p): the geometry of the adjoint workload."""
    d = config2_deck(h_nm=h_nm, n_bands=n_bands, n_phi=n_phi, seed=seed, **kw)
    d.bcs = [b if b.tag != 5 else BC(5, 6, float(specularity)) for b in d.bcs]
    return d


def lognormal_scatter(n_cells: int, sigma: float = 0.2, seed: int = 2) -> np.ndarray:
    """Per-cell scattering multipliers drawn log-normal (median 1)."""
    return np.exp(np.random.default_rng(seed).normal(0.0, sigma, n_cells))


def config3_deck(h_nm: float = 2.5, n_bands: int = 40, n_theta: int = 4, n_phi: int = 4, seed: int = 1,
                 size_nm: Tuple[float, float, float] = (100.0, 100.0, 500.0), **kw) -> Deck:
    """3D hotspot block: size_nm box (100 x 100 x 500 nm by default) of cubes
    of edge h split into 6 tetrahedra each, vertices jittered by up to 20% of
    h (seeded), the config-2 sine-dispersion bands, Gauss-Legendre angles
    (8 * n_theta * n_phi directions: 128 by default), 1e18 W/m^3 generated
    in the top 20 nm (region 2, HeatType REGION), bottom isothermal at
    300 K, sides and top diffuse. Coordinates are in nm (Scale 1e-9)."""
    nx, ny, nz = (int(round(x / h_nm)) for x in size_nm)
    mesh = hex_tet_block_mesh(nx, ny, nz, h_nm, jitter=0.2, seed=seed, region_z=size_nm[2] - 20.0)
    bands = sine_dispersion_bands(n_bands)
    bcs = [BC(1, 1, 300.0), BC(2, 2, 0.0), BC(3, 2, 0.0), BC(4, 2, 0.0), BC(5, 2, 0.0), BC(6, 2, 0.0)]
    kw.setdefault("angle_method", 2)
    kw.setdefault("n_theta", n_theta)
    kw.setdefault("n_phi", n_phi)
    kw.setdefault("material_dim", 3)
    kw.setdefault("tref", 300.0)
    kw.setdefault("mesh_format", "MSH")
    kw.setdefault("region_heat", [0.0, 1e18])
    return Deck(mesh=mesh, bands=bands, bcs=bcs, scale=(1e-9, 1e-9, 1e-9), **kw)


def porous_population_member(i: int, seed: int = 5, h_nm: Tuple[float, float] = (2.0, 6.0),
                             r_nm: Tuple[float, float] = (40.0, 120.0), pores: Tuple[int, int] = (1, 3),
                             n_bands: int = 20, n_phi: int = 8, side_nm: float = 300.0, **kw) -> Deck:
    """Cell i of a seeded population of periodic cells for a batched solve
    (its own random stream, seeded by (seed, i), so any member can be built
    alone): a side_nm square with 1-3 circular diffuse pores of radius
    U(r_nm) placed by rejection sampling (inside the cell, at least one mesh
    spacing from the cell faces and from each other; a pore that does not
    fit after 200 tries is dropped), meshed with spacing U(h_nm); the
    sine-dispersion table of n_bands bands, 4 * n_phi directions,
    x-periodic with a 1 K jump, y-periodic (the config-2 boundary
    conditions)."""
    rng = np.random.default_rng([seed, i])
    bands = sine_dispersion_bands(n_bands)
    h = rng.uniform(*h_nm)
    want = int(rng.integers(pores[0], pores[1] + 1))
    placed: List[Tuple[float, float, float]] = []
    for _ in range(want):
        r = rng.uniform(*r_nm)
        if side_nm - 2 * (r + h) <= 0:
            continue
        for _try in range(200):
            cx, cy = rng.uniform(r + h, side_nm - r - h, size=2)
            if all(np.hypot(cx - px, cy - py) > r + pr + h for px, py, pr in placed):
                placed.append((cx, cy, r))
                break
    if not placed:  # always at least one pore: the smallest radius, centred
        placed.append((side_nm / 2, side_nm / 2, r_nm[0]))
    mesh = porous_cell_mesh(h / side_nm, [(x / side_nm, y / side_nm, r / side_nm) for x, y, r in placed],
                            seed=seed * 100003 + i)
    bcs = [BC(1, -2, 1.0), BC(2, -1, 0.0), BC(3, -4, 0.0), BC(4, -3, 0.0)]
    bcs += [BC(5 + k, 2, 0.0) for k in range(len(placed))]
    kw.setdefault("n_phi", n_phi)
    kw.setdefault("angle_method", 1)
    kw.setdefault("tref", 0.0)
    return Deck(mesh=mesh, bands=bands, bcs=bcs, scale=(side_nm * 1e-9, side_nm * 1e-9), **kw)


def porous_population(n: int, seed: int = 5, **kw) -> List[Deck]:
    """The first n members of the seeded population
    (:func:`porous_population_member`): by default 300 nm cells, 1-3 pores
    of radius U(40, 120) nm, mesh spacing U(2, 6) nm, 20 bands, 32
    directions (the batched-solve workload)."""
    return [porous_population_member(i, seed=seed, **kw) for i in range(n)]
