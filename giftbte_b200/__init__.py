"""giftbte_b200 — B200-native steady synthetic phonon-BTE solver.

Python binding of the C ABI in ``include/giftbte.h`` (the library itself is
C++/CUDA: ``giftbte_b200/_build/libgiftbte_b200.so``). The class
:class:`StaticBTESynthetic` mirrors the reference's solver object
(``includes/StaticBTESynthetic/StaticBTESynthetic.h:24-261``): it is built
from a mesh, boundary conditions, band table and angular quadrature, takes an
initial temperature, and ``solve(max_iter, err_T, err_q)`` runs the outer
source iteration; afterwards ``temperature`` (the macro lattice temperature),
``total_energy`` (Temperature.dat), ``heat_flux`` and ``temperature_band``
hold the results.

There is no CPU fallback: without the compiled library or a CUDA device the
constructor raises.
"""
from __future__ import annotations

import ctypes
import math
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgiftbte_b200.so")

GBTE_OK = 0
GBTE_ERR_NOT_CONVERGED = 1
GBTE_FP64 = 0
GBTE_FP32_MIXED = 1

STATUS = {0: "ok", -1: "invalid argument", -2: "input/output error", -3: "CUDA error", -4: "diverged",
          -5: "device wait timed out", -6: "out of memory", -7: "mesh topology error", -8: "unsupported input",
          -9: "direction shard exchange failed", 1: "not converged within max_iter"}
GBTE_ERR_ARG = -1
GBTE_ERR_IO = -2
GBTE_ERR_CUDA = -3
GBTE_ERR_DIVERGED = -4
GBTE_ERR_TIMEOUT = -5
GBTE_ERR_NOMEM = -6
GBTE_ERR_MESH = -7
GBTE_ERR_UNSUPPORTED = -8
GBTE_ERR_EXCHANGE = -9

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)


class MeshView(ctypes.Structure):
    _fields_ = [("dimension", ctypes.c_int), ("num_nodes", ctypes.c_int), ("num_cells", ctypes.c_int),
                ("num_boundary_elements", ctypes.c_int), ("node_xyz", _c_dbl_p), ("cell_ptr", _c_int_p),
                ("cell_verts", _c_int_p), ("cell_region", _c_int_p), ("belem_ptr", _c_int_p),
                ("belem_verts", _c_int_p), ("belem_tag", _c_int_p), ("scale_x", ctypes.c_double),
                ("scale_y", ctypes.c_double), ("scale_z", ctypes.c_double)]


class BandTableC(ctypes.Structure):
    _fields_ = [("num_materials", ctypes.c_int), ("num_bands", ctypes.c_int), ("group_velocity", _c_dbl_p),
                ("relaxation_time", _c_dbl_p), ("heat_capacity", _c_dbl_p), ("lattice_ratio", _c_dbl_p),
                ("heat_ratio", _c_dbl_p), ("num_regions", ctypes.c_int), ("region_material", _c_int_p),
                ("material_dimension", ctypes.c_int)]


class BCTable(ctypes.Structure):
    _fields_ = [("num", ctypes.c_int), ("tag", _c_int_p), ("type", _c_int_p), ("value", _c_dbl_p),
                ("transmissivity", _c_dbl_p)]


class AngleSpec(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int), ("n_theta", ctypes.c_int), ("n_phi", ctypes.c_int),
                ("num_directions", ctypes.c_int), ("direction_xyz", _c_dbl_p), ("weight", _c_dbl_p),
                ("solid_angle", ctypes.c_double)]


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("use_limiter", ctypes.c_int), ("max_iter", ctypes.c_int),
                ("err_temp", ctypes.c_double), ("err_flux", ctypes.c_double), ("cell_heat", _c_dbl_p),
                ("stream", ctypes.c_void_p), ("device", ctypes.c_int), ("verbose", ctypes.c_int),
                ("macro_rtol", ctypes.c_double), ("profile", ctypes.c_int), ("sweep_bands", ctypes.c_int),
                ("sweep_far_slots", ctypes.c_int), ("direction_batch", ctypes.c_int),
                ("cell_scatter", _c_dbl_p), ("cell_order", ctypes.c_int), ("order", ctypes.c_int),
                ("scheme", ctypes.c_int), ("macro_exact", ctypes.c_int), ("sweep_vector", ctypes.c_int),
                ("sweep_kernel", ctypes.c_int), ("gradient_dirs", ctypes.c_int), ("residual_form", ctypes.c_int),
                ("adjoint_history", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("err_temp", ctypes.c_double), ("err_flux", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("setup_ms", ctypes.c_double), ("transport_ms", ctypes.c_double),
                ("macro_ms", ctypes.c_double), ("macro_cg_iterations", ctypes.c_longlong),
                ("updates", ctypes.c_longlong), ("num_directions", ctypes.c_int), ("num_bands", ctypes.c_int),
                ("num_cells", ctypes.c_int), ("max_levels", ctypes.c_int), ("lagged_faces", ctypes.c_int),
                ("inner_iterations", ctypes.c_int), ("kernel_launches", ctypes.c_longlong),
                ("kernel_ms", ctypes.c_double * 16), ("kernel_count", ctypes.c_longlong * 16),
                ("sweep_bands", ctypes.c_int), ("direction_batch", ctypes.c_int),
                ("sweep_stage_levels", ctypes.c_int), ("sweep_vector", ctypes.c_int),
                ("sweep_threads", ctypes.c_int), ("sweep_kernel", ctypes.c_int), ("gradient_dirs", ctypes.c_int),
                ("residual_form", ctypes.c_int)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("kernel_ms", "kernel_count")}
        lib = library()
        d["kernels"] = {}
        for i in range(16):
            name = lib.gbte_kernel_name(i)
            if name is None:
                break
            if self.kernel_count[i]:
                d["kernels"][name.decode()] = {"ms": self.kernel_ms[i], "launches": self.kernel_count[i]}
        return d


class VjpStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("picard_steps", ctypes.c_int), ("change", ctypes.c_double),
                ("vjp_ms", ctypes.c_double), ("residual", ctypes.c_double)]


class TransientStats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_longlong), ("updates", ctypes.c_longlong), ("err_temp", ctypes.c_double),
                ("err_flux", ctypes.c_double), ("solve_ms", ctypes.c_double)]


class DeckInfo(ctypes.Structure):
    _fields_ = [("dimension", ctypes.c_int), ("num_nodes", ctypes.c_int), ("num_cells", ctypes.c_int),
                ("num_faces", ctypes.c_int), ("num_boundaries", ctypes.c_int),
                ("num_boundary_sides", ctypes.c_int), ("num_bands", ctypes.c_int),
                ("num_directions", ctypes.c_int), ("num_materials", ctypes.c_int), ("max_levels", ctypes.c_int),
                ("lagged_faces", ctypes.c_int), ("kappa_bulk", ctypes.c_double),
                ("capacity_bulk", ctypes.c_double), ("total_volume", ctypes.c_double),
                ("max_iter_or_zero", ctypes.c_double), ("err_temp", ctypes.c_double),
                ("err_flux", ctypes.c_double), ("max_level_width", ctypes.c_int), ("sweep_ring", ctypes.c_int),
                ("far_slots", ctypes.c_int), ("far_refs", ctypes.c_longlong),
                ("index_entries_checked", ctypes.c_longlong), ("transient", ctypes.c_int),
                ("time_step", ctypes.c_double), ("total_time", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


EXPORTS = ["gbte_inspect_deck", "gbte_inspect_mesh", "gbte_default_options", "gbte_create", "gbte_create_from_deck", "gbte_set_initial",
           "gbte_fourier_initial", "gbte_solve", "gbte_get_fields", "gbte_write_outputs", "gbte_get_sizes",
           "gbte_get_geometry", "gbte_last_error", "gbte_status_string", "gbte_destroy", "gbte_kernel_name",
           "gbte_solve_with", "gbte_fourier_initial_noalloc", "gbte_batch_create", "gbte_batch_geometries",
           "gbte_vjp", "gbte_set_profile", "gbte_set_direction_shard", "gbte_options_size", "gbte_transient_solve"]

# int (*gbte_exchange_fn)(void *user, double *buf, size_t count, void *stream)
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)

_lib = None


def library():
    """Load the compiled library (building it first if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        lib = ctypes.CDLL(LIB_PATH)
        lib.gbte_last_error.restype = ctypes.c_char_p
        lib.gbte_last_error.argtypes = [ctypes.c_void_p]
        lib.gbte_status_string.restype = ctypes.c_char_p
        lib.gbte_kernel_name.restype = ctypes.c_char_p
        lib.gbte_options_size.restype = ctypes.c_size_t
        if lib.gbte_options_size() != ctypes.sizeof(Options):
            raise RuntimeError("libgiftbte_b200 was built from another include/giftbte.h (options size "
                               f"{lib.gbte_options_size()} vs {ctypes.sizeof(Options)}); rebuild it")
        lib.gbte_create.argtypes = [ctypes.POINTER(MeshView), ctypes.POINTER(BandTableC), ctypes.POINTER(BCTable),
                                    ctypes.POINTER(AngleSpec), ctypes.POINTER(Options),
                                    ctypes.POINTER(ctypes.c_void_p)]
        lib.gbte_create_from_deck.argtypes = [ctypes.c_char_p, ctypes.POINTER(Options),
                                              ctypes.POINTER(ctypes.c_void_p)]
        lib.gbte_set_initial.argtypes = [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]
        lib.gbte_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(Stats)]
        lib.gbte_solve_with.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.POINTER(Stats)]
        lib.gbte_get_fields.argtypes = [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]
        lib.gbte_write_outputs.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        lib.gbte_get_sizes.argtypes = [ctypes.c_void_p] + [_c_int_p] * 4
        lib.gbte_get_geometry.argtypes = [ctypes.c_void_p, _c_dbl_p, _c_dbl_p]
        lib.gbte_destroy.argtypes = [ctypes.c_void_p]
        lib.gbte_fourier_initial.argtypes = [ctypes.c_void_p]
        lib.gbte_fourier_initial_noalloc.argtypes = [ctypes.c_void_p]
        lib.gbte_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(MeshView), ctypes.POINTER(BandTableC),
                                          ctypes.POINTER(BCTable), ctypes.POINTER(AngleSpec),
                                          ctypes.POINTER(Options), ctypes.POINTER(ctypes.c_void_p)]
        lib.gbte_batch_geometries.argtypes = [ctypes.c_void_p, _c_int_p, _c_int_p]
        lib.gbte_set_profile.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.gbte_set_direction_shard.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, EXCHANGE_FN,
                                                 ctypes.c_void_p]
        lib.gbte_vjp.argtypes = [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, ctypes.c_int, ctypes.c_double, _c_dbl_p,
                                 _c_dbl_p, _c_dbl_p, ctypes.POINTER(VjpStats)]
        lib.gbte_transient_solve.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_int, _c_dbl_p, ctypes.c_longlong,
                                             ctypes.POINTER(TransientStats)]
        lib.gbte_inspect_deck.argtypes = [ctypes.c_char_p, ctypes.POINTER(DeckInfo)]
        lib.gbte_inspect_mesh.argtypes = [ctypes.POINTER(MeshView), ctypes.POINTER(BandTableC),
                                          ctypes.POINTER(BCTable), ctypes.POINTER(AngleSpec),
                                          ctypes.POINTER(DeckInfo)]
        _lib = lib
    return _lib


class GBTEError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t)) if a is not None else None


def default_options(precision: int = GBTE_FP64, **kw) -> Options:
    o = Options()
    library().gbte_default_options(ctypes.byref(o))
    o.precision = precision
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class StaticBTESynthetic:
    """One solver instance on one GPU (see module docstring)."""

    def __init__(self, handle: ctypes.c_void_p, keep=()):
        self._h = handle
        self._keep = keep
        lib = library()
        nc, nb, nd, nbs = (ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int())
        lib.gbte_get_sizes(self._h, ctypes.byref(nc), ctypes.byref(nb), ctypes.byref(nd), ctypes.byref(nbs))
        self.num_cells, self.num_bands, self.num_directions, self.num_boundary_sides = (
            nc.value, nb.value, nd.value, nbs.value)
        self.stats: Optional[dict] = None
        self._n_bc_rows = 0  # boundary-table rows given at creation (known for in-memory decks)

    # --- construction -----------------------------------------------------
    @classmethod
    def from_deck_dir(cls, path: str, precision: int = GBTE_FP64, device: int = 0, verbose: int = 0,
                      **opt) -> "StaticBTESynthetic":
        lib = library()
        o = default_options(precision, device=device, verbose=verbose, **opt)
        h = ctypes.c_void_p()
        rc = lib.gbte_create_from_deck(path.encode(), ctypes.byref(o), ctypes.byref(h))
        if rc != GBTE_OK:
            raise GBTEError(rc, lib.gbte_last_error(None).decode())
        return cls(h)

    @classmethod
    def from_deck(cls, deck, precision: int = GBTE_FP64, device: int = 0, verbose: int = 0,
                  cell_heat: Optional[np.ndarray] = None, cell_scatter: Optional[np.ndarray] = None,
                  **opt) -> "StaticBTESynthetic":
        """Build from a :class:`giftbte_b200.decks.Deck` held in memory.
        ``cell_scatter`` (per cell, > 0) multiplies the scattering rate of
        each cell in the transport (no counterpart in the reference)."""
        lib = library()
        v = _views(deck)
        nc = deck.mesh.n_cells
        if cell_heat is None:
            cell_heat = deck.cell_heat()
        heat = np.ascontiguousarray(cell_heat, dtype=np.float64) if cell_heat is not None else None
        kw = {"max_iter": deck.max_iter, "err_temp": deck.residual_temp, "err_flux": deck.residual_flux,
              "order": 1 if deck.order == "1" else 2, "scheme": 1 if deck.scheme == "Sequential" else 0,
              "use_limiter": 1 if deck.order == "2limit" else 0}
        kw.update(opt)
        o = default_options(precision, device=device, verbose=verbose, **kw)
        o.cell_heat = _ptr(heat, ctypes.c_double)
        scat = np.ascontiguousarray(cell_scatter, dtype=np.float64) if cell_scatter is not None else None
        if scat is not None and scat.shape != (nc,):
            raise ValueError("cell_scatter needs one value per cell")
        o.cell_scatter = _ptr(scat, ctypes.c_double)
        h = ctypes.c_void_p()
        rc = lib.gbte_create(ctypes.byref(v["mv"]), ctypes.byref(v["bt"]), ctypes.byref(v["bc"]),
                             ctypes.byref(v["an"]), ctypes.byref(o), ctypes.byref(h))
        if rc != GBTE_OK:
            raise GBTEError(rc, lib.gbte_last_error(None).decode())
        s = cls(h)
        s._n_bc_rows = len(deck.bcs)
        s.set_initial(np.full(nc, deck.tref))
        return s

    @classmethod
    def from_decks(cls, decks, precision: int = GBTE_FP64, device: int = 0, verbose: int = 0,
                   **opt) -> "StaticBTESynthetic":
        """One batched solve of several independent in-memory decks
        (gbte_batch_create): the band table, quadrature, ScaleX and the
        iteration limits come from the first deck; fields are the decks'
        cell arrays concatenated (see :meth:`geometry_offsets`)."""
        lib = library()
        views = [_views(d) for d in decks]
        n = len(decks)
        meshes = (MeshView * n)(*[v["mv"] for v in views])
        bcs = (BCTable * n)(*[v["bc"] for v in views])
        nreg = max(int(np.max(d.mesh.cell_region)) + 1 for d in decks)
        B = decks[0].bands
        arrs = [np.ascontiguousarray(getattr(B, k), dtype=np.float64)
                for k in ("v", "tau", "C", "lattice_ratio", "heat_ratio")]
        reg = np.zeros(nreg, dtype=np.int32)
        bt = BandTableC(1, B.n_bands, *[_ptr(a, ctypes.c_double) for a in arrs], nreg, _ptr(reg, ctypes.c_int),
                        decks[0].material_dim)
        heats = [d.cell_heat() for d in decks]
        heat = None
        if any(h is not None for h in heats):
            heat = np.ascontiguousarray(np.concatenate([h if h is not None else np.zeros(d.mesh.n_cells)
                                                        for h, d in zip(heats, decks)]), dtype=np.float64)
        d0 = decks[0]
        kw = {"max_iter": d0.max_iter, "err_temp": d0.residual_temp, "err_flux": d0.residual_flux,
              "order": 1 if d0.order == "1" else 2, "scheme": 1 if d0.scheme == "Sequential" else 0}
        kw.update(opt)
        o = default_options(precision, device=device, verbose=verbose, **kw)
        o.cell_heat = _ptr(heat, ctypes.c_double)
        h = ctypes.c_void_p()
        rc = lib.gbte_batch_create(n, meshes, ctypes.byref(bt), bcs, ctypes.byref(views[0]["an"]), ctypes.byref(o),
                                   ctypes.byref(h))
        if rc != GBTE_OK:
            raise GBTEError(rc, lib.gbte_last_error(None).decode())
        s = cls(h)
        s.set_initial(np.concatenate([np.full(d.mesh.n_cells, d.tref) for d in decks]))
        return s

    def geometry_offsets(self) -> np.ndarray:
        """Cell ranges of the geometries of this handle ([num + 1])."""
        lib = library()
        n = ctypes.c_int()
        self._check(lib.gbte_batch_geometries(self._h, ctypes.byref(n), None))
        off = np.zeros(n.value + 1, dtype=np.int32)
        self._check(lib.gbte_batch_geometries(self._h, ctypes.byref(n), _ptr(off, ctypes.c_int)))
        return off

    def split(self, field: np.ndarray) -> list:
        """A concatenated cell field (cells on the last axis for band fields)
        cut into the geometries' pieces."""
        off = self.geometry_offsets()
        if field.ndim == 2 and field.shape[0] == self.num_bands and field.shape[1] == self.num_cells:
            return [field[:, off[k]:off[k + 1]] for k in range(len(off) - 1)]
        return [field[off[k]:off[k + 1]] for k in range(len(off) - 1)]

    # --- the reference's solve interface ----------------------------------
    def set_initial(self, T0: np.ndarray, q0: Optional[np.ndarray] = None,
                    boundary_thermal: Optional[np.ndarray] = None) -> None:
        T0 = np.ascontiguousarray(T0, dtype=np.float64)
        q0 = np.ascontiguousarray(q0, dtype=np.float64) if q0 is not None else None
        bt = np.ascontiguousarray(boundary_thermal, dtype=np.float64) if boundary_thermal is not None else None
        self._check(library().gbte_set_initial(self._h, _ptr(T0, ctypes.c_double), _ptr(q0, ctypes.c_double),
                                               _ptr(bt, ctypes.c_double)))

    def fourier_initial(self) -> None:
        """Replace the initial field by the Fourier pre-solve (kappa_bulk) the
        reference runs before the BTE (StaticFourier::_solve)."""
        self._check(library().gbte_fourier_initial(self._h))

    def fourier_initial_noalloc(self) -> None:
        """The Fourier pre-solve without any device allocation (its scratch
        lives in a static device array of the library; see
        gbte_fourier_initial_noalloc in include/giftbte.h for the limits)."""
        self._check(library().gbte_fourier_initial_noalloc(self._h))

    def solve(self, max_iter: Optional[int] = None, err_temp: Optional[float] = None,
              err_flux: Optional[float] = None, allow_not_converged: bool = True) -> dict:
        """Outer source iteration from the current state (the reference's
        solve(Use_Backup, Num_Max_Iter, Use_Limiter, error_temp_limit,
        error_flux_limit)); limits default to the ones given at creation."""
        st = Stats()
        if max_iter is None and err_temp is None and err_flux is None:
            rc = library().gbte_solve(self._h, ctypes.byref(st))
        else:
            rc = library().gbte_solve_with(self._h, int(max_iter if max_iter is not None else 10000),
                                           float(err_temp if err_temp is not None else 0.0),
                                           float(err_flux if err_flux is not None else 0.0), ctypes.byref(st))
        self.stats = st.as_dict()
        if rc == GBTE_ERR_NOT_CONVERGED and allow_not_converged:
            return self.stats
        self._check(rc)
        return self.stats

    def fields(self, out: Optional[dict] = None) -> dict:
        """The solution in the caller's cell order (gbte_get_fields): ``E``
        and ``T`` (nc,), ``q`` (nc, 3), ``Tband`` (nb, nc). ``out`` may hold
        arrays to fill in place under those keys (float64, C-contiguous,
        writeable, those shapes), e.g. in pinned host memory for faster
        copies; missing keys are allocated."""
        nc, nb = self.num_cells, self.num_bands
        res = {}
        for k, shp in (("E", (nc,)), ("T", (nc,)), ("q", (nc, 3)), ("Tband", (nb, nc))):
            a = None if out is None else out.get(k)
            if a is None:
                a = np.zeros(shp)
            elif (not isinstance(a, np.ndarray) or a.dtype != np.float64 or a.shape != shp
                  or not a.flags.c_contiguous or not a.flags.writeable):
                raise ValueError(f"fields: out[{k!r}] must be a writeable C-contiguous float64 array of shape {shp}")
            res[k] = a
        self._check(library().gbte_get_fields(self._h, _ptr(res["E"], ctypes.c_double),
                                              _ptr(res["T"], ctypes.c_double), _ptr(res["q"], ctypes.c_double),
                                              _ptr(res["Tband"], ctypes.c_double)))
        return res

    @property
    def temperature(self):
        return self.fields()["T"]

    @property
    def total_energy(self):
        return self.fields()["E"]

    @property
    def heat_flux(self):
        return self.fields()["q"]

    @property
    def temperature_band(self):
        return self.fields()["Tband"]

    def geometry(self):
        nc = self.num_cells
        c = np.zeros(3 * nc); v = np.zeros(nc)
        self._check(library().gbte_get_geometry(self._h, _ptr(c, ctypes.c_double), _ptr(v, ctypes.c_double)))
        return c.reshape(nc, 3), v

    def vjp(self, T_bar: Optional[np.ndarray] = None, q_bar: Optional[np.ndarray] = None, max_iter: int = 10000,
            tol: float = 1e-10) -> dict:
        """Gradient of J = <T_bar, T> + <q_bar, q> at the fixed point the last
        solve reached (gbte_vjp): ``tau`` (per band, multiplier on its
        relaxation time), ``scatter`` (per cell, its scattering multiplier),
        ``specularity`` (per boundary-table row; partially specular rows).
        The transposed iteration stops when the residual of the adjoint
        equations relative to dJ/de is <= tol."""
        nc, nb = self.num_cells, self.num_bands
        Tb = np.ascontiguousarray(T_bar, dtype=np.float64) if T_bar is not None else None
        qb = np.ascontiguousarray(q_bar, dtype=np.float64).reshape(-1) if q_bar is not None else None
        if Tb is not None and Tb.shape != (nc,):
            raise ValueError("T_bar needs one value per cell")
        if qb is not None and qb.shape != (3 * nc,):
            raise ValueError("q_bar needs three values per cell")
        g_tau = np.zeros(nb)
        g_cell = np.zeros(nc)
        g_spec = np.zeros(self._n_bc_rows) if self._n_bc_rows else None
        st = VjpStats()
        self._check(library().gbte_vjp(self._h, _ptr(Tb, ctypes.c_double), _ptr(qb, ctypes.c_double), int(max_iter),
                                       float(tol), _ptr(g_tau, ctypes.c_double), _ptr(g_cell, ctypes.c_double),
                                       _ptr(g_spec, ctypes.c_double), ctypes.byref(st)))
        return {"tau": g_tau, "scatter": g_cell, "specularity": g_spec,
                "stats": {k: getattr(st, k) for k, _ in st._fields_}}

    def transient_solve(self, time_step: float, total_time: float, err_temp: float = 0.0, err_flux: float = 0.0,
                        probe_cell: int = 0, history: bool = True, history_cap: int = 1 << 26) -> dict:
        """The explicit transient solver from the thermal grating
        T = cos(2 pi x / ScaleX) (gbte_transient_solve, the reference's
        State=Transient): steps of time_step up to total_time, ending early
        when both margins reach their limits. Returns the stats and, with
        ``history``, the temperature of ``probe_cell`` after every step (the
        reference's TTG.dat column, the first ``history_cap`` steps);
        ``fields()`` then holds the final state."""
        n = min(max(0, math.ceil(total_time / time_step)), int(history_cap))
        hist = np.zeros(n) if history else None
        st = TransientStats()
        self._check(library().gbte_transient_solve(self._h, float(time_step), float(total_time), float(err_temp),
                                                   float(err_flux), int(probe_cell), _ptr(hist, ctypes.c_double),
                                                   n if history else 0, ctypes.byref(st)))
        out = {k: getattr(st, k) for k, _ in st._fields_}
        if history:
            out["history"] = hist[: min(st.steps, n)]
        return out

    def set_direction_shard(self, begin: int, count: int, exchange) -> None:
        """Transport over directions [begin, begin + count) only; the moments
        and boundary values are summed over the shard set every outer
        iteration by ``exchange(buf, count, stream)`` (gbte_set_direction_shard;
        ``giftbte_b200.shard`` has exchanges over torch.distributed and over
        threads of one process). ``exchange`` sums ``count`` doubles of
        device memory at address ``buf`` in place, ordered on the CUDA stream
        ``stream``; an exception makes the solve fail with
        GBTE_ERR_EXCHANGE. count = 0 or exchange = None: all directions."""
        self._xerr = None
        if exchange is None or count == 0:
            self._xcb = None
            self._check(library().gbte_set_direction_shard(self._h, 0, 0, EXCHANGE_FN(), None))
            return

        def cb(user, buf, n, stream):
            try:
                exchange(buf or 0, int(n), stream or 0)
                return 0
            except BaseException as e:  # reported by the solve that called it
                self._xerr = e
                return 1

        self._xcb = EXCHANGE_FN(cb)
        self._check(library().gbte_set_direction_shard(self._h, int(begin), int(count), self._xcb, None))

    def set_profile(self, on: bool) -> None:
        """Per-launch kernel timing for the next solves (gbte_set_profile)."""
        self._check(library().gbte_set_profile(self._h, int(bool(on))))

    def keff_cotangent(self, axis: int = 0, length: float = 1.0, delta_T: float = 1.0) -> np.ndarray:
        """q_bar of the effective conductivity k = <q_axis>_V length / delta_T
        (volume average of the heat flux over the domain)."""
        _, vol = self.geometry()
        qb = np.zeros((self.num_cells, 3))
        qb[:, axis] = vol / vol.sum() * length / delta_T
        return qb

    def write_outputs(self, path: str) -> None:
        self._check(library().gbte_write_outputs(self._h, path.encode()))

    def close(self) -> None:
        if self._h:
            library().gbte_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != GBTE_OK:
            msg = library().gbte_last_error(self._h).decode()
            xerr = getattr(self, "_xerr", None)
            if rc == GBTE_ERR_EXCHANGE and xerr is not None:
                raise GBTEError(rc, f"{msg}: {xerr!r}") from xerr
            raise GBTEError(rc, msg)


def _views(deck) -> dict:
    """C views of an in-memory deck; the returned dict keeps the arrays alive."""
    m = deck.mesh
    nc = m.n_cells
    nn = len(m.nodes)
    xyz = np.zeros((nn, 3))
    xyz[:, 0] = m.nodes[:, 0] * deck.scale[0]
    xyz[:, 1] = m.nodes[:, 1] * deck.scale[1]
    if m.nodes.shape[1] > 2:
        xyz[:, 2] = m.nodes[:, 2] * (deck.scale[2] if len(deck.scale) > 2 else deck.scale[0])
    cells = [np.asarray(c) for c in m.cells]
    cptr = np.zeros(nc + 1, dtype=np.int32)
    cptr[1:] = np.cumsum([len(c) for c in cells])
    cverts = np.ascontiguousarray(np.concatenate(cells), dtype=np.int32)
    creg = np.ascontiguousarray(m.cell_region, dtype=np.int32)
    edges = np.asarray(m.edges)
    nbe = len(edges)
    bptr = (np.arange(nbe + 1) * edges.shape[1]).astype(np.int32)
    bverts = np.ascontiguousarray(edges.ravel(), dtype=np.int32)
    btag = np.ascontiguousarray(m.edge_tags, dtype=np.int32)
    dim = 3 if (m.nodes.shape[1] > 2) else 2
    mv = MeshView(dim, nn, nc, nbe, _ptr(xyz, ctypes.c_double), _ptr(cptr, ctypes.c_int),
                  _ptr(cverts, ctypes.c_int), _ptr(creg, ctypes.c_int), _ptr(bptr, ctypes.c_int),
                  _ptr(bverts, ctypes.c_int), _ptr(btag, ctypes.c_int), deck.scale[0], deck.scale[1],
                  deck.scale[2] if len(deck.scale) > 2 else 1.0)
    mats = deck.materials if hasattr(deck, "materials") else [deck.bands]
    nb = mats[0].n_bands
    arrs = [np.ascontiguousarray(np.concatenate([np.asarray(getattr(B, k), dtype=np.float64) for B in mats]))
            for k in ("v", "tau", "C", "lattice_ratio", "heat_ratio")]
    nreg = max(1, int(np.max(creg)) + 1)
    rmat = deck.region_materials() if hasattr(deck, "region_materials") else [0] * nreg
    reg = np.zeros(nreg, dtype=np.int32)
    reg[:min(nreg, len(rmat))] = np.asarray(rmat, dtype=np.int32)[:nreg]
    bt = BandTableC(len(mats), nb, *[_ptr(a, ctypes.c_double) for a in arrs], len(reg),
                    _ptr(reg, ctypes.c_int), deck.material_dim)
    tags = np.asarray([b.tag for b in deck.bcs], dtype=np.int32)
    types = np.asarray([b.type for b in deck.bcs], dtype=np.int32)
    vals = np.asarray([b.value for b in deck.bcs], dtype=np.float64)
    trans = None
    if any(b.type == 5 for b in deck.bcs):
        trans = np.zeros((len(deck.bcs), len(mats) * nb))
        for i, b in enumerate(deck.bcs):
            if b.type == 5:
                trans[i] = np.asarray(b.trans, dtype=np.float64).reshape(-1)
    bc = BCTable(len(deck.bcs), _ptr(tags, ctypes.c_int), _ptr(types, ctypes.c_int), _ptr(vals, ctypes.c_double),
                 _ptr(trans, ctypes.c_double))
    an = AngleSpec(deck.angle_method, deck.n_theta, deck.n_phi)
    return {"mv": mv, "bt": bt, "bc": bc, "an": an,
            "keep": (xyz, cptr, cverts, creg, bptr, bverts, btag, arrs, reg, tags, types, vals, trans)}


def inspect(deck) -> dict:
    """Host-only summary (no GPU) of what the solver would build for an
    in-memory deck."""
    v = _views(deck)
    info = DeckInfo()
    rc = library().gbte_inspect_mesh(ctypes.byref(v["mv"]), ctypes.byref(v["bt"]), ctypes.byref(v["bc"]),
                                     ctypes.byref(v["an"]), ctypes.byref(info))
    if rc != GBTE_OK:
        raise GBTEError(rc, library().gbte_last_error(None).decode())
    return info.as_dict()


def inspect_deck(path: str) -> dict:
    """Host-only summary of a deck directory (reads input/* like the reference)."""
    info = DeckInfo()
    rc = library().gbte_inspect_deck(path.encode(), ctypes.byref(info))
    if rc != GBTE_OK:
        raise GBTEError(rc, library().gbte_last_error(None).decode())
    return info.as_dict()


def effective_conductivity(q: np.ndarray, volumes: np.ndarray, length: float, delta_T: float, axis: int = 0) -> float:
    """k_eff = <q_axis>_V * L / dT, the volume-averaged flux over the
    temperature difference (the reference computes it in post-processing,
    bin/examples/cross-plane/verify_kappa_crossplane.m:7)."""
    return float(np.sum(q[:, axis] * volumes) / np.sum(volumes) * length / delta_T)
