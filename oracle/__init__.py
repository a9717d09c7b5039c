"""ORACLE — test infrastructure only (never imported by the product).

Python bridge to the CPU restatement in ``oracle/restate/oracle.cpp`` (built
by ``make -C oracle restate`` into ``oracle/_build/liboracle_restate.so``)
and helpers to run the compiled reference binary ``oracle/_ref/BTE_CPU`` on
a deck directory and read back its full-precision result files. Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use this module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle_restate.so")
REF_BIN = os.path.join(HERE, "_ref", "BTE_CPU")
# the reference program with the B200 solver class dropped in (make -C oracle dropin)
DROPIN_BIN = os.path.join(HERE, "_ref", "BTE_B200")

_lib = None


def build(reference_root: Optional[str] = None) -> None:
    """Compile the restatement, and the reference binary when a GiftBTE
    source tree is given (argument, or the environment variable
    GIFTBTE_REFERENCE); machines without the tree use the prebuilt binary."""
    subprocess.check_call(["make", "-s", "-C", HERE, "restate"])
    reference_root = reference_root or os.environ.get("GIFTBTE_REFERENCE", "")
    if reference_root and os.path.isdir(os.path.join(reference_root, "src")):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF={reference_root}", "-j8"])
        subprocess.check_call(["make", "-s", "-C", HERE, "dropin", f"REF={reference_root}", "-j8"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_solve.restype = ctypes.c_int
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t)) if a is not None else None


def solve(deck, T0: Optional[np.ndarray] = None, max_iter: Optional[int] = None,
          err_T: Optional[float] = None, err_q: Optional[float] = None,
          cell_heat: Optional[np.ndarray] = None,
          cell_scatter: Optional[np.ndarray] = None) -> Dict[str, np.ndarray]:
    """Run the restated FP64 solve on a ``giftbte_b200.decks.Deck``.

    Returns the macro temperature ``T`` (TempLattice.dat), the energy
    temperature ``E`` (Temperature.dat), heat flux ``q`` (Nc x 3), band
    temperatures ``Tband`` (Nb x Nc), iteration count and final margins.
    ``cell_scatter`` (extension, no reference counterpart) scales the
    relaxation time of cell c by 1/s_c in the transport.
    """
    m = deck.mesh
    dim = deck.dimension
    nc = m.n_cells
    nn = len(m.nodes)
    xyz = np.zeros((nn, 3))
    for a in range(dim):
        xyz[:, a] = m.nodes[:, a] * deck.scale[a]
    cells = [np.asarray(c) for c in m.cells]
    cptr = np.zeros(nc + 1, dtype=np.int32)
    cptr[1:] = np.cumsum([len(c) for c in cells])
    cverts = np.concatenate(cells).astype(np.int32)
    creg = np.asarray(m.cell_region, dtype=np.int32)
    belems = np.asarray(m.edges, dtype=np.int32)
    nbe = len(belems)
    bptr = (np.arange(nbe + 1) * belems.shape[1]).astype(np.int32)
    bverts = np.ascontiguousarray(belems.ravel())
    btag = np.asarray(m.edge_tags, dtype=np.int32)
    bc_tag = np.asarray([b.tag for b in deck.bcs], dtype=np.int32)
    bc_type = np.asarray([b.type for b in deck.bcs], dtype=np.int32)
    bc_val = np.asarray([b.value for b in deck.bcs], dtype=np.float64)
    B = deck.bands
    nb = B.n_bands
    arr = {k: np.ascontiguousarray(getattr(B, k), dtype=np.float64)
           for k in ("v", "tau", "C", "lattice_ratio", "heat_ratio")}
    reg_mat = np.zeros(deck.n_regions, dtype=np.int32)
    if T0 is None:
        T0 = np.full(nc, deck.tref)
    T0 = np.ascontiguousarray(T0, dtype=np.float64)
    if cell_heat is None:
        cell_heat = deck.cell_heat()
    if cell_heat is not None:
        cell_heat = np.ascontiguousarray(cell_heat, dtype=np.float64)
    if cell_scatter is not None:
        cell_scatter = np.ascontiguousarray(cell_scatter, dtype=np.float64)
    out_T = np.zeros(nc); out_E = np.zeros(nc); out_q = np.zeros(3 * nc); out_Tb = np.zeros(nb * nc)
    iters = ctypes.c_int(0)
    err = np.zeros(2)
    rc = lib().oracle_solve(
        dim, nn, _p(xyz, ctypes.c_double), nc, _p(cptr, ctypes.c_int), _p(cverts, ctypes.c_int),
        _p(creg, ctypes.c_int), nbe, _p(bptr, ctypes.c_int), _p(bverts, ctypes.c_int), _p(btag, ctypes.c_int),
        len(deck.bcs), _p(bc_tag, ctypes.c_int), _p(bc_type, ctypes.c_int), _p(bc_val, ctypes.c_double),
        1, nb, _p(arr["v"], ctypes.c_double), _p(arr["tau"], ctypes.c_double), _p(arr["C"], ctypes.c_double),
        _p(arr["lattice_ratio"], ctypes.c_double), _p(arr["heat_ratio"], ctypes.c_double),
        _p(reg_mat, ctypes.c_int), len(reg_mat), deck.material_dim, deck.angle_method, deck.n_theta, deck.n_phi,
        ctypes.c_double(deck.scale[0]), _p(cell_heat, ctypes.c_double), _p(T0, ctypes.c_double), None,
        int(max_iter if max_iter is not None else deck.max_iter),
        ctypes.c_double(err_T if err_T is not None else deck.residual_temp),
        ctypes.c_double(err_q if err_q is not None else deck.residual_flux),
        1 if getattr(deck, "order", "2") == "2limit" else 0,
        _p(out_T, ctypes.c_double), _p(out_E, ctypes.c_double), _p(out_q, ctypes.c_double),
        _p(out_Tb, ctypes.c_double), ctypes.byref(iters), _p(err, ctypes.c_double),
        _p(cell_scatter, ctypes.c_double), 1 if getattr(deck, "order", "2") == "1" else 2,
        1 if getattr(deck, "scheme", "Synthetic") == "Sequential" else 0)
    if rc != 0:
        raise RuntimeError(f"oracle_solve failed with code {rc}")
    return {"T": out_T, "E": out_E, "q": out_q.reshape(nc, 3), "Tband": out_Tb.reshape(nb, nc),
            "iters": int(iters.value), "err": err}


def run_reference(deck_root: str, timeout: float = 3600.0, binary: Optional[str] = None) -> Dict[str, np.ndarray]:
    """Run the compiled reference (or ``binary``, e.g. DROPIN_BIN) in
    ``deck_root`` (which holds ``input/``) and parse its result files (17
    significant digits, see oracle/ref_shim/full_precision.cpp)."""
    binary = binary or REF_BIN
    if not os.path.exists(binary):
        raise FileNotFoundError(binary)
    logp = os.path.join(deck_root, "ref_run.log")
    with open(logp, "w") as log:
        rc = subprocess.run([binary], cwd=deck_root, stdout=log, stderr=subprocess.STDOUT, timeout=timeout).returncode
    if rc != 0:
        with open(logp, errors="replace") as f:
            tail = f.read()[-2000:]
        raise RuntimeError(f"{os.path.basename(binary)} exited with {rc}; end of its log:\n{tail}")
    return read_reference_outputs(deck_root)


def read_reference_outputs(deck_root: str) -> Dict[str, np.ndarray]:
    if not os.path.exists(os.path.join(deck_root, "TempLattice.dat")) and \
            os.path.exists(os.path.join(deck_root, "TTG.dat")):
        return read_transient_outputs(deck_root)
    T = np.loadtxt(os.path.join(deck_root, "TempLattice.dat"))
    E = np.loadtxt(os.path.join(deck_root, "Temperature.dat"))
    q = np.loadtxt(os.path.join(deck_root, "HeatFlux.dat"))
    tb = np.loadtxt(os.path.join(deck_root, "Tempband.dat"))
    nb = int(tb[:, 0].max())
    out = {"xyz": T[:, :3], "T": T[:, 3], "E": E[:, 3], "q": q[:, 3:6],
           "Tband": tb[:, 4].reshape(nb, -1)}
    fm = os.path.join(deck_root, "Temperature_macro.dat")
    if os.path.exists(fm):
        out["Tf"] = np.loadtxt(fm)[:, 3]
        out["qf"] = np.loadtxt(os.path.join(deck_root, "HeatFlux_macro.dat"))[:, 3:6]
    iters = 0
    margins = []
    logp = os.path.join(deck_root, "ref_run.log")
    if os.path.exists(logp):
        with open(logp) as f:
            for line in f:
                if line.startswith("Iteration #"):
                    iters += 1
                    t = line.split("Temperature:")[1].split()[0]
                    q = line.split("Heat Flux:")[1].split()[0]
                    margins.append((float(t), float(q)))
    out["iters"] = iters
    out["margins"] = np.asarray(margins).reshape(-1, 2)
    return out


def read_transient_outputs(deck_root: str) -> Dict[str, np.ndarray]:
    """Outputs of the reference's transient solver (Transient::_print_out,
    src/TransientBTE/transient.cpp:865-889, and TransientSolver.cpp:158):
    Tempcell.dat (cell centre, lattice temperature), HeatFlux.dat (centre,
    flux) and TTG.dat (time, temperature of cell 0 after each step); the
    per-step margins from the log."""
    T = np.loadtxt(os.path.join(deck_root, "Tempcell.dat"))
    q = np.loadtxt(os.path.join(deck_root, "HeatFlux.dat"))
    ttg = np.loadtxt(os.path.join(deck_root, "TTG.dat")).reshape(-1, 2)
    margins = []
    logp = os.path.join(deck_root, "ref_run.log")
    if os.path.exists(logp):
        with open(logp) as f:
            for line in f:
                if line.startswith("Iteration #"):
                    margins.append((float(line.split("Temperature:")[1].split()[0]),
                                    float(line.split("Heat Flux:")[1].split()[0])))
    return {"xyz": T[:, :3], "T": T[:, 3], "q": q[:, 3:6], "ttg": ttg, "iters": len(margins),
            "margins": np.asarray(margins).reshape(-1, 2)}
