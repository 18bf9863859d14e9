"""ORACLE -- test infrastructure only (checker for tests/, smoke() and bench.py's
cpu_baseline leg; the product never imports it).

ctypes front end of oracle/liboracle.so (oracle.c, a CPU FP64 restatement of the
reference nonbonded evaluation) plus the reference's particle binning
(src/space.c:403-423: cell index by truncating (x - origin) * (1/h) in double, position
stored relative to the cell origin in float).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "liboracle.so")
REF_DIR = os.path.join(_HERE, "_ref")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", _HERE, "liboracle.so"], check=True, capture_output=True)
        L = C.CDLL(LIB)
        P = C.POINTER
        L.oracle_nonbond.restype = C.c_int
        L.oracle_nonbond.argtypes = [C.c_int, P(C.c_float), P(C.c_int), P(C.c_int), P(C.c_double), P(C.c_double),
                                     P(C.c_int), C.c_double, C.c_uint, C.c_int, P(C.c_int), P(C.c_float),
                                     P(C.c_float), P(C.c_int), P(C.c_int), C.c_int, P(C.c_int), P(C.c_double),
                                     P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_longlong),
                                     P(C.c_longlong), P(C.c_double), C.c_int]
        L.oracle_bonds.restype = C.c_int
        L.oracle_bonds.argtypes = [C.c_int, P(C.c_int), P(C.c_float), P(C.c_int), P(C.c_int), P(C.c_double),
                                   P(C.c_float), P(C.c_float), C.c_int, P(C.c_double), P(C.c_double),
                                   P(C.c_double)]
        L.oracle_rigid.restype = C.c_int
        L.oracle_rigid.argtypes = [C.c_int] + [C.c_void_p] * 14 + [C.c_double, C.c_double, C.c_int, C.c_int,
                                                                    C.c_void_p]
        L.oracle_sortkeys.restype = C.c_int
        L.oracle_sortkeys.argtypes = [C.c_int, P(C.c_float), P(C.c_double), C.c_int, P(C.c_uint)]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def bin_system(sysm):
    """Cell grid and the reference's cell assignment / cell-local float positions."""
    cdim = np.floor(sysm.dim / sysm.L).astype(np.int32)
    h = sysm.dim / cdim
    ih = 1.0 / h
    ind = ((sysm.x - sysm.origin) * ih).astype(np.int64)      # truncation, values >= 0
    cell = ((ind[:, 0] * cdim[1] + ind[:, 1]) * cdim[2] + ind[:, 2]).astype(np.int32)
    corigin = sysm.origin + ind * h
    xrel = (sysm.x - corigin).astype(np.float32)
    return dict(cdim=cdim, h=h, cell=cell, xrel=xrel)


def pack_tables(sysm, tables):
    """tables[k] = (n, alpha[4] float32, coef[(n+1)*8] float32) for sysm.pots[k], then, for a
    system with explicit electrostatics (sysm.ep), the table of sysm.ep last."""
    mt = len(sysm.masses)
    potidx = -np.ones((mt, mt), np.int32)
    coef, alpha, coff, potn = [], [], [], []
    off = 0
    for k, (n, a, c) in enumerate(tables):
        if k < len(sysm.pots):
            spec = sysm.pots[k]
            potidx[spec.ti, spec.tj] = k
            potidx[spec.tj, spec.ti] = k
        coef.append(np.asarray(c, np.float32))
        alpha.append(np.asarray(a, np.float32)[:4])
        coff.append(off)
        potn.append(n)
        off += len(c)
    return dict(potidx=potidx.reshape(-1), coef=np.concatenate(coef).astype(np.float32),
                alpha=np.concatenate(alpha).astype(np.float32), coff=np.array(coff, np.int32),
                potn=np.array(potn, np.int32))


def nonbond(sysm, tables, binned=None):
    """FP64 forces (by id), energy, virial, the sums over pairs of |e| (epot_abs) and |r.F|
    (virial_abs), pair and excluded-pair counts."""
    b = binned or bin_system(sysm)
    t = pack_tables(sysm, tables)
    N = sysm.n
    f = np.zeros((N, 3), np.float64)
    epot, eabs, vir, vabs = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    npairs, nex = C.c_longlong(), C.c_longlong()
    xrel = np.ascontiguousarray(b["xrel"], np.float32)
    cell = np.ascontiguousarray(b["cell"], np.int32)
    typ = np.ascontiguousarray(sysm.type, np.int32)
    org = np.ascontiguousarray(sysm.origin, np.float64)
    dim = np.ascontiguousarray(sysm.dim, np.float64)
    cdim = np.ascontiguousarray(b["cdim"], np.int32)
    excl = np.ascontiguousarray(sysm.excl, np.int32).reshape(-1)
    ep = len(sysm.pots) if getattr(sysm, "ep", None) is not None else -1
    if ep >= 0 and len(tables) != len(sysm.pots) + 1:
        raise ValueError("a system with explicit electrostatics needs the ep table after the type tables")
    q = np.ascontiguousarray(sysm.q if getattr(sysm, "q", None) is not None else np.zeros(N), np.float64)
    rc = lib().oracle_nonbond(N, _p(xrel, C.c_float), _p(cell, C.c_int), _p(typ, C.c_int), _p(org, C.c_double),
                              _p(dim, C.c_double), _p(cdim, C.c_int), float(sysm.cutoff), sysm.period,
                              len(sysm.masses), _p(t["potidx"], C.c_int), _p(t["coef"], C.c_float),
                              _p(t["alpha"], C.c_float), _p(t["coff"], C.c_int), _p(t["potn"], C.c_int),
                              len(sysm.excl), _p(excl, C.c_int) if excl.size else None, _p(f, C.c_double),
                              C.byref(epot), C.byref(eabs), C.byref(vir), C.byref(vabs), C.byref(npairs),
                              C.byref(nex), _p(q, C.c_double) if ep >= 0 else None, ep)
    if rc != 0:
        raise RuntimeError("oracle_nonbond failed")
    return dict(f=f, epot=epot.value, epot_abs=eabs.value, virial=vir.value, virial_abs=vabs.value,
                pairs=npairs.value, excluded=nex.value)


def bonds(sysm, table, binned=None):
    """FP64 bond forces (by id) and energy of sysm.bonds with one bond table (n, alpha, coef)
    of potential sysm.bond_pot (oracle_bonds)."""
    b = binned or bin_system(sysm)
    n, alpha, coef = table
    N = sysm.n
    f = np.zeros((N, 3), np.float64)
    e = C.c_double()
    bij = np.ascontiguousarray(sysm.bonds, np.int32).reshape(-1)
    xrel = np.ascontiguousarray(b["xrel"], np.float32)
    cell = np.ascontiguousarray(b["cell"], np.int32)
    cdim = np.ascontiguousarray(b["cdim"], np.int32)
    dim = np.ascontiguousarray(sysm.dim, np.float64)
    coef = np.ascontiguousarray(coef, np.float32)
    alpha = np.ascontiguousarray(alpha, np.float32)
    spec = sysm.bond_pot
    ab2 = np.array([spec.a * spec.a, spec.b * spec.b], np.float64)
    lib().oracle_bonds(len(bij) // 2, _p(bij, C.c_int), _p(xrel, C.c_float), _p(cell, C.c_int), _p(cdim, C.c_int),
                       _p(dim, C.c_double), _p(coef, C.c_float), _p(alpha, C.c_float), int(n), _p(ab2, C.c_double),
                       _p(f, C.c_double), C.byref(e))
    return dict(f=f, epot=e.value)


def _bonded(fn, terms, width, sysm, tables, xrel, cell, cdim):
    """Calls oracle_angles / oracle_dihedrals: terms (M, width) ids and table index; tables
    [(n, alpha, coef, a, b)] by potential index."""
    N = sysm.n
    f = np.zeros((N, 3), np.float64)
    e = C.c_double()
    t = np.ascontiguousarray(np.asarray(terms, np.int32).reshape(-1, width))
    coef = np.ascontiguousarray(np.concatenate([np.asarray(tb[2], np.float32) for tb in tables]), np.float32)
    coff = np.ascontiguousarray(np.cumsum([0] + [len(tb[2]) for tb in tables[:-1]]), np.int32)
    alpha = np.ascontiguousarray(np.concatenate([np.asarray(tb[1], np.float32) for tb in tables]), np.float32)
    potn = np.ascontiguousarray([tb[0] for tb in tables], np.int32)
    ab = np.ascontiguousarray([[tb[3], tb[4]] for tb in tables], np.float64).reshape(-1)
    xrel = np.ascontiguousarray(xrel, np.float32)
    cell = np.ascontiguousarray(cell, np.int32)
    cdim = np.ascontiguousarray(cdim, np.int32)
    dim = np.ascontiguousarray(sysm.dim, np.float64)
    fn(len(t), _p(t, C.c_int), _p(xrel, C.c_float), _p(cell, C.c_int), _p(cdim, C.c_int), _p(dim, C.c_double),
       _p(coef, C.c_float), _p(coff, C.c_int), _p(alpha, C.c_float), _p(potn, C.c_int), _p(ab, C.c_double),
       _p(f, C.c_double), C.byref(e))
    return dict(f=f, epot=e.value)


def angles(sysm, tables, binned=None, xrel=None, cell=None):
    """FP64 angle forces (by id) and energy of sysm.angles (oracle_angles); tables
    [(n, alpha, coef, a, b)] of sysm.angle_pots.  Positions from bin_system(sysm) unless
    xrel and cell are given."""
    b = binned or bin_system(sysm)
    return _bonded(lib().oracle_angles, sysm.angles, 4, sysm, tables, b["xrel"] if xrel is None else xrel,
                   b["cell"] if cell is None else cell, b["cdim"])


def dihedrals(sysm, tables, binned=None, xrel=None, cell=None):
    """FP64 dihedral forces (by id) and energy of sysm.dihedrals (oracle_dihedrals)."""
    b = binned or bin_system(sysm)
    return _bonded(lib().oracle_dihedrals, sysm.dihedrals, 5, sysm, tables, b["xrel"] if xrel is None else xrel,
                   b["cell"] if cell is None else cell, b["cdim"])


def sortkeys(xrel_cell: np.ndarray, h, sid: int) -> np.ndarray:
    n = len(xrel_cell)
    keys = np.zeros(max(n, 1), np.uint32)
    x = np.ascontiguousarray(xrel_cell, np.float32)
    hh = np.ascontiguousarray(h, np.float64)
    lib().oracle_sortkeys(n, _p(x, C.c_float), _p(hh, C.c_double), sid, _p(keys, C.c_uint))
    return keys[:n]


def rigid(groups, x, v, f, cell, cdim, h, mass, dt, tol, pshake, a_update):
    """One rigid-constraint evaluation (oracle_rigid) on particle state by id.

    groups: list of (parts: list of ids, constraints: list of (i, j, d2), a: nc x nc float32).
    x, v, f: (N, 3) float32 cell-relative positions, velocities, forces; cell: (N,) cell
    index; cdim: cell grid; h: cell edge; mass: (N,) per-particle mass.
    Returns (x, v, f, [a], iters) after the evaluation (inputs are not modified)."""
    roff = np.cumsum([0] + [len(g[0]) for g in groups]).astype(np.int32)
    coff = np.cumsum([0] + [len(g[1]) for g in groups]).astype(np.int32)
    parts = np.array([i for g in groups for i in g[0]], np.int32)
    con = np.array([c for g in groups for c in g[1]], np.float64).reshape(-1, 3)
    ci = np.ascontiguousarray(con[:, 0], np.int32)
    cj = np.ascontiguousarray(con[:, 1], np.int32)
    d2 = np.ascontiguousarray(con[:, 2], np.float64)
    a = np.concatenate([np.asarray(g[2], np.float32).reshape(-1) for g in groups]).astype(np.float32)
    cdim = np.asarray(cdim, np.int64)
    ncells = int(np.prod(cdim))
    cid = np.arange(ncells)
    loc = np.stack([cid // (cdim[1] * cdim[2]), (cid // cdim[2]) % cdim[1], cid % cdim[2]], 1).astype(np.int32)
    xo, vo, fo = (np.ascontiguousarray(t, np.float32).copy() for t in (x, v, f))
    cell = np.ascontiguousarray(cell, np.int32)
    hh = np.ascontiguousarray(h, np.float64)
    m = np.ascontiguousarray(mass, np.float64)
    iters = np.zeros(len(groups), np.int32)
    rc = lib().oracle_rigid(len(groups), roff.ctypes.data, parts.ctypes.data, coff.ctypes.data, ci.ctypes.data,
                            cj.ctypes.data, d2.ctypes.data, a.ctypes.data, cell.ctypes.data, loc.ctypes.data,
                            hh.ctypes.data, m.ctypes.data, xo.ctypes.data, vo.ctypes.data, fo.ctypes.data,
                            float(dt), float(tol), int(pshake), int(a_update), iters.ctypes.data)
    if rc != 0:
        raise RuntimeError("oracle_rigid failed")
    mats, off = [], 0
    for g in groups:
        n = len(g[1])
        mats.append(a[off:off + n * n].reshape(n, n).copy())
        off += n * n
    return xo, vo, fo, mats, iters


def ref_available(strict: bool = True) -> bool:
    return os.path.exists(os.path.join(REF_DIR, "ref_driver_strict" if strict else "ref_driver"))


def run_ref_forces(sysm, workdir, runners=4, strict=True):
    """Runs the compiled reference (oracle/_ref) on `sysm`; returns workloads.read_refout()."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(_HERE), "mdcore-history_b200"))
    import workloads as W
    sysf = os.path.join(workdir, sysm.name + ".sys")
    outf = os.path.join(workdir, sysm.name + ".out")
    W.write_sysfile(sysm, sysf)
    exe = os.path.join(REF_DIR, "ref_driver_strict" if strict else "ref_driver")
    subprocess.run([exe, "forces", sysf, outf, str(runners)], check=True, capture_output=True)
    return W.read_refout(outf, sysm)
