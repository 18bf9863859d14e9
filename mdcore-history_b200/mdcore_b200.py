"""ctypes binding of libmdcore_b200.so (the C engine API declared in include/mdcore_b200.h).

The calls mirror a reference mdcore driver (examples/argon/argon.c): engine_init,
engine_addtype, potential_create_*, engine_addpot, engine_load, engine_exclusion_add,
engine_start, engine_step.  The library runs every force evaluation on the GPU and fails
loudly when it cannot: there is no CPU fallback.
"""
from __future__ import annotations

import collections
import ctypes as C
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmdcore_b200.so")

MLP_IN = 10
MLP_HIDDEN = 32
MLP_NPARAM = MLP_HIDDEN * MLP_IN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_HIDDEN + 1
# count-product heuristic weights of the reference's partitioner (src/engine.c:574-576)
CLASS_WEIGHT = (0.50004, 0.16176, 0.036213)

engine_flag_none = 0
engine_flag_cuda = 4
engine_flag_verlet = 16
engine_flag_verlet_pseudo = 256
engine_flag_unsorted = 512
engine_flag_shake = 1024
space_periodic_full = 7


class Potential(C.Structure):
    """struct potential (src/potential.h:57-74)."""
    _fields_ = [("alpha", C.c_float * 4), ("c", C.POINTER(C.c_float)), ("a", C.c_double),
                ("b", C.c_double), ("flags", C.c_uint), ("n", C.c_int)]

    def table(self):
        n = self.n
        c = np.ctypeslib.as_array(self.c, shape=((n + 1) * 8,)).copy()
        return n, np.array(self.alpha[:], dtype=np.float32), c


class RigidConstr(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int), ("d2", C.c_double)]


class Rigid(C.Structure):
    """struct rigid (src/rigid.h:39-59)."""
    _fields_ = [("nr_parts", C.c_int), ("parts", C.c_int * 10), ("nr_constr", C.c_int),
                ("constr", RigidConstr * 30), ("a", C.c_float * 900)]

    def constraints(self):
        """(i, j, d2) of every constraint, group-local indices."""
        return [(self.constr[k].i, self.constr[k].j, self.constr[k].d2) for k in range(self.nr_constr)]

    def matrix(self) -> np.ndarray:
        n = self.nr_constr
        return np.array(self.a[:n * n], np.float32).reshape(n, n)


class NbStats(C.Structure):
    _fields_ = [("pairs", C.c_int64), ("excluded", C.c_int64), ("candidates", C.c_int64),
                ("epot", C.c_double), ("virial", C.c_double), ("status", C.c_int),
                ("ms_kernels", C.c_float), ("ms_pack", C.c_float), ("ms_device", C.c_float),
                ("ms_unpack", C.c_float)]


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Loads the library (once); raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C mdcore-history_b200`")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    dp, ip, vp = P(C.c_double), P(C.c_int), C.c_void_p
    sig = {
        "engine_sizeof": (C.c_size_t, []),
        "engine_init": (C.c_int, [vp, dp, dp, dp, C.c_double, C.c_uint, C.c_int, C.c_uint]),
        "engine_addtype": (C.c_int, [vp, C.c_double, C.c_double, C.c_char_p, C.c_char_p]),
        "engine_addpot": (C.c_int, [vp, P(Potential), C.c_int, C.c_int]),
        "engine_load": (C.c_int, [vp, dp, dp, ip, ip, ip, dp, P(C.c_uint), C.c_int]),
        "engine_unload": (C.c_int, [vp, dp, dp, ip, ip, ip, dp, P(C.c_uint), dp, C.c_int]),
        "engine_exclusion_add": (C.c_int, [vp, C.c_int, C.c_int]),
        "engine_exclusion_shrink": (C.c_int, [vp]),
        "engine_rigid_add": (C.c_int, [vp, C.c_int, C.c_int, C.c_double]),
        "engine_start": (C.c_int, [vp, C.c_int, C.c_int]),
        "engine_step": (C.c_int, [vp]),
        "engine_step_host": (C.c_int, [vp]),
        "engine_setexplepot": (C.c_int, [vp, P(Potential)]),
        "engine_bond_addpot": (C.c_int, [vp, P(Potential), C.c_int, C.c_int]),
        "engine_bond_add": (C.c_int, [vp, C.c_int, C.c_int]),
        "engine_energies": (C.c_int, [vp, dp]),
        "engine_angle_addpot": (C.c_int, [vp, P(Potential)]),
        "engine_angle_add": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int]),
        "engine_dihedral_addpot": (C.c_int, [vp, P(Potential)]),
        "engine_dihedral_add": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
        "potential_create_harmonic_angle": (P(Potential), [C.c_double] * 5),
        "potential_create_harmonic_dihedral": (P(Potential), [C.c_double, C.c_int, C.c_double, C.c_double]),
        "engine_batch_step_host": (C.c_int, [vp]),
        "engine_advance": (C.c_int, [vp]),
        "engine_finalize": (C.c_int, [vp]),
        "engine_cuda_setdevice": (C.c_int, [vp, C.c_int]),
        "engine_cuda_load": (C.c_int, [vp]),
        "engine_nonbond_cuda": (C.c_int, [vp]),
        "engine_nonbond_cuda_fresh": (C.c_int, [vp]),
        "engine_batch_nonbond_fresh": (C.c_int, [vp]),
        "engine_cuda_load_parts": (C.c_int, [vp]),
        "engine_cuda_unload_parts": (C.c_int, [vp]),
        "engine_nonbond_cuda_resident": (C.c_int, [vp]),
        "engine_cuda_setstream": (C.c_int, [vp, vp]),
        "engine_cuda_settune": (C.c_int, [vp, C.c_int, C.c_int]),
        "engine_cuda_getsort": (C.c_int, [vp, C.c_int, P(C.c_uint), C.c_int]),
        "engine_getforces": (C.c_int, [vp, dp, C.c_int]),
        "engine_getcells": (C.c_int, [vp, ip, C.c_int]),
        "engine_nonbond_stats": (C.c_int, [vp, P(NbStats)]),
        "engine_set_dt": (C.c_int, [vp, C.c_double]),
        "engine_cuda_kernel_times": (C.c_int, [vp, P(C.c_float), P(C.c_float)]),
        "engine_cuda_setorder": (C.c_int, [vp, ip, C.c_int]),
        "engine_cuda_taskclocks": (C.c_int, [vp, C.c_int, P(C.c_longlong), ip, C.c_int]),
        "engine_cuda_ntasks": (C.c_int, [vp]),
        "engine_cuda_fp32_peak": (C.c_int, [C.c_int, P(C.c_float)]),
        "engine_zero_forces": (C.c_int, [vp]),
        "engine_cuda_setwindow": (C.c_int, [vp, C.c_int]),
        "engine_rigid_eval": (C.c_int, [vp]),
        "engine_rigid_stats": (C.c_int, [vp, ip, ip]),
        "engine_rigid_getmatrices": (C.c_int, [vp]),
        "engine_rigid_get": (C.c_int, [vp, C.c_int, vp]),
        "engine_getparts": (C.c_int, [vp, vp, vp, vp, vp, C.c_int]),
        "engine_cuda_graph": (C.c_int, [vp, C.c_int]),
        "engine_cuda_autotune": (C.c_int, [vp, C.c_int, ip, ip, ip, ip, P(C.c_float)]),
        "engine_cuda_setlayout": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
        "engine_batch_setlayout": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
        "engine_batch_create": (C.c_int, [P(vp), C.c_int, P(vp)]),
        "engine_batch_free": (C.c_int, [vp]),
        "engine_batch_nonbond": (C.c_int, [vp]),
        "engine_batch_step": (C.c_int, [vp]),
        "engine_batch_setgroups": (C.c_int, [vp, C.c_int]),
        "engine_batch_sched_order": (C.c_int, [vp, C.c_int]),
        "engine_batch_load_parts": (C.c_int, [vp]),
        "engine_batch_resident": (C.c_int, [vp]),
        "engine_batch_unload_parts": (C.c_int, [vp]),
        "engine_batch_stats": (C.c_int, [vp, P(NbStats)]),
        "engine_batch_zero_forces": (C.c_int, [vp]),
        "engine_batch_setstream": (C.c_int, [vp, vp]),
        "engine_batch_kernel_times": (C.c_int, [vp, P(C.c_float), P(C.c_float)]),
        "engine_batch_settune": (C.c_int, [vp, C.c_int, C.c_int]),
        "engine_batch_graph": (C.c_int, [vp, C.c_int]),
        "engine_batch_autotune": (C.c_int, [vp, C.c_int, ip, ip, ip, ip, P(C.c_float)]),
        "engine_batch_ntasks": (C.c_int, [vp]),
        "engine_cuda_resident_begin": (C.c_int, [vp, C.c_int]),
        "engine_cuda_resident_steps": (C.c_int, [vp, C.c_int]),
        "engine_cuda_resident_sync": (C.c_int, [vp]),
        "engine_cuda_resident_end": (C.c_int, [vp]),
        "engine_batch_resident_begin": (C.c_int, [vp, C.c_int]),
        "engine_batch_resident_steps": (C.c_int, [vp, C.c_int]),
        "engine_batch_resident_sync": (C.c_int, [vp]),
        "engine_batch_resident_end": (C.c_int, [vp]),
        "engine_cuda_resident_info": (C.c_int, [vp, ip, ip, P(C.c_longlong), P(C.c_longlong), ip]),
        "engine_batch_resident_info": (C.c_int, [vp, ip, ip, P(C.c_longlong), P(C.c_longlong), ip]),
        "engine_cuda_minimize": (C.c_int, [vp, C.c_double, C.c_double]),
        "engine_cuda_energylog": (C.c_int, [vp, C.c_int]),
        "engine_cuda_energylog_read": (C.c_int, [vp, dp, C.c_int]),
        "engine_cuda_setaccum": (C.c_int, [vp, C.c_int]),
        "engine_cuda_setspin": (C.c_int, [vp, C.c_int]),
        "engine_cuda_verlet_rebuilds": (C.c_int, [vp, ip]),
        "engine_cuda_copytimeout_test": (C.c_int, [vp, C.c_int]),
        "engine_sched_record": (C.c_int, [vp, C.c_int]),
        "engine_sched_features": (C.c_int, [vp, P(C.c_float), C.c_int]),
        "engine_sched_targets": (C.c_int, [vp, P(C.c_float), C.c_int]),
        "engine_sched_train": (C.c_int, [vp, C.c_int, C.c_int, C.c_float, C.c_uint, P(C.c_float)]),
        "engine_sched_predict": (C.c_int, [vp, P(C.c_float), C.c_int]),
        "engine_sched_apply": (C.c_int, [vp, C.c_int]),
        "engine_sched_order": (C.c_int, [vp, C.c_int, C.c_int]),
        "engine_cuda_getorder": (C.c_int, [vp, ip, C.c_int]),
        "nb_mlp_predict": (C.c_int, [vp, C.c_int, vp, vp, vp]),
        "nb_mlp_grad": (C.c_int, [vp, vp, vp, C.c_int, vp, vp, vp, vp]),
        "nb_mlp_adam": (C.c_int, [vp, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, vp]),
        "potential_create_LJ126": (P(Potential), [C.c_double] * 5),
        "potential_create_LJ126_Coulomb": (P(Potential), [C.c_double] * 6),
        "potential_create_Coulomb": (P(Potential), [C.c_double] * 4),
        "potential_create_harmonic": (P(Potential), [C.c_double] * 5),
        "potential_create_Ewald": (P(Potential), [C.c_double] * 5),
        "potential_create_LJ126_Ewald": (P(Potential), [C.c_double] * 7),
        "errs_dump": (C.c_int, [vp]),
        "errs_clear": (None, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class MdcoreError(RuntimeError):
    pass


def _check(rc: int, what: str):
    if rc is not None and rc < 0:
        import io, tempfile
        libc = C.CDLL(None)
        msg = ""
        with tempfile.TemporaryFile(mode="w+") as tf:
            fp = libc.fdopen(os.dup(tf.fileno()), b"w")
            lib().errs_dump(fp)
            libc.fflush(fp)
            libc.fclose(fp)
            tf.seek(0)
            msg = tf.read()
        raise MdcoreError(f"{what} failed with {rc}: {msg.strip()}")
    return rc


def create_potential(spec):
    """Builds a table with the library's potential_create_* (spec: workloads.PotSpec)."""
    L = lib()
    k, a, b, tol, p = spec.kind, spec.a, spec.b, spec.tol, spec.p
    if k == 1:
        ptr = L.potential_create_LJ126(a, b, p[0], p[1], tol)
    elif k == 2:
        ptr = L.potential_create_LJ126_Coulomb(a, b, p[0], p[1], p[2], tol)
    elif k == 3:
        ptr = L.potential_create_Coulomb(a, b, p[0], tol)
    elif k == 4:
        ptr = L.potential_create_Ewald(a, b, p[0], p[1], tol)
    elif k == 5:
        ptr = L.potential_create_LJ126_Ewald(a, b, p[0], p[1], p[2], p[3], tol)
    elif k == 7:
        ptr = L.potential_create_harmonic(a, b, p[0], p[1], tol)
    else:
        raise ValueError(f"potential kind {k} has no library constructor")
    if not ptr:
        _check(-17, f"potential_create kind {k}")
    return ptr


def create_angle_potential(a, b, K, theta0, tol):
    """potential_create_harmonic_angle (one entry of workloads.System.angle_pots)."""
    ptr = lib().potential_create_harmonic_angle(a, b, K, theta0, tol)
    if not ptr:
        _check(-17, "potential_create_harmonic_angle")
    return ptr


def create_dihedral_potential(K, n, delta, tol):
    """potential_create_harmonic_dihedral (one entry of workloads.System.dihedral_pots)."""
    ptr = lib().potential_create_harmonic_dihedral(K, int(n), delta, tol)
    if not ptr:
        _check(-17, "potential_create_harmonic_dihedral")
    return ptr


def bonded_tables(ptrs):
    """(n, alpha, coef, a, b) of each potential: the oracle's table arguments."""
    out = []
    for p in ptrs:
        n, alpha, c = p.contents.table()
        out.append((n, alpha, c, p.contents.a, p.contents.b))
    return out


class Engine:
    """Owns one struct engine allocated in Python memory, as a C driver would on its stack."""

    def __init__(self, origin, dim, L, cutoff, period=space_periodic_full, max_type=1, flags=engine_flag_cuda):
        self.lib = lib()
        size = self.lib.engine_sizeof()
        self._buf = C.create_string_buffer(size + 64)
        addr = C.addressof(self._buf)
        self.ptr = C.c_void_p((addr + 63) & ~63)
        o = np.ascontiguousarray(origin, np.float64)
        d = np.ascontiguousarray(dim, np.float64)
        l = np.ascontiguousarray(L, np.float64)
        _check(self.lib.engine_init(self.ptr, _dptr(o), _dptr(d), _dptr(l), float(cutoff), period, max_type, flags),
               "engine_init")
        self.pots = []
        self.n = 0
        self.closed = False

    @classmethod
    def from_system(cls, sysm, flags=engine_flag_cuda, device=0, start=True):
        e = cls(sysm.origin, sysm.dim, sysm.L, sysm.cutoff, sysm.period, len(sysm.masses), flags)
        for m, q in zip(sysm.masses, sysm.charges):
            _check(e.lib.engine_addtype(e.ptr, m, q, None, None), "engine_addtype")
        for spec in sysm.pots:
            ptr = create_potential(spec)
            e.pots.append(ptr)
            _check(e.lib.engine_addpot(e.ptr, ptr, spec.ti, spec.tj), "engine_addpot")
        x = np.ascontiguousarray(sysm.x, np.float64)
        t = np.ascontiguousarray(sysm.type, np.int32)
        v = None if sysm.v is None else np.ascontiguousarray(sysm.v, np.float64)
        q = None if getattr(sysm, "q", None) is None else np.ascontiguousarray(sysm.q, np.float64)
        _check(e.lib.engine_load(e.ptr, _dptr(x), None if v is None else _dptr(v), _iptr(t), None, None,
                                 None if q is None else _dptr(q), None, sysm.n), "engine_load")
        if getattr(sysm, "ep", None) is not None:
            ep = create_potential(sysm.ep)
            e.pots.append(ep)
            _check(e.lib.engine_setexplepot(e.ptr, ep), "engine_setexplepot")
        if getattr(sysm, "bonds", None) is not None and len(sysm.bonds):
            bp = create_potential(sysm.bond_pot)
            e.pots.append(bp)
            bt = np.asarray(sysm.type)[np.asarray(sysm.bonds)]
            for ti, tj in {(int(min(a, b)), int(max(a, b))) for a, b in bt}:
                _check(e.lib.engine_bond_addpot(e.ptr, bp, ti, tj), "engine_bond_addpot")
            for i, j in np.asarray(sysm.bonds):
                _check(e.lib.engine_bond_add(e.ptr, int(i), int(j)), "engine_bond_add")
        e.angle_pots, e.dihedral_pots = [], []
        if getattr(sysm, "angles", None) is not None and len(sysm.angles):
            for spec in sysm.angle_pots:
                ptr = create_angle_potential(*spec)
                e.angle_pots.append(ptr)
                _check(e.lib.engine_angle_addpot(e.ptr, ptr), "engine_angle_addpot")
            for i, j, k, pid in np.asarray(sysm.angles):
                _check(e.lib.engine_angle_add(e.ptr, int(i), int(j), int(k), int(pid)), "engine_angle_add")
        if getattr(sysm, "dihedrals", None) is not None and len(sysm.dihedrals):
            for spec in sysm.dihedral_pots:
                ptr = create_dihedral_potential(*spec)
                e.dihedral_pots.append(ptr)
                _check(e.lib.engine_dihedral_addpot(e.ptr, ptr), "engine_dihedral_addpot")
            for i, j, k, l, pid in np.asarray(sysm.dihedrals):
                _check(e.lib.engine_dihedral_add(e.ptr, int(i), int(j), int(k), int(l), int(pid)),
                       "engine_dihedral_add")
        e.n = sysm.n
        if sysm.rigid is not None:
            for i, j, d in np.asarray(sysm.rigid):
                _check(e.lib.engine_rigid_add(e.ptr, int(i), int(j), float(d)), "engine_rigid_add")
        for i, j in np.asarray(sysm.excl).reshape(-1, 2):
            _check(e.lib.engine_exclusion_add(e.ptr, int(i), int(j)), "engine_exclusion_add")
        if len(sysm.excl):
            _check(e.lib.engine_exclusion_shrink(e.ptr), "engine_exclusion_shrink")
        _check(e.lib.engine_set_dt(e.ptr, sysm.dt), "engine_set_dt")
        if start:
            _check(e.lib.engine_cuda_setdevice(e.ptr, device), "engine_cuda_setdevice")
            _check(e.lib.engine_start(e.ptr, 1, 1), "engine_start")
        return e

    # -- force evaluation ----------------------------------------------------------
    def nonbond(self):
        """One force evaluation at the current positions (host buffers in and out): the
        cells' forces and energies become this evaluation's (engine_nonbond_cuda_fresh)."""
        _check(self.lib.engine_nonbond_cuda_fresh(self.ptr), "engine_nonbond_cuda_fresh")
        return self

    def step(self):
        """engine_step: one time step on the device, host particles in and out."""
        _check(self.lib.engine_step(self.ptr), "engine_step")
        return self

    def step_host(self):
        """engine_step_host: re-binning and integration on the host, forces and constraints
        through host buffers."""
        _check(self.lib.engine_step_host(self.ptr), "engine_step_host")
        return self

    # -- device-resident time steps --------------------------------------------------
    def resident_begin(self, margin: int = -1):
        """Uploads the particles into per-cell device blocks (engine_cuda_resident_begin)."""
        _check(self.lib.engine_cuda_resident_begin(self.ptr, margin), "engine_cuda_resident_begin")
        return self

    def resident_steps(self, nsteps: int = 1):
        """nsteps engine_step equivalents entirely on the device."""
        _check(self.lib.engine_cuda_resident_steps(self.ptr, nsteps), "engine_cuda_resident_steps")
        return self

    def resident_sync(self):
        """Host cells, energies and stats as of the last resident step."""
        _check(self.lib.engine_cuda_resident_sync(self.ptr), "engine_cuda_resident_sync")
        return self

    def resident_end(self):
        _check(self.lib.engine_cuda_resident_end(self.ptr), "engine_cuda_resident_end")
        return self

    def resident_info(self):
        """ResidentInfo(capc, mcap, steps, pairs, regrows): slots per cell, leavers per cell
        and step, completed steps and their accepted pairs, re-blockings."""
        return _resident_info(self.lib.engine_cuda_resident_info, self.ptr)

    def minimize(self, gamma: float, dmax: float = 0.01):
        """Resident steps become steepest-descent moves x += gamma f (at most dmax nm per
        particle, velocities zeroed); gamma <= 0 restores the time step."""
        _check(self.lib.engine_cuda_minimize(self.ptr, gamma, dmax), "engine_cuda_minimize")
        return self

    def energy_log(self, cap: int):
        """Per-step energy log of the resident steps, a ring of `cap` records (0: off)."""
        _check(self.lib.engine_cuda_energylog(self.ptr, cap), "engine_cuda_energylog")
        return self

    def energy_log_read(self, cap: int) -> np.ndarray:
        """Records in step order: (step, potential, kinetic, total) per row, kJ/mol."""
        out = np.zeros((max(cap, 1), 4))
        n = _check(self.lib.engine_cuda_energylog_read(self.ptr, _dptr(out), cap), "engine_cuda_energylog_read")
        return out[:n]

    def set_accum(self, fp32: bool):
        """Force accumulation of the plain form: FP32 float atomics (True) or fixed point."""
        _check(self.lib.engine_cuda_setaccum(self.ptr, int(fp32)), "engine_cuda_setaccum")
        return self

    def verlet_rebuilds(self) -> int:
        """Re-binning + sort steps of the resident steps since the upload (engine_flag_verlet)."""
        r = C.c_int()
        _check(self.lib.engine_cuda_verlet_rebuilds(self.ptr, C.byref(r)), "engine_cuda_verlet_rebuilds")
        return r.value

    def set_spin(self, polls: int):
        """Polls per bounded wait of the sweeps on this engine's device (<= 0: default)."""
        _check(self.lib.engine_cuda_setspin(self.ptr, polls), "engine_cuda_setspin")
        return self

    def copytimeout_test(self, enable: bool):
        """Test hook: the sweeps' staging copies are not issued, so their waits run out."""
        _check(self.lib.engine_cuda_copytimeout_test(self.ptr, int(enable)), "engine_cuda_copytimeout_test")
        return self

    def load_parts(self):
        _check(self.lib.engine_cuda_load_parts(self.ptr), "engine_cuda_load_parts")

    def resident(self):
        _check(self.lib.engine_nonbond_cuda_resident(self.ptr), "engine_nonbond_cuda_resident")

    def unload_parts(self):
        _check(self.lib.engine_zero_forces(self.ptr), "engine_zero_forces")
        _check(self.lib.engine_cuda_unload_parts(self.ptr), "engine_cuda_unload_parts")

    def set_stream(self, stream_ptr: int):
        _check(self.lib.engine_cuda_setstream(self.ptr, C.c_void_p(stream_ptr)), "engine_cuda_setstream")

    def kernel_times(self):
        a, b = C.c_float(), C.c_float()
        _check(self.lib.engine_cuda_kernel_times(self.ptr, C.byref(a), C.byref(b)), "engine_cuda_kernel_times")
        return a.value, b.value

    # -- learned scheduler ----------------------------------------------------------
    def sched_record(self, nsteps: int):
        _check(self.lib.engine_sched_record(self.ptr, nsteps), "engine_sched_record")

    def sched_features(self) -> np.ndarray:
        n = self.ntasks()
        X = np.zeros((n, MLP_IN), np.float32)
        _check(self.lib.engine_sched_features(self.ptr, X.ctypes.data_as(C.POINTER(C.c_float)), n),
               "engine_sched_features")
        return X

    def sched_targets(self) -> np.ndarray:
        n = self.ntasks()
        y = np.zeros(n, np.float32)
        _check(self.lib.engine_sched_targets(self.ptr, y.ctypes.data_as(C.POINTER(C.c_float)), n),
               "engine_sched_targets")
        return y

    def sched_train(self, epochs: int = 100, batch: int = 1024, lr: float = 3e-3, seed: int = 0) -> float:
        loss = C.c_float()
        _check(self.lib.engine_sched_train(self.ptr, epochs, batch, lr, seed, C.byref(loss)), "engine_sched_train")
        return loss.value

    def sched_predict(self) -> np.ndarray:
        n = self.ntasks()
        p = np.zeros(n, np.float32)
        _check(self.lib.engine_sched_predict(self.ptr, p.ctypes.data_as(C.POINTER(C.c_float)), n),
               "engine_sched_predict")
        return p

    def sched_order(self, source: int, tile: int = 0):
        """Cost-class tiles in cell-major order (source 0: count-product, 1: the network)."""
        _check(self.lib.engine_sched_order(self.ptr, source, tile), "engine_sched_order")

    def sched_apply(self, use_mlp: bool):
        _check(self.lib.engine_sched_apply(self.ptr, int(use_mlp)), "engine_sched_apply")

    def tune(self, warps: int = 0, plain: bool = False):
        """warps per block (0 = default); plain=True selects the one-block-per-task form."""
        _check(self.lib.engine_cuda_settune(self.ptr, warps, 1 if plain else 0), "engine_cuda_settune")

    def set_window(self, window: int):
        """Sweep steps per register reduce-scatter of the persistent sweep (4 or 8)."""
        _check(self.lib.engine_cuda_setwindow(self.ptr, window), "engine_cuda_setwindow")

    def graph(self, enable: bool = True):
        """CUDA-graph replay of each evaluation's launches."""
        _check(self.lib.engine_cuda_graph(self.ptr, int(enable)), "engine_cuda_graph")

    def set_layout(self, layout: int, stages: int = 1, occupancy: int = 640):
        """Persistent sweep shape: lane layout 0 = 32 i per warp, 1 = 8 i x 4 j tile;
        stages = staging buffers per worker warp (1 or 2); occupancy = resident threads per
        SM the registers are sized for (640, 768, 1024)."""
        _check(self.lib.engine_cuda_setlayout(self.ptr, layout, stages, occupancy), "engine_cuda_setlayout")

    def autotune(self, reps: int = 5):
        """Keeps the fastest persistent launch shape; returns (warps, layout, stages,
        occupancy, ms)."""
        w, lay, stg, occ, ms = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_float()
        _check(self.lib.engine_cuda_autotune(self.ptr, reps, C.byref(w), C.byref(lay), C.byref(stg), C.byref(occ),
                                             C.byref(ms)), "engine_cuda_autotune")
        return w.value, lay.value, stg.value, occ.value, ms.value

    def ntasks(self) -> int:
        return _check(self.lib.engine_cuda_ntasks(self.ptr), "engine_cuda_ntasks")

    def get_order(self) -> np.ndarray:
        o = np.zeros(self.ntasks(), np.int32)
        _check(self.lib.engine_cuda_getorder(self.ptr, _iptr(o), len(o)), "engine_cuda_getorder")
        return o

    def set_order(self, order):
        o = np.ascontiguousarray(order, np.int32)
        _check(self.lib.engine_cuda_setorder(self.ptr, _iptr(o), len(o)), "engine_cuda_setorder")

    def task_clocks(self, enable: bool = True, read: bool = False):
        """Enables per-task clock64 records; with read=True returns (clocks[n,2], sm[n]) of
        the last launch."""
        if not read:
            _check(self.lib.engine_cuda_taskclocks(self.ptr, int(enable), None, None, 0), "engine_cuda_taskclocks")
            return None
        n = self.ntasks()
        clk = np.zeros((n, 2), np.int64)
        sm = np.zeros(n, np.int32)
        _check(self.lib.engine_cuda_taskclocks(self.ptr, int(enable), clk.ctypes.data_as(C.POINTER(C.c_longlong)),
                                               _iptr(sm), n), "engine_cuda_taskclocks")
        return clk, sm

    # -- rigid constraints -----------------------------------------------------------
    def rigid_eval(self):
        """engine_rigid_eval: SHAKE or P-SHAKE of every rigid group on the device."""
        _check(self.lib.engine_rigid_eval(self.ptr), "engine_rigid_eval")

    def rigid_stats(self):
        """(largest iteration count, unconverged groups) of the last evaluation."""
        a, b = C.c_int(), C.c_int()
        _check(self.lib.engine_rigid_stats(self.ptr, C.byref(a), C.byref(b)), "engine_rigid_stats")
        return a.value, b.value

    def rigid_groups(self):
        """Every rigid group as a Rigid structure, P-SHAKE matrices synced from the device."""
        _check(self.lib.engine_rigid_getmatrices(self.ptr), "engine_rigid_getmatrices")
        n = _check(self.lib.engine_rigid_get(self.ptr, 0, None), "engine_rigid_get")
        out = []
        for g in range(n):
            r = Rigid()
            _check(self.lib.engine_rigid_get(self.ptr, g, C.byref(r)), "engine_rigid_get")
            out.append(r)
        return out

    def parts(self):
        """Cell-relative float positions, velocities, forces (N x 3 each) and cells by id."""
        x = np.zeros((self.n, 3), np.float32); v = np.zeros((self.n, 3), np.float32)
        f = np.zeros((self.n, 3), np.float32); c = np.zeros(self.n, np.int32)
        _check(self.lib.engine_getparts(self.ptr, x.ctypes.data, v.ctypes.data, f.ctypes.data, c.ctypes.data,
                                        self.n), "engine_getparts")
        return x, v, f, c

    # -- readback --------------------------------------------------------------------
    def forces(self) -> np.ndarray:
        f = np.zeros((self.n, 3), np.float64)
        _check(self.lib.engine_getforces(self.ptr, _dptr(f), self.n), "engine_getforces")
        return f

    def cells(self) -> np.ndarray:
        c = np.zeros(self.n, np.int32)
        _check(self.lib.engine_getcells(self.ptr, _iptr(c), self.n), "engine_getcells")
        return c

    def stats(self) -> NbStats:
        s = NbStats()
        _check(self.lib.engine_nonbond_stats(self.ptr, C.byref(s)), "engine_nonbond_stats")
        return s

    def sortkeys(self, cid: int, count: int) -> np.ndarray:
        buf = np.zeros(13 * max(count, 1), np.uint32)
        _check(self.lib.engine_cuda_getsort(self.ptr, cid, buf.ctypes.data_as(C.POINTER(C.c_uint)), buf.size),
               "engine_cuda_getsort")
        return buf[:13 * count].reshape(13, count)

    def energies(self):
        """e->s.epot and its parts after the last step or evaluation (engine_energies)."""
        out = np.zeros(6)
        _check(self.lib.engine_energies(self.ptr, _dptr(out)), "engine_energies")
        return dict(zip(("total", "nonbond", "bond", "angle", "dihedral", "exclusion"), (float(v) for v in out)))

    def unload(self):
        x = np.zeros((self.n, 3)); t = np.zeros(self.n, np.int32); pid = np.zeros(self.n, np.int32)
        epot = np.zeros(1)
        _check(self.lib.engine_unload(self.ptr, _dptr(x), None, _iptr(t), _iptr(pid), None, None, None,
                                      _dptr(epot), self.n), "engine_unload")
        return x, t, pid, float(epot[0])

    def close(self):
        if not self.closed:
            self.lib.engine_finalize(self.ptr)
            self.closed = True

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def leapfrog_energy(log: np.ndarray, dt_ps: float):
    """Total energy of the leap-frog steps of an energy log (rows: step, U, K after the step,
    U + K): E_t = U_t + (K(v_(t-1/2)) + K(v_(t+1/2))) / 2 for every record after the first,
    the times in ns, and the least-squares drift of E (kJ/mol/ns)."""
    E = log[1:, 1] + 0.5 * (log[:-1, 2] + log[1:, 2])
    t_ns = log[1:, 0] * dt_ps * 1e-3
    slope = float(np.polyfit(t_ns, E, 1)[0]) if len(E) > 2 else 0.0
    return E, t_ns, slope


def fp32_peak_tflops(device: int = 0) -> float:
    v = C.c_float()
    _check(lib().engine_cuda_fp32_peak(device, C.byref(v)), "engine_cuda_fp32_peak")
    return v.value


ResidentInfo = collections.namedtuple("ResidentInfo", "capc mcap steps pairs regrows")


def _resident_info(fn, ptr):
    a, b, c, d, g = C.c_int(), C.c_int(), C.c_longlong(), C.c_longlong(), C.c_int()
    _check(fn(ptr, C.byref(a), C.byref(b), C.byref(c), C.byref(d), C.byref(g)), fn.__name__)
    return ResidentInfo(a.value, b.value, c.value, d.value, g.value)


class Batch:
    """Many engines (replicas) evaluated together: one sort and one persistent sweep
    launch over all of them (engine_batch_*).  The engines need no device state of their
    own (Engine.from_system(..., start=False)) and must stay open while the batch is."""

    def __init__(self, engines, device: Optional[int] = None):
        self.lib = lib()
        self.engines = list(engines)
        self.closed = True
        if device is not None:
            for e in self.engines:
                _check(self.lib.engine_cuda_setdevice(e.ptr, device), "engine_cuda_setdevice")
        self._arr = (C.c_void_p * len(self.engines))(*[e.ptr.value for e in self.engines])
        h = C.c_void_p()
        _check(self.lib.engine_batch_create(self._arr, len(self.engines), C.byref(h)), "engine_batch_create")
        self.ptr = h
        self.closed = False

    def _zero(self):
        _check(self.lib.engine_batch_zero_forces(self.ptr), "engine_batch_zero_forces")

    def nonbond(self):
        """One force evaluation of every engine (host buffers in and out)."""
        _check(self.lib.engine_batch_nonbond_fresh(self.ptr), "engine_batch_nonbond_fresh")
        return self

    def step(self):
        _check(self.lib.engine_batch_step(self.ptr), "engine_batch_step")
        return self

    def sched_order(self, tile: int = 0):
        """Count-product costs in locality tiles (engine_batch_sched_order; 0: automatic)."""
        _check(self.lib.engine_batch_sched_order(self.ptr, tile), "engine_batch_sched_order")
        return self

    def set_groups(self, groups: int):
        """Groups of engines engine_batch_step pipelines (0: automatic)."""
        _check(self.lib.engine_batch_setgroups(self.ptr, groups), "engine_batch_setgroups")
        return self

    def step_host(self):
        _check(self.lib.engine_batch_step_host(self.ptr), "engine_batch_step_host")
        return self

    def resident_begin(self, margin: int = -1):
        _check(self.lib.engine_batch_resident_begin(self.ptr, margin), "engine_batch_resident_begin")
        return self

    def resident_steps(self, nsteps: int = 1):
        _check(self.lib.engine_batch_resident_steps(self.ptr, nsteps), "engine_batch_resident_steps")
        return self

    def resident_sync(self):
        _check(self.lib.engine_batch_resident_sync(self.ptr), "engine_batch_resident_sync")
        return self

    def resident_end(self):
        _check(self.lib.engine_batch_resident_end(self.ptr), "engine_batch_resident_end")
        return self

    def resident_info(self):
        return _resident_info(self.lib.engine_batch_resident_info, self.ptr)

    def load_parts(self):
        _check(self.lib.engine_batch_load_parts(self.ptr), "engine_batch_load_parts")

    def resident(self):
        _check(self.lib.engine_batch_resident(self.ptr), "engine_batch_resident")

    def unload_parts(self):
        self._zero()
        _check(self.lib.engine_batch_unload_parts(self.ptr), "engine_batch_unload_parts")

    def stats(self) -> NbStats:
        s = NbStats()
        _check(self.lib.engine_batch_stats(self.ptr, C.byref(s)), "engine_batch_stats")
        return s

    def set_stream(self, stream_ptr: int):
        _check(self.lib.engine_batch_setstream(self.ptr, C.c_void_p(stream_ptr)), "engine_batch_setstream")

    def kernel_times(self):
        a, b = C.c_float(), C.c_float()
        _check(self.lib.engine_batch_kernel_times(self.ptr, C.byref(a), C.byref(b)), "engine_batch_kernel_times")
        return a.value, b.value

    def tune(self, warps: int = 0, plain: bool = False):
        _check(self.lib.engine_batch_settune(self.ptr, warps, 1 if plain else 0), "engine_batch_settune")

    def graph(self, enable: bool = True):
        _check(self.lib.engine_batch_graph(self.ptr, int(enable)), "engine_batch_graph")

    def set_layout(self, layout: int, stages: int = 1, occupancy: int = 640):
        _check(self.lib.engine_batch_setlayout(self.ptr, layout, stages, occupancy), "engine_batch_setlayout")

    def autotune(self, reps: int = 5):
        """Keeps the fastest persistent launch shape; returns (warps, layout, stages,
        occupancy, ms)."""
        w, lay, stg, occ, ms = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_float()
        _check(self.lib.engine_batch_autotune(self.ptr, reps, C.byref(w), C.byref(lay), C.byref(stg), C.byref(occ),
                                              C.byref(ms)), "engine_batch_autotune")
        return w.value, lay.value, stg.value, occ.value, ms.value

    def ntasks(self) -> int:
        return _check(self.lib.engine_batch_ntasks(self.ptr), "engine_batch_ntasks")

    def close(self):
        if not self.closed:
            self.lib.engine_batch_free(self.ptr)
            self.closed = True

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
