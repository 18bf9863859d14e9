"""CPU tests of the product's host code (no GPU needed): the C library loads and exports
every function its header declares, builds bit-identical potential tables, bins particles
like the reference and refuses what it does not implement."""
import os
import re

import numpy as np
import pytest

import mdcore_b200 as M
import workloads as W
from helpers import GOLDEN, load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "mdcore_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "for", "while", "sizeof")))


def test_library_exports_every_declared_function():
    lib = M.lib()
    names = header_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_tables_bit_identical_to_reference():
    z = np.load(os.path.join(GOLDEN, "tables.npz"))
    for k in range(int(z["ncases"])):
        kind, a, b, tol, p0, p1, p2, p3 = z[f"case{k}"]
        spec = W.PotSpec(int(kind), 0, 0, a, b, tol, (p0, p1, p2, p3))
        n, alpha, c = M.create_potential(spec).contents.table()
        assert n == int(z[f"case{k}_n"]), (k, n)
        assert np.array_equal(alpha.view(np.uint32), z[f"case{k}_alpha"].view(np.uint32)), k
        assert np.array_equal(c.view(np.uint32), z[f"case{k}_c"].view(np.uint32)), k


@pytest.mark.parametrize("fname", ["argon_1372.npz", "water_3000.npz"])
def test_system_tables_bit_identical(fname):
    sysm, ref = load_golden(fname)
    for spec, (n, alpha, c) in zip(sysm.pots, ref["tables"]):
        n2, a2, c2 = M.create_potential(spec).contents.table()
        assert n2 == n
        assert np.array_equal(a2.view(np.uint32), alpha.view(np.uint32))
        assert np.array_equal(c2.view(np.uint32), c.view(np.uint32))


@pytest.mark.parametrize("fname", ["argon_1372.npz", "water_3000.npz"])
def test_engine_cell_assignment_matches_reference(fname):
    sysm, ref = load_golden(fname)
    e = M.Engine.from_system(sysm, start=False)
    assert np.array_equal(e.cells(), ref["cell"])
    x, t, pid, _ = e.unload()
    order = np.argsort(pid)
    assert np.array_equal(pid[order], np.arange(sysm.n))
    assert np.allclose(x[order], sysm.x, atol=1e-6)
    assert np.array_equal(t[order], sysm.type)
    e.close()


def test_space_getpos_and_prepare():
    """space_getpos (src/space.c:447-466): cell origin + relative position of a local id,
    the same doubles engine_unload returns; space_err_range past nr_parts.  space_prepare
    (src/space.c:186-219) zeroes the energies and forces."""
    import ctypes as C
    sysm, _ = load_golden("argon_1372.npz")
    e = M.Engine.from_system(sysm, start=False)
    lib = M.lib()
    lib.space_getpos.restype = C.c_int
    lib.space_getpos.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
    lib.space_prepare.restype = C.c_int
    lib.space_prepare.argtypes = [C.c_void_p]
    sp = e.ptr.value + 8                       # struct engine: unsigned flags, then struct space
    x, _, pid, _ = e.unload()
    out = (C.c_double * 3)()
    for row in range(0, sysm.n, 97):
        assert lib.space_getpos(sp, int(pid[row]), out) == 0
        assert list(out) == list(x[row])
    assert lib.space_getpos(sp, sysm.n, out) < 0
    M.lib().errs_clear()
    assert lib.space_prepare(sp) == 0
    assert not e.forces().any()
    assert e.energies()["total"] == 0.0
    e.close()


def test_engine_refuses_unimplemented_flags():
    with pytest.raises(M.MdcoreError):
        M.Engine(np.zeros(3), np.full(3, 4.0), np.ones(3), 1.0, flags=16384)   # engine_flag_dpd


def test_engine_refuses_too_few_cells():
    """A periodic box of fewer than 3 cells per dimension would pair cells twice."""
    with pytest.raises(M.MdcoreError):
        M.Engine(np.zeros(3), np.full(3, 2.5), np.ones(3), 1.0)


def test_potential_range_errors():
    lib = M.lib()
    # Too tight a tolerance cannot be met within 320 intervals.
    p = lib.potential_create_LJ126(0.1, 1.0, *W.lj_AB(0.996, 0.3405), 1e-13)
    assert not p
    lib.errs_clear()


def test_batch_refuses_engines_with_other_potentials():
    """A batch evaluates every replica with one set of tables: engines with other types or
    potentials are refused before any device call."""
    a, _ = load_golden("argon_1372.npz")
    w, _ = load_golden("water_3000.npz")
    ea, ew = M.Engine.from_system(a, start=False), M.Engine.from_system(w, start=False)
    with pytest.raises(M.MdcoreError, match="differ"):
        M.Batch([ea, ew])
    b = W.argon_fcc(7)
    b.pots = [W.PotSpec(p.kind, p.ti, p.tj, p.a, p.b, 1e-3, p.p) for p in b.pots]
    eb = M.Engine.from_system(b, start=False)
    with pytest.raises(M.MdcoreError, match="potentials"):
        M.Batch([ea, eb])
    M.lib().errs_clear()
    for e in (ea, ew, eb):
        e.close()


def test_replica_ensemble_shapes():
    systems = W.argon_replicas(nrep=64, seed=1)
    assert len(systems) == 64
    for s in systems:
        assert 500 <= s.n <= 8000
        assert (s.dim >= 3 * s.cutoff).all()
        assert (s.x >= 0).all() and (s.x < s.dim).all()
        assert len(np.unique(np.round(s.x / 1e-4))) > 0


@pytest.mark.parametrize("std", ["gnu99", "c11"])
def test_headers_compile_cleanly(std, tmp_path):
    """include/mdcore.h (and through it mdcore_b200.h and cycle.h) compiles in C with every
    warning an error, as a driver built with -Wall -Werror includes it."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    src = tmp_path / "inc.c"
    src.write_text('#include "mdcore.h"\nint main(void) { struct engine e; (void)e; return engine_timer_last > 0 ? 0 : 1; }\n')
    r = subprocess.run(["gcc", f"-std={std}", "-D_GNU_SOURCE", "-Wall", "-Wextra", "-Werror", "-c",
                        "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(tmp_path / "inc.o")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
