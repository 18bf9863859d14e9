"""The topology and parameter readers (engine_read_psf, engine_read_cpf, engine_read_xplor)
against the reference's, on the synthetic CHARMM-style system of tests/golden/topo
(make_topology.py): tests/drivers/topo_driver.c, compiled unchanged against
libmdcore_b200, must print what the same driver printed against the reference library --
the same types (name, charge, mass, epsilon, Rmin), bonds, rigid constraints, angle and
dihedral potential assignments, bit-identical bonded and pair tables, and particles -- for
CHARMM and XPLOR files with Ewald, plain LJ and shifted-Coulomb pair forms.  On the GPU the
energies of two engine_step calls (exclusions as the reference's JAC example adds them)
follow the reference's."""
import gzip
import importlib.util
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOPO = os.path.join(ROOT, "tests", "golden", "topo")
LIBDIR = os.path.join(ROOT, "mdcore-history_b200")

_spec = importlib.util.spec_from_file_location("make_topology", os.path.join(ROOT, "tests", "golden",
                                                                          "make_topology.py"))
MT = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(MT)


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("topo") / "topo_driver")
    cmd = ["gcc", "-std=gnu99", "-O2", "-Wall", "-Werror", "-DENGINE_FLAGS=engine_flag_cuda",
           os.path.join(ROOT, "tests", "drivers", "topo_driver.c"), "-I", os.path.join(ROOT, "include"),
           "-L", LIBDIR, "-lmdcore_b200", f"-Wl,-rpath,{LIBDIR}", "-lm", "-lpthread", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def run(driver, case, steps):
    name, par, fmt, kappa, tol, rigid, sw, _, dt = case
    args = [driver, os.path.join(TOPO, "small.psf"), os.path.join(TOPO, "small.pdb"), os.path.join(TOPO, par),
            fmt, repr(kappa), repr(tol), str(rigid), repr(sw), repr(MT.BOX_NM), repr(MT.CUTOFF), str(steps),
            repr(dt)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return [l for l in r.stdout.splitlines() if l.split(" ", 1)[0] in MT.TAGS]


def reference(case):
    with gzip.open(os.path.join(TOPO, f"ref_{case[0]}.txt.gz"), "rt") as f:
        return f.read().splitlines()


@pytest.mark.parametrize("case", MT.CASES, ids=[c[0] for c in MT.CASES])
def test_reader_builds_what_the_reference_builds(case, driver):
    ours = run(driver, case, 0)
    ref = [l for l in reference(case) if not l.startswith(("energy", "exclusions"))]
    assert len(ours) == len(ref), (len(ours), len(ref))
    bad = [(a, b) for a, b in zip(ours, ref) if a != b]
    assert not bad, bad[:5]
    kinds = {l.split(" ", 1)[0] for l in ours}
    assert {"type", "bond", "angle", "dihedral", "pair", "part"} <= kinds
    if case[5]:
        assert any(l.startswith("constraint") for l in ours)


def test_reader_rejects_a_file_that_is_not_a_psf(tmp_path):
    import ctypes as C
    import mdcore_b200 as M
    bad = tmp_path / "bad.psf"
    bad.write_text("NOT A PSF\n")
    lib = M.lib()
    lib.engine_read_psf.restype = C.c_int
    lib.engine_read_psf.argtypes = [C.c_void_p, C.c_int, C.c_int]
    e = M.Engine([0.0, 0.0, 0.0], [3.0, 3.0, 3.0], [1.0, 1.0, 1.0], 0.9, max_type=10)
    fd = os.open(str(bad), os.O_RDONLY)
    fd2 = os.open(os.path.join(TOPO, "small.pdb"), os.O_RDONLY)
    try:
        assert lib.engine_read_psf(e.ptr, fd, fd2) == -14            # engine_err_psf
    finally:
        os.close(fd)
        os.close(fd2)
        lib.errs_clear()
        e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", [c for c in MT.CASES if c[7] > 0], ids=[c[0] for c in MT.CASES if c[7] > 0])
def test_engine_steps_of_a_read_system_follow_the_reference(case, driver):
    ours = run(driver, case, case[7])
    ref = reference(case)
    ex = [l for l in ours if l.startswith("exclusions")]
    assert ex and ex == [l for l in ref if l.startswith("exclusions")]
    eo = [float(l.split()[3]) for l in ours if l.startswith("energy")]
    er = [float(l.split()[3]) for l in ref if l.startswith("energy")]
    assert len(eo) == len(er) == case[7]
    for a, b in zip(eo, er):
        assert abs(a - b) <= 1e-5 * abs(b), (eo, er)
