"""The drop-in boundary from C: tests/drivers/md_driver.c, a driver written the way the
reference's examples are (engine API calls, space_addpart, velocity loops over
e.s.cells[].parts[], e.time, e.dt, e.s.epot), compiled unchanged with gcc against
include/mdcore.h and libmdcore_b200, runs 20 steps on the GPU; its energies follow the same
driver compiled against the reference's own headers and CPU library (oracle/_ref)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "tests", "drivers", "md_driver.c")
LIBDIR = os.path.join(ROOT, "mdcore-history_b200")
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "md_driver_ref")


def build_driver(out, flags="engine_flag_cuda"):
    """gcc on the unchanged driver source against include/ and libmdcore_b200.so."""
    cmd = ["gcc", "-std=gnu99", "-O2", "-Wall", "-Werror", f"-DENGINE_FLAGS={flags}", DRIVER,
           "-I", os.path.join(ROOT, "include"), "-L", LIBDIR, "-lmdcore_b200", f"-Wl,-rpath,{LIBDIR}",
           "-lm", "-lpthread", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def steps_of(stdout):
    rows = [l.split() for l in stdout.splitlines() if l.startswith("step ")]
    return np.array([[float(v) for v in r[1:5]] for r in rows])     # time, epot, ekin, temperature


def test_driver_compiles_and_links_against_the_library(tmp_path):
    exe = build_driver(str(tmp_path / "md_driver"))
    assert os.access(exe, os.X_OK)


@pytest.mark.gpu
def test_driver_runs_on_the_gpu_and_follows_the_reference(tmp_path):
    if not os.path.exists(REF_DRIVER):
        pytest.skip("reference CPU build (oracle/_ref) not present")
    exe = build_driver(str(tmp_path / "md_driver"))
    nsteps, nparts = 20, 32000
    ours = subprocess.run([exe, "1", str(nsteps), str(nparts)], capture_output=True, text=True, timeout=300,
                          cwd=str(tmp_path))
    assert ours.returncode == 0, ours.stdout[-2000:] + ours.stderr[-2000:]
    threads = str(min(16, os.cpu_count() or 1))
    ref = subprocess.run([REF_DRIVER, threads, str(nsteps), str(nparts)], capture_output=True, text=True,
                         timeout=600, cwd=str(tmp_path), env=dict(os.environ, OMP_NUM_THREADS=threads))
    assert ref.returncode == 0, ref.stdout[-2000:]
    a, b = steps_of(ours.stdout), steps_of(ref.stdout)
    assert a.shape == b.shape == (nsteps, 4)
    assert np.array_equal(a[:, 0], np.arange(1, nsteps + 1)) and np.array_equal(b[:, 0], a[:, 0])
    # FP32 pair forces in both, FP64 energy sums here: the same trajectory to FP32 rounding
    rel_e = np.abs(a[:, 1] - b[:, 1]) / np.abs(b[:, 1])
    rel_k = np.abs(a[:, 2] - b[:, 2]) / np.abs(b[:, 2])
    assert rel_e.max() <= 1e-5 and rel_k.max() <= 1e-5, (rel_e, rel_k)
