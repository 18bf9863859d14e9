"""The drop-in boundary from C, at compile and link time: the reference's own example
drivers for the systems this library runs (examples/argon/argon.c, the LJ argon box;
examples/bulk/bulk.c, rigid SPC/E water; examples/neon/neon.c) compile unchanged against
include/ (mdcore.h, cycle.h) and link against libmdcore_b200.so -- every engine field they
touch (e.s.cells[].parts[], e.s.cid_real, e.s.nr_swaps, e.timers[engine_timer_*], e.time,
e.dt, ...) and every function they call exists with the reference's types.  The drivers are
read from the reference checkout at test time (skipped where it is absent); running them
needs a GPU (tests/test_gpu_cdriver.py runs a driver of the same shape)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_root():
    import importlib.util
    spec = importlib.util.spec_from_file_location("graft_entry", os.path.join(ROOT, "__graft_entry__.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.REFERENCE


@pytest.mark.parametrize("name", ["argon", "bulk", "neon"])
def test_reference_example_compiles_and_links(name, tmp_path):
    src = os.path.join(reference_root(), "examples", name, name + ".c")
    if not os.path.exists(src):
        pytest.skip("reference checkout not present")
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    # the drivers include "../config.h" (the autotools configuration): an empty one
    work = tmp_path / "ex"
    work.mkdir()
    (tmp_path / "config.h").write_text("")
    shutil.copy(src, work / (name + ".c"))
    libdir = os.path.join(ROOT, "mdcore-history_b200")
    r = subprocess.run(["gcc", "-std=gnu99", "-O1", "-w", "-D_GNU_SOURCE", "-fopenmp", "-I" + os.path.join(ROOT, "include"),
                        name + ".c", "-L" + libdir, "-lmdcore_b200", "-lm", "-lpthread", "-o", name],
                       cwd=work, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    assert (work / name).exists()
