"""GPU tests of the Verlet skin of the resident steps (engine_flag_verlet, implied by
engine_flag_verlet_pseudo): between rebuilds particles stay in their cells and the sort keys
of the last rebuild are reused with the projection bound widened by the cells'
displacements (src/engine.c:193-315, src/runner_dopair.c:583).  Over a 50-step trajectory
every step's accepted and excluded pair counts equal the FP64 oracle's on the same
particles, energies and forces stay within FP32 rounding of it, and fewer than one step in
two re-bins and sorts."""
import numpy as np
import pytest

import mdcore_b200 as M
import oracle as O
import workloads as W
from helpers import force_errors, tables_of

pytestmark = pytest.mark.gpu

VERLET = M.engine_flag_cuda | M.engine_flag_verlet_pseudo


def systems():
    argon = W.argon_fcc(8, seed=3)
    argon.v = W.maxwell_velocities(argon, 100.0, seed=3)
    water = W.with_rigid_water(W.water_spce(12), 300.0, seed=5)
    return {"argon": argon, "water": water}


@pytest.mark.parametrize("name", ["argon", "water"])
@pytest.mark.parametrize("layout", [0, 1, "plain"])
def test_skin_steps_match_the_oracle(name, layout):
    sysm = systems()[name]
    tables = tables_of(sysm)
    e = M.Engine.from_system(sysm, flags=VERLET)
    if layout == "plain":
        e.tune(0, plain=True)
    else:
        e.set_layout(layout)
    e.graph(True)
    e.resident_begin()
    cdim = np.floor(np.asarray(sysm.dim) / np.asarray(sysm.L)).astype(np.int32)
    h = np.asarray(sysm.dim) / cdim
    nsteps = 50
    for t in range(nsteps):
        e.resident_sync()
        x, _, _, c = e.parts()
        o = O.nonbond(sysm, tables, binned=dict(cdim=cdim, h=h, cell=c, xrel=x))
        p0 = e.resident_info().pairs
        e.resident_steps(1)
        assert e.resident_info().pairs - p0 == o["pairs"], (t, e.resident_info().pairs - p0, o["pairs"])
        if t % 10 == 9:
            e.resident_sync()
            st = e.stats()
            assert st.status == 0 and st.excluded == o["excluded"]
            assert abs(st.epot - o["epot"]) <= 1e-6 * o["epot_abs"], (st.epot, o["epot"])
            err = force_errors(e.forces(), o["f"])       # the step's forces before the constraints
            assert err["global_rel"] <= 2e-6 and err["max_over_frms"] <= 2e-5, err
    rebuilds = e.verlet_rebuilds()
    assert 1 <= rebuilds < nsteps // 2, rebuilds
    e.resident_end()
    e.close()


def test_skin_follows_the_sorted_every_step_trajectory():
    """The same 40 steps with and without the skin: the sort keys and the sweep's summation
    order differ, the trajectories only by FP32 rounding."""
    sysm = systems()["argon"]
    out = {}
    for flags in (M.engine_flag_cuda, VERLET):
        e = M.Engine.from_system(sysm, flags=flags)
        e.graph(True)
        e.energy_log(64)
        e.resident_begin()
        e.resident_steps(40)
        out[flags] = e.energy_log_read(64)
        e.resident_end()
        e.close()
    a, b = out[M.engine_flag_cuda], out[VERLET]
    assert np.array_equal(a[:, 0], b[:, 0])
    assert np.abs(a[:, 1] - b[:, 1]).max() <= 1e-5 * np.abs(a[:, 1]).max()
    assert np.abs(a[:, 2] - b[:, 2]).max() <= 1e-5 * np.abs(a[:, 2]).max()
