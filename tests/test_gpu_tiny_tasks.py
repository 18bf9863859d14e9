"""GPU tests of the persistent sweeps' tiny-task path: in systems of fewer than 8 particles
per cell on average, the kernels of 1024 threads per SM evaluate a task of at most 32
candidate pairs (a self task of at most 8 particles, a pair task with n_i n_j <= 32) one pair
per lane without staging or sort keys, beside the staged sorted sweep of the larger tasks.
Systems with both kinds -- dilute rigid water (exclusions, type tables in shared memory), a
liquid slab in its vapour (two types), dilute argon (one table), dilute solvated chains
(global tables, per-particle charges, exclusions) -- against the FP64 oracle for both lane
layouts and both staging depths; the full-size slab; forces independent of the queue order;
resident steps equal to engine_step."""
import numpy as np
import pytest

import mdcore_b200 as M
import oracle as O
import workloads as W
from helpers import force_errors, tables_of

pytestmark = pytest.mark.gpu

HALF_SHELL = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1),
              (0, 1, 1), (0, 1, -1), (1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1)]


def systems():
    return {
        "water": W.water_spce(nside=8, density=1.0, seed=3),
        "slab": W.lj_slab(nx=22, nz=11, n_total=22 * 22 * 11 + 1000, box=(8.0, 8.0, 24.0), slab=4.0, seed=4),
        "argon": W.argon_fcc(6, density=2.0, jitter=0.2, seed=5),
        "chains": W.chains_water(nchains=4, length=20, nwater=150, box=(6.0, 6.0, 6.0), seed=2,
                                 angles_dihedrals=False),
    }


def task_kinds(sysm):
    """(tiny, staged) live task counts of the periodic cell grid (cells of at least 3 per side)."""
    b = O.bin_system(sysm)
    cdim = b["cdim"]
    cnt = np.bincount(b["cell"], minlength=int(np.prod(cdim))).reshape(cdim)
    tiny = int(((cnt >= 2) & (cnt <= 8)).sum())
    staged = int((cnt > 8).sum())
    for d in HALF_SHELL:
        nj = np.roll(cnt, tuple(-np.array(d)), axis=(0, 1, 2))
        live = (cnt > 0) & (nj > 0)
        tiny += int((live & (cnt * nj <= 32)).sum())
        staged += int((live & (cnt * nj > 32)).sum())
    return tiny, staged


_ORACLE = {}


def oracle_of(name, sysm):
    if name not in _ORACLE:
        _ORACLE[name] = O.nonbond(sysm, tables_of(sysm))
    return _ORACLE[name]


@pytest.mark.parametrize("stages", [1, 2])
@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("name", ["water", "slab", "argon", "chains"])
def test_tiny_and_staged_tasks_vs_oracle(name, layout, stages):
    sysm = systems()[name]
    tiny, staged = task_kinds(sysm)
    assert tiny > 0 and (staged > 0 or name == "argon"), (tiny, staged)
    o = oracle_of(name, sysm)
    e = M.Engine.from_system(sysm)
    e.set_layout(layout, stages, 1024)             # the shapes that carry the tiny path
    e.nonbond()
    f, st = e.forces(), e.stats()
    err = force_errors(f, o["f"])
    print(name, layout, stages, "tiny", tiny, "staged", staged, "pairs", st.pairs, err)
    assert st.status == 0
    assert st.pairs == o["pairs"] and st.excluded == o["excluded"], (st.pairs, o["pairs"], st.excluded, o["excluded"])
    assert abs(st.epot - o["epot"]) <= 1e-6 * o["epot_abs"], (st.epot, o["epot"])
    assert abs(st.virial - o["virial"]) <= 1e-6 * o["virial_abs"], (st.virial, o["virial"])
    assert err["global_rel"] <= 2e-6, err
    assert err["max_over_frms"] <= 2e-5, err
    e.close()


@pytest.mark.parametrize("layout", [0, 1])
def test_tiny_tasks_independent_of_task_order(layout):
    """Fixed point: any queue order gives bit-identical forces, energy and virial."""
    sysm = systems()["slab"]
    e = M.Engine.from_system(sysm)
    e.set_layout(layout, 1, 1024)
    e.nonbond()
    f1, s1 = e.forces(), e.stats()
    rng = np.random.default_rng(11)
    for _ in range(3):
        e.set_order(rng.permutation(e.ntasks()))
        e.nonbond()
        f2, s2 = e.forces(), e.stats()
        assert np.array_equal(f1, f2)
        assert s1.epot == s2.epot and s1.virial == s2.virial and s1.pairs == s2.pairs
    e.close()


def test_tiny_tasks_resident_steps_equal_engine_step():
    """Ten MD steps of the slab in its vapour at 90 K: device-resident steps and engine_step
    give the same positions and energy bit for bit."""
    sysm = systems()["slab"]
    sysm.v = W.maxwell_velocities(sysm, 90.0, seed=6)
    out = []
    for resident in (False, True):
        e = M.Engine.from_system(sysm)
        if resident:
            e.graph(True)
            e.resident_begin().resident_steps(10).resident_end()
        else:
            for _ in range(10):
                e.step()
        x, t, pid, epot = e.unload()
        pos = np.zeros((sysm.n, 3))
        pos[pid] = x
        out.append((pos, epot))
        e.close()
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]


@pytest.mark.parametrize("layout", [0, 1])
def test_full_size_slab_with_tiny_path_vs_oracle(layout):
    """The 1,048,576-atom slab (4.1 particles per cell: the tiny path is on) with the
    1024-thread shapes that carry it, two staging buffers: counts bit-exact, energy, virial
    and forces as the oracle's."""
    sysm = W.lj_slab()
    o = oracle_of("slab-1048576", sysm)
    e = M.Engine.from_system(sysm)
    e.set_layout(layout, 2, 1024)
    e.nonbond()
    f, st = e.forces(), e.stats()
    err = force_errors(f, o["f"])
    print("slab-1048576", layout, "pairs", st.pairs, err)
    assert st.status == 0
    assert st.pairs == o["pairs"] and st.excluded == o["excluded"]
    assert abs(st.epot - o["epot"]) <= 1e-6 * abs(o["epot"])
    assert abs(st.virial - o["virial"]) <= 1e-6 * o["virial_abs"]
    assert err["global_rel"] <= 2e-6, err
    assert err["max_over_frms"] <= 2e-5, err
    e.close()
