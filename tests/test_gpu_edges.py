"""GPU edge cases of the sweep against the oracle: empty and single-particle systems, pairs at
exactly the cutoff distance, a cell at the largest supported size, a cell beyond it
(refused before any launch), exclusions between far-apart ids (the list path rather than
the id-window bit mask) and a box with no pair inside the cutoff."""
import numpy as np
import pytest

import mdcore_b200 as M
import oracle as O
import workloads as W
from helpers import force_errors, load_golden

pytestmark = pytest.mark.gpu


def lj_system(x, L=3.0, scale=1.0, name="edge", excl=None):
    A, B = W.lj_AB(0.996, 0.3405)
    x = np.asarray(x, np.float64).reshape(-1, 3)
    return W.System(name=name, origin=np.zeros(3), dim=np.full(3, L), L=np.full(3, 1.0), cutoff=1.0,
                    masses=[39.948], charges=[0.0],
                    pots=[W.PotSpec(W.KIND_LJ126, 0, 0, 0.25, 1.0, 1e-4, (A * scale, B * scale, 0.0, 0.0))],
                    x=x, type=np.zeros(len(x), np.int32),
                    excl=np.zeros((0, 2), np.int32) if excl is None else np.asarray(excl, np.int32), dt=0.005)


def run(sysm, layout=1):
    e = M.Engine.from_system(sysm)
    e.set_layout(layout)
    e.nonbond()
    return e, e.forces(), e.stats()


def oracle_of(sysm):
    tables = [M.create_potential(p).contents.table() for p in sysm.pots]
    return O.nonbond(sysm, tables)


@pytest.mark.parametrize("n", [0, 1])
def test_empty_and_single_particle(n):
    sysm = lj_system(np.full((n, 3), 0.5))
    e, f, st = run(sysm)
    assert st.status == 0 and st.pairs == 0 and st.excluded == 0 and st.epot == 0.0
    assert f.shape == (n, 3) and not f.any()
    e.close()


def test_dilute_box_without_pairs():
    """Particles farther apart than the cutoff in every direction: candidates, no pairs."""
    g = np.stack(np.meshgrid(np.arange(3), np.arange(3), np.arange(3), indexing="ij"), -1).reshape(-1, 3)
    sysm = lj_system((g + 0.5) * 1.1, L=3.3)
    e, f, st = run(sysm)
    assert st.status == 0 and st.pairs == 0 and st.epot == 0.0 and not f.any()
    e.close()


@pytest.mark.parametrize("layout", [0, 1])
def test_pairs_at_exactly_the_cutoff(layout):
    """r^2 == cutoff^2 in float is inside (the reference tests r2 <= rc^2); the next float
    distance outside.  Counts as the oracle's, per axis and across a cell face."""
    xs, expect_in = [], 0
    for k, axis in enumerate((0, 1, 2)):
        a = np.array([0.5, 0.5, 0.5]) + 0.001 * k
        b = a.copy()
        b[axis] += 1.0                                        # exactly 1.0 apart, next cell
        c = a.copy()
        c[(axis + 1) % 3] += 1.5                              # far from a and b
        d = c.copy()
        d[axis] += np.nextafter(np.float32(1.0), np.float32(2.0))   # just beyond the cutoff
        xs += [a, b, c, d]
    sysm = lj_system(np.array(xs), L=3.0, scale=1e-3)
    e, f, st = run(sysm, layout)
    o = oracle_of(sysm)
    assert st.status == 0
    assert st.pairs == o["pairs"]
    err = force_errors(f, o["f"])
    assert err["global_rel"] <= 2e-6, err
    e.close()


def test_largest_cell():
    """A cell of 1,000 particles (the limit is 1,024) next to sparse cells: two worker warps
    per block fit its shared-memory slices; results as the oracle's."""
    rng = np.random.default_rng(3)
    dense = rng.uniform(0.0, 1.0, size=(1000, 3))
    sparse = rng.uniform(0.0, 3.0, size=(200, 3))
    sparse = sparse[(sparse >= 1.0).any(axis=1)]
    sysm = lj_system(np.concatenate([dense, sparse]), L=3.0, scale=1e-4)
    e, f, st = run(sysm)
    o = oracle_of(sysm)
    assert st.status == 0 and st.pairs == o["pairs"]
    assert abs(st.epot - o["epot"]) <= 1e-6 * o["epot_abs"]
    err = force_errors(f, o["f"])
    assert err["global_rel"] <= 2e-6, err
    e.close()


def test_oversized_cell_is_refused():
    """More than 1,024 particles in one cell: engine_err_maxparts from the host, no launch."""
    rng = np.random.default_rng(4)
    sysm = lj_system(rng.uniform(0.0, 1.0, size=(1100, 3)), L=3.0, scale=1e-4)
    e = M.Engine.from_system(sysm)
    with pytest.raises(M.MdcoreError, match="-24"):
        e.nonbond()
    M.lib().errs_clear()
    # the engine stays usable once the particles are spread out
    x = rng.uniform(0.0, 3.0, size=(1100, 3))
    e.close()
    e = M.Engine.from_system(lj_system(x, L=3.0, scale=1e-4))
    e.nonbond()
    assert e.stats().status == 0
    e.close()


def test_far_exclusions_use_the_list():
    """Exclusions between ids more than 16 apart (list path) and within 16 (bit mask), mixed:
    excluded counts and forces as the oracle's."""
    base, _ = load_golden("argon_1372.npz")
    rng = np.random.default_rng(5)
    # partners within the cutoff, chosen from the oracle's own cell binning
    b = O.bin_system(base)
    pos = base.x
    pairs = []
    while len(pairs) < 300:
        i, j = rng.integers(0, base.n, size=2)
        if i == j:
            continue
        d = pos[i] - pos[j]
        d -= np.round(d / base.dim) * base.dim
        if (d ** 2).sum() < 0.8 and (len(pairs) % 2 == 0) == (abs(int(i) - int(j)) > 16):
            pairs.append((int(i), int(j)))
    sysm = W.System(**{**base.__dict__, "excl": np.array(pairs, np.int32), "name": "argon-far-excl"})
    e, f, st = run(sysm)
    o = oracle_of(sysm)
    assert st.status == 0
    assert st.excluded == o["excluded"] and st.pairs == o["pairs"]
    assert abs(st.epot - o["epot"]) <= 1e-6 * abs(o["epot"])
    err = force_errors(f, o["f"])
    assert err["global_rel"] <= 2e-6, err
    e.close()
