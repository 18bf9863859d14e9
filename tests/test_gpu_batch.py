"""GPU tests of replica batches (engine_batch_*): many independent engines evaluated by one
sort launch and one persistent sweep over their concatenated task lists.

Each replica's forces, energy and virial must equal those of the same engine evaluated
alone, bit for bit (fixed-point accumulation, and every task computes the same float
partials whichever engine list it belongs to), and match the oracle within the parity
tolerances of the single-engine tests; the batch's pair and exclusion counts are the sums
over the replicas.
"""
import numpy as np
import pytest

import mdcore_b200 as M
import oracle as O
import workloads as W
from helpers import force_errors, load_golden

pytestmark = pytest.mark.gpu


def engines_of(systems, start=False):
    return [M.Engine.from_system(s, start=start) for s in systems]


def check_replica_vs_oracle(sysm, tables, f, st, max_over_frms=2e-5):
    o = O.nonbond(sysm, tables)
    err = force_errors(f, o["f"])
    # A replica's net energy and virial can be small remainders of cancelling pair terms
    # (dilute or near-zero-pressure replicas): their FP32 rounding errors are bounded
    # against the sums of |e| and |r.F| over pairs.
    assert abs(st.epot - o["epot"]) <= 1e-6 * o["epot_abs"], (sysm.name, st.epot, o["epot"])
    assert abs(st.virial - o["virial"]) <= 1e-6 * o["virial_abs"], (sysm.name, st.virial, o["virial"])
    assert err["global_rel"] <= 2e-6, (sysm.name, err)
    assert err["max_over_frms"] <= max_over_frms, (sysm.name, err)
    return o


@pytest.mark.parametrize("plain", [False, True], ids=["tuned", "plain"])
def test_batch_equals_single_engines(plain):
    systems = W.argon_replicas(nrep=12, seed=3)
    tables = [M.create_potential(p).contents.table() for p in systems[0].pots]
    singles = []
    for s in systems:
        e = M.Engine.from_system(s)
        if plain:
            e.tune(0, True)
        e.nonbond()
        singles.append((e.forces(), e.stats()))
        e.close()
    engines = engines_of(systems)
    b = M.Batch(engines)
    if plain:
        b.tune(0, True)
    b.nonbond()
    bs = b.stats()
    assert bs.status == 0
    pairs = excluded = 0
    for s, e, (f1, s1) in zip(systems, engines, singles):
        f2, s2 = e.forces(), e.stats()
        assert np.array_equal(f1, f2), s.name
        assert s1.epot == s2.epot and s1.virial == s2.virial, s.name
        pairs += s1.pairs
        excluded += s1.excluded
        o = check_replica_vs_oracle(s, tables, f2, s2)
        assert o["pairs"] == s1.pairs
    assert bs.pairs == pairs and bs.excluded == excluded
    assert abs(bs.epot - sum(e.stats().epot for e in engines)) <= 1e-9 * abs(bs.epot)
    b.close()
    for e in engines:
        e.close()


def test_batch_of_water_and_exclusions():
    """Replicas with exclusions: particle ids of replica k are offset in the batch, so each
    replica's exclusions must still remove exactly its own pairs."""
    sysm, ref = load_golden("water_3000.npz")
    e1 = M.Engine.from_system(sysm)
    e1.nonbond()
    f1, s1 = e1.forces(), e1.stats()
    e1.close()
    engines = engines_of([sysm, sysm, sysm])
    b = M.Batch(engines)
    b.nonbond()
    bs = b.stats()
    assert bs.status == 0
    for e in engines:
        assert np.array_equal(e.forces(), f1)
        assert e.stats().epot == s1.epot
    assert bs.pairs == 3 * s1.pairs and bs.excluded == 3 * s1.excluded
    b.close()
    for e in engines:
        e.close()


def test_full_replica_ensemble_vs_oracle():
    """The 512-replica benchmark ensemble (1.45 M atoms): every replica against the oracle,
    batch pair count equal to the oracle's total.  The largest per-atom force error over
    1.45 M atoms is the far tail of the FP32 rounding distribution, bounded at 3e-5 F_rms
    (the reference's own FP32 forces reach 2e-5 F_rms against the oracle on 1,372 argon
    atoms)."""
    systems = W.argon_replicas()
    tables = [M.create_potential(p).contents.table() for p in systems[0].pots]
    engines = engines_of(systems)
    b = M.Batch(engines)
    b.nonbond()
    bs = b.stats()
    assert bs.status == 0
    pairs = 0
    for s, e in zip(systems, engines):
        o = check_replica_vs_oracle(s, tables, e.forces(), e.stats(), max_over_frms=3e-5)
        pairs += o["pairs"]
    assert bs.pairs == pairs
    b.close()
    for e in engines:
        e.close()


def test_batch_steps_equal_single_steps():
    """engine_batch_step: re-binning, one batch force evaluation, integration -- the same
    trajectories as engine_step on each engine alone."""
    systems = W.argon_replicas(nrep=6, seed=5)
    single = []
    for s in systems:
        e = M.Engine.from_system(s)
        for _ in range(5):
            e.step_host()
        single.append(e.unload())
        e.close()
    engines = engines_of(systems)
    b = M.Batch(engines)
    for _ in range(5):
        b.step()
        assert b.stats().status == 0
    for e, (x1, t1, p1, ep1) in zip(engines, single):
        x2, t2, p2, ep2 = e.unload()
        o1, o2 = np.argsort(p1), np.argsort(p2)
        assert np.array_equal(p1[o1], p2[o2])
        assert np.array_equal(x1[o1], x2[o2])
        assert ep1 == ep2
    b.close()
    for e in engines:
        e.close()


def test_batch_graph_and_autotune_keep_results():
    """The autotuned shape gives the oracle's results; CUDA-graph replays of it are
    bit-identical to direct launches of the same shape."""
    systems = W.argon_replicas(nrep=16, seed=7)
    tables = [M.create_potential(p).contents.table() for p in systems[0].pots]
    engines = engines_of(systems)
    b = M.Batch(engines)
    b.nonbond()
    warps, layout, stages, occ, ms = b.autotune(reps=2)
    assert warps in (2, 4, 8) and layout in (0, 1) and stages in (1, 2) and occ in (640, 768, 1024) and ms > 0
    b.nonbond()
    ref = [e.forces() for e in engines]
    e_ref = [e.stats().epot for e in engines]
    for s, e, f in zip(systems, engines, ref):
        check_replica_vs_oracle(s, tables, f, e.stats())
    b.graph(True)
    for _ in range(4):                 # direct, capture, replay, replay
        b.nonbond()
        assert b.stats().status == 0
        for e, f, ep in zip(engines, ref, e_ref):
            assert np.array_equal(e.forces(), f)
            assert e.stats().epot == ep
    b.close()
    for e in engines:
        e.close()


def _state(e):
    x, v, f, c = e.parts()                 # by particle id
    return x, v, f, c, e.energies()["total"]


@pytest.mark.parametrize("groups", [2, 3, 64])
def test_grouped_batch_steps_equal_one_group(groups):
    """engine_batch_step in groups of engines (own device blocks and stream per group,
    pipelined packing and unpacking): every engine's trajectory equals the one-group step
    bit for bit -- positions, velocities, forces, cells and energy -- over argon replicas
    and rigid-water replicas (P-SHAKE); more groups than engines means one per engine."""
    def systems():
        argon = W.argon_replicas(nrep=7, seed=11)
        water = [W.with_rigid_water(W.water_spce(10, seed=k), 300.0, seed=k) for k in range(2)]
        return argon, water

    out = {}
    for k in (1, groups):
        runs = []
        for sset in systems():
            engines = engines_of(sset)
            b = M.Batch(engines)
            b.set_groups(k)
            for _ in range(6):
                b.step()
                assert b.stats().status == 0
            runs.append(([_state(e) for e in engines], b.stats()))
            b.close()
            for e in engines:
                e.close()
        out[k] = runs
    for (s1, b1), (s2, b2) in zip(out[1], out[groups]):
        assert (b1.pairs, b1.excluded) == (b2.pairs, b2.excluded)
        assert b1.epot == b2.epot or abs(b1.epot - b2.epot) <= 1e-12 * abs(b1.epot)
        for a, b in zip(s1, s2):
            for u, w in zip(a[:4], b[:4]):
                assert np.array_equal(u, w)
            assert a[4] == b[4]


def test_grouped_steps_then_resident_steps():
    """A batch that stepped in groups still starts resident steps from the host cells, and
    while it holds resident particles its engine_batch_step runs as one group."""
    systems = W.argon_replicas(nrep=5, seed=13)
    ref_engines = engines_of(systems)
    ref = M.Batch(ref_engines)
    ref.set_groups(1)
    engines = engines_of(systems)
    b = M.Batch(engines)
    b.set_groups(3)
    for bb in (ref, b):
        for _ in range(3):
            bb.step()
        bb.resident_begin()
        bb.resident_steps(4)
        bb.resident_end()
        bb.step()
    for e1, e2 in zip(ref_engines, engines):
        for u, w in zip(_state(e1)[:4], _state(e2)[:4]):
            assert np.array_equal(u, w)
    for bb in (ref, b):
        bb.close()
    for e in ref_engines + engines:
        e.close()


def test_batch_sched_order_keeps_results():
    """engine_batch_sched_order (locality tiles of the count-product costs, any tile size)
    only reorders the queue: forces and energies bit-identical to the default order."""
    systems = W.argon_replicas(nrep=9, seed=17)
    engines = engines_of(systems)
    b = M.Batch(engines)
    b.nonbond()
    ref = [(e.forces().copy(), e.stats().epot) for e in engines]
    pairs = b.stats().pairs
    for tile in (1, 7, 0, 100000):
        b.sched_order(tile)
        b.nonbond()
        assert b.stats().status == 0 and b.stats().pairs == pairs
        for e, (f, ep) in zip(engines, ref):
            assert np.array_equal(e.forces(), f) and e.stats().epot == ep
    with pytest.raises(M.MdcoreError):
        b.sched_order(-1)
    b.close()
    for e in engines:
        e.close()


def test_full_ensemble_grouped_steps_equal_one_group():
    """The 512-replica ensemble (1,451,403 atoms): three engine_batch_step calls in the
    automatic grouping (4 groups) and in one group give every replica the same particles
    bit for bit, and the batch totals agree."""
    systems = W.argon_replicas()
    out = []
    for groups in (1, 0):
        engines = engines_of(systems)
        b = M.Batch(engines)
        b.set_groups(groups)
        for _ in range(3):
            b.step()
            assert b.stats().status == 0
        st = b.stats()
        out.append(([e.parts()[:3] for e in engines[::37]], (st.pairs, st.excluded, st.epot)))
        b.close()
        for e in engines:
            e.close()
    (p1, t1), (p2, t2) = out
    assert t1[0] == t2[0] and t1[1] == t2[1] and abs(t1[2] - t2[2]) <= 1e-12 * abs(t1[2])
    for a, b in zip(p1, p2):
        for u, w in zip(a, b):
            assert np.array_equal(u, w)
