"""CPU tests: the oracle and the product's host code against the reference's golden outputs.

The fixtures in tests/golden were produced by the reference mdcore library itself
(tests/golden/make_golden.py); these tests need no GPU.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from helpers import force_errors, load_golden, sort_cells_of

SYSTEMS = ["argon_1372.npz", "water_3000.npz"]


@pytest.mark.parametrize("fname", SYSTEMS)
def test_oracle_binning_matches_reference(fname):
    """Cell index and cell-local float position of every particle, bit for bit."""
    sysm, ref = load_golden(fname)
    b = O.bin_system(sysm)
    assert np.array_equal(b["cell"], ref["cell"])
    assert np.array_equal(b["xrel"].view(np.uint32), ref["xrel"].astype(np.float32).view(np.uint32))


@pytest.mark.parametrize("fname", SYSTEMS)
def test_oracle_pair_and_exclusion_counts_match_reference(fname):
    """The oracle's pair set is the reference sweep's, counted with counter tables."""
    sysm, ref = load_golden(fname)
    r = O.nonbond(sysm, ref["tables"])
    assert r["excluded"] == int(ref["excl_in_cut"])
    assert r["pairs"] + r["excluded"] == int(ref["pairs_swept"])


@pytest.mark.parametrize("fname,etol,gtol,atol", [
    # argon: the reference FP32 sum agrees with the FP64 oracle to 5e-10 in energy.
    ("argon_1372.npz", 1e-8, 3e-6, 2e-5),
    # water: the reference sweeps the excluded O-H/H-H pairs (|e| ~ 770 kJ/mol each summed)
    # and subtracts them again in FP32, so its own energy carries ~1e-5 relative error.
    ("water_3000.npz", 2e-5, 1e-5, 1e-4),
])
def test_oracle_energy_and_forces_match_reference(fname, etol, gtol, atol):
    sysm, ref = load_golden(fname)
    r = O.nonbond(sysm, ref["tables"])
    assert abs(r["epot"] - float(ref["epot"])) <= etol * abs(float(ref["epot"]))
    err = force_errors(ref["f"], r["f"])
    assert err["global_rel"] <= gtol, err
    assert err["max_over_frms"] <= atol, err


@pytest.mark.parametrize("fname", SYSTEMS)
def test_oracle_sort_keys_match_reference(fname):
    """Projected-distance keys of every needed sort direction: same distances in the same
    order, same set of (index, distance) keys (ties may be ordered differently: the
    reference quicksort is not stable)."""
    sysm, ref = load_golden(fname)
    b = O.bin_system(sysm)
    checked = 0
    for cid, mask, ids, keys in sort_cells_of(ref):
        xr = b["xrel"][ids]
        for sid in range(13):
            if not (mask >> sid) & 1:
                continue
            k = O.sortkeys(xr, b["h"], sid)
            assert np.array_equal(k & 0xffff, keys[sid] & 0xffff)
            assert np.array_equal(np.sort(k), np.sort(keys[sid]))
            checked += 1
    assert checked > 0


def test_oracle_pshake_matches_reference_bit_exact():
    """P-SHAKE (src/rigid.c:279-523): three evaluations of the oracle from the fixture's
    state reproduce the reference's positions, velocities, constraint forces and refined
    mixing matrices bit for bit."""
    from helpers import load_rigid_golden, rigid_oracle_steps
    sysm, z, groups = load_rigid_golden()
    b = O.bin_system(sysm)
    assert np.array_equal(b["cell"], z["cell"])
    res = rigid_oracle_steps(sysm, groups, b["xrel"], z["v"].astype(np.float32),
                             np.zeros((sysm.n, 3), np.float32), True, 3)
    assert res[0][4].max() > 5                          # the first evaluation iterates
    for k, (x, v, f, a, it) in enumerate(res):
        assert np.array_equal(x.view(np.uint32), z["px"][k].view(np.uint32)), k
        assert np.array_equal(v.view(np.uint32), z["pv"][k].view(np.uint32)), k
        assert np.array_equal(f.view(np.uint32), z["pf"][k].view(np.uint32)), k
        assert np.array_equal(a.view(np.uint32), z["pa"][k].view(np.uint32)), k


def test_oracle_shake_close_to_reference():
    """SHAKE (src/rigid.c:81-277): the oracle iterates in FP64, the reference's single
    build keeps the multiplier, gradients and tolerance in float; both converge to
    |d^2 - r^2| < 1e-6 and the positions agree to a float ulp, velocities to 1e-6 nm/ps."""
    from helpers import load_rigid_golden, rigid_oracle_steps
    sysm, z, groups = load_rigid_golden()
    b = O.bin_system(sysm)
    (x, v, f, a, it), = rigid_oracle_steps(sysm, groups, b["xrel"], z["v"].astype(np.float32),
                                           np.zeros((sysm.n, 3), np.float32), False, 1)
    assert it.max() > 5
    assert np.abs(x - z["sx"][0]).max() <= 1.2e-7
    assert np.abs(v - z["sv"][0]).max() <= 1e-6
    assert np.array_equal(f, z["sf"][0])                 # SHAKE leaves forces alone


def test_rigid_groups_match_reference():
    """engine_rigid_add (src/engine_rigid.c:78-229): the same groups, particle order and
    group-local constraint ends as the reference, identity mixing matrices."""
    import mdcore_b200 as M
    from helpers import load_rigid_golden
    sysm, z, groups = load_rigid_golden()
    e = M.Engine.from_system(sysm, start=False)
    ours = []
    n = M.lib().engine_rigid_get(e.ptr, 0, None)
    for g in range(n):
        r = M.Rigid()
        assert M.lib().engine_rigid_get(e.ptr, g, C.byref(r)) == n
        ours.append(r)
    assert len(ours) == len(groups)
    for r, (parts, con, a) in zip(ours, groups):
        assert list(r.parts[:r.nr_parts]) == parts
        assert r.constraints() == con
        assert np.array_equal(r.matrix(), a)
    e.close()


def test_rigid_add_merges_groups():
    """Two groups joined by a constraint become one group whose constraint ends index the
    merged particle list."""
    import mdcore_b200 as M
    import workloads as W
    s = W.argon_fcc(7)
    e = M.Engine.from_system(s, start=False)
    L = M.lib()
    for i, j in ((0, 1), (2, 3), (1, 2)):
        assert L.engine_rigid_add(e.ptr, i, j, 0.3) == 0
    n = L.engine_rigid_get(e.ptr, 0, None)
    assert n == 1
    r = M.Rigid()
    L.engine_rigid_get(e.ptr, 0, C.byref(r))
    parts = list(r.parts[:r.nr_parts])
    assert sorted(parts) == [0, 1, 2, 3]
    ends = {(parts[i], parts[j]) for i, j, _ in r.constraints()}
    assert ends == {(0, 1), (2, 3), (1, 2)}
    assert np.array_equal(r.matrix(), np.eye(3, dtype=np.float32))
    e.close()
