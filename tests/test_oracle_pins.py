"""CPU tests: the oracle and the product's host code against the reference's golden outputs.

The fixtures in tests/golden were produced by the reference mdcore library itself
(tests/golden/make_golden.py); these tests need no GPU.
"""
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
