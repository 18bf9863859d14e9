"""Explicit electrostatics in the oracle, on the CPU (no GPU).

The reference stores the explicit electrostatic potential (engine_setexplepot) but never
evaluates it, so there is no reference output to pin against.  The oracle's restatement is
checked against the reference's own way of expressing the same physics: SPC/E water with
the charges baked into per-type-pair tables (O-O LJ + Coulomb, O-H and H-H Coulomb) must
give the same pair counts, energy and forces as LJ-only type tables plus q_i q_j times one
unit-charge Coulomb table, up to the fit error of the tables: the two forms interpolate
different functions (LJ + q_O^2 Coulomb in one table against LJ and Coulomb apart, and a
Coulomb table built for charge q is not q times the unit-charge one), whose forces differ by
up to ~1e-4 per pair near the cutoff at tolerance 1e-5.  A wrong charge, sign or pair set
would show as errors of order one."""
import dataclasses

import numpy as np

import oracle as O
import workloads as W
from helpers import force_errors, tables_of


def explicit_form(sysm):
    """The same water with LJ type tables and explicit per-particle charges."""
    A, B = W.lj_AB(0.650, 0.3166)
    qO, qH = -0.8476, 0.4238
    lj = [W.PotSpec(W.KIND_LJ126, 0, 0, sysm.pots[0].a, sysm.cutoff, sysm.pots[0].tol, (A, B, 0.0, 0.0))]
    q = np.where(sysm.type == 0, qO, qH) * W.QSCALE
    coul = sysm.pots[1]
    ep = W.PotSpec(W.KIND_COULOMB, 0, 0, coul.a, sysm.cutoff, coul.tol, (1.0, 0.0, 0.0, 0.0))
    return dataclasses.replace(sysm, pots=lj, q=q, ep=ep, name=sysm.name + "-explicit")


def test_explicit_charges_equal_baked_tables():
    base = W.water_spce(6, seed=3)
    base = dataclasses.replace(base, pots=[dataclasses.replace(p, tol=1e-5) for p in base.pots])
    ob = O.nonbond(base, tables_of(base))
    ex = explicit_form(base)
    oe = O.nonbond(ex, tables_of(ex))
    assert oe["pairs"] == ob["pairs"] and oe["excluded"] == ob["excluded"]
    assert abs(oe["epot"] - ob["epot"]) <= 1e-5 * ob["epot_abs"]
    err = force_errors(oe["f"], ob["f"])
    assert err["global_rel"] <= 1e-3, err      # the table fits, summed with cancellation


def test_pairs_without_type_potential_interact_through_charges():
    """H-H and O-H have no type table in the explicit form: the pair set is still every
    non-excluded pair within the cutoff."""
    base = W.water_spce(5, seed=4)
    ex = explicit_form(base)
    counting = O.nonbond(dataclasses.replace(base, ep=None, q=None), tables_of(base))
    oe = O.nonbond(ex, tables_of(ex))
    assert oe["pairs"] == counting["pairs"]


def test_chain_system_shape():
    s = W.chains_water(nchains=4, length=20, nwater=300, box=(3.6, 3.6, 3.6), seed=2)
    assert s.n == 80 + 900
    assert len(s.pots) == 22 * 23 // 2 and s.ep is not None
    q = s.q[900:].reshape(4, 20)
    assert np.allclose(q.sum(1), 0.0, atol=1e-9)                 # neutral chains
    assert len(s.excl) == 3 * 300 + 4 * (19 + 18)
    o = O.nonbond(s, tables_of(s))
    assert o["pairs"] > 0 and o["excluded"] > 0 and np.isfinite(o["epot"])
