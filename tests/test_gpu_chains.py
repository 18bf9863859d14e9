"""GPU tests of the heterogeneous solvated-chain system (20 bead types + water, 253 type
tables read from global memory, explicit electrostatics q_i q_j ep(r) with per-particle
charges, 1-2/1-3 chain exclusions, rigid water): forces, energy, virial and counts against
the FP64 oracle, every launch shape, the plain form, and device steps against host steps."""
import dataclasses

import numpy as np
import pytest

import mdcore_b200 as M
import oracle as O
import workloads as W
from helpers import force_errors, tables_of

pytestmark = pytest.mark.gpu


def small():
    return W.chains_water(nchains=4, length=20, nwater=300, box=(3.6, 3.6, 3.6), seed=2)


def check(sysm, f, st, o, max_over_frms=2e-5):
    assert st.status == 0
    assert st.pairs == o["pairs"] and st.excluded == o["excluded"], (st.pairs, o["pairs"], st.excluded, o["excluded"])
    assert abs(st.epot - o["epot"]) <= 1e-6 * o["epot_abs"], (st.epot, o["epot"])
    assert abs(st.virial - o["virial"]) <= 1e-6 * o["virial_abs"], (st.virial, o["virial"])
    err = force_errors(f, o["f"])
    assert err["global_rel"] <= 2e-6, err
    assert err["max_over_frms"] <= max_over_frms, err


@pytest.mark.parametrize("shape", [(4, 1, 1, 640), (2, 0, 1, 640), (4, 1, 2, 1024), (8, 1, 1, 768), "plain"])
def test_small_chain_system_vs_oracle(shape):
    sysm = small()
    o = O.nonbond(sysm, tables_of(sysm))
    e = M.Engine.from_system(sysm)
    if shape == "plain":
        e.tune(0, plain=True)
    else:
        e.tune(shape[0])
        e.set_layout(shape[1], shape[2], shape[3])
    e.nonbond()
    check(sysm, e.forces(), e.stats(), o)
    e.close()


def test_full_size_chain_system_vs_oracle():
    """220 chains of 100 beads and 23,400 waters (92,200 atoms), cutoff 1.2 nm."""
    sysm = W.chains_water()
    o = O.nonbond(sysm, tables_of(sysm))
    e = M.Engine.from_system(sysm)
    e.nonbond()
    check(sysm, e.forces(), e.stats(), o, max_over_frms=3e-5)
    e.close()


def test_chain_device_steps_equal_host_steps():
    """Without the chain bonds (engine_step_host has no bonds): explicit electrostatics,
    global tables and rigid water, host steps against device steps bit for bit."""
    sysm = dataclasses.replace(W.chains_water(nchains=4, length=20, nwater=300, box=(3.6, 3.6, 3.6), seed=2, gap=0.3),
                               bonds=None, bond_pot=None)
    sysm.v = W.maxwell_velocities(sysm, 300.0, seed=3)
    out = []
    for device in (False, True):
        e = M.Engine.from_system(sysm)
        for _ in range(6):
            e.step() if device else e.step_host()
        out.append((e.parts(), e.stats()))
        e.close()
    (xa, va, _, ca), sa = out[0]
    (xb, vb, _, cb), sb = out[1]
    assert np.array_equal(ca, cb)
    assert np.array_equal(xa.view(np.uint32), xb.view(np.uint32))
    assert np.array_equal(va.view(np.uint32), vb.view(np.uint32))
    assert sa.epot == sb.epot


def test_bond_forces_vs_oracle():
    """Chains alone (no water): one device step with dt = 0 leaves the particles in place and
    returns the forces of the sweep plus the harmonic chain bonds; against the oracle's
    nonbonded and bond forces.  The engine's potential energy is the sum of both."""
    sysm = W.chains_water(nchains=12, length=40, nwater=0, box=(3.6, 3.6, 3.6), seed=5)
    sysm.dt = 0.0
    e = M.Engine.from_system(sysm)
    e.step()
    _, _, f, _ = e.parts()
    o = O.nonbond(sysm, tables_of(sysm))
    ob = O.bonds(sysm, M.create_potential(sysm.bond_pot).contents.table())
    ftot = o["f"] + ob["f"]
    err = force_errors(f.astype(np.float64), ftot)
    assert err["global_rel"] <= 2e-6, err
    _, _, _, epot = e.unload()
    assert abs(epot - (o["epot"] + ob["epot"])) <= 1e-6 * (o["epot_abs"] + abs(ob["epot"])), (epot, o["epot"], ob["epot"])
    assert e.stats().pairs == o["pairs"]
    e.close()


def test_bonded_chains_hold_together():
    """Thirty device steps of bonded chains in water at 300 K (dt 2 fs): every bond stays
    within 20 % of its 0.15 nm length, resident and engine_step trajectories agree."""
    sysm = W.chains_water(nchains=4, length=20, nwater=300, box=(3.6, 3.6, 3.6), seed=2, gap=0.3)
    sysm.v = W.maxwell_velocities(sysm, 300.0, seed=3)
    out = []
    for resident in (False, True):
        e = M.Engine.from_system(sysm)
        if resident:
            e.graph(True)
            e.resident_begin().resident_steps(30).resident_end()
        else:
            for _ in range(30):
                e.step()
        x, t, pid, epot = e.unload()
        pos = np.zeros((sysm.n, 3))
        pos[pid] = x
        out.append((pos, epot))
        e.close()
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]
    pos = out[0][0]
    d = pos[sysm.bonds[:, 0]] - pos[sysm.bonds[:, 1]]
    d -= np.round(d / sysm.dim) * sysm.dim
    r = np.linalg.norm(d, axis=1)
    assert np.all(np.abs(r - 0.15) < 0.03), (r.min(), r.max())


def test_host_step_refuses_bonds():
    sysm = W.chains_water(nchains=2, length=10, nwater=0, box=(3.6, 3.6, 3.6), seed=1)
    e = M.Engine.from_system(sysm)
    with pytest.raises(M.MdcoreError, match="-30"):
        e.step_host()
    M.lib().errs_clear()
    e.close()
