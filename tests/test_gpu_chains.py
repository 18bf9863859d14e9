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
    sysm = W.chains_water(nchains=4, length=20, nwater=300, box=(3.6, 3.6, 3.6), seed=2, gap=0.3,
                          angles_dihedrals=False)
    sysm = dataclasses.replace(sysm, bonds=None, bond_pot=None)
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
    sysm = W.chains_water(nchains=12, length=40, nwater=0, box=(3.6, 3.6, 3.6), seed=5, angles_dihedrals=False)
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


def bonded_oracle(sysm):
    """Oracle nonbonded + bond + angle + dihedral forces (by id) and the energies."""
    o = O.nonbond(sysm, tables_of(sysm))
    ob = O.bonds(sysm, M.create_potential(sysm.bond_pot).contents.table())
    oa = O.angles(sysm, M.bonded_tables([M.create_angle_potential(*p) for p in sysm.angle_pots]))
    od = O.dihedrals(sysm, M.bonded_tables([M.create_dihedral_potential(*p) for p in sysm.dihedral_pots]))
    return o, ob, oa, od


def test_angle_dihedral_forces_vs_oracle():
    """Chains with bonds, angles (bond angles 100-150 degrees) and dihedrals, no solvent:
    one device step with dt = 0 returns the sweep's forces plus the three bonded terms',
    against the oracle's (FP32 on the device, FP64 in the oracle); the potential energy is
    the sum of the four.  The largest single-atom error comes from FP32 pair forces at the
    close contacts of chains that cross one another (the nonbonded part), hence the F_rms
    bound of 5e-5; the bonded terms alone are checked in the next test."""
    sysm = W.bonded_chains(nchains=4, seed=3)
    sysm.dt = 0.0
    e = M.Engine.from_system(sysm)
    e.step()
    _, _, f, _ = e.parts()
    o, ob, oa, od = bonded_oracle(sysm)
    ftot = o["f"] + ob["f"] + oa["f"] + od["f"]
    err = force_errors(f.astype(np.float64), ftot)
    print("bonded chains", err)
    assert err["global_rel"] <= 1e-5, err
    assert err["max_over_frms"] <= 5e-5, err
    en = e.energies()
    print("energies", en, "oracle", o["epot"], ob["epot"], oa["epot"], od["epot"])
    assert abs(en["nonbond"] - o["epot"]) <= 1e-6 * o["epot_abs"]
    assert abs(en["bond"] - ob["epot"]) <= 1e-6 * abs(oa["epot"])
    assert abs(en["angle"] - oa["epot"]) <= 1e-6 * abs(oa["epot"])
    assert abs(en["dihedral"] - od["epot"]) <= 1e-6 * abs(od["epot"])
    assert en["total"] == en["nonbond"] + en["bond"] + en["angle"] + en["dihedral"]
    assert e.stats().status == 0
    e.close()


def test_angle_dihedral_forces_alone():
    """The same step without the angles and dihedrals: the difference of the two steps'
    forces (each a fixed-point sum, rounded once to float) is the angles' and dihedrals'
    forces, against the oracle's."""
    full = W.bonded_chains(nchains=4, seed=3)
    full.dt = 0.0
    bare = dataclasses.replace(full, angles=None, angle_pots=None, dihedrals=None, dihedral_pots=None)
    out = []
    for sysm in (full, bare):
        e = M.Engine.from_system(sysm)
        e.step()
        _, _, f, _ = e.parts()
        out.append(f.astype(np.float64))
        e.close()
    _, _, oa, od = bonded_oracle(full)
    df = out[0] - out[1]
    err = force_errors(df, oa["f"] + od["f"])
    print("angles + dihedrals", err)
    assert err["global_rel"] <= 1e-5, err
    assert err["max_over_frms"] <= 3e-5, err


def test_bonded_resident_steps_equal_engine_step():
    """Twenty steps of bonded chains at 300 K (dt 1 fs): device-resident steps and
    engine_step give the same trajectory bit for bit."""
    sysm = W.bonded_chains(nchains=4, seed=3)
    sysm.dt = 0.001
    sysm.v = W.maxwell_velocities(sysm, 300.0, seed=4)
    out = []
    for resident in (False, True):
        e = M.Engine.from_system(sysm)
        if resident:
            e.graph(True)
            e.resident_begin().resident_steps(20).resident_end()
        else:
            for _ in range(20):
                e.step()
        x, t, pid, epot = e.unload()
        pos = np.zeros((sysm.n, 3))
        pos[pid] = x
        out.append((pos, epot))
        e.close()
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]


@pytest.mark.parametrize("groups", [1, 3])
def test_bonded_batch_equals_single_engines(groups):
    """Three bonded-chain systems stepped as one batch (engine_batch_step, in one group or
    one group per engine) and each alone (engine_step): the same positions and energies bit
    for bit (the angle and dihedral records carry their engine)."""
    systems = [W.bonded_chains(nchains=4, seed=s) for s in (3, 4, 5)]
    for k, s in enumerate(systems):
        s.v = W.maxwell_velocities(s, 300.0, seed=10 + k)
        s.dt = 0.001
    single = []
    for s in systems:
        e = M.Engine.from_system(s)
        for _ in range(4):
            e.step()
        single.append(e.unload())
        e.close()
    engines = [M.Engine.from_system(s, start=False) for s in systems]
    b = M.Batch(engines)
    b.set_groups(groups)                 # 3: one group per engine (own device blocks and stream)
    for _ in range(4):
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


def test_host_step_refuses_angles():
    sysm = dataclasses.replace(W.bonded_chains(nchains=2, seed=1), bonds=None, bond_pot=None)
    e = M.Engine.from_system(sysm)
    with pytest.raises(M.MdcoreError, match="-30"):
        e.step_host()
    M.lib().errs_clear()
    e.close()
