"""GPU tests of the heterogeneous solvated-chain system (20 bead types + water, 231 type
tables read from global memory, explicit electrostatics q_i q_j ep(r) with per-particle
charges, 1-2/1-3 chain exclusions, rigid water): forces, energy, virial and counts against
the FP64 oracle, every launch shape, the plain form, and device steps against host steps."""
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
    sysm = W.chains_water(nchains=4, length=20, nwater=300, box=(3.6, 3.6, 3.6), seed=2, gap=0.3)
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
