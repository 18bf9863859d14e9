"""GPU tests of device-resident time steps (engine_cuda_resident_* / engine_batch_resident_*):
re-binning, sort, sweep, integration and rigid constraints as device launches only, the
host cells brought up to date on request.

The device restates engine_step's float expressions (space_shuffle's shift, engine_advance's
update, the constraint corrections) and sums forces in fixed point, so its trajectories
must equal engine_step's bit for bit: positions, velocities, cells and energies by particle
id, with and without CUDA-graph replay, for single engines and batches of replicas.  A
cell that outgrows its device block ends the call with engine_err_maxparts and leaves the
host copy untouched.
"""
import numpy as np
import pytest

import mdcore_b200 as M
import workloads as W

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def warm_argon(ncell=8, temperature=1200.0, seed=4):
    sysm = W.argon_fcc(ncell, seed=seed)
    sysm.v = W.maxwell_velocities(sysm, temperature, seed=seed)
    return sysm


def host_run(sysm, nsteps, flags=M.engine_flag_cuda, layout=None, device_steps=False):
    """nsteps of engine_step_host (re-binning and integration on the host), or of
    engine_step (one device step per call, host particles in and out)."""
    e = M.Engine.from_system(sysm, flags=flags)
    if layout is not None:
        e.set_layout(layout)
    for _ in range(nsteps):
        if device_steps:
            e.step()
        else:
            e.step_host()
    out = e.parts(), e.stats()
    rig = e.rigid_stats() if sysm.rigid is not None else None
    e.close()
    return out, rig


def same_state(a, b, forces=True):
    (xa, va, fa, ca), sa = a
    (xb, vb, fb, cb), sb = b
    assert np.array_equal(ca, cb)
    assert np.array_equal(bits(xa), bits(xb))
    assert np.array_equal(bits(va), bits(vb))
    if forces:
        assert np.array_equal(bits(fa), bits(fb))
        assert sa.epot == sb.epot and sa.virial == sb.virial


@pytest.mark.parametrize("graph", [False, True], ids=["direct", "graph"])
@pytest.mark.parametrize("layout", [0, 1])
def test_resident_steps_equal_engine_step(graph, layout):
    sysm = warm_argon()
    nsteps = 30
    ref, _ = host_run(sysm, nsteps, layout=layout)       # the lane layouts round partial sums differently
    e = M.Engine.from_system(sysm)
    e.set_layout(layout)
    e.graph(graph)
    e.resident_begin()
    e.resident_steps(10).resident_steps(nsteps - 10).resident_sync()
    assert e.stats().status == 0
    info = e.resident_info()
    assert info.steps == nsteps and info.regrows == 0
    assert info.pairs > nsteps * 0.9 * e.stats().pairs
    got = e.parts(), e.stats()
    # particles did cross cell faces
    e0 = M.Engine.from_system(sysm)
    assert (got[0][3] != e0.parts()[3]).sum() > 20
    e0.close()
    same_state(ref, got)
    e.resident_end()
    e.close()


def test_resident_sync_without_steps_keeps_the_host_state():
    sysm = warm_argon(6)
    e = M.Engine.from_system(sysm)
    e.nonbond()
    before = e.parts()
    e.resident_begin().resident_sync()
    x, v, _, c = e.parts()
    assert np.array_equal(c, before[3])
    assert np.array_equal(bits(x), bits(before[0])) and np.array_equal(bits(v), bits(before[1]))
    e.close()


def test_host_steps_continue_after_resident_steps():
    """resident_end hands the particles back: host and device steps carry on from the device
    state."""
    sysm = warm_argon(6)
    ref, _ = host_run(sysm, 12)
    e = M.Engine.from_system(sysm)
    for _ in range(4):
        e.step_host()
    e.resident_begin().resident_steps(5).resident_end()
    e.step()
    e.step_host()
    e.step()
    same_state(ref, (e.parts(), e.stats()))
    e.close()


@pytest.mark.parametrize("graph", [False, True], ids=["direct", "graph"])
def test_engine_step_on_the_device_equals_host_steps(graph):
    """engine_step (upload, one device step, download per call) against engine_step_host."""
    sysm = warm_argon(7)
    ref, _ = host_run(sysm, 15)
    e = M.Engine.from_system(sysm)
    e.graph(graph)
    for _ in range(15):
        e.step()
    same_state(ref, (e.parts(), e.stats()))
    e.close()


def test_engine_step_on_the_device_rigid_water():
    sysm = W.with_rigid_water(W.water_spce(10), 300.0, seed=4)
    ref, rig_ref = host_run(sysm, 24)
    got, rig = host_run(sysm, 24, device_steps=True)
    same_state(ref, got, forces=False)
    assert got[1].epot == ref[1].epot and rig == rig_ref


@pytest.mark.parametrize("flags", [M.engine_flag_cuda, M.engine_flag_cuda | M.engine_flag_shake],
                         ids=["pshake", "shake"])
def test_resident_rigid_water_equals_engine_step(flags):
    """Rigid water through and past the P-SHAKE matrix refinement steps (direct launches),
    then graph replay: positions and velocities bit for bit, same iteration statistics."""
    sysm = W.with_rigid_water(W.water_spce(10), 300.0, seed=2)
    nsteps = 26
    ref, rig_ref = host_run(sysm, nsteps, flags)
    e = M.Engine.from_system(sysm, flags=flags)
    e.graph(True)
    e.resident_begin().resident_steps(nsteps).resident_sync()
    got = e.parts(), e.stats()
    same_state(ref, got, forces=False)
    assert got[1].epot == ref[1].epot
    assert e.rigid_stats() == rig_ref
    e.close()


def test_batch_resident_steps_equal_engine_step():
    systems = W.argon_replicas(nrep=6, seed=7)
    for k, s in enumerate(systems):
        s.v = W.maxwell_velocities(s, 900.0, seed=k)
    nsteps = 12
    refs = [host_run(s, nsteps)[0] for s in systems]
    engines = [M.Engine.from_system(s, start=False) for s in systems]
    b = M.Batch(engines)
    b.graph(True)
    b.resident_begin().resident_steps(nsteps).resident_sync()
    assert b.stats().status == 0
    for e, ref in zip(engines, refs):
        got = e.parts(), e.stats()
        same_state(ref, got)
    b.resident_end()
    b.close()
    for e in engines:
        e.close()


def test_batch_step_on_the_device_equals_host_steps():
    systems = W.argon_replicas(nrep=5, seed=9)
    for k, s in enumerate(systems):
        s.v = W.maxwell_velocities(s, 900.0, seed=k)
    out = []
    for device in (False, True):
        engines = [M.Engine.from_system(s, start=False) for s in systems]
        b = M.Batch(engines)
        for _ in range(6):
            b.step() if device else b.step_host()
        out.append([(e.parts(), e.stats()) for e in engines])
        b.close()
        for e in engines:
            e.close()
    for ref, got in zip(*out):
        same_state(ref, got)


def crowding_system():
    """Eight particles of cell (0,0,0) heading into cell (1,0,0), which holds eight of its
    own: the second step's re-binning puts 16 into a block of 12 slots."""
    A, B = W.lj_AB(0.996, 0.3405)
    yz = np.stack(np.meshgrid([0.15, 0.45, 0.75], [0.15, 0.45, 0.75], indexing="ij"), -1).reshape(-1, 2)[:8]
    movers = np.concatenate([np.full((8, 1), 0.95), yz], axis=1)     # near the +x face of cell 0
    g = np.stack(np.meshgrid([1.4, 1.7], [0.2, 0.5], [0.2, 0.5], indexing="ij"), -1).reshape(-1, 3)
    resting = g                                                       # inside cell (1, 0, 0)
    x = np.concatenate([movers, resting])
    v = np.zeros_like(x)
    v[:8, 0] = 20.0                                   # 0.1 nm in one step of 0.005 ps
    return W.System(name="crowding", origin=np.zeros(3), dim=np.full(3, 3.0), L=np.full(3, 1.0), cutoff=1.0,
                    masses=[39.948], charges=[0.0],
                    pots=[W.PotSpec(W.KIND_LJ126, 0, 0, 0.25, 1.0, 1e-4, (A * 1e-6, B * 1e-6, 0.0, 0.0))],
                    x=x, type=np.zeros(len(x), np.int32), excl=np.zeros((0, 2), np.int32), dt=0.005, v=v)


def test_block_overflow_regrows_and_matches_engine_step():
    """Twelve slots per cell: the second step's re-binning would put 16 particles into one
    block.  The step is aborted on the device, the particles of step 1 are re-blocked with
    more room and step 2 runs again: the same result as engine_step."""
    sysm = crowding_system()
    ref, _ = host_run(sysm, 3)
    e = M.Engine.from_system(sysm)
    e.resident_begin(margin=0)
    assert e.resident_info()[0] == 12
    e.resident_steps(3).resident_sync()
    info = e.resident_info()
    assert info.regrows == 1 and info.steps == 3 and info.capc >= 16
    same_state(ref, (e.parts(), e.stats()))
    e.close()


def test_many_leavers_regrow_the_lists():
    """The whole box drifts by 0.6 nm per step: two layers of nine particles leave every
    cell in the same step (more than 16), the leaver lists double and the steps match
    engine_step."""
    rng = np.random.default_rng(11)
    A, B = W.lj_AB(0.996, 0.3405)
    g = np.stack(np.meshgrid(*[np.arange(3)] * 3, indexing="ij"), -1).reshape(-1, 3).astype(float)
    sub = np.stack(np.meshgrid(*[[0.1, 0.4, 0.7]] * 3, indexing="ij"), -1).reshape(-1, 3)
    x = (g[:, None, :] + sub[None, :, :]).reshape(-1, 3) + rng.uniform(0, 0.02, size=(27 * 27, 3))
    v = np.tile([[120.0, 0.0, 0.0]], (len(x), 1))         # 0.6 nm per step of 0.005 ps: 18 leave a cell
    sysm = W.System(name="drift", origin=np.zeros(3), dim=np.full(3, 3.0), L=np.full(3, 1.0), cutoff=1.0,
                    masses=[39.948], charges=[0.0],
                    pots=[W.PotSpec(W.KIND_LJ126, 0, 0, 0.25, 1.0, 1e-4, (A * 1e-6, B * 1e-6, 0.0, 0.0))],
                    x=x, type=np.zeros(len(x), np.int32), excl=np.zeros((0, 2), np.int32), dt=0.005, v=v)
    ref, _ = host_run(sysm, 8)
    e = M.Engine.from_system(sysm)
    e.graph(True)
    e.resident_begin().resident_steps(8).resident_sync()
    info = e.resident_info()
    assert info.mcap > 16 and info.regrows >= 1 and info.steps == 8
    same_state(ref, (e.parts(), e.stats()))
    e.close()


def test_engine_step_retries_an_aborted_step():
    """engine_step with more than 16 leavers per cell: the device step is aborted, the host
    cells are untouched, the step runs again with longer leaver lists; same trajectory as
    engine_step_host."""
    rng = np.random.default_rng(11)
    A, B = W.lj_AB(0.996, 0.3405)
    g = np.stack(np.meshgrid(*[np.arange(3)] * 3, indexing="ij"), -1).reshape(-1, 3).astype(float)
    sub = np.stack(np.meshgrid(*[[0.1, 0.4, 0.7]] * 3, indexing="ij"), -1).reshape(-1, 3)
    x = (g[:, None, :] + sub[None, :, :]).reshape(-1, 3) + rng.uniform(0, 0.02, size=(27 * 27, 3))
    v = np.tile([[120.0, 0.0, 0.0]], (len(x), 1))
    sysm = W.System(name="drift", origin=np.zeros(3), dim=np.full(3, 3.0), L=np.full(3, 1.0), cutoff=1.0,
                    masses=[39.948], charges=[0.0],
                    pots=[W.PotSpec(W.KIND_LJ126, 0, 0, 0.25, 1.0, 1e-4, (A * 1e-6, B * 1e-6, 0.0, 0.0))],
                    x=x, type=np.zeros(len(x), np.int32), excl=np.zeros((0, 2), np.int32), dt=0.005, v=v)
    ref, _ = host_run(sysm, 8)
    got, _ = host_run(sysm, 8, device_steps=True)
    same_state(ref, got)
