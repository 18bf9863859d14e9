"""GPU tests of the rigid constraints (engine_rigid_eval on the device, FP64 iterations).

  P-SHAKE (default)  device == oracle == reference, bit for bit: positions, velocities,
                     constraint forces and refined mixing matrices, three evaluations.
  SHAKE              device == oracle bit for bit (both FP64); the reference's single
                     build (float multiplier) agrees to a float ulp in position.
  steps              engine_step (device) and engine_step_host with rigid water keep every
                     constraint within the tolerance, no group fails to converge.
"""
import dataclasses

import numpy as np
import pytest

import mdcore_b200 as M
import oracle as O
import workloads as W
from helpers import load_rigid_golden, rigid_oracle_steps

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def device_evals(sysm, flags, nevals):
    e = M.Engine.from_system(sysm, flags=flags)
    out = []
    for _ in range(nevals):
        e.rigid_eval()
        x, v, f, _ = e.parts()
        a = np.concatenate([r.matrix().reshape(-1) for r in e.rigid_groups()])
        out.append((x, v, f, a, e.rigid_stats()))
    e.close()
    return out


def test_device_pshake_bit_exact():
    sysm, z, groups = load_rigid_golden()
    dev = device_evals(sysm, M.engine_flag_cuda, 3)
    b = O.bin_system(sysm)
    ora = rigid_oracle_steps(sysm, groups, b["xrel"], z["v"].astype(np.float32), np.zeros((sysm.n, 3), np.float32),
                             True, 3)
    for k, ((x, v, f, a, (itmax, bad)), (xo, vo, fo, ao, ito)) in enumerate(zip(dev, ora)):
        assert bad == 0 and itmax == ito.max(), (k, itmax, ito.max())
        for mine, theirs, ref in ((x, xo, z["px"][k]), (v, vo, z["pv"][k]), (f, fo, z["pf"][k]), (a, ao, z["pa"][k])):
            assert np.array_equal(bits(mine), bits(theirs)), k
            assert np.array_equal(bits(mine), bits(ref)), k


def test_device_shake_bit_exact_vs_oracle():
    sysm, z, groups = load_rigid_golden()
    (x, v, f, _, (itmax, bad)), = device_evals(sysm, M.engine_flag_cuda | M.engine_flag_shake, 1)
    b = O.bin_system(sysm)
    (xo, vo, fo, _, ito), = rigid_oracle_steps(sysm, groups, b["xrel"], z["v"].astype(np.float32),
                                               np.zeros((sysm.n, 3), np.float32), False, 1)
    assert bad == 0 and itmax == ito.max()
    assert np.array_equal(bits(x), bits(xo)) and np.array_equal(bits(v), bits(vo)) and np.array_equal(bits(f), bits(fo))
    assert np.abs(x - z["sx"][0]).max() <= 1.2e-7
    assert np.abs(v - z["sv"][0]).max() <= 1e-6


def constraint_residuals(e, sysm):
    """|r_ij^2 - d^2| of every constraint from the engine's positions (minimum image)."""
    xs, t, pid, _ = e.unload()
    pos = np.zeros((sysm.n, 3))
    pos[pid] = xs
    rig = np.asarray(sysm.rigid)
    i, j, d = rig[:, 0].astype(int), rig[:, 1].astype(int), rig[:, 2]
    dx = pos[i] - pos[j]
    dx -= np.round(dx / sysm.dim) * sysm.dim
    return np.abs((dx ** 2).sum(1) - d ** 2)


@pytest.mark.parametrize("device_steps", [True, False], ids=["engine_step", "engine_step_host"])
@pytest.mark.parametrize("flags", [M.engine_flag_cuda, M.engine_flag_cuda | M.engine_flag_shake],
                         ids=["pshake", "shake"])
def test_rigid_water_steps_keep_constraints(flags, device_steps):
    sysm = W.with_rigid_water(W.water_spce(10), 300.0, seed=2)
    e = M.Engine.from_system(sysm, flags=flags)
    for _ in range(25):                      # crosses the 20 matrix-refinement steps
        if device_steps:
            e.step()
        else:
            e.step_host()
        assert e.stats().status == 0
        itmax, bad = e.rigid_stats()
        assert bad == 0 and 0 < itmax < 100
        # tolerance 1e-6 on d^2 - r^2 plus the float rounding of the stored positions
        assert constraint_residuals(e, sysm).max() < 2e-6
    e.close()


def test_full_size_rigid_water_vs_oracle():
    """SPC/E water, 32,768 rigid molecules: one P-SHAKE evaluation after a free step, device
    against oracle bit for bit."""
    base = W.with_rigid_water(W.water_spce(32), 300.0, seed=3)
    sysm = dataclasses.replace(base, x=W.wrap_positions(base.x + base.dt * base.v, base.dim))
    e = M.Engine.from_system(sysm)
    groups = [(list(r.parts[:r.nr_parts]), r.constraints(), r.matrix()) for r in e.rigid_groups()]
    e.rigid_eval()
    x, v, f, _ = e.parts()
    b = O.bin_system(sysm)
    (xo, vo, fo, _, ito), = rigid_oracle_steps(sysm, groups, b["xrel"], sysm.v.astype(np.float32),
                                               np.zeros((sysm.n, 3), np.float32), True, 1)
    assert ito.max() > 5 and e.rigid_stats() == (ito.max(), 0)
    assert np.array_equal(bits(x), bits(xo)) and np.array_equal(bits(v), bits(vo)) and np.array_equal(bits(f), bits(fo))
    e.close()


def _timers(e):
    """struct engine's last field: unsigned long long timers[engine_timer_last] (18)."""
    import ctypes as C
    n = 18
    off = M.lib().engine_sizeof() - 8 * n
    return np.array((C.c_ulonglong * n).from_address(e.ptr.value + off))


def test_rigid_unsort_timers_and_reset():
    """engine_rigid_unsort (the groups in a random order) leaves the trajectory bit for bit
    unchanged -- each group's constraints are solved alone; engine_step fills the step and
    transfer timers (CPU ticks) and engine_timers_reset zeroes them."""
    import ctypes as C
    sysm = W.with_rigid_water(W.water_spce(10), 300.0, seed=3)
    lib = M.lib()
    lib.engine_rigid_unsort.restype = C.c_int
    lib.engine_rigid_unsort.argtypes = [C.c_void_p]
    lib.engine_timers_reset.restype = C.c_int
    lib.engine_timers_reset.argtypes = [C.c_void_p]
    out = []
    for unsort in (False, True):
        e = M.Engine.from_system(sysm)
        if unsort:
            assert lib.engine_rigid_unsort(e.ptr) == 0
        assert lib.engine_timers_reset(e.ptr) == 0
        for _ in range(4):
            e.step()
        t = _timers(e)
        assert t[0] > 0 and t[15] > 0 and t[16] > 0 and t[17] > 0     # step, cuda_load, unload, dopairs
        assert t[0] >= max(t[15], t[16], t[17])
        assert lib.engine_timers_reset(e.ptr) == 0
        assert not _timers(e).any()
        x, v, f, c = e.parts()
        out.append((x, v, c, e.energies()["total"]))
        e.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
