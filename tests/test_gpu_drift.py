"""GPU tests of the pieces the solvated-chain trajectory run is built from: the per-step
energy log of the resident steps against the host's energies, the steepest-descent
resident steps, FP32 force accumulation of the plain form against the FP64 oracle, and a
short NVE trajectory of a small solvated-chain system (both accumulation arms) whose total
energy stays bounded."""
import dataclasses

import numpy as np
import pytest

import mdcore_b200 as M
import oracle as O
import workloads as W
from helpers import force_errors, load_golden

pytestmark = pytest.mark.gpu


def kinetic(sysm, e):
    """sum m v^2 / 2 of the engine's host velocities (after a sync)."""
    _, v, _, _ = e.parts()
    m = np.asarray(sysm.masses, np.float64)[sysm.type]
    return 0.5 * float((m[:, None] * v.astype(np.float64) ** 2).sum())


def test_energy_log_matches_host_energies():
    sysm = W.with_rigid_water(W.water_spce(10), 300.0, seed=3)
    e = M.Engine.from_system(sysm)
    e.graph(True)
    e.energy_log(16)
    e.resident_begin()
    for nsteps in (3, 25):                      # through the P-SHAKE refinement steps
        e.resident_steps(nsteps)
        e.resident_sync()
        log = e.energy_log_read(16)
        assert log[-1, 0] == (3 if nsteps == 3 else 28)
        assert np.all(np.diff(log[:, 0]) == 1)
        u = e.energies()["total"]
        assert abs(log[-1, 1] - u) <= 1e-9 * abs(u), (log[-1, 1], u)
        k = kinetic(sysm, e)
        assert abs(log[-1, 2] - k) <= 1e-9 * k, (log[-1, 2], k)
        assert log[-1, 3] == log[-1, 1] + log[-1, 2]
    e.resident_end()
    e.close()


def test_minimizer_lowers_the_energy_and_caps_moves():
    sysm = W.argon_fcc(6, jitter=0.04, seed=5)
    e = M.Engine.from_system(sysm)
    e.energy_log(64)
    e.resident_begin()
    e.minimize(1e-5, 0.002)
    x0 = None
    us = []
    for _ in range(6):
        e.resident_steps(5)
        e.resident_sync()
        x, _, pid, _ = e.unload()
        xg = np.zeros_like(x)
        xg[pid] = x
        if x0 is not None:
            d = xg - x0
            d -= np.round(d / sysm.dim) * sysm.dim
            assert np.linalg.norm(d, axis=1).max() <= 5 * 0.002 * (1 + 1e-5)
        x0 = xg
        _, v, _, _ = e.parts()
        assert not v.any()                      # steepest descent: velocities zero
        us.append(e.energies()["total"])
    log = e.energy_log_read(64)
    assert len(log) == 30 and np.all(np.diff(log[:, 1]) < 0), log[:, 1]
    assert us[-1] < us[0]
    e.minimize(0.0)
    e.resident_end()
    e.close()


def test_fp32_accumulation_against_oracle():
    sysm, ref = load_golden("water_3000.npz")
    o = O.nonbond(sysm, ref["tables"])
    out = {}
    for arm in ("fp32", "fixed"):
        e = M.Engine.from_system(sysm)
        if arm == "fp32":
            e.tune(0, plain=True)
            e.set_accum(True)
        e.graph(True)
        for _ in range(3):                      # direct, capture, replay
            e.nonbond()
            st = e.stats()
            assert st.status == 0
            assert st.pairs == o["pairs"] and st.excluded == o["excluded"]
            assert abs(st.epot - o["epot"]) <= 1e-6 * abs(o["epot"])
            err = force_errors(e.forces(), o["f"])
            assert err["global_rel"] <= 2e-6 and err["max_over_frms"] <= 2e-5, (arm, err)
        out[arm] = e.forces()
        e.close()
    # the two arms differ only by rounding
    assert force_errors(out["fp32"], out["fixed"])["global_rel"] <= 2e-6


def small_chains():
    return W.chains_water(nchains=6, length=20, nwater=1000, box=(3.6, 3.6, 3.6), seed=4)


def relaxed_small_chains():
    """The small system after 300 steepest-descent steps, with 300 K velocities."""
    sysm = small_chains()
    e = M.Engine.from_system(sysm)
    e.energy_log(400)
    e.resident_begin()
    e.minimize(2e-6, 0.003)
    e.resident_steps(100)
    e.minimize(1e-6, 0.001)
    e.resident_steps(200)
    lg = e.energy_log_read(400)
    assert len(lg) == 300 and np.isfinite(lg).all()
    assert lg[-1, 1] < lg[0, 1]
    e.minimize(0.0)
    e.resident_end()
    x, _, pid, _ = e.unload()
    e.close()
    xr = np.zeros_like(x)
    xr[pid] = x
    relaxed = dataclasses.replace(sysm, x=W.wrap_positions(xr, np.asarray(sysm.dim)))
    relaxed.v = W.maxwell_velocities(relaxed, 300.0, seed=11)
    return relaxed


def nve(relaxed, dt, nsteps, fp32=False):
    """Energy log and final particles (by id) of nsteps NVE steps from the relaxed state."""
    eng = M.Engine.from_system(dataclasses.replace(relaxed, dt=dt))
    if fp32:
        eng.tune(0, plain=True)
        eng.set_accum(True)
    eng.graph(True)
    eng.energy_log(nsteps + 8)
    eng.resident_begin()
    eng.resident_steps(nsteps)
    log = eng.energy_log_read(nsteps + 8)
    eng.resident_end()
    x, _, pid, _ = eng.unload()
    eng.close()
    assert len(log) == nsteps
    xs = np.zeros_like(x)
    xs[pid] = x
    return log, xs


def test_short_trajectory_of_relaxed_chain_system():
    """NVE steps of the relaxed small solvated-chain system over 0.4 ps: the drift of the
    leap-frog total energy is set by the time step (it falls at least 2x from 2 fs to 1 fs)
    and stays within a few per cent of the kinetic energy; the FP32 arm follows the
    fixed-point arm over the first steps; the fixed-point arm repeats bit for bit."""
    relaxed = relaxed_small_chains()
    dev = {}
    for dt in (0.002, 0.001):
        log, _ = nve(relaxed, dt, int(round(0.4 / dt)))
        Et, _, _ = M.leapfrog_energy(log, dt)
        dev[dt] = np.abs(Et - Et[0]).max() / log[:, 2].mean()
    assert dev[0.001] <= 0.5 * dev[0.002], dev
    assert dev[0.002] <= 0.03 and dev[0.001] <= 0.01, dev
    log_fix, x_fix = nve(relaxed, 0.002, 100)
    log_f32, _ = nve(relaxed, 0.002, 100, fp32=True)
    E_fix, _, _ = M.leapfrog_energy(log_fix, 0.002)
    E_f32, _, _ = M.leapfrog_energy(log_f32, 0.002)
    assert np.abs(E_f32[:10] - E_fix[:10]).max() <= 1e-4 * np.abs(E_fix[:10]).max()
    log_fix2, x_fix2 = nve(relaxed, 0.002, 100)
    assert np.array_equal(log_fix, log_fix2) and np.array_equal(x_fix, x_fix2)
