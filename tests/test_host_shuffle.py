"""Host re-binning (space_shuffle) order, on the CPU: every cell keeps its remaining
particles in their order and appends the arrivals from its 26 neighbours by direction
index (dx+1)*9 + (dy+1)*3 + (dz+1), each neighbour's leavers in their order; a leaver's
position is shifted by -delta*h in float.  The device-resident re-binning follows the same
rule, which is what keeps host and device trajectories equal bit for bit."""
import ctypes as C

import numpy as np
import pytest

import mdcore_b200 as M
import workloads as W

SPACE_OFFSET = 8            # struct engine: unsigned flags, then struct space (8-byte aligned)


def space_fields(e):
    base = e.ptr.value + SPACE_OFFSET
    dim = np.frombuffer((C.c_double * 3).from_address(base), np.float64).copy()
    cdim = np.frombuffer((C.c_int * 3).from_address(base + 48), np.int32).copy()
    h = np.frombuffer((C.c_double * 3).from_address(base + 72), np.float64).copy()
    return dim, cdim, h


def expected_shuffle(order, cell_of, xrel, cdim, h):
    """Particle order and cell-relative positions after re-binning, by the rule above."""
    hf = h.astype(np.float32)
    nc = int(np.prod(cdim))
    stay = [[] for _ in range(nc)]
    leave = [[] for _ in range(nc)]
    newx = xrel.copy()
    for pid in order:
        c = cell_of[pid]
        x = xrel[pid]
        delta = (x >= hf).astype(int) - (x < np.float32(0)).astype(int)
        if not delta.any():
            stay[c].append(pid)
            continue
        newx[pid] = (x - (delta.astype(np.float32) * hf).astype(np.float32)).astype(np.float32)
        leave[c].append((pid, int((delta[0] + 1) * 9 + (delta[1] + 1) * 3 + (delta[2] + 1))))
    out = []
    for c in range(nc):
        loc = np.array([c // (cdim[1] * cdim[2]), (c // cdim[2]) % cdim[1], c % cdim[2]])
        seq = list(stay[c])
        for d in range(27):
            if d == 13:
                continue
            delta = np.array([d // 9 - 1, (d // 3) % 3 - 1, d % 3 - 1])
            sl = (loc - delta) % cdim
            src = (sl[0] * cdim[1] + sl[1]) * cdim[2] + sl[2]
            seq += [pid for pid, dd in leave[src] if dd == d]
        out += seq
    return np.array(out), newx


@pytest.mark.parametrize("seed", [0, 1])
def test_shuffle_order_and_shift(seed):
    sysm = W.argon_fcc(8, seed=seed)
    rng = np.random.default_rng(seed)
    sysm.v = rng.normal(0.0, 6.0, size=(sysm.n, 3))
    sysm.dt = 0.02
    e = M.Engine.from_system(sysm, start=False)
    dim, cdim, h = space_fields(e)
    assert np.allclose(dim, sysm.dim)
    lib = M.lib()
    lib.engine_advance(e.ptr)
    xrel, _, _, cell_of = e.parts()
    _, _, order, _ = e.unload()
    want_order, want_x = expected_shuffle(order, cell_of, xrel, cdim, h)
    assert (want_order != np.sort(want_order)).any()
    moved = lib.space_shuffle(C.c_void_p(e.ptr.value + SPACE_OFFSET))
    assert moved == 1
    _, _, got_order, _ = e.unload()
    got_x, _, _, got_cell = e.parts()
    assert np.array_equal(got_order, want_order)
    assert np.array_equal(got_x.view(np.uint32), want_x.astype(np.float32).view(np.uint32))
    assert (got_cell != cell_of).sum() > 50
    e.close()
