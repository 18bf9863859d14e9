"""GPU test of engine_nonbond_cuda_noalloc, the entry point for callers that cannot
allocate device memory when they need forces (a host program that hands the engine a fixed,
pre-reserved device budget, or code running between set-up and a stream capture).

The entry point is called through the C ABI on device buffers this test provides, twice in
a row, and its forces, energy and counts are checked against the ordinary entry point
(engine_nonbond_cuda) within the force tolerance the parity tests use.  Its scratch lives
in a static device array shared by all calls, so the second call also checks that nothing
of the first call's state leaks into the next.  The file sorts last so that a run that
stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import mdcore_b200 as M
import oracle as O
from helpers import force_errors, load_golden

pytestmark = pytest.mark.gpu


def device_layout(sysm):
    """Cell-major slots as engine_cuda_load_parts lays them out: cells in index order,
    particles of a cell in load (id) order, cell starts padded to multiples of 4."""
    b = O.bin_system(sysm)
    ncells = int(np.prod(b["cdim"]))
    counts = np.bincount(b["cell"], minlength=ncells).astype(np.int32)
    pads = (counts + 3) // 4 * 4
    cstart = np.zeros(ncells + 1, np.int32)
    cstart[1:] = np.cumsum(pads)
    nslots = int(cstart[-1])
    xq = np.zeros((nslots, 4), np.float32)
    pid = np.zeros(nslots, np.int32)
    fill = cstart[:-1].copy()
    for i in range(sysm.n):                       # ids in load order
        c = b["cell"][i]
        s = fill[c]
        fill[c] += 1
        xq[s, :3] = b["xrel"][i]
        pid[s] = i
    xq.view(np.int32)[:, 3] = np.where(pid >= 0, sysm.type[pid], 0)
    return xq, pid, cstart, counts, nslots, ncells


def test_noalloc_matches_ordinary_entry_point():
    torch = pytest.importorskip("torch")
    sysm, _ = load_golden("water_3000.npz")
    e = M.Engine.from_system(sysm)
    e.nonbond()
    f_ref, st_ref = e.forces(), e.stats()

    xq, pid, cstart, counts, nslots, ncells = device_layout(sysm)
    dev = torch.device("cuda", 0)
    d_xq = torch.from_numpy(xq).to(dev)
    d_pid = torch.from_numpy(pid).to(dev)
    d_cstart = torch.from_numpy(cstart).to(dev)
    d_count = torch.from_numpy(counts).to(dev)
    d_force = torch.zeros(3 * nslots, dtype=torch.int64, device=dev)
    d_epot = torch.zeros(ncells, dtype=torch.int64, device=dev)
    d_acc = torch.zeros(8, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)

    fn = noalloc_fn()

    results = []
    for _ in range(2):
        rc = fn(e.ptr, d_xq.data_ptr(), d_pid.data_ptr(), d_cstart.data_ptr(), d_count.data_ptr(), nslots,
                int(counts.max()), d_force.data_ptr(), d_epot.data_ptr(), d_acc.data_ptr(), stream.cuda_stream)
        assert rc == 0
        torch.cuda.synchronize(dev)
        fx = d_force.cpu().numpy().reshape(nslots, 3).astype(np.float64) / 2.0 ** 24
        acc = d_acc.cpu().numpy()
        f = np.zeros((sysm.n, 3))
        occupied = np.zeros(nslots, bool)
        for c in range(ncells):
            occupied[cstart[c]:cstart[c] + counts[c]] = True
        f[pid[occupied]] = fx[occupied]
        epot = d_epot.cpu().numpy().astype(np.float64).sum() / 2.0 ** 32
        results.append((f, epot, acc))

        assert acc[5] == 0                                  # device status
        assert acc[2] == st_ref.pairs and acc[3] == st_ref.excluded and acc[4] == st_ref.candidates
        assert abs(epot - st_ref.epot) <= 1e-6 * abs(st_ref.epot)
        err = force_errors(f, f_ref)
        assert err["global_rel"] <= 2e-6, err
        assert err["max_over_frms"] <= 2e-5, err

    # The shared scratch carries nothing from one call into the next.
    assert np.array_equal(results[0][0], results[1][0])
    assert results[0][1] == results[1][1]
    e.close()


def noalloc_fn():
    fn = M.lib().engine_nonbond_cuda_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def test_noalloc_rejects_bad_arguments_before_any_launch():
    """Sizes beyond the scratch, cells beyond 1,024 particles and misaligned buffers are
    refused on the host: the pointers below are never dereferenced."""
    sysm, _ = load_golden("argon_1372.npz")
    e = M.Engine.from_system(sysm)
    lib = M.lib()
    fn = noalloc_fn()
    d16, d4 = C.c_void_p(16), C.c_void_p(20)
    assert fn(e.ptr, d16, d16, d16, d16, 65537, 32, d16, d16, d16, None) == -6     # engine_err_range
    assert fn(e.ptr, d16, d16, d16, d16, 1024, 1025, d16, d16, d16, None) == -24   # engine_err_maxparts
    assert fn(e.ptr, d4, d16, d16, d16, 1024, 32, d16, d16, d16, None) == -6       # xq not 16-byte aligned
    assert fn(e.ptr, d16, d4, d16, d16, 1024, 32, d16, d16, d16, None) == -6       # pid not 16-byte aligned
    assert fn(e.ptr, d16, d16, d16, d16, 1024, 32, d4, d16, d16, None) == -6       # force not 8-byte aligned
    lib.errs_clear()
    e.close()


class Buffers:
    def __init__(self, sysm):
        torch = pytest.importorskip("torch")
        self.xq, self.pid, self.cstart, self.counts, self.nslots, self.ncells = device_layout(sysm)
        dev = torch.device("cuda", 0)
        self.dev = dev
        self.d_xq = torch.from_numpy(self.xq).to(dev)
        self.d_pid = torch.from_numpy(self.pid).to(dev)
        self.d_cstart = torch.from_numpy(self.cstart).to(dev)
        self.d_count = torch.from_numpy(self.counts).to(dev)
        self.d_force = torch.zeros(3 * self.nslots, dtype=torch.int64, device=dev)
        self.d_epot = torch.zeros(self.ncells, dtype=torch.int64, device=dev)
        self.d_acc = torch.zeros(8, dtype=torch.int64, device=dev)
        self.stream = torch.cuda.current_stream(dev)

    def call(self, e, maxcount, cstart=None):
        torch = pytest.importorskip("torch")
        cs = self.d_cstart if cstart is None else cstart
        rc = noalloc_fn()(e.ptr, self.d_xq.data_ptr(), self.d_pid.data_ptr(), cs.data_ptr(),
                          self.d_count.data_ptr(), self.nslots, maxcount, self.d_force.data_ptr(),
                          self.d_epot.data_ptr(), self.d_acc.data_ptr(), self.stream.cuda_stream)
        torch.cuda.synchronize(self.dev)
        return rc, self.d_force.cpu().numpy().copy(), self.d_acc.cpu().numpy().copy()


def test_noalloc_reports_undersized_maxcount_and_bad_layout():
    sysm, _ = load_golden("water_3000.npz")
    e = M.Engine.from_system(sysm)
    B = Buffers(sysm)
    # a maxcount below the largest cell: the call returns 0 and the device status says so
    rc, _, acc = B.call(e, 8)
    assert rc == 0 and acc[5] & 2, acc
    # a cell start that is not a multiple of 4: nothing is swept, status bit 128
    torch = pytest.importorskip("torch")
    bad = B.cstart.copy()
    bad[B.ncells // 2] += 1
    rc, f, acc = B.call(e, int(B.counts.max()), torch.from_numpy(bad).to(B.dev))
    assert rc == 0 and acc[5] & 128, acc
    assert not f.any() and acc[2] == 0
    # and a correct call right after it is unaffected
    rc, _, acc = B.call(e, int(B.counts.max()))
    assert rc == 0 and acc[5] == 0 and acc[2] > 0
    e.close()


def test_noalloc_between_ordinary_graph_evaluations():
    """An ordinary evaluation, then an allocation-free call with a smaller maxcount, then
    ordinary evaluations that capture and replay their CUDA graph: the allocation-free call
    leaves the ordinary path's launch state alone, so the graph evaluations succeed and give
    the first evaluation's forces bit for bit."""
    sysm, _ = load_golden("water_3000.npz")
    for layout in (0, 1):
        e = M.Engine.from_system(sysm)
        e.set_layout(layout, 1, 640)
        e.graph(True)
        e.nonbond()                                  # direct launch
        f0, st0 = e.forces(), e.stats()
        B = Buffers(sysm)
        rc, _, acc = B.call(e, 8)                    # smaller shared memory than the ordinary sweep's
        assert rc == 0 and acc[5] & 2
        for _ in range(3):                           # capture, then replays
            e.nonbond()
            assert e.stats().status == 0
            assert np.array_equal(e.forces(), f0)
            assert e.stats().pairs == st0.pairs
        rc, _, acc = B.call(e, int(B.counts.max()))
        assert rc == 0 and acc[5] == 0 and acc[2] == st0.pairs
        e.close()
