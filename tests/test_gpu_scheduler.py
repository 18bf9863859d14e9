"""GPU tests of the learned task-cost scheduler.

* The hand-written MLP kernels (forward, backward, Adam) against a float64 numpy restatement
  on the same BF16-rounded weights.
* Trained on clock64 task durations of the water system, the network predicts task cost
  better than the reference's count-product heuristic (least-squares scaled), and the
  queue order it produces leaves the forces bit-identical.
"""
import ctypes as C

import numpy as np
import pytest

import mdcore_b200 as M
import workloads as W

pytestmark = pytest.mark.gpu

IN, H, NP = M.MLP_IN, M.MLP_HIDDEN, M.MLP_NPARAM


def bf16_round(a):
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32)


def unpack(w):
    o = 0
    W1 = w[o:o + H * IN].reshape(H, IN); o += H * IN
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + H * H].reshape(H, H); o += H * H
    b2 = w[o:o + H]; o += H
    w3 = w[o:o + H]; o += H
    return W1, b1, W2, b2, w3, w[o]


def numpy_grad(w, X, y):
    W1, b1, W2, b2, w3, b3 = unpack(w.astype(np.float64))
    X = X.astype(np.float64)
    z1 = X @ W1.T + b1; h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2; h2 = np.maximum(z2, 0)
    out = h2 @ w3 + b3
    r = out - y
    n = len(y)
    loss = (r ** 2).mean()
    dy = 2 * r / n
    g_w3 = h2.T @ dy; g_b3 = dy.sum()
    dh2 = np.outer(dy, w3) * (z2 > 0)
    g_W2 = dh2.T @ h1; g_b2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (z1 > 0)
    g_W1 = dh1.T @ X; g_b1 = dh1.sum(0)
    return out, loss, np.concatenate([g_W1.ravel(), g_b1, g_W2.ravel(), g_b2, g_w3, [g_b3]])


def test_mlp_kernels_match_numpy():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    n = 777
    X = rng.uniform(0, 2, size=(n, IN)).astype(np.float32)
    y = rng.uniform(0, 3, size=n).astype(np.float32)
    w = bf16_round(rng.normal(0, 0.3, size=NP).astype(np.float32))
    dev = torch.device("cuda", 0)
    dX = torch.from_numpy(X).to(dev)
    dy = torch.from_numpy(y).to(dev)
    dwb = torch.from_numpy(w).to(dev).to(torch.bfloat16)
    dgrad = torch.zeros(NP, dtype=torch.float32, device=dev)
    dloss = torch.zeros(1, dtype=torch.float32, device=dev)
    dout = torch.zeros(n, dtype=torch.float32, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    L = M.lib()
    assert L.nb_mlp_predict(dX.data_ptr(), n, dwb.data_ptr(), dout.data_ptr(), s) == 0
    assert L.nb_mlp_grad(dX.data_ptr(), dy.data_ptr(), None, n, dwb.data_ptr(), dgrad.data_ptr(),
                         dloss.data_ptr(), s) == 0
    torch.cuda.synchronize(dev)
    out_ref, loss_ref, g_ref = numpy_grad(w, X, y)
    assert np.allclose(dout.cpu().numpy(), out_ref, rtol=1e-5, atol=1e-5)
    assert abs(dloss.item() - loss_ref) <= 1e-5 * loss_ref
    g = dgrad.cpu().numpy()
    assert np.abs(g - g_ref).max() <= 1e-4 * np.abs(g_ref).max()

    # One Adam step from zero moments moves every weight by -lr * sign(g) (bias-corrected).
    wm = torch.from_numpy(w.copy()).to(dev)
    m = torch.zeros(NP, device=dev)
    v = torch.zeros(NP, device=dev)
    assert L.nb_mlp_adam(wm.data_ptr(), dwb.data_ptr(), dgrad.data_ptr(), m.data_ptr(), v.data_ptr(), 1e-3, 0.9,
                         0.999, 1e-12, 1, s) == 0
    torch.cuda.synchronize(dev)
    step = wm.cpu().numpy() - w
    nz = np.abs(g) > 1e-6
    assert np.allclose(step[nz], -1e-3 * np.sign(g[nz]), rtol=1e-3)
    assert np.array_equal(dwb.float().cpu().numpy(), bf16_round(wm.cpu().numpy()))


def heuristic_cost(X):
    ni, nj = X[:, 0] * 32, X[:, 1] * 32
    cls = X[:, 6:10].argmax(1)
    w = np.where(cls == 3, ni * ni - ni, ni * nj * np.array(M.CLASS_WEIGHT + (0.0,))[cls])
    return w


def test_learned_cost_beats_count_product_and_keeps_forces():
    sysm = W.water_spce(32)
    e = M.Engine.from_system(sysm)
    e.nonbond()
    f0 = e.forces()
    e.load_parts()
    e.sched_record(4)
    X = e.sched_features()
    y = e.sched_targets()
    loss = e.sched_train(epochs=150, batch=512, lr=3e-3, seed=1)
    p = e.sched_predict()
    h = heuristic_cost(X)
    a = (h @ y) / (h @ h)                       # least-squares scale of the heuristic
    mse_mlp = float(((p - y) ** 2).mean())
    mse_heur = float(((a * h - y) ** 2).mean())
    print(f"tasks {len(y)} mse mlp {mse_mlp:.4f} (train loss {loss:.4f}) count-product {mse_heur:.4f}")
    assert mse_mlp < 0.5 * mse_heur
    e.sched_apply(True)
    e.nonbond()
    assert np.array_equal(e.forces(), f0)
    e.sched_apply(False)
    e.nonbond()
    assert np.array_equal(e.forces(), f0)
    e.close()


def test_learned_order_shortens_the_water_sweep():
    """Full-size SPC/E water (10,206 tasks of ~135-particle cells, a few per worker warp,
    their costs shaped by exclusions and type mix as well as by the counts): the network's
    longest-first order sweeps faster than the count-product order.  Median sweep time of
    21 device-resident evaluations per order, L2 flushed before each."""
    torch = pytest.importorskip("torch")
    sysm = W.water_spce(32)
    e = M.Engine.from_system(sysm)
    e.nonbond()
    e.load_parts()
    e.autotune(reps=3)
    e.graph(True)
    e.sched_record(4)
    e.sched_features()
    e.sched_targets()
    e.sched_train(epochs=150, batch=512, lr=3e-3, seed=1)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def median_sweep():
        for _ in range(3):                      # direct launch, capture, replay
            e.resident()
        ts = []
        for _ in range(21):
            flush.zero_()
            torch.cuda.synchronize()
            e.resident()
            ts.append(e.kernel_times()[1])
        return float(np.median(ts))

    e.sched_apply(False)
    t_heur = median_sweep()
    e.sched_apply(True)
    t_mlp = median_sweep()
    print(f"sweep: count-product {t_heur:.4f} ms, learned {t_mlp:.4f} ms")
    assert t_mlp < t_heur, (t_mlp, t_heur)
    e.close()
