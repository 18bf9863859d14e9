// Persistent sweeps over a device task queue (sm_100a): sweep_tuned (one i particle per
// lane, 32 per warp) and sweep_tiled (8 i x 4 j lanes per warp).
//
// Differences from the plain sweep (nb_kernels.cuh), none of which changes the pair set:
//  * persistent blocks (as many as fit on every SM) of independent worker warps: every
//    warp pops whole tasks from a device queue (an atomic counter over a permutation of the
//    task list, so a scheduler can order it, e.g. longest task first), stages the j cell
//    (positions, ids, sort keys) and the i cell's sort keys in its own shared-memory slice
//    with TMA bulk copies completed on an mbarrier (bounded waits), sweeps the task and
//    writes its forces; the tables are staged into shared memory once per block;
//  * f = U'(r) * (1/halfwidth) * rsqrt(r2) with one Newton step instead of an IEEE
//    division (r itself stays correctly rounded, and the cutoff test uses the exactly
//    rounded r2);
//  * Newton's third law through a register reduce-scatter: each lane keeps its j
//    contributions of 4 or 8 consecutive sweep steps and one reduce-scatter across the warp
//    sums them, after which distinct lanes hold the totals of distinct j.  The order of
//    additions is fixed, so task partials stay independent of scheduling;
//  * energy is summed per pair in double (float partial sums of cancelling Coulomb terms
//    would cost ~1e-6 of the total); the virial per particle and task from the partial
//    forces: sum over pairs of r_ij.F_ij = sum_i (x_i - shift).F_i + sum_j x_j.F_j;
//  * tasks of at most 32 candidate pairs (a few particles per cell, as in a vapour) are not
//    staged: one pair per lane, each accepted pair's force added to both particles;
//  * optional per-task clock64 records (start, end, SM) for the learned scheduler.
#pragma once
#include "nb_kernels.cuh"

// TPSM, a template parameter of both persistent sweeps: resident threads per SM their
// register allocation is sized for (launch bounds).  640 threads leave 96 registers per
// thread, 768 leave 80, 1024 leave 64: large cells (long sweeps) run best with 96,
// small cells (short tasks, latency-bound) with more warps per SM.

namespace nb {

struct TunedParams {
    Params p;
    const int* order;            // queue: task indices in scheduling order
    const int* qcount;           // number of queue entries (device), or nullptr: p.ntasks
    int* counter;                // queue head (zeroed before each launch)
    long long* task_clock;       // 2 * ntasks: start, end (clock64) or nullptr
    int* task_sm;                // SM id per task or nullptr
};

__device__ __forceinline__ unsigned smid() {
    unsigned r;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
    return r;
}

// Table evaluation with fused multiply-adds (interval index included: a different
// rounding can only move r to the neighbouring interval at a node, where the two pieces
// agree), 1/r supplied by the caller.
__device__ __forceinline__ void eval_table_fast(const float* __restrict__ coef, float4 info, int nmax, float r,
                                                float rinv, float& e, float& f) {
    const float t = fmaf(r, fmaf(r, info.z, info.y), info.x);
    const int ind = min(__float2int_rz(fmaxf(0.0f, t)), nmax);
    const float4* c = reinterpret_cast<const float4*>(coef + (__float_as_int(info.w) & 0xfffff) + 8 * ind);
    const float4 c0 = c[0], c1 = c[1];
    const float x = (r - c0.x) * c0.y;
    float ee = fmaf(c0.z, x, c0.w);
    float eff = c0.z;
    eff = fmaf(eff, x, ee); ee = fmaf(ee, x, c1.x);
    eff = fmaf(eff, x, ee); ee = fmaf(ee, x, c1.y);
    eff = fmaf(eff, x, ee); ee = fmaf(ee, x, c1.z);
    eff = fmaf(eff, x, ee); ee = fmaf(ee, x, c1.w);
    e = ee;
    f = eff * c0.y * rinv;
}

// Warp reduce-scatter of 4 values per lane: afterwards lane l holds the sum over the warp
// of v[l & 3] (lanes l, l+4, ..., l+28 hold the same total).  Six shuffles.
__device__ __forceinline__ float reduce_scatter4(const float (&v)[4], int lane) {
    constexpr unsigned FULL = 0xffffffffu;
    const bool b0 = lane & 1, b1 = lane & 2;
    float a[2];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const float send = b0 ? v[2 * m] : v[2 * m + 1];
        const float keep = b0 ? v[2 * m + 1] : v[2 * m];
        a[m] = keep + __shfl_xor_sync(FULL, send, 1);
    }
    const float send = b1 ? a[0] : a[1];
    const float keep = b1 ? a[1] : a[0];
    float d = keep + __shfl_xor_sync(FULL, send, 2);
    d += __shfl_xor_sync(FULL, d, 4);
    d += __shfl_xor_sync(FULL, d, 8);
    d += __shfl_xor_sync(FULL, d, 16);
    return d;
}

// Warp reduce-scatter of 8 values per lane: afterwards lane l holds sum over the warp of
// v[l & 7] (lanes l, l+8, l+16, l+24 hold the same total).
__device__ __forceinline__ float reduce_scatter8(const float (&v)[8], int lane) {
    constexpr unsigned FULL = 0xffffffffu;
    const bool b0 = lane & 1, b1 = lane & 2, b2 = lane & 4;
    float a[4], c[2], d;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const float send = b0 ? v[2 * m] : v[2 * m + 1];
        const float keep = b0 ? v[2 * m + 1] : v[2 * m];
        a[m] = keep + __shfl_xor_sync(FULL, send, 1);
    }
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const float send = b1 ? a[2 * m] : a[2 * m + 1];
        const float keep = b1 ? a[2 * m + 1] : a[2 * m];
        c[m] = keep + __shfl_xor_sync(FULL, send, 2);
    }
    {
        const float send = b2 ? c[0] : c[1];
        const float keep = b2 ? c[1] : c[0];
        d = keep + __shfl_xor_sync(FULL, send, 4);
    }
    d += __shfl_xor_sync(FULL, d, 8);
    d += __shfl_xor_sync(FULL, d, 16);
    return d;
}

// ---------------------------------------------------------------- queue compaction
// Each step the queue is rebuilt from the scheduling order, keeping (in order) only tasks
// whose cells are both non-empty: a block-wise flag count, a one-block scan of the block
// totals, and a scatter.  Deterministic and stable.
constexpr int kQueueBlock = 1024;

__device__ __forceinline__ bool task_live(const TaskRec& r, const int* __restrict__ ccount) {
    const int ni = ccount[r.ci], nj = ccount[r.cj];
    return r.sid < 0 ? ni >= 2 : (ni > 0 && nj > 0);
}

// Exclusive scan of one flag per thread over the block; returns the block total.
__device__ __forceinline__ int block_scan_flag(int flag, int& excl, int* warp_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned ball = __ballot_sync(0xffffffffu, flag);
    const int in_warp = __popc(ball & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[warp] = __popc(ball);
    __syncthreads();
    if (warp == 0) {
        const int v = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        warp_tot[lane] = incl - v;          // exclusive prefix of warps
        if (lane == 31) warp_tot[32] = incl;
    }
    __syncthreads();
    excl = warp_tot[warp] + in_warp;
    const int total = warp_tot[32];
    __syncthreads();
    return total;
}

__global__ void __launch_bounds__(kQueueBlock) queue_count(const int* __restrict__ order, const TaskRec* __restrict__ tasks,
                                                           const int* __restrict__ ccount, int ntasks, int* __restrict__ bsum) {
    __shared__ int warp_tot[33];
    const int q = blockIdx.x * kQueueBlock + threadIdx.x;
    const int flag = q < ntasks ? task_live(tasks[order[q]], ccount) : 0;
    int excl;
    const int total = block_scan_flag(flag, excl, warp_tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kQueueBlock) queue_offsets(int* __restrict__ bsum, int nblocks, int* __restrict__ qcount) {
    __shared__ int warp_tot[33];
    int run = 0;
    for (int base = 0; base < nblocks; base += kQueueBlock) {
        const int b = base + threadIdx.x;
        const int v = b < nblocks ? bsum[b] : 0;
        // inclusive-of-others exclusive scan via the flag scan applied to counts: do it in
        // two steps: warp scan of values, then warps
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const int wv = warp_tot[lane];
            int wi = wv;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += t;
            }
            warp_tot[lane] = wi - wv;
            if (lane == 31) warp_tot[32] = wi;
        }
        __syncthreads();
        if (b < nblocks) bsum[b] = run + warp_tot[warp] + incl - v;
        run += warp_tot[32];
        __syncthreads();
    }
    if (threadIdx.x == 0) *qcount = run;
}

__global__ void __launch_bounds__(kQueueBlock) queue_scatter(const int* __restrict__ order, const TaskRec* __restrict__ tasks,
                                                             const int* __restrict__ ccount, int ntasks,
                                                             const int* __restrict__ bsum, int* __restrict__ queue) {
    __shared__ int warp_tot[33];
    const int q = blockIdx.x * kQueueBlock + threadIdx.x;
    const int t = q < ntasks ? order[q] : 0;
    const int flag = q < ntasks ? task_live(tasks[t], ccount) : 0;
    int excl;
    block_scan_flag(flag, excl, warp_tot);
    if (flag) queue[bsum[blockIdx.x] + excl] = t;
}

// Shared memory of one worker warp (cap = largest cell rounded up to 4, plus 8 spare rows
// that the sweep windows may read past the end of the j list): two mbarriers, the j list
// in sweep order (js, jid: 20 B per row) and STAGES staging buffers for the raw bulk copies
// of a task (xraw, pidraw, keyj, keyi: 28 B per row).  The j list's slots and sort
// distances are read from the copied keys (keyj, in descending distance order), which stay
// in place while the task is swept.  With two stages the copies of the next task land
// while the warp sweeps the current one.
__host__ __device__ inline size_t warp_slice_bytes(int cap, int stages) {
    return 16 + (size_t)cap * (20 + 28 * (size_t)stages);
}

__host__ __device__ inline size_t warps_smem_bytes(int cap, int nw, int ncoef, int npots, int mt, int stages) {
    size_t b = (size_t)nw * warp_slice_bytes(cap, stages);
    b += (size_t)npots * 16;
    b += (size_t)((ncoef + 3) & ~3) * 4;
    b += (size_t)((npots + 3) & ~3) * 4;
    b += (size_t)((mt * mt + 3) & ~3) * 4;
    return b;
}

// Shared tables (one copy per block, after the warp slices).
struct SharedTables {
    float4* potinfo;
    float* coef;
    int* potn;
    int* potidx;
    float4 one;         // kTabOne: the one table's interval transform and offsets, in registers
};

// Table modes of the persistent sweeps: kTabShared (tables staged in shared memory, a lookup
// per pair), kTabOne (one table for every type pair), kTabGlobal (tables read from global
// memory through L1, for systems whose tables do not fit in shared memory, and explicit
// electrostatics).
constexpr int kTabShared = 0, kTabOne = 1, kTabGlobal = 2;

template <int NW, int STAGES, int TAB>
__device__ __forceinline__ SharedTables stage_tables(const Params& P, unsigned char* smem_raw, int cap) {
    SharedTables S;
    S.one = TAB == kTabOne ? P.potinfo[0] : make_float4(0.f, 0.f, 0.f, 0.f);
    if (TAB == kTabGlobal) {
        S.potinfo = const_cast<float4*>(P.potinfo);
        S.coef = const_cast<float*>(P.coef);
        S.potn = const_cast<int*>(P.potn);
        S.potidx = const_cast<int*>(P.potidx);
        return S;
    }
    unsigned char* sp = smem_raw + (size_t)NW * warp_slice_bytes(cap, STAGES);
    S.potinfo = reinterpret_cast<float4*>(sp); sp += (size_t)P.npots * 16;
    S.coef = reinterpret_cast<float*>(sp); sp += (size_t)((P.ncoef + 3) & ~3) * 4;
    S.potn = reinterpret_cast<int*>(sp); sp += (size_t)((P.npots + 3) & ~3) * 4;
    S.potidx = reinterpret_cast<int*>(sp);
    const int tid = threadIdx.x;
    for (int k = tid; k < P.ncoef; k += NW * 32) S.coef[k] = P.coef[k];
    for (int k = tid; k < P.npots; k += NW * 32) { S.potinfo[k] = P.potinfo[k]; S.potn[k] = P.potn[k]; }
    for (int k = tid; k < P.max_type * P.max_type; k += NW * 32) S.potidx[k] = P.potidx[k];
    return S;
}

// One worker warp's shared-memory slice, viewed through staging buffer `stage`.
struct WarpSlice {
    uint64_t* bar;      // mbarrier of this stage
    float4* xraw;       // j cell as copied
    float4* js;         // j cell in sweep order (w: type bits)
    float4* fj;         // j (and self) partial forces; aliases xraw once js is built
    int* pidraw;
    unsigned* keyj;
    unsigned* keyi;
    int* jid;
};

// Slot in cell j and sort distance of the j list's k-th entry (sweep order: ascending
// distance, the reverse of the copied keys).
__device__ __forceinline__ int jlist_loc(const WarpSlice& W, int nj, int k) { return W.keyj[nj - 1 - k] >> 16; }
__device__ __forceinline__ int jlist_dist(const WarpSlice& W, int nj, int k) {
    return W.keyj[nj - 1 - k] & 0xffff;
}

__device__ __forceinline__ WarpSlice warp_slice(unsigned char* smem_raw, int cap, int warp, int stages, int stage) {
    unsigned char* wp = smem_raw + (size_t)warp * warp_slice_bytes(cap, stages);
    WarpSlice W;
    W.bar = reinterpret_cast<uint64_t*>(wp) + stage;
    wp += 16;
    W.js = reinterpret_cast<float4*>(wp); wp += (size_t)cap * 16;
    W.jid = reinterpret_cast<int*>(wp); wp += (size_t)cap * 4;
    wp += (size_t)stage * cap * 28;
    W.xraw = reinterpret_cast<float4*>(wp); wp += (size_t)cap * 16;
    W.fj = W.xraw;
    W.pidraw = reinterpret_cast<int*>(wp); wp += (size_t)cap * 4;
    W.keyj = reinterpret_cast<unsigned*>(wp); wp += (size_t)cap * 4;
    W.keyi = reinterpret_cast<unsigned*>(wp);
    return W;
}

// Pops the next task index of this warp from the device queue (`batch` entries at a time);
// returns -1 when the queue is drained.
struct QueueCursor {
    int q = 0, qend = 0;
};

__device__ __forceinline__ int pop_task(const TunedParams& T, QueueCursor& c, int nq, int batch, int lane) {
    if (c.q >= c.qend) {
        int q0 = 0;
        if (lane == 0) q0 = atomicAdd(T.counter, batch);
        c.q = __shfl_sync(0xffffffffu, q0, 0);
        c.qend = min(c.q + batch, nq);
        if (c.q >= nq) return -1;
    }
    return T.order[c.q++];
}

// A task as the warp sees it.
struct TaskDesc {
    int t;                  // task index, -1 when the queue is drained
    TaskRec tr;
    int ni, nj, si, sj;     // particle counts and first slots of cells i and j
};

// Pops the next task and starts loading its description, spread over the lanes (lane k
// holds field k: t, ci, cj, sid, dbits, ni, nj, si, sj), so that the dependent loads stay
// in flight while the warp works on the current task.
__device__ __forceinline__ int desc_fetch(const Params& P, const TunedParams& T, QueueCursor& c, int nq, int batch,
                                          int lane) {
    const int t = pop_task(T, c, nq, batch, lane);
    if (t < 0) return -1;
    if (lane == 0) return t;
    if (lane <= 4) return reinterpret_cast<const int*>(P.tasks + t)[lane - 1];
    if (lane <= 8) {
        const int cell = (lane & 1) ? P.tasks[t].ci : P.tasks[t].cj;    // lanes 5, 7: ci; 6, 8: cj
        return lane <= 6 ? P.ccount[cell] : P.cstart[cell];
    }
    return 0;
}

__device__ __forceinline__ TaskDesc desc_get(int f) {
    constexpr unsigned FULL = 0xffffffffu;
    TaskDesc d;
    d.t = __shfl_sync(FULL, f, 0);
    d.tr.ci = __shfl_sync(FULL, f, 1);
    d.tr.cj = __shfl_sync(FULL, f, 2);
    d.tr.sid = __shfl_sync(FULL, f, 3);
    d.tr.dbits = __shfl_sync(FULL, f, 4);
    d.ni = __shfl_sync(FULL, f, 5);
    d.nj = __shfl_sync(FULL, f, 6);
    d.si = __shfl_sync(FULL, f, 7);
    d.sj = __shfl_sync(FULL, f, 8);
    return d;
}

// A task with pairs to sweep that fits the slice.
__device__ __forceinline__ bool desc_runnable(const TaskDesc& d, int cap) {
    const bool self = d.tr.sid < 0;
    return d.ni > 0 && d.nj > 0 && !(self && d.ni < 2) && d.ni + 8 <= cap && d.nj + 8 <= cap;
}

__device__ __forceinline__ bool desc_oversized(const TaskDesc& d, int cap) {
    return d.ni + 8 > cap || d.nj + 8 > cap;
}

// A task of at most 32 candidate pairs (a self task of at most 8 particles, a pair task with
// n_i n_j <= 32: the vapour of an inhomogeneous system), evaluated one pair per lane
// without staging (tiny_task).
__device__ __forceinline__ bool desc_tiny(const TaskDesc& d) {
    return d.tr.sid < 0 ? d.ni <= 8 : d.ni * d.nj <= 32;
}

// A task that is staged in the warp's slice and swept: every runnable one, except the tiny
// ones when the kernel has the tiny path (TINY) and the system asks for it (P.tiny).
template <bool TINY>
__device__ __forceinline__ bool desc_staged(const Params& P, const TaskDesc& d, int cap) {
    if constexpr (TINY) return desc_runnable(d, cap) && !(P.tiny && desc_tiny(d));
    return desc_runnable(d, cap);
}

// Lane 0 issues the bulk copies of task d into the staging buffer of W: the j cell's
// positions and ids, and for pair tasks the sort keys of both cells along the task's axis.
__device__ __forceinline__ void issue_copies(const Params& P, const TaskDesc& d, const WarpSlice& W, int lane) {
    __syncwarp();                      // earlier generic accesses of the buffer are done
    if (lane == 0) {
        const bool self = d.tr.sid < 0;
        const int padi = (d.ni + 3) & ~3, padj = (d.nj + 3) & ~3;
        // test hook: no arrival and no copy, so the wait on W.bar runs out with no
        // transaction pending on the barrier
        if (c_skip_copies) return;
        fence_proxy_async();
        mbar_arrive_expect_tx(W.bar, self ? (uint32_t)padj * 20u : (uint32_t)padj * 24u + (uint32_t)padi * 4u);
        bulk_g2s(W.xraw, P.xq + d.sj, padj * 16, W.bar);
        bulk_g2s(W.pidraw, P.pid + d.sj, padj * 4, W.bar);
        if (!self) {
            bulk_g2s(W.keyj, P.keys + 13 * (size_t)d.sj + (size_t)d.tr.sid * padj, padj * 4, W.bar);
            bulk_g2s(W.keyi, P.keys + 13 * (size_t)d.si + (size_t)d.tr.sid * padi, padi * 4, W.bar);
        }
    }
}

// After the copies of d landed in W: the j list in sweep order (ascending sort distance
// for pair tasks, storage order for self tasks) and zeroed j partial forces.
__device__ __forceinline__ void build_jlist(const TaskDesc& d, const WarpSlice& W, int lane) {
    const bool self = d.tr.sid < 0;
    const int nj = d.nj;
    if (!self) {
        for (int k = lane; k < nj; k += 32) {
            const unsigned key = W.keyj[nj - 1 - k];
            const int loc = key >> 16;
            W.js[k] = W.xraw[loc];
            W.jid[k] = W.pidraw[loc];
        }
    } else {
        for (int k = lane; k < nj; k += 32) W.js[k] = W.xraw[k];
    }
    __syncwarp();
    const int nout = self ? d.ni : nj;
    for (int k = lane; k < nout; k += 32) W.fj[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncwarp();
}

// The task loop of a worker warp: pops tasks, stages them (STAGES = 2: the next task's
// copies are issued before the current task is swept) and calls
// sweep(task, slice, t_start) for every task with pairs to sweep, or tiny(task, slice,
// t_start) for a task of at most 32 candidate pairs, which is not staged.  Returns when the
// queue is drained or a bulk copy timed out (status set).
//
// With many tasks per worker warp (at least 16), or two stages, the next task is popped
// and its description loaded while the current one is swept.  With few, large tasks the
// warp pops only when it is done: a task reserved early would wait behind the current one
// while other warps run dry at the end of the queue.
template <int STAGES, bool TINY, typename Sweep, typename Tiny>
__device__ __forceinline__ void run_tasks(const Params& P, const TunedParams& T, unsigned char* smem_raw, int cap,
                                          int nw, unsigned& status, Sweep&& sweep, Tiny&& tiny) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nq = T.qcount ? *T.qcount : P.ntasks;
    const int workers = (int)gridDim.x * nw;
    // queue entries per pop: up to 8 (16 and more measured slower on small-cell systems)
    const int batch = max(1, min(8, nq / (8 * workers)));
    const bool early = STAGES == 2 || nq >= 16 * workers;     // warp-uniform
    QueueCursor cur;
    unsigned phases = 0;               // bit s: parity of completed phases of stage s
    int s = 0;
    TaskDesc d = desc_get(desc_fetch(P, T, cur, nq, batch, lane));
    bool issued = d.t >= 0 && desc_staged<TINY>(P, d, cap);
    if (issued) issue_copies(P, d, warp_slice(smem_raw, cap, warp, STAGES, s), lane);
    while (d.t >= 0) {
        long long t_start = 0;
        if (T.task_clock && lane == 0) t_start = clock64();
        int fnext = early ? desc_fetch(P, T, cur, nq, batch, lane) : 0;
        if (!issued) {                 // empty, single-particle, oversized or tiny task
            if (!early) fnext = desc_fetch(P, T, cur, nq, batch, lane);
            // No copy of this warp is in flight here (only the task marked issued has
            // copies), so the tiny path may use the slice's j arrays.
            if (desc_oversized(d, cap)) status |= kStatusCellOverflow;
            else if (TINY && desc_runnable(d, cap)) tiny(d, warp_slice(smem_raw, cap, warp, STAGES, s), t_start);
            d = desc_get(fnext);
            issued = d.t >= 0 && desc_staged<TINY>(P, d, cap);
            if (issued) issue_copies(P, d, warp_slice(smem_raw, cap, warp, STAGES, s), lane);
            continue;
        }
        const WarpSlice W = warp_slice(smem_raw, cap, warp, STAGES, s);
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(W.bar, (phases >> s) & 1))) {
            // A copy that has not landed after a whole bounded wait: flag it, give the copies
            // still in flight a second bounded wait (their destination is this warp's
            // slice, which must outlive them), and stop popping tasks.  These are the only
            // copies this warp can have in flight: with two staging buffers the next task's
            // copies are issued only after the current task's have landed.  If even the
            // second wait runs out, the block may exit with a copy outstanding; the status
            // makes the evaluation fail.
            status |= kStatusCopyTimeout;
            mbar_wait_bounded(W.bar, (phases >> s) & 1);
            return;
        }
        phases ^= 1u << s;
        build_jlist(d, W, lane);
        bool n_issued = false;
        if (STAGES == 2) {
            const TaskDesc n = desc_get(fnext);
            if (n.t >= 0 && desc_staged<TINY>(P, n, cap)) {
                issue_copies(P, n, warp_slice(smem_raw, cap, warp, STAGES, s ^ 1), lane);
                n_issued = true;
            }
        }
        // Only the lane-spread description of the next task (one register) stays live
        // through the sweep.
        sweep(d, W, t_start);
        if (!early) fnext = desc_fetch(P, T, cur, nq, batch, lane);
        d = desc_get(fnext);
        if (STAGES == 2) {
            s ^= 1;
            issued = n_issued;
        } else {
            issued = d.t >= 0 && desc_staged<TINY>(P, d, cap);
            if (issued) issue_copies(P, d, warp_slice(smem_raw, cap, warp, STAGES, s), lane);
        }
    }
}

// Length of the sorted j prefix lane's particle i (sort distance di) interacts with: j
// whose distance is below dmaxdist - dnshift + di (src/runner_dopair.c:606-612).  keyj
// holds cell j's keys in descending distance order; the prefix is its tail.
__device__ __forceinline__ int sorted_prefix(const unsigned* __restrict__ keyj, int nj, int lim) {
    int lo = 0, hi = nj;          // first key (descending) whose distance is below lim
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((int)(keyj[mid] & 0xffff) >= lim) lo = mid + 1; else hi = mid;
    }
    return nj - lo;
}

// The pair interaction of lane's particle i with j at sweep position k: cutoff test on the
// exactly rounded r^2, potential lookup, exclusion test, table evaluation.  Returns the
// force contribution on j (w) and adds -w to the i force; counts candidates, pairs and
// excluded pairs.
// The exclusions of lane's particle i, for the sweep: its bit mask of partners at id
// offsets -16..16, the range [lo, lo + span] of offsets the mask covers (an empty range
// when the mask is empty), and its CSR list of farther partners.
struct IExcl {
    int pid;
    unsigned emask;
    int lo, span;
    int exlo, exhi;
};

__device__ __forceinline__ IExcl load_iexcl(const Params& P, int pid) {
    IExcl x;
    x.pid = pid;
    x.emask = P.emask[pid];
    x.exlo = P.exoff[pid];
    x.exhi = P.exoff[pid + 1];
    if (x.emask) {                     // bit b <-> offset b - 16 (b < 16) or b - 15 (b >= 16)
        const int bl = __ffs(x.emask) - 1, bh = 31 - __clz(x.emask);
        x.lo = bl < 16 ? bl - 16 : bl - 15;
        x.span = (bh < 16 ? bh - 16 : bh - 15) - x.lo;
    } else {
        x.lo = 0x40000000;             // no offset d satisfies 0 <= d - lo <= span
        x.span = 0;
    }
    return x;
}

__device__ __forceinline__ IExcl no_iexcl() {
    IExcl x;
    x.pid = 0; x.emask = 0u; x.lo = 0x40000000; x.span = 0; x.exlo = 0; x.exhi = 0;
    return x;
}

// 1/sqrt(x) from the hardware approximation (x is never denormal here: r^2 of two
// particles is at least ~1e-3 nm^2), refined by the caller.
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Candidates a lane examines in a strip: the sweep positions k < len of its column
// (stride = lanes per row of j: 4 in the 8 x 4 tile, 1 with 32 i per warp).
__device__ __forceinline__ unsigned strip_candidates(int len, int col, int stride) {
    return len > col ? (unsigned)((len - col + stride - 1) / stride) : 0u;
}

template <bool HAS_EXCL, int TAB>
__device__ __forceinline__ void pair_force(const Params& P, const SharedTables& S, const float4 xj,
                                           const int* __restrict__ jids, int k, bool act,
                                           float pix, float piy, float piz, int prow, float qi, const IExcl& ix,
                                           float cut2, float& fix, float& fiy, float& fiz,
                                           float& wx, float& wy, float& wz, double& e_task, unsigned& npairs,
                                           unsigned& nexcl, bool& any_acc) {
    constexpr unsigned FULL = 0xffffffffu;
    const float dx = __fsub_rn(pix, xj.x), dy = __fsub_rn(piy, xj.y), dz = __fsub_rn(piz, xj.z);
    const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    int pot = 0;
    if (TAB != kTabOne) pot = act ? S.potidx[prow + __float_as_int(xj.w)] : -1;
    bool acc = act && (pot >= 0 || (TAB == kTabGlobal && P.ep_pot >= 0)) && r2 <= cut2;
    if (HAS_EXCL) {
        // One window test per candidate; the mask bit or the list is looked at only for
        // ids inside the particle's exclusion window (or when it has far partners).
        const int d = jids[k] - ix.pid;
        const bool inwin = (unsigned)(d - ix.lo) <= (unsigned)ix.span;
        if (acc && (inwin || ix.exhi > ix.exlo)) {
            bool ex;
            if (inwin)
                ex = (ix.emask >> (d + 16 - (d > 0))) & 1u;
            else {
                ex = false;
                for (int qx = ix.exlo; qx < ix.exhi; ++qx) ex |= (P.exlist[qx] == ix.pid + d);
            }
            if (ex) { acc = false; ++nexcl; }
        }
    }
    wx = 0.f; wy = 0.f; wz = 0.f;
    if (__any_sync(FULL, acc)) {
        any_acc = true;
        if (acc) {
            // 1/r: rsqrt plus one Newton step; r: r2/r corrected by one residual step,
            // which gives the correctly rounded square root (the water energy is ~250x
            // smaller than the sum of |pair energies|, so unbiased 1-ulp errors in r would
            // show at 1e-6).
            float rinv = rsqrt_approx(r2);
            rinv = fmaf(-0.5f * rinv, fmaf(r2 * rinv, rinv, -1.0f), rinv);
            float r = r2 * rinv;
            r = fmaf(fmaf(-r, r, r2), 0.5f * rinv, r);
            float e, f;
            if (TAB == kTabGlobal) {
                e = 0.f;
                f = 0.f;
                if (pot >= 0) {
                    const float4 info = S.potinfo[pot];
                    eval_table_fast(S.coef, info, __float_as_int(info.w) >> 20, r, rinv, e, f);
                }
                if (P.ep_pot >= 0) {            // + q_i q_j ep(r)
                    const float qq = qi * P.qid[jids[k]];
                    const float4 info = S.potinfo[P.ep_pot];
                    float ee, fe;
                    eval_table_fast(S.coef, info, __float_as_int(info.w) >> 20, r, rinv, ee, fe);
                    e = fmaf(qq, ee, e);
                    f = fmaf(qq, fe, f);
                }
            } else {
                const float4 info = TAB == kTabOne ? S.one : S.potinfo[pot];
                eval_table_fast(S.coef, info, __float_as_int(info.w) >> 20, r, rinv, e, f);
            }
            wx = f * dx; wy = f * dy; wz = f * dz;
            fix -= wx; fiy -= wy; fiz -= wz;
            e_task += (double)e;
            ++npairs;
        }
    }
}

// Exact warp sum of 64-bit fixed-point values: three 32-bit reductions (the low and middle
// 16 bits, the signed high 32 bits) and a recombination; the same total in any lane order.
// Per-lane values stay far below 2^62, so the high words sum without overflow.
__device__ __forceinline__ long long warp_sum_fixed(long long v) {
    constexpr unsigned FULL = 0xffffffffu;
    const unsigned lo = __reduce_add_sync(FULL, (unsigned)(v & 0xffff));
    const unsigned mid = __reduce_add_sync(FULL, (unsigned)((v >> 16) & 0xffff));
    const int hi = __reduce_add_sync(FULL, (int)(v >> 32));
    return ((long long)hi << 32) + ((long long)mid << 16) + (long long)lo;
}

// End of a task: the j partial forces (and, for self tasks, the i forces) go to the
// fixed-point accumulators, the j side of the virial is added, the warp sums energy and
// virial exactly in fixed point and lane 0 adds them to the i cell (per-task clock64 record).
__device__ __forceinline__ void finish_task(const Params& P, const TunedParams& T, const WarpSlice& W,
                                            const TaskDesc& d, double e_task, double v_task, long long t_start,
                                            unsigned& status, int lane) {
    constexpr unsigned FULL = 0xffffffffu;
    const bool self = d.tr.sid < 0;
    const int nout = self ? d.ni : d.nj;
    __syncwarp();
    for (int k = lane; k < nout; k += 32) {
        const float4 a = W.fj[k];
        const float4 xk = W.js[k];
        v_task += (double)xk.x * a.x + (double)xk.y * a.y + (double)xk.z * a.z;
        unsigned long long* fp = P.force + 3 * (size_t)(self ? (d.si + k) : (d.sj + jlist_loc(W, d.nj, k)));
        atomic_add_fixed(fp + 0, to_fixed(a.x, status));
        atomic_add_fixed(fp + 1, to_fixed(a.y, status));
        atomic_add_fixed(fp + 2, to_fixed(a.z, status));
    }
    // Energy and virial: each lane's FP64 partial to fixed point, summed exactly.
    const long long e_fix = warp_sum_fixed(__double2ll_rn(e_task * kEnergyScale));
    const long long v_fix = warp_sum_fixed(__double2ll_rn(-v_task * kEnergyScale));
    if (lane == 0) {
        atomicAdd(&P.cell_epot[d.tr.ci], (unsigned long long)e_fix);
        atomicAdd(P.cell_vir ? &P.cell_vir[d.tr.ci] : &P.acc[kAccVirial], (unsigned long long)v_fix);
        if (T.task_clock) {
            T.task_clock[2 * d.t] = t_start;
            T.task_clock[2 * d.t + 1] = clock64();
            T.task_sm[d.t] = (int)smid();
        }
    }
    __syncwarp();
}

// Warp totals of the counters, one atomic per warp.
__device__ __forceinline__ void flush_counters(const Params& P, unsigned npairs, unsigned nexcl, unsigned ncand,
                                               unsigned status, int lane) {
    constexpr unsigned FULL = 0xffffffffu;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        npairs += __shfl_xor_sync(FULL, npairs, o);
        nexcl += __shfl_xor_sync(FULL, nexcl, o);
        ncand += __shfl_xor_sync(FULL, ncand, o);
        status |= __shfl_xor_sync(FULL, status, o);
    }
    if (lane == 0) {
        if (npairs) atomicAdd(&P.acc[kAccPairs], (unsigned long long)npairs);
        if (nexcl) atomicAdd(&P.acc[kAccExcl], (unsigned long long)nexcl);
        if (ncand) atomicAdd(&P.acc[kAccCand], (unsigned long long)ncand);
        if (status) atomicOr(&P.acc[kAccStatus], (unsigned long long)status);
    }
}




// A tiny task (desc_tiny): one candidate pair per lane, the two particles read from global
// memory, no staging and no sort keys.  All n_i n_j pairs of a pair task are tested: the
// sorted sweep's bound is conservative (a j past a particle's sorted prefix lies beyond the
// cutoff), so the accepted pairs are the same.  Each accepted pair's force goes to both
// particles in fixed point (-w on i, +w on j; order-independent like every other partial),
// the pair energy and virial d.w into the task's FP64 sums as in finish_task.  Self tasks
// map lane l to the pair (i, j), j < i, of the triangle's rows i = 1, 2, ...
template <bool HAS_EXCL, int TAB>
__device__ __forceinline__ void tiny_task(const Params& P, const TunedParams& T, const SharedTables& S,
                                          const TaskDesc& d, const WarpSlice& W, long long t_start, int mt,
                                          unsigned& npairs, unsigned& nexcl, unsigned& ncand, unsigned& status,
                                          int lane) {
    const bool self = d.tr.sid < 0;
    const int ni = d.ni, nj = d.nj;
    const int npair = self ? ni * (ni - 1) / 2 : ni * nj;
    const bool act = lane < npair;
    int i = 0, j = 0;
    if (act) {
        if (self) {
            int l = lane;
            i = 1;
            while (l >= i) { l -= i; ++i; }
            j = l;
        } else {
            i = lane / nj;
            j = lane - i * nj;
        }
    }
    const int slot_i = d.si + i, slot_j = (self ? d.si : d.sj) + j;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f), xj = xi;
    IExcl ix = no_iexcl();
    float qi = 0.f;
    if (act) {
        xi = P.xq[slot_i];
        xj = P.xq[slot_j];
        if (HAS_EXCL || TAB == kTabGlobal) {
            const int pi = P.pid[slot_i];
            if (HAS_EXCL) ix = load_iexcl(P, pi);
            if (TAB == kTabGlobal && P.ep_pot >= 0) qi = P.qid[pi];
            // slot `lane` of the j-id list (pair_force reads the partner's id there); with
            // cap < 32 it runs past the list into this warp's own staging area (32 ids need
            // 4 cap + 28 cap >= 128 bytes there, cap >= 9), which has no copy in flight
            // while a tiny task runs
            W.jid[lane] = P.pid[slot_j];
        }
    }
    __syncwarp();
    const float4 sh = self ? make_float4(0.f, 0.f, 0.f, 0.f) : P.tshift[d.t];
    const float pix = __fsub_rn(xi.x, sh.x), piy = __fsub_rn(xi.y, sh.y), piz = __fsub_rn(xi.z, sh.z);
    const int prow = __float_as_int(xi.w) * mt;
    float fix = 0.f, fiy = 0.f, fiz = 0.f, wx, wy, wz;
    double e_task = 0.0;
    bool any_acc = false;
    pair_force<HAS_EXCL, TAB>(P, S, xj, W.jid, lane, act, pix, piy, piz, prow, qi, ix, self ? P.cutoff2s : P.cutoff2,
                              fix, fiy, fiz, wx, wy, wz, e_task, npairs, nexcl, any_acc);
    ncand += act ? 1u : 0u;
    const float dx = __fsub_rn(pix, xj.x), dy = __fsub_rn(piy, xj.y), dz = __fsub_rn(piz, xj.z);
    const double v_pair = (double)dx * wx + (double)dy * wy + (double)dz * wz;      // 0 unless accepted
    if (act) {
        const long long fx = to_fixed(wx, status), fy = to_fixed(wy, status), fz = to_fixed(wz, status);
        unsigned long long* fpi = P.force + 3 * (size_t)slot_i;
        unsigned long long* fpj = P.force + 3 * (size_t)slot_j;
        atomic_add_fixed(fpi + 0, -fx);
        atomic_add_fixed(fpi + 1, -fy);
        atomic_add_fixed(fpi + 2, -fz);
        atomic_add_fixed(fpj + 0, fx);
        atomic_add_fixed(fpj + 1, fy);
        atomic_add_fixed(fpj + 2, fz);
    }
    const long long e_fix = warp_sum_fixed(__double2ll_rn(e_task * kEnergyScale));
    const long long v_fix = warp_sum_fixed(__double2ll_rn(v_pair * kEnergyScale));
    if (lane == 0) {
        atomicAdd(&P.cell_epot[d.tr.ci], (unsigned long long)e_fix);
        atomicAdd(P.cell_vir ? &P.cell_vir[d.tr.ci] : &P.acc[kAccVirial], (unsigned long long)v_fix);
        if (T.task_clock) {
            T.task_clock[2 * d.t] = t_start;
            T.task_clock[2 * d.t + 1] = clock64();
            T.task_sm[d.t] = (int)smid();
        }
    }
    __syncwarp();
}

// Sum of (x, y, z) over the 4 columns of a row of the 8 x 4 lane tile, scattered: column 0
// gets the x sum, 1 the y sum, 2 the z sum, each as (c0 + c1) + (c2 + c3).
__device__ __forceinline__ float reduce_scatter_cols3(float x, float y, float z, int col) {
    constexpr unsigned FULL = 0xffffffffu;
    const bool b0 = col & 1, b1 = col & 2;
    const float a0 = (b0 ? y : x) + __shfl_xor_sync(FULL, b0 ? x : y, 1);
    const float a1 = (b0 ? 0.f : z) + __shfl_xor_sync(FULL, b0 ? z : 0.f, 1);
    return (b1 ? a1 : a0) + __shfl_xor_sync(FULL, b1 ? a0 : a1, 2);
}

// Warp reduce-scatter of two window steps over the 8 i rows of the 8 x 4 lane tile: the
// lane of row q holds, for its column, the sum over the 8 rows of step q & 1.  Fixed order
// of additions.
__device__ __forceinline__ float reduce_scatter_rows2(const float (&v)[2], int lane) {
    constexpr unsigned FULL = 0xffffffffu;
    const bool b2 = lane & 4;
    const float send = b2 ? v[0] : v[1];
    const float keep = b2 ? v[1] : v[0];
    float a = keep + __shfl_xor_sync(FULL, send, 4);
    a += __shfl_xor_sync(FULL, a, 8);
    a += __shfl_xor_sync(FULL, a, 16);
    return a;
}

// Warp reduce-scatter over the 8 i rows of the 8 x 4 lane tile (lane = 4 * row + column):
// each lane holds WIN values (window steps m); afterwards the lane of row q holds, for its
// column, the sum over the 8 rows of step m = q (WIN = 8) or m = q & 3 (WIN = 4).  Fixed
// order of additions.
template <int WIN>
__device__ __forceinline__ float reduce_scatter_rows(const float (&v)[WIN], int lane) {
    constexpr unsigned FULL = 0xffffffffu;
    const bool b2 = lane & 4, b3 = lane & 8, b4 = lane & 16;
    if constexpr (WIN == 8) {
        float a[4], c[2];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const float send = b2 ? v[2 * m] : v[2 * m + 1];
            const float keep = b2 ? v[2 * m + 1] : v[2 * m];
            a[m] = keep + __shfl_xor_sync(FULL, send, 4);
        }
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const float send = b3 ? a[2 * m] : a[2 * m + 1];
            const float keep = b3 ? a[2 * m + 1] : a[2 * m];
            c[m] = keep + __shfl_xor_sync(FULL, send, 8);
        }
        const float send = b4 ? c[0] : c[1];
        const float keep = b4 ? c[1] : c[0];
        return keep + __shfl_xor_sync(FULL, send, 16);
    } else {
        float a[2];
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const float send = b2 ? v[2 * m] : v[2 * m + 1];
            const float keep = b2 ? v[2 * m + 1] : v[2 * m];
            a[m] = keep + __shfl_xor_sync(FULL, send, 4);
        }
        const float send = b3 ? a[0] : a[1];
        const float keep = b3 ? a[1] : a[0];
        float c = keep + __shfl_xor_sync(FULL, send, 8);
        c += __shfl_xor_sync(FULL, c, 16);
        return c;
    }
}

// Persistent worker warps, one i particle per lane: every warp pops whole tasks from the
// device queue, stages them in its own shared-memory slice and sweeps the i particles in
// chunks of 32; the j contributions of WIN consecutive sweep steps are kept per lane and
// summed across the warp by one reduce-scatter.  Warps never wait for each other.
//
// WIN (4 or 8): sweep steps per reduce-scatter; 8 halves the shuffles per step but holds
// twice the registers.  STAGES (1 or 2): staging buffers per warp.
template <int NW, bool HAS_EXCL, int TAB, int WIN, int STAGES, int TPSM, bool TINY>
__global__ void __launch_bounds__(NW * 32, TPSM / (NW * 32)) sweep_tuned(TunedParams T, int cap) {
    static_assert(WIN == 4 || WIN == 8, "sweep window of 4 or 8 steps");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr unsigned FULL = 0xffffffffu;
    const Params& P = T.p;
    if (step_aborted(P.abort)) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = P.max_type;
    const SharedTables S = stage_tables<NW, STAGES, TAB>(P, smem_raw, cap);
    if (lane < STAGES) {
        mbar_init(warp_slice(smem_raw, cap, warp, STAGES, lane).bar, 1);
        mbar_fence_init();
    }
    __syncthreads();

    unsigned npairs = 0, nexcl = 0, ncand = 0, status = 0;
    run_tasks<STAGES, TINY>(P, T, smem_raw, cap, NW, status, [&](const TaskDesc& d, const WarpSlice& W, long long t_start) {
        const bool self = d.tr.sid < 0;
        const int ni = d.ni, nj = d.nj, si = d.si;
        const float4* __restrict__ jpos = W.js;
        const int* __restrict__ jids = self ? W.pidraw : W.jid;
        const float4 sh = self ? make_float4(0.f, 0.f, 0.f, 0.f) : P.tshift[d.t];
        const float cut2 = self ? P.cutoff2s : P.cutoff2;
        const int dnshift = task_dnshift(d.tr);
        const int dmaxdist = task_dmax_skin(P, d.tr);
        double e_task = 0.0, v_task = 0.0;
        const int nchunks = (ni + 31) >> 5;
        const int jd0 = self ? 0 : jlist_dist(W, nj, 0);

        for (int ch = 0; ch < nchunks; ++ch) {
            const int ii = ch * 32 + lane;
            bool valid = ii < ni;
            int loc = ii, len = 0;
            if (self) {
                len = valid ? ii : 0;                       // pairs j < i
            } else {
                const unsigned key = valid ? W.keyi[ii] : 0u;
                loc = key >> 16;
                const int di = key & 0xffff;
                if (!P.unsorted) valid = valid && (jd0 + dnshift - di <= dmaxdist);
                if (!__any_sync(FULL, valid)) break;        // later chunks lie farther from cell j
                if (valid) len = P.unsorted ? nj : sorted_prefix(W.keyj, nj, dmaxdist - dnshift + di);
            }
            const int kmax = (int)__reduce_max_sync(FULL, (unsigned)len);
            float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
            IExcl ix = no_iexcl();
            float qi = 0.f;
            if (valid) {
                xi = self ? W.js[loc] : P.xq[si + loc];
                if (HAS_EXCL) ix = load_iexcl(P, self ? W.pidraw[loc] : P.pid[si + loc]);
                if (TAB == kTabGlobal && P.ep_pot >= 0) qi = P.qid[self ? W.pidraw[loc] : P.pid[si + loc]];
            }
            const float pix = __fsub_rn(xi.x, sh.x), piy = __fsub_rn(xi.y, sh.y), piz = __fsub_rn(xi.z, sh.z);
            const int prow = __float_as_int(xi.w) * mt;
            ncand += strip_candidates(len, 0, 1);
            float fix = 0.f, fiy = 0.f, fiz = 0.f;
            for (int k0 = 0; k0 < kmax; k0 += WIN) {
                float vx[WIN], vy[WIN], vz[WIN];
                bool any_acc = false;
#pragma unroll
                for (int m = 0; m < WIN; ++m) {
                    const int k = k0 + m;
                    pair_force<HAS_EXCL, TAB>(P, S, jpos[k], jids, k, k < len, pix, piy, piz, prow, qi, ix, cut2,
                                                  fix, fiy, fiz, vx[m], vy[m], vz[m], e_task, npairs, nexcl,
                                                  any_acc);
                }
                if (any_acc) {
                    float tx, ty, tz;
                    if constexpr (WIN == 8) {
                        tx = reduce_scatter8(vx, lane);
                        ty = reduce_scatter8(vy, lane);
                        tz = reduce_scatter8(vz, lane);
                    } else {
                        tx = reduce_scatter4(vx, lane);
                        ty = reduce_scatter4(vy, lane);
                        tz = reduce_scatter4(vz, lane);
                    }
                    if (lane < WIN && k0 + lane < kmax) {
                        float4 a = W.fj[k0 + lane];
                        a.x += tx; a.y += ty; a.z += tz;
                        W.fj[k0 + lane] = a;
                    }
                }
            }
            __syncwarp();
            if (valid) {
                if (self) {
                    float4 a = W.fj[loc];
                    a.x += fix; a.y += fiy; a.z += fiz;
                    W.fj[loc] = a;
                } else {
                    // virial, i side: sum over pairs of r_ij.F_ij = sum_i (x_i - shift).F_i + sum_j x_j.F_j
                    v_task += (double)pix * fix + (double)piy * fiy + (double)piz * fiz;
                    unsigned long long* fp = P.force + 3 * (size_t)(si + loc);
                    atomic_add_fixed(fp + 0, to_fixed(fix, status));
                    atomic_add_fixed(fp + 1, to_fixed(fiy, status));
                    atomic_add_fixed(fp + 2, to_fixed(fiz, status));
                }
            }
            __syncwarp();
        }
        finish_task(P, T, W, d, e_task, v_task, t_start, status, lane);
    }, [&](const TaskDesc& d, const WarpSlice& W, long long t_start) {
        tiny_task<HAS_EXCL, TAB>(P, T, S, d, W, t_start, mt, npairs, nexcl, ncand, status, lane);
    });
    flush_counters(P, npairs, nexcl, ncand, status, lane);
}

// Persistent worker warps on an 8 x 4 lane tile: lane 4 q + c sweeps i particle q of a
// strip of 8 consecutive i (in sort order) against the j of its column c, j = k0 + 4 m + c.
// Eight i of neighbouring sort distance have similar sorted-prefix lengths, so far fewer
// lane slots fall outside a particle's prefix than with 32 i per warp (on ~20-particle
// cells about 0.6 of the lane slots carry a candidate instead of ~0.25).  The j
// contributions of WIN steps (4 WIN consecutive j) are summed over the 8 rows by one
// reduce-scatter, after which the 32 (or 16) lanes write distinct j; the i forces are
// summed over the 4 columns at the end of the strip.
template <int NW, bool HAS_EXCL, int TAB, int WIN, int STAGES, int TPSM, bool TINY>
__global__ void __launch_bounds__(NW * 32, TPSM / (NW * 32)) sweep_tiled(TunedParams T, int cap) {
    static_assert(WIN == 4 || WIN == 8, "sweep window of 4 or 8 steps");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr unsigned FULL = 0xffffffffu;
    const Params& P = T.p;
    if (step_aborted(P.abort)) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = lane >> 2, col = lane & 3;
    const int mt = P.max_type;
    const SharedTables S = stage_tables<NW, STAGES, TAB>(P, smem_raw, cap);
    if (lane < STAGES) {
        mbar_init(warp_slice(smem_raw, cap, warp, STAGES, lane).bar, 1);
        mbar_fence_init();
    }
    __syncthreads();

    unsigned npairs = 0, nexcl = 0, ncand = 0, status = 0;
    run_tasks<STAGES, TINY>(P, T, smem_raw, cap, NW, status, [&](const TaskDesc& d, const WarpSlice& W, long long t_start) {
        const bool self = d.tr.sid < 0;
        const int ni = d.ni, nj = d.nj, si = d.si;
        const float4* __restrict__ jpos = W.js;
        const int* __restrict__ jids = self ? W.pidraw : W.jid;
        const int tshift_t = d.t;        // the task's shift is read at each strip, not held
        const float cut2 = self ? P.cutoff2s : P.cutoff2;
        const int dnshift = task_dnshift(d.tr);
        const int dmaxdist = task_dmax_skin(P, d.tr);
        double e_task = 0.0, v_task = 0.0;
        const int nstrips = (ni + 7) >> 3;
        const int jd0 = self ? 0 : jlist_dist(W, nj, 0);
        // Pair tasks: every fourth strip, each lane finds the slot, validity and sorted-prefix
        // length of one i of the next 32 (one search per lane instead of one per row and
        // strip, where the row's four lanes repeat it); the strips take their rows' values
        // from those lanes.
        int c_loc = 0, c_len = 0, c_valid = 0;

        for (int st = 0; st < nstrips; ++st) {
            const int ii = st * 8 + row;
            bool valid = ii < ni;
            int loc = ii, len = 0;
            if (self) {
                len = valid ? ii : 0;                       // pairs j < i
            } else {
                if ((st & 3) == 0) {                        // warp-uniform
                    const int ic = st * 8 + lane;
                    bool v = ic < ni;
                    const unsigned key = v ? W.keyi[ic] : 0u;
                    c_loc = key >> 16;
                    const int di = key & 0xffff;
                    if (!P.unsorted) v = v && (jd0 + dnshift - di <= dmaxdist);
                    c_valid = v;
                    c_len = v ? (P.unsorted ? nj : sorted_prefix(W.keyj, nj, dmaxdist - dnshift + di)) : 0;
                }
                const int src = ((st & 3) << 3) + row;
                valid = __shfl_sync(FULL, c_valid, src) != 0;
                if (!__any_sync(FULL, valid)) break;        // later strips lie farther from cell j
                loc = __shfl_sync(FULL, c_loc, src);
                len = __shfl_sync(FULL, c_len, src);
            }
            const int kmax = (int)__reduce_max_sync(FULL, (unsigned)len);
            float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
            IExcl ix = no_iexcl();
            float qi = 0.f;
            if (valid) {
                xi = self ? W.js[loc] : P.xq[si + loc];
                if (HAS_EXCL) ix = load_iexcl(P, self ? W.pidraw[loc] : P.pid[si + loc]);
                if (TAB == kTabGlobal && P.ep_pot >= 0) qi = P.qid[self ? W.pidraw[loc] : P.pid[si + loc]];
            }
            const float4 sh = self ? make_float4(0.f, 0.f, 0.f, 0.f) : P.tshift[tshift_t];
            const float pix = __fsub_rn(xi.x, sh.x), piy = __fsub_rn(xi.y, sh.y), piz = __fsub_rn(xi.z, sh.z);
            const int prow = __float_as_int(xi.w) * mt;
            ncand += strip_candidates(len, col, 4);
            float fix = 0.f, fiy = 0.f, fiz = 0.f;
            for (int k0 = 0; k0 < kmax; k0 += 4 * WIN) {
                if (WIN == 4 && kmax - k0 <= 8) {
                    // The last window, with at most two live steps (the usual case on cells
                    // of ~20 particles, where a strip sweeps ~10 j): two steps and a
                    // reduce-scatter of two values instead of four.
                    float vx[2], vy[2], vz[2];
                    bool any_acc = false;
#pragma unroll
                    for (int m = 0; m < 2; ++m) {
                        if (k0 + 4 * m < kmax) {             // warp-uniform
                            const int k = k0 + 4 * m + col;
                            pair_force<HAS_EXCL, TAB>(P, S, jpos[k], jids, k, k < len, pix, piy, piz, prow, qi,
                                                          ix, cut2, fix, fiy, fiz, vx[m], vy[m], vz[m], e_task,
                                                          npairs, nexcl, any_acc);
                        } else {
                            vx[m] = 0.f; vy[m] = 0.f; vz[m] = 0.f;
                        }
                    }
                    if (any_acc) {
                        const float tx = reduce_scatter_rows2(vx, lane);
                        const float ty = reduce_scatter_rows2(vy, lane);
                        const float tz = reduce_scatter_rows2(vz, lane);
                        const int k = k0 + 4 * (row & 1) + col;
                        if (row < 2 && k < kmax) {
                            float4 a = W.fj[k];
                            a.x += tx; a.y += ty; a.z += tz;
                            W.fj[k] = a;
                        }
                    }
                    break;
                }
                float vx[WIN], vy[WIN], vz[WIN];
                bool any_acc = false;
#pragma unroll
                for (int m = 0; m < WIN; ++m) {
                    if (k0 + 4 * m < kmax) {                 // warp-uniform
                        const int k = k0 + 4 * m + col;
                        pair_force<HAS_EXCL, TAB>(P, S, jpos[k], jids, k, k < len, pix, piy, piz, prow, qi, ix,
                                                      cut2, fix, fiy, fiz, vx[m], vy[m], vz[m], e_task, npairs,
                                                      nexcl, any_acc);
                    } else {
                        vx[m] = 0.f; vy[m] = 0.f; vz[m] = 0.f;
                    }
                }
                if (any_acc) {
                    const float tx = reduce_scatter_rows<WIN>(vx, lane);
                    const float ty = reduce_scatter_rows<WIN>(vy, lane);
                    const float tz = reduce_scatter_rows<WIN>(vz, lane);
                    const int k = k0 + 4 * (WIN == 8 ? row : (row & 3)) + col;
                    if ((WIN == 8 || row < 4) && k < kmax) {
                        float4 a = W.fj[k];
                        a.x += tx; a.y += ty; a.z += tz;
                        W.fj[k] = a;
                    }
                }
            }
            // i force: sum over the 4 columns, scattered so that column c holds component c
            // ((c0 + c1) + (c2 + c3) for every component, the same float sums in any lane)
            const float fi = reduce_scatter_cols3(fix, fiy, fiz, col);
            __syncwarp();
            if (valid && col < 3) {
                if (self) {
                    float* a = &W.fj[loc].x + col;
                    *a += fi;
                } else {
                    const float pc = col == 0 ? pix : (col == 1 ? piy : piz);
                    v_task += (double)pc * fi;
                    atomic_add_fixed(P.force + 3 * (size_t)(si + loc) + col, to_fixed(fi, status));
                }
            }
            __syncwarp();
        }
        finish_task(P, T, W, d, e_task, v_task, t_start, status, lane);
    }, [&](const TaskDesc& d, const WarpSlice& W, long long t_start) {
        tiny_task<HAS_EXCL, TAB>(P, T, S, d, W, t_start, mt, npairs, nexcl, ncand, status, lane);
    });
    flush_counters(P, npairs, nexcl, ncand, status, lane);
}

}  // namespace nb
