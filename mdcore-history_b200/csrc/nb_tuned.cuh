// Tuned sweep: persistent CTAs over a device task queue (sm_100a).
//
// Differences from the plain sweep (nb_kernels.cuh), none of which changes the pair set:
//  * persistent CTAs (a multiple of the SM count) pull task indices from a device queue
//    (an atomic counter over a permutation of the task list, so a scheduler can order the
//    queue, e.g. longest task first); the tables are staged into shared memory once per CTA;
//  * two shared-memory stages: while a CTA sweeps one task, the TMA bulk copies of the next
//    task's cells are already in flight;
//  * f = U'(r) * (1/halfwidth) * rsqrt(r2) with one Newton step instead of an IEEE
//    division (r itself stays correctly rounded, and the cutoff test uses the exactly
//    rounded r2);
//  * Newton's third law through a register reduce-scatter: each lane keeps its j
//    contributions of 8 consecutive sweep steps and the warp sums them with 9 shuffles per
//    component (xor 1, 2, 4 exchange halves; xor 8, 16 add), after which lane m holds the
//    warp total for step m.  The order of additions is fixed, so task partials stay
//    independent of scheduling;
//  * the j record carries its sort distance and type in one 16-byte shared-memory word;
//  * energy is summed per pair in double (float partial sums of cancelling Coulomb terms
//    would cost ~1e-6 of the total); the virial per particle and task from the partial
//    forces: sum over pairs of r_ij.F_ij = sum_i (x_i - shift).F_i + sum_j x_j.F_j;
//  * optional per-task clock64 records (start, end, SM) for the learned scheduler.
#pragma once
#include "nb_kernels.cuh"

// Resident threads per SM the register allocation of sweep_tuned is sized for (launch
// bounds): 640 threads = 20 warps leaves ~100 registers per thread.
#ifndef MDB_TUNED_THREADS_PER_SM
#define MDB_TUNED_THREADS_PER_SM 640
#endif

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

// Shared-memory layout of one stage (raw copies of the two cells of a task).
struct Stage {
    float4 *xi, *xj;
    int *pidi, *pidj;
    unsigned *keyi, *keyj;
};

__host__ __device__ inline size_t tuned_stage_bytes(int cap) { return (size_t)cap * 48; }

__host__ __device__ inline size_t tuned_smem_bytes(int cap, int nw, int ncoef, int npots, int mt) {
    size_t b = 64;                                   // 2 mbarriers + queue slots
    b += 2 * tuned_stage_bytes(cap);                 // double-buffered raw cells
    b += (size_t)cap * 16 * 2;                       // js (sorted j, dist|type in w), fi
    b += (size_t)cap * 4 * 3;                        // jid, jloc, jdist
    b += (size_t)nw * cap * 16;                      // per-warp j partial forces
    b += (size_t)npots * 16;
    b += (size_t)((ncoef + 3) & ~3) * 4;
    b += (size_t)((npots + 3) & ~3) * 4;
    b += (size_t)((mt * mt + 3) & ~3) * 4;
    b += (size_t)nw * 16 + (size_t)nw * 32;
    return b;
}

__device__ __forceinline__ Stage stage_at(unsigned char* base, int cap, int s) {
    unsigned char* p = base + (size_t)s * tuned_stage_bytes(cap);
    Stage st;
    st.xi = reinterpret_cast<float4*>(p); p += (size_t)cap * 16;
    st.xj = reinterpret_cast<float4*>(p); p += (size_t)cap * 16;
    st.pidi = reinterpret_cast<int*>(p); p += (size_t)cap * 4;
    st.pidj = reinterpret_cast<int*>(p); p += (size_t)cap * 4;
    st.keyi = reinterpret_cast<unsigned*>(p); p += (size_t)cap * 4;
    st.keyj = reinterpret_cast<unsigned*>(p);
    return st;
}

template <bool SELF>
__device__ __forceinline__ uint32_t stage_bytes(int padi, int padj) {
    return SELF ? (uint32_t)padj * 20u : (uint32_t)(padi + padj) * 24u;
}

// Thread 0: issue the bulk copies of task t into stage st.
__device__ __forceinline__ void issue_task(const Params& P, int t, const Stage& st, uint64_t* bar) {
    const TaskRec tr = P.tasks[t];
    const int ni = P.ccount[tr.ci], nj = P.ccount[tr.cj];
    const int padi = (ni + 3) & ~3, padj = (nj + 3) & ~3;
    const int si = P.cstart[tr.ci], sj = P.cstart[tr.cj];
    const bool self = tr.sid < 0;
    fence_proxy_async();
    if (ni == 0 || nj == 0) {          // nothing to copy; complete the phase by arrival alone
        mbar_arrive_expect_tx(bar, 0);
        return;
    }
    mbar_arrive_expect_tx(bar, self ? stage_bytes<true>(padi, padj) : stage_bytes<false>(padi, padj));
    bulk_g2s(st.xj, P.xq + sj, padj * 16, bar);
    bulk_g2s(st.pidj, P.pid + sj, padj * 4, bar);
    if (!self) {
        bulk_g2s(st.keyj, P.keys + 13 * (size_t)sj + (size_t)tr.sid * padj, padj * 4, bar);
        bulk_g2s(st.xi, P.xq + si, padi * 16, bar);
        bulk_g2s(st.pidi, P.pid + si, padi * 4, bar);
        bulk_g2s(st.keyi, P.keys + 13 * (size_t)si + (size_t)tr.sid * padi, padi * 4, bar);
    }
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
// that the 4- or 8-step sweep windows may read past the end of the j list).
__host__ __device__ inline size_t warp_slice_bytes(int cap) { return 16 + (size_t)cap * 56; }

__host__ __device__ inline size_t warps_smem_bytes(int cap, int nw, int ncoef, int npots, int mt) {
    size_t b = (size_t)nw * warp_slice_bytes(cap);
    b += (size_t)npots * 16;
    b += (size_t)((ncoef + 3) & ~3) * 4;
    b += (size_t)((npots + 3) & ~3) * 4;
    b += (size_t)((mt * mt + 3) & ~3) * 4;
    return b;
}

// Persistent worker warps: every warp pops whole tasks from the device queue, stages the
// j cell (positions, ids, sort keys) and the i cell's sort keys in its own shared-memory
// slice with TMA bulk copies, sweeps all i chunks of the task itself and writes the
// task's forces and energy.  Warps never wait for each other.
//
// WIN (4 or 8) is the number of consecutive sweep steps whose j contributions a lane keeps
// in registers before the warp reduce-scatter: 8 halves the shuffles per step but holds
// twice the registers.
template <int NW, bool HAS_EXCL, bool ONE_POT, int WIN>
__global__ void __launch_bounds__(NW * 32, MDB_TUNED_THREADS_PER_SM / (NW * 32)) sweep_tuned(TunedParams T, int cap) {
    static_assert(WIN == 4 || WIN == 8, "sweep window of 4 or 8 steps");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr unsigned FULL = 0xffffffffu;
    const Params& P = T.p;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mt = P.max_type;

    // ---- shared tables (once per block), then the warp's slice
    unsigned char* sp = smem_raw + (size_t)NW * warp_slice_bytes(cap);
    float4* potinfo = reinterpret_cast<float4*>(sp); sp += (size_t)P.npots * 16;
    float* coef = reinterpret_cast<float*>(sp); sp += (size_t)((P.ncoef + 3) & ~3) * 4;
    int* potn = reinterpret_cast<int*>(sp); sp += (size_t)((P.npots + 3) & ~3) * 4;
    int* potidx = reinterpret_cast<int*>(sp);
    for (int k = tid; k < P.ncoef; k += NW * 32) coef[k] = P.coef[k];
    for (int k = tid; k < P.npots; k += NW * 32) { potinfo[k] = P.potinfo[k]; potn[k] = P.potn[k]; }
    for (int k = tid; k < mt * mt; k += NW * 32) potidx[k] = P.potidx[k];

    unsigned char* wp = smem_raw + (size_t)warp * warp_slice_bytes(cap);
    uint64_t* bar = reinterpret_cast<uint64_t*>(wp); wp += 16;
    float4* xraw = reinterpret_cast<float4*>(wp); wp += (size_t)cap * 16;   // j cell as copied
    float4* js = reinterpret_cast<float4*>(wp); wp += (size_t)cap * 16;     // j cell, sweep order
    float4* fj = xraw;            // j (and self) forces, once js has been built from xraw
    int* pidraw = reinterpret_cast<int*>(wp); wp += (size_t)cap * 4;
    unsigned* keyj = reinterpret_cast<unsigned*>(wp); wp += (size_t)cap * 4;
    unsigned* keyi = reinterpret_cast<unsigned*>(wp); wp += (size_t)cap * 4;
    int* jid = reinterpret_cast<int*>(wp); wp += (size_t)cap * 4;
    int* jloc = reinterpret_cast<int*>(wp); wp += (size_t)cap * 4;
    int* jdist = reinterpret_cast<int*>(wp);
    if (lane == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    __syncthreads();

    unsigned npairs = 0, nexcl = 0, ncand = 0, status = 0;
    unsigned phase = 0;                   // completed phases of this warp's mbarrier
    const int nq = T.qcount ? *T.qcount : P.ntasks;
    // Queue entries are taken `batch` at a time: one when there are few tasks per worker
    // (load balance), up to 16 on systems with millions of small tasks (the queue head is
    // a single atomic counter).
    const int workers = gridDim.x * NW;
    const int batch = max(1, min(16, nq / (8 * workers)));
    int q = 0, qend = 0;
    for (;;) {
        if (q >= qend) {
            int q0 = 0;
            if (lane == 0) q0 = atomicAdd(T.counter, batch);
            q = __shfl_sync(FULL, q0, 0);
            qend = min(q + batch, nq);
            if (q >= nq) break;
        }
        const int t = T.order[q++];
        const TaskRec tr = P.tasks[t];
        const bool self = tr.sid < 0;
        const int ni = P.ccount[tr.ci], nj = P.ccount[tr.cj];
        if (ni == 0 || nj == 0 || (self && ni < 2)) continue;
        if (ni + 8 > cap || nj + 8 > cap) { status |= kStatusCellOverflow; continue; }
        const int si = P.cstart[tr.ci], sj = P.cstart[tr.cj];
        const int padi = (ni + 3) & ~3, padj = (nj + 3) & ~3;
        long long t_start = 0;
        __syncwarp();
        if (lane == 0) {
            if (T.task_clock) t_start = clock64();
            fence_proxy_async();
            mbar_arrive_expect_tx(bar, self ? (uint32_t)padj * 20u : (uint32_t)padj * 24u + (uint32_t)padi * 4u);
            bulk_g2s(xraw, P.xq + sj, padj * 16, bar);
            bulk_g2s(pidraw, P.pid + sj, padj * 4, bar);
            if (!self) {
                bulk_g2s(keyj, P.keys + 13 * (size_t)sj + (size_t)tr.sid * padj, padj * 4, bar);
                bulk_g2s(keyi, P.keys + 13 * (size_t)si + (size_t)tr.sid * padi, padi * 4, bar);
            }
        }
        const int nout = self ? ni : nj;
        if (!__all_sync(FULL, mbar_wait_bounded(bar, phase & 1))) {
            status |= kStatusCopyTimeout;
            mbar_wait_bounded(bar, phase & 1);   // second bounded chance for copies in flight
            break;
        }
        ++phase;
        if (!self) {
            for (int k = lane; k < nj; k += 32) {
                const unsigned key = keyj[nj - 1 - k];
                const int loc = key >> 16;
                js[k] = xraw[loc];
                jid[k] = pidraw[loc];
                jloc[k] = loc;
                jdist[k] = key & 0xffff;
            }
        } else {
            for (int k = lane; k < nj; k += 32) js[k] = xraw[k];
        }
        __syncwarp();
        for (int k = lane; k < nout; k += 32) fj[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncwarp();
        const float4* __restrict__ jpos = js;
        const int* __restrict__ jids = self ? pidraw : jid;

        const float4 sh = self ? make_float4(0.f, 0.f, 0.f, 0.f) : P.tshift[t];
        const float cut2 = self ? P.cutoff2s : P.cutoff2;
        const int dnshift = task_dnshift(tr);
        const int dmaxdist = task_dmax(tr);
        double e_task = 0.0, v_task = 0.0;
        const int nchunks = (ni + 31) >> 5;
        const int jd0 = self ? 0 : jdist[0];

        for (int ch = 0; ch < nchunks; ++ch) {
            const int ii = ch * 32 + lane;
            bool valid = ii < ni;
            int loc = ii, len = 0;
            if (self) {
                len = valid ? ii : 0;                       // pairs j < i
            } else {
                const unsigned key = valid ? keyi[ii] : 0u;
                loc = key >> 16;
                const int di = key & 0xffff;
                if (!P.unsorted) valid = valid && (jd0 + dnshift - di <= dmaxdist);
                if (!__any_sync(FULL, valid)) break;        // later chunks lie farther from cell j
                if (valid) {
                    if (P.unsorted) {
                        len = nj;
                    } else {                                // j with dist < lim form a prefix
                        const int lim = dmaxdist - dnshift + di;
                        int lo = 0, hi = nj;
                        while (lo < hi) {
                            const int mid = (lo + hi) >> 1;
                            if (jdist[mid] < lim) lo = mid + 1; else hi = mid;
                        }
                        len = lo;
                    }
                }
            }
            const int kmax = (int)__reduce_max_sync(FULL, (unsigned)len);
            float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
            int pidi = 0, exlo = 0, exhi = 0;
            unsigned emask = 0u;
            if (valid) {
                xi = self ? js[loc] : P.xq[si + loc];
                if (HAS_EXCL) {
                    pidi = self ? pidraw[loc] : P.pid[si + loc];
                    emask = P.emask[pidi];
                    exlo = P.exoff[pidi];
                    exhi = P.exoff[pidi + 1];
                }
            }
            const float pix = __fsub_rn(xi.x, sh.x), piy = __fsub_rn(xi.y, sh.y), piz = __fsub_rn(xi.z, sh.z);
            const int prow = __float_as_int(xi.w) * mt;
            float fix = 0.f, fiy = 0.f, fiz = 0.f;
            for (int k0 = 0; k0 < kmax; k0 += WIN) {
                float vx[WIN], vy[WIN], vz[WIN];
                bool any_acc = false;
#pragma unroll
                for (int m = 0; m < WIN; ++m) {
                    const int k = k0 + m;
                    const float4 xj = jpos[k];
                    const bool act = k < len;
                    const float dx = __fsub_rn(pix, xj.x), dy = __fsub_rn(piy, xj.y), dz = __fsub_rn(piz, xj.z);
                    const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
                    int pot = 0;
                    if (!ONE_POT) pot = act ? potidx[prow + __float_as_int(xj.w)] : -1;
                    bool acc = act && pot >= 0 && r2 <= cut2;
                    ncand += act;
                    if (HAS_EXCL && acc) {
                        const int d = jids[k] - pidi;
                        bool ex;
                        if ((unsigned)(d + 16) <= 32u)
                            ex = (emask >> (d + 16 - (d > 0))) & (d != 0);
                        else {
                            ex = false;
                            for (int qx = exlo; qx < exhi; ++qx) ex |= (P.exlist[qx] == pidi + d);
                        }
                        if (ex) { acc = false; ++nexcl; }
                    }
                    float wx = 0.f, wy = 0.f, wz = 0.f;
                    if (__any_sync(FULL, acc)) {
                        any_acc = true;
                        if (acc) {
                            // 1/r: rsqrt plus one Newton step; r: r2/r corrected by one
                            // residual step, which gives the correctly rounded square root
                            // (the water energy is ~250x smaller than the sum of |pair
                            // energies|, so unbiased 1-ulp errors in r would show at 1e-6).
                            float rinv = rsqrtf(r2);
                            rinv = fmaf(-0.5f * rinv, fmaf(r2 * rinv, rinv, -1.0f), rinv);
                            float r = r2 * rinv;
                            r = fmaf(fmaf(-r, r, r2), 0.5f * rinv, r);
                            float e, f;
                            const float4 info = potinfo[pot];
                            eval_table_fast(coef, info, __float_as_int(info.w) >> 20, r, rinv, e, f);
                            wx = f * dx; wy = f * dy; wz = f * dz;
                            fix -= wx; fiy -= wy; fiz -= wz;
                            e_task += (double)e;
                            ++npairs;
                        }
                    }
                    vx[m] = wx; vy[m] = wy; vz[m] = wz;
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
                        float4 a = fj[k0 + lane];
                        a.x += tx; a.y += ty; a.z += tz;
                        fj[k0 + lane] = a;
                    }
                }
            }
            __syncwarp();
            if (valid) {
                if (self) {
                    float4 a = fj[loc];
                    a.x += fix; a.y += fiy; a.z += fiz;
                    fj[loc] = a;
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

        for (int k = lane; k < nout; k += 32) {
            const float4 a = fj[k];
            const float4 xk = jpos[k];
            v_task += (double)xk.x * a.x + (double)xk.y * a.y + (double)xk.z * a.z;
            unsigned long long* fp = P.force + 3 * (size_t)(self ? (si + k) : (sj + jloc[k]));
            atomic_add_fixed(fp + 0, to_fixed(a.x, status));
            atomic_add_fixed(fp + 1, to_fixed(a.y, status));
            atomic_add_fixed(fp + 2, to_fixed(a.z, status));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            e_task += __shfl_xor_sync(FULL, e_task, o);
            v_task += __shfl_xor_sync(FULL, v_task, o);
        }
        if (lane == 0) {
            atomicAdd(&P.cell_epot[tr.ci], (unsigned long long)__double2ll_rn(e_task * kEnergyScale));
            atomicAdd(P.cell_vir ? &P.cell_vir[tr.ci] : &P.acc[kAccVirial],
                      (unsigned long long)__double2ll_rn(-v_task * kEnergyScale));
            if (T.task_clock) {
                T.task_clock[2 * t] = t_start;
                T.task_clock[2 * t + 1] = clock64();
                T.task_sm[t] = (int)smid();
            }
        }
    }

    // Counters: warp sums, one atomic per warp.
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

}  // namespace nb
