// Tuned sweep: persistent CTAs over a device task queue (sm_100a).
//
// Differences from the plain sweep (nb_kernels.cuh), none of which changes the pair set:
//  * persistent CTAs (a multiple of the SM count) pull task indices from a device queue
//    (an atomic counter over a permutation of the task list, so a scheduler can order the
//    queue, e.g. longest task first); the tables are staged into shared memory once per CTA;
//  * two shared-memory stages: while a CTA sweeps one task, the TMA bulk copies of the next
//    task's cells are already in flight;
//  * r = r2 * rsqrt(r2), f = U'(r) * (1/halfwidth) * rsqrt(r2): one MUFU op instead of an
//    IEEE square root and division (the cutoff test still uses the exactly rounded r2);
//  * Newton's third law through a register reduce-scatter: each lane keeps its j
//    contributions of 8 consecutive sweep steps and the warp sums them with 9 shuffles per
//    component (xor 1, 2, 4 exchange halves; xor 8, 16 add), after which lane m holds the
//    warp total for step m.  The order of additions is fixed, so task partials stay
//    independent of scheduling;
//  * the j record carries its sort distance and type in one 16-byte shared-memory word;
//  * energy and virial are summed in float over an 8-step window and in double beyond;
//  * optional per-task clock64 records (start, end, SM) for the learned scheduler.
#pragma once
#include "nb_kernels.cuh"

namespace nb {

struct TunedParams {
    Params p;
    const int* order;            // queue: task indices in scheduling order
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
    b += (size_t)cap * 4 * 2;                        // jid, jloc
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

// Fast table evaluation: index as the reference computes it (rounded ops), r from rsqrt.
__device__ __forceinline__ void eval_table_fast(const float* __restrict__ coef, float4 info, int nmax, float r,
                                                float rinv, float& e, float& f) {
    float t = __fadd_rn(info.x, __fmul_rn(r, __fadd_rn(info.y, __fmul_rn(r, info.z))));
    int ind = __float2int_rz(fmaxf(0.0f, t));
    ind = min(ind, nmax);
    const float4* c = reinterpret_cast<const float4*>(coef + __float_as_int(info.w) + 8 * ind);
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

template <int NW, bool HAS_EXCL>
__global__ void __launch_bounds__(NW * 32) sweep_tuned(TunedParams T, int cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr unsigned FULL = 0xffffffffu;
    const Params& P = T.p;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mt = P.max_type;

    // ---- shared memory carve-up
    unsigned char* sp = smem_raw;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sp);
    int* qslot = reinterpret_cast<int*>(sp + 16);
    sp += 64;
    unsigned char* const stage_base = sp;
    sp += 2 * tuned_stage_bytes(cap);
    float4* js = reinterpret_cast<float4*>(sp); sp += (size_t)cap * 16;     // cap includes 8 spare rows
    float4* fis = reinterpret_cast<float4*>(sp); sp += (size_t)cap * 16;
    int* jid = reinterpret_cast<int*>(sp); sp += (size_t)cap * 4;
    int* jloc = reinterpret_cast<int*>(sp); sp += (size_t)cap * 4;
    float4* fj = reinterpret_cast<float4*>(sp); sp += (size_t)NW * cap * 16;
    float4* potinfo = reinterpret_cast<float4*>(sp); sp += (size_t)P.npots * 16;
    float* coef = reinterpret_cast<float*>(sp); sp += (size_t)((P.ncoef + 3) & ~3) * 4;
    int* potn = reinterpret_cast<int*>(sp); sp += (size_t)((P.npots + 3) & ~3) * 4;
    int* potidx = reinterpret_cast<int*>(sp); sp += (size_t)((mt * mt + 3) & ~3) * 4;
    double* wred = reinterpret_cast<double*>(sp); sp += (size_t)NW * 16;
    unsigned long long* cred = reinterpret_cast<unsigned long long*>(sp);

    for (int k = tid; k < P.ncoef; k += NW * 32) coef[k] = P.coef[k];
    for (int k = tid; k < P.npots; k += NW * 32) { potinfo[k] = P.potinfo[k]; potn[k] = P.potn[k]; }
    for (int k = tid; k < mt * mt; k += NW * 32) potidx[k] = P.potidx[k];
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0) {
        const int q0 = atomicAdd(T.counter, 1);
        qslot[0] = q0;
        if (q0 < P.ntasks) issue_task(P, T.order[q0], stage_at(stage_base, cap, 0), &bars[0]);
    }
    __syncthreads();

    unsigned npairs = 0, nexcl = 0, ncand = 0, status = 0;
    for (int it = 0;; ++it) {
        const int s = it & 1;
        const int q = qslot[s];
        if (q >= P.ntasks) break;
        const int t = T.order[q];
        if (tid == 0) {                       // prefetch the next task into the other stage
            const int q1 = atomicAdd(T.counter, 1);
            qslot[s ^ 1] = q1;
            if (q1 < P.ntasks) issue_task(P, T.order[q1], stage_at(stage_base, cap, s ^ 1), &bars[s ^ 1]);
        }
        const TaskRec tr = P.tasks[t];
        const bool self = tr.sid < 0;
        const int ni = P.ccount[tr.ci], nj = P.ccount[tr.cj];
        const int si = P.cstart[tr.ci], sj = P.cstart[tr.cj];
        const bool ok = mbar_wait_bounded(&bars[s], (it >> 1) & 1);
        if (__syncthreads_or(!ok)) {
            status |= kStatusCopyTimeout;
            if (tid == 0) mbar_wait_bounded(&bars[s ^ 1], ((it + 1) >> 1) & 1);
            break;
        }
        if (ni == 0 || nj == 0 || (self && ni < 2)) {
            __syncthreads();
            continue;
        }
        if (ni + 8 > cap || nj + 8 > cap) {   // host sizes cap; guard anyway
            status |= kStatusCellOverflow;
            __syncthreads();
            continue;
        }
        long long t_start = 0;
        if (tid == 0 && T.task_clock) t_start = clock64();
        const Stage S = stage_at(stage_base, cap, s);

        // j records in ascending projected distance: xyz, w = type | dist << 16.
        if (!self) {
            for (int k = tid; k < nj; k += NW * 32) {
                const unsigned key = S.keyj[nj - 1 - k];
                const int loc = key >> 16;
                float4 x = S.xj[loc];
                x.w = __int_as_float((__float_as_int(x.w) & 0xffff) | (int)((key & 0xffffu) << 16));
                js[k] = x;
                jid[k] = S.pidj[loc];
                jloc[k] = loc;
            }
        } else {
            for (int k = tid; k < nj; k += NW * 32) {
                js[k] = S.xj[k];
                jid[k] = S.pidj[k];
            }
        }
        for (int k = tid; k < NW * nj; k += NW * 32) {
            const int w = k / nj, kk = k - w * nj;
            fj[w * cap + kk] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncthreads();

        const float4 sh = self ? make_float4(0.f, 0.f, 0.f, 0.f) : P.tshift[t];
        const float cut2 = self ? P.cutoff2s : P.cutoff2;
        const int dnshift = tr.dnshift;
        float4* myfj = fj + warp * cap;
        double e_task = 0.0, v_task = 0.0;
        const int nchunks = (ni + 31) >> 5;
        const int jd0 = self ? 0 : (int)((unsigned)__float_as_int(js[0].w) >> 16);

        for (int ch = warp; ch < nchunks; ch += NW) {
            const int ii = ch * 32 + lane;
            bool valid = ii < ni;
            int loc = ii, di = 0;
            if (!self) {
                const unsigned key = valid ? S.keyi[ii] : 0u;
                loc = key >> 16;
                di = key & 0xffff;
                if (!P.unsorted) valid = valid && (jd0 + dnshift - di <= P.dmaxdist);
                if (!__any_sync(FULL, valid)) break;
            }
            float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
            int pidi = -1, exlo = 0, exhi = 0;
            unsigned emask = 0u;
            if (valid) {
                xi = self ? S.xj[loc] : S.xi[loc];
                if (HAS_EXCL) {
                    pidi = self ? S.pidj[loc] : S.pidi[loc];
                    emask = P.emask[pidi];
                    exlo = P.exoff[pidi];
                    exhi = P.exoff[pidi + 1];
                }
            }
            const float pix = __fsub_rn(xi.x, sh.x), piy = __fsub_rn(xi.y, sh.y), piz = __fsub_rn(xi.z, sh.z);
            const int prow = (__float_as_int(xi.w) & 0xffff) * mt;
            const int lim = P.dmaxdist - dnshift + di;
            const int kend = self ? min(ch * 32 + 32, ni) - 1 : nj;
            float fix = 0.f, fiy = 0.f, fiz = 0.f;
            for (int k0 = 0; k0 < kend; k0 += 8) {
                if (!self && !P.unsorted) {
                    const int dk = (int)((unsigned)__float_as_int(js[k0].w) >> 16);
                    if (!__any_sync(FULL, valid && dk < lim)) break;   // distances only grow with k
                }
                float vx[8], vy[8], vz[8];
                float ew = 0.f, vw = 0.f;
                bool any_acc = false;
#pragma unroll
                for (int m = 0; m < 8; ++m) {
                    const int k = k0 + m;
                    const float4 xj = js[k];
                    const int wbits = __float_as_int(xj.w);
                    const int dk = (int)((unsigned)wbits >> 16);
                    const bool act = valid && k < kend && (self ? (k < ii) : (P.unsorted || dk < lim));
                    const float dx = __fsub_rn(pix, xj.x), dy = __fsub_rn(piy, xj.y), dz = __fsub_rn(piz, xj.z);
                    const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
                    const int pot = act ? potidx[prow + (wbits & 0xffff)] : -1;
                    bool acc = act && pot >= 0 && r2 <= cut2;
                    ncand += act;
                    if (HAS_EXCL && acc && excluded_pair(pidi, jid[k], emask, exlo, exhi, P.exlist)) {
                        acc = false;
                        ++nexcl;
                    }
                    float wx = 0.f, wy = 0.f, wz = 0.f;
                    if (__any_sync(FULL, acc)) {
                        any_acc = true;
                        if (acc) {
                            const float rinv = rsqrtf(r2);
                            float e, f;
                            eval_table_fast(coef, potinfo[pot], potn[pot], r2 * rinv, rinv, e, f);
                            wx = f * dx; wy = f * dy; wz = f * dz;
                            fix -= wx; fiy -= wy; fiz -= wz;
                            ew += e;
                            vw = fmaf(f, r2, vw);
                            ++npairs;
                        }
                    }
                    vx[m] = wx; vy[m] = wy; vz[m] = wz;
                }
                if (any_acc) {
                    const float tx = reduce_scatter8(vx, lane);
                    const float ty = reduce_scatter8(vy, lane);
                    const float tz = reduce_scatter8(vz, lane);
                    if (lane < 8 && k0 + lane < kend) {
                        float4 a = myfj[k0 + lane];
                        a.x += tx; a.y += ty; a.z += tz;
                        myfj[k0 + lane] = a;
                    }
                    e_task += (double)ew;
                    v_task += (double)vw;
                }
            }
            if (valid) {
                if (self) {
                    fis[loc] = make_float4(fix, fiy, fiz, 0.f);
                } else {
                    unsigned long long* fp = P.force + 3 * (size_t)(si + loc);
                    atomic_add_fixed(fp + 0, to_fixed(fix, status));
                    atomic_add_fixed(fp + 1, to_fixed(fiy, status));
                    atomic_add_fixed(fp + 2, to_fixed(fiz, status));
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            e_task += __shfl_xor_sync(FULL, e_task, o);
            v_task += __shfl_xor_sync(FULL, v_task, o);
        }
        if (lane == 0) {
            wred[2 * warp] = e_task;
            wred[2 * warp + 1] = v_task;
        }
        __syncthreads();

        const int nout = self ? ni : nj;
        for (int k = tid; k < nout; k += NW * 32) {
            float4 a = self ? fis[k] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                const float4 b = fj[w * cap + k];
                a.x += b.x; a.y += b.y; a.z += b.z;
            }
            unsigned long long* fp = P.force + 3 * (size_t)(self ? (si + k) : (sj + jloc[k]));
            atomic_add_fixed(fp + 0, to_fixed(a.x, status));
            atomic_add_fixed(fp + 1, to_fixed(a.y, status));
            atomic_add_fixed(fp + 2, to_fixed(a.z, status));
        }
        if (tid == 0) {
            double e = 0.0, v = 0.0;
            for (int w = 0; w < NW; ++w) { e += wred[2 * w]; v += wred[2 * w + 1]; }
            atomicAdd(&P.cell_epot[tr.ci], (unsigned long long)__double2ll_rn(e * kEnergyScale));
            atomicAdd(&P.acc[kAccVirial], (unsigned long long)__double2ll_rn(v * kEnergyScale));
            if (T.task_clock) {
                T.task_clock[2 * t] = t_start;
                T.task_clock[2 * t + 1] = clock64();
                T.task_sm[t] = (int)smid();
            }
        }
        __syncthreads();
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
