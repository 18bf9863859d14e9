// Device-side data layout and small PTX helpers of the nonbonded engine (sm_100a).
//
// Particle data in HBM is cell-major: cell c owns the slots [start[c], start[c]+count[c])
// of every per-particle array, with start[c] a multiple of 4 so that every cell's block
// of 4-byte and 16-byte records starts on a 16-byte boundary and can be moved into shared
// memory with one cp.async.bulk (TMA bulk copy) per array.
//
//   xq[slot]    float4  {x, y, z} relative to the cell origin (the reference's FPTYPE
//                       cell-local coordinates, src/space.c:421-423) and w = type (int bits)
//   pid[slot]   int     global particle id
//   keys[13*start[c] + sid*cpad[c] + k]   uint32 sort keys of cell c along direction sid,
//                       (k_local << 16) | projected distance (src/runner_dosort.c:148-149),
//                       sorted by descending distance; cpad[c] = count rounded up to 4.
//   force[3*slot+k]  int64 fixed-point force, 2^24 units per kJ/mol/nm.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nb {

constexpr float kForceScale = 16777216.0f;          // 2^24
constexpr double kEnergyScale = 4294967296.0;       // 2^32
constexpr int kMaxPartsPerCell = 1024;
constexpr int kSpinLimit = 1 << 22;                 // bounded waits: default polls per wait
// Polls per bounded wait of the sweeps (engine_cuda_setspin; kSpinLimit by default), and a
// test hook (engine_cuda_copytimeout_test): when set, the sweeps neither arrive on their
// staging mbarriers nor issue a copy, so every such wait (a phase that nothing completes)
// runs out and reports kStatusCopyTimeout with nothing in flight and no transaction
// pending on any barrier.
__constant__ int c_spin_limit = kSpinLimit;
__constant__ int c_skip_copies = 0;

// Status bits of the device status word.
enum : unsigned {
    kStatusOk = 0,
    kStatusCopyTimeout = 1u,
    kStatusCellOverflow = 2u,
    kStatusTableIndex = 4u,
    kStatusForceOverflow = 8u,
    kStatusNonFinite = 64u,        // a particle's position or velocity stopped being finite
    kStatusLayout = 128u,          // a caller-given cell start or count breaks the slot layout
};

// Accumulator slots (unsigned long long each).
enum { kAccEpot = 0, kAccVirial, kAccPairs, kAccExcl, kAccCand, kAccStatus, kAccCount = 8 };

struct TaskRec {        // one cell pair (or self) task
    int ci, cj, sid;              // sid = -1 for self tasks
    int dbits;                    // discretised shift norm | sweep bound << 16 (pair tasks)
};

// The reference's discretised |shift| (src/runner_dopair.c:593-597) and projection bound
// dmaxdist (src/runner_dopair.c:583), per task because replicas of a batch have their own
// cell sizes.
__host__ __device__ __forceinline__ int task_dnshift(const TaskRec& r) { return r.dbits & 0xffff; }
__host__ __device__ __forceinline__ int task_dmax(const TaskRec& r) { return (int)((unsigned)r.dbits >> 16); }

struct Params {
    const float4* xq;
    const int* pid;
    const unsigned* keys;
    const int* cstart;
    const int* ccount;
    unsigned long long* force;
    unsigned long long* acc;
    unsigned long long* cell_epot;  // per-cell fixed-point energy (2^32 units per kJ/mol)
    unsigned long long* cell_vir;   // per-cell fixed-point virial, or nullptr: summed in acc
    const TaskRec* tasks;
    const float4* tshift;       // per-task shift of cell j relative to cell i
    int ntasks;
    const float* coef;          // concatenated tables, (n+1)*8 floats each
    const float4* potinfo;      // {alpha0, alpha1, alpha2, int_bits(offset of chunk 0)}
    const int* potn;            // n of each table (largest valid chunk index)
    const int* potidx;          // max_type*max_type -> table index or -1
    int max_type, npots, ncoef;
    const unsigned* emask;      // by particle id: excluded partners at id offsets +-1..16
    const int* exoff;           // by particle id: CSR of the other excluded partners
    const int* exlist;
    float cutoff2;              // pair tasks: float(cutoff)^2 in float (src/runner_dopair.c:578-579)
    float cutoff2s;             // self tasks: float(cutoff^2) (src/runner_dopair.c:896)
    int unsorted;               // 1: sweep every candidate (engine_flag_unsorted)
    const unsigned long long* abort;   // device-resident steps: nonzero = skip this launch
    // Explicit electrostatics (engine_setexplepot): every pair within the cutoff that is not
    // excluded also interacts through q_i q_j ep(r), ep being table ep_pot (-1: none), q by
    // particle id.  tab_global: the tables are read from global memory (through L1) instead
    // of being staged in shared memory (many type pairs).
    const float* qid;
    int ep_pot;
    int tab_global;
    // 1: the persistent sweeps evaluate tasks of at most 32 candidate pairs one pair per lane
    // without staging (systems of few particles per cell); 0: every task is staged.
    int tiny = 0;
    // Plain form only: when set, each task's partial forces are added to these floats with
    // float atomics (FP32 accumulation, order-dependent, as the reference's GPU runner adds
    // them) instead of to the fixed-point accumulators.
    float* force32 = nullptr;
    // Verlet skin (resident steps with engine_flag_verlet): the sort keys are those of the
    // last rebuild, and each cell's particles have moved since by at most cell_mdx[c] key
    // units; a pair task's projection bound widens by cell_mdx[ci] + cell_mdx[cj]
    // (src/runner_dopair.c:583: cutoff + maxdx_i + maxdx_j).  nullptr: fresh keys.
    const int* cell_mdx = nullptr;
};

// The projection bound of a pair task, widened by the cells' displacements since the keys
// were made (Verlet skin).
__device__ __forceinline__ int task_dmax_skin(const Params& P, const TaskRec& r) {
    int d = task_dmax(r);
    if (P.cell_mdx != nullptr && r.sid >= 0) d += P.cell_mdx[r.ci] + P.cell_mdx[r.cj];
    return d;
}

// A device-resident step that was aborted (see nb_resident.cuh) launches nothing more.
__device__ __forceinline__ bool step_aborted(const unsigned long long* abort) {
    return abort != nullptr && *(const volatile unsigned long long*)abort != 0;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// One-dimensional TMA bulk copy global -> shared, completion counted on `bar`.
// dst and src must be 16-byte aligned and bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of `bar` to complete, at most c_spin_limit polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    const int limit = c_spin_limit;
    for (int it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Float -> 64-bit fixed point, flagging values outside the representable range.
__device__ __forceinline__ long long to_fixed(float v, unsigned& status) {
    float s = v * kForceScale;
    if (!(fabsf(s) < 9.0e18f)) status |= kStatusForceOverflow;
    return __float2ll_rn(s);
}

__device__ __forceinline__ void atomic_add_fixed(unsigned long long* p, long long v) {
    if (v != 0) atomicAdd(p, static_cast<unsigned long long>(v));
}

}  // namespace nb
