// Device-resident time steps (sm_100a): the particles stay in HBM between steps and the
// whole step -- re-binning, sort, sweep, integration, rigid constraints -- runs as device
// launches (one CUDA graph per step), the host state being brought up to date only on
// request.
//
// Layout: every cell owns a fixed block of `capc` slots (cell c: slots c*capc ..
// c*capc + count[c]), so slot offsets never change and every launch has a fixed size.
// Re-binning (the device form of space_shuffle, src/space.c:235-291) keeps each cell's
// remaining particles in their order and appends the arrivals from the 26 neighbours in a
// fixed direction order, each neighbour's leavers in their order: the result does not depend
// on thread scheduling.
//
// Overflow: a cell that would exceed its capacity, or more than `mcap` leavers of one cell
// in one step, sets a sticky abort word.  Every later kernel of that step and of the steps
// after it returns at once, so the side the step read from keeps the last completed step
// intact; integrate_cells counts the completed steps (and their accepted pairs), from which
// the host finds that side,
// re-blocks the particles with more room and runs the remaining steps again.  Nothing is
// written out of bounds.  A position or velocity that is no longer finite (a system blowing
// up) stops the steps after the step that produced it, and the host reports an error.
#pragma once
#include "nb_device.cuh"
#include "nb_kernels.cuh"

namespace nb {

constexpr unsigned kStatusResidentOverflow = 1u << 4;   // a cell outgrew its block
constexpr unsigned kStatusMoverOverflow = 1u << 5;      // too many leavers of one cell

struct Mover {
    float4 x;        // position relative to the destination cell, w = type bits
    float4 v;        // velocity, w = direction index (bits)
    int pid;
    int pad[3];
};

struct ResidentCells {
    int ncells, capc, mcap;  // cells, slots per cell, leavers per cell and step
    const int* nbr;          // 27 per cell: global index of the neighbour in direction d (13 = self)
    const float4* cell_h;    // per cell: edge lengths (float, as the host keeps them)
};

// Direction index of a cell offset (dx, dy, dz) in {-1, 0, 1}^3.
__device__ __forceinline__ int dir_index(int dx, int dy, int dz) { return (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1); }

// Phase 1, one warp per cell: particles still inside [0, h) keep their order and are
// written to the same cell of the output side; leavers go to the cell's mover list,
// shifted into their destination cell's frame (src/space.c: x -= delta*h).
__global__ void __launch_bounds__(256) rebin_split(ResidentCells RC, const float4* __restrict__ xq,
                                                   const float4* __restrict__ v, const int* __restrict__ pid,
                                                   const int* __restrict__ count, float4* __restrict__ xq_out,
                                                   float4* __restrict__ v_out, int* __restrict__ pid_out,
                                                   int* __restrict__ nstay, int* __restrict__ nmove,
                                                   Mover* __restrict__ movers, unsigned long long* status) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= RC.ncells || *(volatile unsigned long long*)status != 0) return;
    const int n = min(count[c], RC.capc);
    const size_t base = (size_t)c * RC.capc;
    const float4 h = RC.cell_h[c];
    int stays = 0, moves = 0;
    for (int k0 = 0; k0 < n; k0 += 32) {
        const int k = k0 + lane;
        const bool active = k < n;
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f), vv = x;
        int id = 0;
        if (active) {
            x = xq[base + k];
            vv = v[base + k];
            id = pid[base + k];
        }
        const int dx = (x.x >= h.x) - (x.x < 0.0f), dy = (x.y >= h.y) - (x.y < 0.0f), dz = (x.z >= h.z) - (x.z < 0.0f);
        const bool stay = active && dx == 0 && dy == 0 && dz == 0;
        const bool move = active && !stay;
        const unsigned bs = __ballot_sync(FULL, stay), bm = __ballot_sync(FULL, move);
        const unsigned below = (1u << lane) - 1u;
        if (stay) {
            const int o = stays + __popc(bs & below);
            xq_out[base + o] = x;
            v_out[base + o] = vv;
            pid_out[base + o] = id;
        }
        if (move) {
            const int m = moves + __popc(bm & below);
            if (m < RC.mcap) {
                Mover mv;
                mv.x = make_float4(__fsub_rn(x.x, __fmul_rn((float)dx, h.x)), __fsub_rn(x.y, __fmul_rn((float)dy, h.y)),
                                   __fsub_rn(x.z, __fmul_rn((float)dz, h.z)), x.w);
                mv.v = make_float4(vv.x, vv.y, vv.z, __int_as_float(dir_index(dx, dy, dz)));
                mv.pid = id;
                mv.pad[0] = mv.pad[1] = mv.pad[2] = 0;
                movers[(size_t)c * RC.mcap + m] = mv;
            } else {
                atomicOr(status, (unsigned long long)kStatusMoverOverflow);
            }
        }
        stays += __popc(bs);
        moves += __popc(bm);
    }
    if (lane == 0) {
        nstay[c] = stays;
        nmove[c] = min(moves, RC.mcap);
    }
}

// Phase 2, one warp per destination cell: after its stayers, the arrivals from the
// neighbours in direction order 0..26 (a particle that moved by d arrives from the
// neighbour at -d), each neighbour's leavers in their order; with slot_of, the slot of
// every particle id of the cell.
__global__ void __launch_bounds__(256) rebin_gather(ResidentCells RC, const Mover* __restrict__ movers,
                                                    const int* __restrict__ nstay, const int* __restrict__ nmove,
                                                    float4* __restrict__ xq_out, float4* __restrict__ v_out,
                                                    int* __restrict__ pid_out, int* __restrict__ count,
                                                    unsigned long long* status, int* __restrict__ slot_of) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= RC.ncells || *(volatile unsigned long long*)status != 0) return;
    const size_t base = (size_t)c * RC.capc;
    int off = nstay[c];
    bool over = false;
    // lane d (< 27) looks up the neighbour a particle moving by direction d comes from and
    // whether it has leavers; only those directions are walked, in order
    int my_src = 0, my_nm = 0;
    if (lane < 27 && lane != 13) {
        my_src = RC.nbr[(size_t)c * 27 + (26 - lane)];
        my_nm = nmove[my_src];
    }
    unsigned todo = __ballot_sync(FULL, my_nm > 0);
    while (todo) {
        const int d = __ffs(todo) - 1;
        todo &= todo - 1;
        const int src = __shfl_sync(FULL, my_src, d);
        const int nm = __shfl_sync(FULL, my_nm, d);
        for (int m0 = 0; m0 < nm; m0 += 32) {
            const int m = m0 + lane;
            Mover mv;
            bool match = false;
            if (m < nm) {
                mv = movers[(size_t)src * RC.mcap + m];
                match = __float_as_int(mv.v.w) == d;
            }
            const unsigned bmatch = __ballot_sync(FULL, match);
            if (match) {
                const int o = off + __popc(bmatch & ((1u << lane) - 1u));
                if (o < RC.capc) {
                    xq_out[base + o] = mv.x;
                    v_out[base + o] = make_float4(mv.v.x, mv.v.y, mv.v.z, 0.f);
                    pid_out[base + o] = mv.pid;
                } else {
                    over = true;
                }
            }
            off += __popc(bmatch);
        }
    }
    if (__any_sync(FULL, over) && lane == 0) atomicOr(status, (unsigned long long)kStatusResidentOverflow);
    const int n = min(off, RC.capc);
    if (lane == 0) count[c] = n;
    if (slot_of != nullptr) {          // rigid systems: the slot of every particle id in this cell
        __syncwarp();
        for (int k = lane; k < n; k += 32) slot_of[pid_out[base + k]] = (int)(base + k);
    }
}

// Slot of every particle id after re-binning (for the rigid constraints).
__global__ void __launch_bounds__(256) slot_of_ids(ResidentCells RC, const int* __restrict__ pid,
                                                   const int* __restrict__ count, int* __restrict__ slot_of,
                                                   const unsigned long long* __restrict__ status) {
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= RC.ncells || (status != nullptr && *status != 0)) return;
    const int n = min(count[c], RC.capc);
    const size_t base = (size_t)c * RC.capc;
    for (int k = lane; k < n; k += 32) slot_of[pid[base + k]] = (int)(base + k);
}

// Symplectic Euler update of every particle (engine_advance, src/engine.c:1975-1979), with
// the float expressions the host integrator evaluates: w = (float)(dt * 1/m),
// v += f*w, x += dt*v; forces from the fixed-point accumulators of the sweep.  One thread
// per slot (grid: ncells * capc threads).
__global__ void __launch_bounds__(256) integrate_cells(ResidentCells RC, const int* __restrict__ count,
                                                       const unsigned long long* __restrict__ force,
                                                       const int* __restrict__ cell_engine,
                                                       const float* __restrict__ engine_dt,
                                                       const double* __restrict__ engine_imass, int max_type,
                                                       float4* __restrict__ xq, float4* __restrict__ v,
                                                       unsigned long long* __restrict__ status,
                                                       const unsigned long long* __restrict__ acc,
                                                       unsigned long long* __restrict__ done) {
    if (*status != 0) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {          // completed steps, accepted pairs
        done[0] += 1ull;
        done[1] += acc[kAccPairs];
    }
    // one thread per slot of every block (the slots past a cell's count do nothing)
    const size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= (size_t)RC.ncells * RC.capc) return;
    const int c = (int)(s / (unsigned)RC.capc);
    if ((int)(s - (size_t)c * RC.capc) >= min(count[c], RC.capc)) return;
    const int k_eng = cell_engine[c];
    const float dt = engine_dt[k_eng];
    {
        float4 x = xq[s], vv = v[s];
        const int type = __float_as_int(x.w);
        const float w = (float)((double)dt * engine_imass[(size_t)k_eng * max_type + type]);
        const float fx = (float)((double)(long long)force[3 * s + 0] * (1.0 / (double)kForceScale));
        const float fy = (float)((double)(long long)force[3 * s + 1] * (1.0 / (double)kForceScale));
        const float fz = (float)((double)(long long)force[3 * s + 2] * (1.0 / (double)kForceScale));
        vv.x = __fadd_rn(vv.x, __fmul_rn(fx, w));
        vv.y = __fadd_rn(vv.y, __fmul_rn(fy, w));
        vv.z = __fadd_rn(vv.z, __fmul_rn(fz, w));
        x.x = __fadd_rn(x.x, __fmul_rn(dt, vv.x));
        x.y = __fadd_rn(x.y, __fmul_rn(dt, vv.y));
        x.z = __fadd_rn(x.z, __fmul_rn(dt, vv.z));
        xq[s] = x;
        v[s] = vv;
        if (!isfinite(x.x + x.y + x.z + vv.x + vv.y + vv.z))      // a system blowing up: stop
            atomicOr(status, (unsigned long long)kStatusNonFinite);
    }
}

// Bonds (bond_eval, src/bond.c:81-250) of the particles in the device cells: one thread per
// bond, the two particles found through slot_of, the distance from their cell-relative
// positions and the periodic offset of their cells (held to -1..1), r^2 held to the table's
// [a^2, b^2]; the pair force goes into the fixed-point accumulators like the sweep's, the
// energy into a fixed-point sum per engine.
struct BondArgs {
    const int4* bonds;           // global id i, global id j, bond table, engine
    int nbonds;
    const float* coef;           // bond tables, the sweep's format
    const float4* potinfo;
    const int* potn;
    const double2* ab2;          // per table: a^2, b^2
    const int* slot_of;
    const float4* xq;
    unsigned long long* force;
    const int* eng_cell0;        // per engine: first global cell, cell grid, cell edge
    const int4* eng_cdim;
    const double4* eng_h;
    int capc;
    unsigned long long* ebond;   // per engine, 2^32 units per kJ/mol
    unsigned long long* acc;     // status bits
    const unsigned long long* abort;
};

__global__ void __launch_bounds__(128) bond_forces(BondArgs B) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B.nbonds || (B.abort != nullptr && *(const volatile unsigned long long*)B.abort != 0)) return;
    const int4 b = B.bonds[t];
    const int si = B.slot_of[b.x], sj = B.slot_of[b.y];
    const float4 xi = B.xq[si], xj = B.xq[sj];
    const int4 cd = B.eng_cdim[b.w];
    const double4 h = B.eng_h[b.w];
    const int ci = si / B.capc - B.eng_cell0[b.w], cj = sj / B.capc - B.eng_cell0[b.w];
    const int li[3] = {ci / (cd.y * cd.z), (ci / cd.z) % cd.y, ci % cd.z};
    const int lj[3] = {cj / (cd.y * cd.z), (cj / cd.z) % cd.y, cj % cd.z};
    const double hh[3] = {h.x, h.y, h.z};
    const float xiv[3] = {xi.x, xi.y, xi.z}, xjv[3] = {xj.x, xj.y, xj.z};
    float dx[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        int sh = li[k] - lj[k];
        if (sh > 1) sh = -1;
        else if (sh < -1) sh = 1;
        const float pix = (float)((double)xiv[k] + hh[k] * sh);
        dx[k] = __fsub_rn(pix, xjv[k]);
    }
    float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx[0], dx[0]), __fmul_rn(dx[1], dx[1])), __fmul_rn(dx[2], dx[2]));
    const double2 ab2 = B.ab2[b.z];
    if ((double)r2 < ab2.x || (double)r2 > ab2.y) r2 = (float)fmax(ab2.x, fmin(ab2.y, (double)r2));
    float e, f;
    unsigned status = 0;
    eval_table(B.coef, B.potinfo[b.z], B.potn[b.z], r2, e, f, status);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float w = f * dx[k];
        atomic_add_fixed(B.force + 3 * (size_t)si + k, to_fixed(-w, status));
        atomic_add_fixed(B.force + 3 * (size_t)sj + k, to_fixed(w, status));
    }
    atomicAdd(&B.ebond[b.w], (unsigned long long)__double2ll_rn((double)e * kEnergyScale));
    if (status) atomicOr(&B.acc[kAccStatus], (unsigned long long)status);
}

// Cell offsets of the compacted download: an exclusive scan of min(count, capc) over the
// cells in three launches of kScanBlock-thread blocks (block sums, their scan, the scan).
constexpr int kScanBlock = 1024;

__device__ __forceinline__ int block_scan_int(int v, int& excl, int* warp_tot) {
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
        const int w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        warp_tot[lane] = wi - w;
        if (lane == 31) warp_tot[32] = wi;
    }
    __syncthreads();
    excl = warp_tot[warp] + incl - v;
    const int total = warp_tot[32];
    __syncthreads();
    return total;
}

__global__ void __launch_bounds__(kScanBlock) scan_counts_sums(const int* __restrict__ count, int n, int capc,
                                                              int* __restrict__ bsum) {
    __shared__ int warp_tot[33];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    int excl;
    const int total = block_scan_int(i < n ? min(count[i], capc) : 0, excl, warp_tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) scan_counts_blocks(int* __restrict__ bsum, int nblocks) {
    __shared__ int warp_tot[33];
    int run = 0;
    for (int base = 0; base < nblocks; base += kScanBlock) {
        const int b = base + threadIdx.x;
        const int v = b < nblocks ? bsum[b] : 0;
        int excl;
        const int total = block_scan_int(v, excl, warp_tot);
        if (b < nblocks) bsum[b] = run + excl;
        run += total;
    }
}

__global__ void __launch_bounds__(kScanBlock) scan_counts_apply(const int* __restrict__ count, int n, int capc,
                                                               const int* __restrict__ bsum, int* __restrict__ off) {
    __shared__ int warp_tot[33];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    const int v = i < n ? min(count[i], capc) : 0;
    int excl;
    block_scan_int(v, excl, warp_tot);
    if (i < n) off[i] = bsum[blockIdx.x] + excl;
}

}  // namespace nb
