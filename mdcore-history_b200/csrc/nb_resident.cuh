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
                                                   Mover* __restrict__ movers, unsigned long long* status,
                                                   const int* __restrict__ rebuild) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= RC.ncells || *(volatile unsigned long long*)status != 0) return;
    const int n = min(count[c], RC.capc);
    const size_t base = (size_t)c * RC.capc;
    // Verlet skin between rebuilds: nobody leaves (particles stay in their cells, in their
    // slots, up to half the skin outside the cell), the block is copied in order.
    const bool moving = rebuild == nullptr || *rebuild != 0;
    const float4 h = moving ? RC.cell_h[c] : make_float4(INFINITY, INFINITY, INFINITY, 0.f);
    int stays = 0, moves = 0;
    // the next 32 particles are loaded while these are written (latency of one load, not of
    // one per 32 particles)
    float4 xn = make_float4(0.f, 0.f, 0.f, 0.f), vn = xn;
    int idn = 0;
    if (lane < n) {
        xn = xq[base + lane];
        vn = v[base + lane];
        idn = pid[base + lane];
    }
    for (int k0 = 0; k0 < n; k0 += 32) {
        const int k = k0 + lane;
        const bool active = k < n;
        const float4 x = xn, vv = vn;
        const int id = idn;
        if (k + 32 < n) {
            xn = xq[base + k + 32];
            vn = v[base + k + 32];
            idn = pid[base + k + 32];
        }
        const int dx = moving ? (x.x >= h.x) - (x.x < 0.0f) : 0, dy = moving ? (x.y >= h.y) - (x.y < 0.0f) : 0,
                  dz = moving ? (x.z >= h.z) - (x.z < 0.0f) : 0;
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
    // The candidates of all those directions as one list, direction-major: lane d's movers
    // occupy [pre_d, pre_d + nm_d).  Each pass loads 32 of them at once (one load latency
    // for many directions instead of one per direction) and keeps those that moved by d.
    int incl = my_nm;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    const int my_pre = incl - my_nm;
    const int total = __shfl_sync(FULL, incl, 31);
    for (int t0 = 0; t0 < total; t0 += 32) {
        const int t = t0 + lane;
        // the direction holding candidate t: the last lane whose list starts at or before t
        int d = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const int pre = __shfl_sync(FULL, my_pre, d + step);
            if (pre <= t) d += step;
        }
        const int src = __shfl_sync(FULL, my_src, d);
        const int m = t - __shfl_sync(FULL, my_pre, d);
        Mover mv;
        bool match = false;
        if (t < total) {
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

// ---------------------------------------------------------------- Verlet skin
// engine_verlet_update (src/engine.c:193-315) for the resident steps: the particles are
// re-binned and sorted only when the largest displacement since the last rebuild exceeds
// half the skin (min h - cutoff) or a quarter of the cutoff; in between, each pair task's
// projection bound carries the two cells' displacements.  Device words (vw): [0] rebuild
// this step (1) or not (0), [1] largest displacement of the step (float bits, >= 0),
// [2] rebuilds so far.

// After re-binning: on a rebuild step, the positions the keys are made from become the
// reference positions and the displacements restart from zero.
__global__ void __launch_bounds__(256) verlet_mark(ResidentCells RC, const int* __restrict__ count,
                                                  const float4* __restrict__ xq, float4* __restrict__ oldx,
                                                  int* __restrict__ cell_mdx, const int* __restrict__ vw,
                                                  const unsigned long long* __restrict__ status) {
    if (*status != 0 || vw[0] == 0) return;
    const size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < (size_t)RC.ncells && s < (size_t)RC.ncells * RC.capc) cell_mdx[s] = 0;
    if (s >= (size_t)RC.ncells * RC.capc) return;
    const int c = (int)(s / (unsigned)RC.capc);
    if ((int)(s - (size_t)c * RC.capc) < min(count[c], RC.capc)) oldx[s] = xq[s];
}

// After the step: each cell's largest displacement from the reference positions (one warp
// per cell), in key units of its engine's sort scale for the next step's bounds, and the
// largest of all.
__global__ void __launch_bounds__(256) verlet_check(ResidentCells RC, const int* __restrict__ count,
                                                   const float4* __restrict__ xq, const float4* __restrict__ oldx,
                                                   const float2* __restrict__ cscale, int* __restrict__ cell_mdx,
                                                   int* __restrict__ vw, const unsigned long long* __restrict__ status) {
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= RC.ncells || *status != 0) return;
    const int n = min(count[c], RC.capc);
    const size_t base = (size_t)c * RC.capc;
    float d2 = 0.f;
    for (int k = lane; k < n; k += 32) {
        const float4 x = xq[base + k], o = oldx[base + k];
        const float dx = x.x - o.x, dy = x.y - o.y, dz = x.z - o.z;
        d2 = fmaxf(d2, dx * dx + dy * dy + dz * dz);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, o));
    if (lane == 0) {
        // rounded up, plus one unit for the floor of either key
        const float md = sqrtf(d2) * 1.0001f;
        cell_mdx[c] = (int)ceilf(cscale[c].x * md) + 1;
        atomicMax(&vw[1], __float_as_int(md));
    }
}

// The rebuild decision for the next step (src/engine.c:262): 2 maxdx > skin or
// maxdx > cutoff / 4 (engine_maxdxratio, src/engine.h:83).
__global__ void verlet_decide(int* __restrict__ vw, float skin, float cutoff,
                              const unsigned long long* __restrict__ status) {
    if (*status != 0) return;
    const float md = __int_as_float(vw[1]);
    const int rebuild = (2.0f * md > skin) || (md > 0.25f * cutoff);
    vw[0] = rebuild;
    vw[1] = 0;
    if (rebuild) vw[2] += 1;
}

// Symplectic Euler update of every particle (engine_advance, src/engine.c:1975-1979), with
// the float expressions the host integrator evaluates: w = (float)(dt * 1/m),
// v += f*w, x += dt*v; forces from the fixed-point accumulators of the sweep.  One thread
// per slot (grid: ncells * capc threads).
//
// With sd_gamma > 0 the update is a steepest-descent move instead (an energy minimiser for
// unrelaxed starts; no counterpart in the reference's step): x += g f with g = sd_gamma,
// held so that no particle moves farther than sd_dmax, and v = 0.
__global__ void __launch_bounds__(256) integrate_cells(ResidentCells RC, const int* __restrict__ count,
                                                       const unsigned long long* __restrict__ force,
                                                       const int* __restrict__ cell_engine,
                                                       const float* __restrict__ engine_dt,
                                                       const double* __restrict__ engine_imass, int max_type,
                                                       float4* __restrict__ xq, float4* __restrict__ v,
                                                       unsigned long long* __restrict__ status,
                                                       const unsigned long long* __restrict__ acc,
                                                       unsigned long long* __restrict__ done, float sd_gamma,
                                                       float sd_dmax) {
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
        if (sd_gamma > 0.f) {
            const float fn = sqrtf(fx * fx + fy * fy + fz * fz);
            const float g = fn * sd_gamma > sd_dmax ? sd_dmax / fn : sd_gamma;
            x.x += g * fx;
            x.y += g * fy;
            x.z += g * fz;
            xq[s] = x;
            v[s] = make_float4(0.f, 0.f, 0.f, vv.w);
            if (!isfinite(x.x + x.y + x.z)) atomicOr(status, (unsigned long long)kStatusNonFinite);
            return;
        }
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

// Per-step energy log (no counterpart in the reference; drivers such as
// examples/argon/argon.c sum the kinetic energy on the host every step): the kinetic
// energy of every particle's velocity after the step, sum of m v^2 / 2 in FP64 per thread,
// to 2^32 fixed point per block and one integer atomic; then one block sums the cells'
// fixed-point energies and the bonded energies and writes the record of the step.
__global__ void __launch_bounds__(256) kinetic_cells(ResidentCells RC, const int* __restrict__ count,
                                                     const int* __restrict__ cell_engine,
                                                     const double* __restrict__ engine_imass, int max_type,
                                                     const float4* __restrict__ xq, const float4* __restrict__ v,
                                                     const unsigned long long* __restrict__ status,
                                                     unsigned long long* __restrict__ ekin) {
    __shared__ long long part[8];
    if (*status != 0) return;
    const size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (s < (size_t)RC.ncells * RC.capc) {
        const int c = (int)(s / (unsigned)RC.capc);
        if ((int)(s - (size_t)c * RC.capc) < min(count[c], RC.capc)) {
            const float4 vv = v[s];
            const double im = engine_imass[(size_t)cell_engine[c] * max_type + __float_as_int(xq[s].w)];
            e = 0.5 * ((double)vv.x * vv.x + (double)vv.y * vv.y + (double)vv.z * vv.z) / im;
        }
    }
    long long q = __double2ll_rn(e * kEnergyScale);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = q;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
        if (t != 0) atomicAdd(ekin, (unsigned long long)t);
    }
}

__global__ void __launch_bounds__(1024) energy_record(const unsigned long long* __restrict__ cell_epot, int ncells,
                                                      const unsigned long long* __restrict__ ebond, int nbond,
                                                      const unsigned long long* __restrict__ ekin,
                                                      const unsigned long long* __restrict__ base,
                                                      const unsigned long long* __restrict__ done,
                                                      const unsigned long long* __restrict__ status,
                                                      unsigned long long* __restrict__ log, int cap) {
    __shared__ long long part[32];
    if (*status != 0) return;
    long long q = 0;
    for (int c = threadIdx.x; c < ncells; c += blockDim.x) q += (long long)cell_epot[c];
    for (int k = threadIdx.x; k < nbond; k += blockDim.x) q += (long long)ebond[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = q;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
        const unsigned long long n = *base + done[0];
        unsigned long long* r = log + 4 * (size_t)((n - 1) % (unsigned long long)cap);
        r[0] = n;
        r[1] = (unsigned long long)t;
        r[2] = *ekin;
        r[3] = 0ull;
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
    unsigned long long* ebond;   // bond, angle, dihedral energy per engine (3 x nengines), 2^32 units per kJ/mol
    unsigned long long* acc;     // status bits
    const unsigned long long* abort;
    int nengines;
    const int4* angles;          // global ids i, j, k; engine << 16 | table
    int nangles;
    const int4* dihedrals;       // global ids i, j, k, l
    const int* dihedral_te;      // engine << 16 | table, by dihedral
    int ndihedrals;
    const double2* ab;           // per table: its range [a, b] (angles, dihedrals: of the cosine)
};

// Position of the particle in slot s relative to the cell of slot sref (both of engine eng):
// its cell-relative position plus the cell edge times the cells' offset, the offset held to
// -1..1 in each dimension (the periodic image next to sref's cell), as src/angle.c:141-158
// and src/dihedral.c:146-171 place i, k (and l) relative to j's cell.
__device__ __forceinline__ void pos_near(const BondArgs& B, int eng, int s, int sref, float out[3]) {
    const int4 cd = B.eng_cdim[eng];
    const double4 h = B.eng_h[eng];
    const int c = s / B.capc - B.eng_cell0[eng], cr = sref / B.capc - B.eng_cell0[eng];
    const int l[3] = {c / (cd.y * cd.z), (c / cd.z) % cd.y, c % cd.z};
    const int lr[3] = {cr / (cd.y * cd.z), (cr / cd.z) % cd.y, cr % cd.z};
    const double hh[3] = {h.x, h.y, h.z};
    const float4 x = B.xq[s];
    const float xv[3] = {x.x, x.y, x.z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        int sh = l[k] - lr[k];
        if (sh > 1) sh = -1;
        else if (sh < -1) sh = 1;
        out[k] = (float)((double)xv[k] + hh[k] * sh);
    }
}

__device__ __forceinline__ float dot3(const float a[3], const float b[3]) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1])), __fmul_rn(a[2], b[2]));
}

__device__ __forceinline__ void cross3(const float a[3], const float b[3], float out[3]) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

// The cosine held to the table's range (the reference warns and clamps,
// src/angle.c:183-187, src/dihedral.c:254-260), the table read at it.
__device__ __forceinline__ void eval_cosine(const BondArgs& B, int tab, float c, float& e, float& f,
                                            unsigned& status) {
    const double2 ab = B.ab[tab];
    if ((double)c < ab.x || (double)c > ab.y) c = (float)fmax(ab.x, fmin(ab.y, (double)c));
    eval_table_r(B.coef, B.potinfo[tab], B.potn[tab], c, e, f, status);
}

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

// Angles (angle_eval, src/angle.c:81-300): one thread per angle i-j-k.  With u = x_i - x_j
// and w = x_k - x_j (positions near j's cell), cos = u.w / (|u| |w|) held to [-1, 1], and
// its gradients d cos/d x_i = (w/|w| - cos u/|u|) / |u|, d cos/d x_k = (u/|u| - cos w/|w|) / |w|,
// d cos/d x_j = -(both); the force on each particle is -dE/dcos times its gradient.
__global__ void __launch_bounds__(128) angle_forces(BondArgs B) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B.nangles || (B.abort != nullptr && *(const volatile unsigned long long*)B.abort != 0)) return;
    const int4 a = B.angles[t];
    const int eng = a.w >> 16, tab = a.w & 0xffff;
    const int si = B.slot_of[a.x], sj = B.slot_of[a.y], sk = B.slot_of[a.z];
    float xi[3], xj[3], xk[3], u[3], w[3];
    pos_near(B, eng, si, sj, xi);
    pos_near(B, eng, sj, sj, xj);
    pos_near(B, eng, sk, sj, xk);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        u[k] = __fsub_rn(xi[k], xj[k]);
        w[k] = __fsub_rn(xk[k], xj[k]);
    }
    const float iu = __fdiv_rn(1.0f, __fsqrt_rn(dot3(u, u)));
    const float iw = __fdiv_rn(1.0f, __fsqrt_rn(dot3(w, w)));
    const float c = fminf(1.0f, fmaxf(-1.0f, dot3(u, w) * iu * iw));
    float gi[3], gk[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float uh = u[k] * iu, wh = w[k] * iw;
        gi[k] = (wh - c * uh) * iu;
        gk[k] = (uh - c * wh) * iw;
    }
    float e, f;
    unsigned status = 0;
    eval_cosine(B, tab, c, e, f, status);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float wi = f * gi[k], wk = f * gk[k];
        atomic_add_fixed(B.force + 3 * (size_t)si + k, to_fixed(-wi, status));
        atomic_add_fixed(B.force + 3 * (size_t)sk + k, to_fixed(-wk, status));
        atomic_add_fixed(B.force + 3 * (size_t)sj + k, to_fixed(wi + wk, status));
    }
    atomicAdd(&B.ebond[B.nengines + eng], (unsigned long long)__double2ll_rn((double)e * kEnergyScale));
    if (status) atomicOr(&B.acc[kAccStatus], (unsigned long long)status);
}

// Dihedrals (dihedral_eval, src/dihedral.c:81-380): one thread per dihedral i-j-k-l.  With
// b1 = x_j - x_i, b2 = x_k - x_j, b3 = x_l - x_k (positions near j's cell), the plane normals
// n1 = b1 x b2 and n2 = b2 x b3, cos = n1.n2 / (|n1| |n2|) held to [-1, 1].  Gradients by the
// chain rule through the normals: g1 = d cos/d n1 = (n2/|n2| - cos n1/|n1|) / |n1|,
// g2 = (n1/|n1| - cos n2/|n2|) / |n2|; d cos/d b1 = b2 x g1, d cos/d b3 = g2 x b2,
// d cos/d b2 = g1 x b1 + b3 x g2; then x_i: -d/db1, x_j: d/db1 - d/db2, x_l: d/db3, and x_k
// takes minus the sum of the other three.
__global__ void __launch_bounds__(128) dihedral_forces(BondArgs B) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B.ndihedrals || (B.abort != nullptr && *(const volatile unsigned long long*)B.abort != 0)) return;
    const int4 d = B.dihedrals[t];
    const int te = B.dihedral_te[t];
    const int eng = te >> 16, tab = te & 0xffff;
    const int si = B.slot_of[d.x], sj = B.slot_of[d.y], sk = B.slot_of[d.z], sl = B.slot_of[d.w];
    float xi[3], xj[3], xk[3], xl[3], b1[3], b2[3], b3[3];
    pos_near(B, eng, si, sj, xi);
    pos_near(B, eng, sj, sj, xj);
    pos_near(B, eng, sk, sj, xk);
    pos_near(B, eng, sl, sj, xl);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        b1[k] = __fsub_rn(xj[k], xi[k]);
        b2[k] = __fsub_rn(xk[k], xj[k]);
        b3[k] = __fsub_rn(xl[k], xk[k]);
    }
    float n1[3], n2[3];
    cross3(b1, b2, n1);
    cross3(b2, b3, n2);
    const float i1 = __fdiv_rn(1.0f, __fsqrt_rn(dot3(n1, n1)));
    const float i2 = __fdiv_rn(1.0f, __fsqrt_rn(dot3(n2, n2)));
    const float c = fminf(1.0f, fmaxf(-1.0f, dot3(n1, n2) * i1 * i2));
    float g1[3], g2[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float h1 = n1[k] * i1, h2 = n2[k] * i2;
        g1[k] = (h2 - c * h1) * i1;
        g2[k] = (h1 - c * h2) * i2;
    }
    float db1[3], db2[3], db3[3], t1[3], t2[3];
    cross3(b2, g1, db1);
    cross3(g2, b2, db3);
    cross3(g1, b1, t1);
    cross3(b3, g2, t2);
    float e, f;
    unsigned status = 0;
    eval_cosine(B, tab, c, e, f, status);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        db2[k] = t1[k] + t2[k];
        const float wi = f * -db1[k], wj = f * (db1[k] - db2[k]), wl = f * db3[k];
        atomic_add_fixed(B.force + 3 * (size_t)si + k, to_fixed(-wi, status));
        atomic_add_fixed(B.force + 3 * (size_t)sj + k, to_fixed(-wj, status));
        atomic_add_fixed(B.force + 3 * (size_t)sl + k, to_fixed(-wl, status));
        atomic_add_fixed(B.force + 3 * (size_t)sk + k, to_fixed(wi + wj + wl, status));
    }
    atomicAdd(&B.ebond[2 * B.nengines + eng], (unsigned long long)__double2ll_rn((double)e * kEnergyScale));
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
