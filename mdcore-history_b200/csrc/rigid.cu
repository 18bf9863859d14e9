// Rigid constraints on the device: engine_rigid_eval (src/engine_rigid.c:352-583) with
// SHAKE (src/rigid.c:81-277, engine_flag_shake) and P-SHAKE (src/rigid.c:279-523, the
// default).  One thread per rigid group iterates in FP64; the P-SHAKE mixing matrices stay
// on the device between steps.
//
// Per evaluation (after the position update of a step): the host packs every group's
// particles -- cell-relative float position, velocity, and the cell offset of the particle
// relative to the group's first particle (the reference's periodic shift of -1, 0 or +1
// cell per dimension) -- into pinned buffers; one copy up; the kernel; one copy down of
// the corrected positions (FP64, relative to the first particle's cell); the host applies
// the reference's position, velocity and (P-SHAKE) force corrections to the cells.
//
// This file is compiled with --fmad=false: the iterations round every operation as the
// C expressions of the reference do (no fused multiply-adds), so the result can be
// compared bit for bit with a CPU restatement compiled without contraction.
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#include <cuda_runtime.h>
#include "mdcore_b200.h"
#include "internal.h"
#include "host_pool.h"

using nb::HostPool;

namespace {

struct RigidArgs {
    int nrig;
    const int* roff;            // nrig+1: first particle slot of each group
    const int* coff;            // nrig+1: first constraint of each group
    const int* aoff;            // nrig+1: first matrix entry of each group (sum of nc^2)
    const int2* cij;            // constraint ends, group-local indices
    const double* d2;           // squared constraint lengths
    const double* mass;         // per slot
    const float4* x;            // per slot: cell-relative position, w = shift code bits
    const float4* v;            // per slot: velocity
    float* a;                   // P-SHAKE matrices (read and refined in place)
    double* xp;                 // per slot: corrected position (3 doubles)
    int* stat;                  // [0] largest iteration count, [1] unconverged groups
    double h0, h1, h2;          // cell edge
    double dt, tol;
    int a_update;               // P-SHAKE: refine the matrices this step
    // Resident steps (RES kernels): particles read and written in place in the device
    // cells instead of the packed slots above.
    const int* rpid;            // per group slot: particle id
    const int* slot_of;         // global particle id -> device slot
    int id0;                    // this engine's first global id
    float4* rxq;                // device cells: cell-relative position, w = type
    float4* rv;                 // device cells: velocity
    int capc, cell0;            // slots per cell, this engine's first global cell
    int cd0, cd1, cd2;          // cell grid
    const unsigned long long* abort;   // resident: nonzero = the step was aborted
    // Resident steps of an engine whose every particle is in a rigid group: the update of
    // engine_advance (integrate_cells' arithmetic) runs here on each group's particles
    // before the constraints, and no separate update kernel is launched.
    int fuse;
    const unsigned long long* force;   // fixed-point forces by slot (2^24 per kJ/mol/nm)
    const double* imass;               // 1/mass by type
    float dtf;                         // the time step as the update uses it
    unsigned long long* status;        // the step's status word (non-finite result: bit 64)
    unsigned long long* done;          // completed steps, their accepted pairs
    const unsigned long long* pairs;   // this step's accepted pairs
};

// Cell grid coordinates of a resident slot.
__device__ __forceinline__ void slot_loc(const RigidArgs& A, int slot, int* loc) {
    const int c = slot / A.capc - A.cell0;
    loc[0] = c / (A.cd1 * A.cd2);
    loc[1] = (c / A.cd2) % A.cd1;
    loc[2] = c % A.cd2;
}

// Periodic cell offset -1/0/+1 of loc relative to loc0 per dimension (src/rigid.c:133-141).
__device__ __forceinline__ int shift_dim(int a, int b) {
    int s = a - b;
    if (s > 1) s = -1;
    else if (s < -1) s = 1;
    return s;
}

// Position (relative to the group's first cell), position before the step and mass of every
// particle of a group; packed slots carry the shift code (sx+1) + 3 (sy+1) + 9 (sz+1) in w
// (-1: a group to skip), resident ones derive it from the cells.  Returns the shifts.
template <bool RES>
__device__ __forceinline__ void load_group(const RigidArgs& A, int p0, int np, double* xp, double* xo, double* m,
                                           int* shifts) {
    int loc0[3] = {0, 0, 0};
    if (RES) slot_loc(A, A.slot_of[A.id0 + A.rpid[p0]], loc0);
    for (int k = 0; k < np; k++) {
        float4 x, v;
        int sh[3];
        if (RES) {
            const int slot = A.slot_of[A.id0 + A.rpid[p0 + k]];
            x = A.rxq[slot];
            v = A.rv[slot];
            if (A.fuse) {   // symplectic Euler, as integrate_cells: v += f w, x += dt v
                const float w = (float)((double)A.dtf * A.imass[__float_as_int(x.w)]);
                const float f0 = (float)((double)(long long)A.force[3 * (size_t)slot + 0] * (1.0 / 16777216.0));
                const float f1 = (float)((double)(long long)A.force[3 * (size_t)slot + 1] * (1.0 / 16777216.0));
                const float f2 = (float)((double)(long long)A.force[3 * (size_t)slot + 2] * (1.0 / 16777216.0));
                v.x = __fadd_rn(v.x, __fmul_rn(f0, w));
                v.y = __fadd_rn(v.y, __fmul_rn(f1, w));
                v.z = __fadd_rn(v.z, __fmul_rn(f2, w));
                x.x = __fadd_rn(x.x, __fmul_rn(A.dtf, v.x));
                x.y = __fadd_rn(x.y, __fmul_rn(A.dtf, v.y));
                x.z = __fadd_rn(x.z, __fmul_rn(A.dtf, v.z));
                A.rxq[slot] = x;
                A.rv[slot] = v;
                if (!isfinite(x.x + x.y + x.z + v.x + v.y + v.z)) atomicOr(A.status, 64ull);
            }
            int loc[3];
            slot_loc(A, slot, loc);
            for (int j = 0; j < 3; j++) sh[j] = shift_dim(loc[j], loc0[j]);
        } else {
            x = A.x[p0 + k];
            v = A.v[p0 + k];
            const int code = __float_as_int(x.w);
            sh[0] = code % 3 - 1;
            sh[1] = (code / 3) % 3 - 1;
            sh[2] = code / 9 - 1;
        }
        for (int j = 0; j < 3; j++) shifts[3 * k + j] = sh[j];
        const double s[3] = {(double)sh[0], (double)sh[1], (double)sh[2]};
        const double h[3] = {A.h0, A.h1, A.h2};
        const float xv[3] = {x.x, x.y, x.z}, vv[3] = {v.x, v.y, v.z};
        for (int j = 0; j < 3; j++) {
            // src/rigid.c:133-146: xp = x + h*shift; position before the step xp - dt*v
            xp[3 * k + j] = (double)xv[j] + h[j] * s[j];
            xo[3 * k + j] = xp[3 * k + j] - A.dt * (double)vv[j];
        }
        m[k] = A.mass[p0 + k];
    }
}

// The corrected positions: packed, to the FP64 output slots (the host applies them);
// resident, applied in place with the host's expressions (src/rigid.c:236-262):
// xn = xp - h*shift, v += (xn - x)/dt, x = xn.  The P-SHAKE constraint forces, which no
// later step reads, are not kept on the device.
template <bool RES>
__device__ __forceinline__ void store_group(const RigidArgs& A, int p0, int np, const double* xp, const int* shifts) {
    if (!RES) {
        for (int k = 0; k < 3 * np; k++) A.xp[3 * (size_t)p0 + k] = xp[k];
        return;
    }
    const double h[3] = {A.h0, A.h1, A.h2};
    const double idt = 1.0 / A.dt;
    for (int k = 0; k < np; k++) {
        const int slot = A.slot_of[A.id0 + A.rpid[p0 + k]];
        float4 x = A.rxq[slot], v = A.rv[slot];
        float* xs = &x.x;
        float* vs = &v.x;
        for (int j = 0; j < 3; j++) {
            const double xn = xp[3 * k + j] - h[j] * shifts[3 * k + j];
            vs[j] = (float)((double)vs[j] + idt * (xn - (double)xs[j]));
            xs[j] = (float)xn;
        }
        A.rxq[slot] = x;
        A.rv[slot] = v;
    }
}

// SHAKE, src/rigid.c:148-213, with every quantity in FP64.
template <int MP, int MC, bool RES>
__global__ void __launch_bounds__(128) rigid_shake(RigidArgs A) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.nrig) return;
    if (RES && A.abort != nullptr && *(const volatile unsigned long long*)A.abort != 0) return;
    if (RES && A.fuse && r == 0) {     // completed steps, accepted pairs (integrate_cells' job)
        A.done[0] += 1ull;
        A.done[1] += *A.pairs;
    }
    const int p0 = A.roff[r], np = A.roff[r + 1] - p0;
    const int c0 = A.coff[r], nc = A.coff[r + 1] - c0;
    if (np > MP || nc > MC || (!RES && __float_as_int(A.x[p0].w) < 0)) return;
    double xp[3 * MP], xo[3 * MP], m[MP], vc[3 * MC], wvc[3 * MC], res[MC];
    int shifts[3 * MP];
    load_group<RES>(A, p0, np, xp, xo, m, shifts);
    for (int k = 0; k < nc; k++) {
        const int2 c = A.cij[c0 + k];
        for (int j = 0; j < 3; j++) {
            vc[3 * k + j] = xo[3 * c.x + j] - xo[3 * c.y + j];
            wvc[3 * k + j] = 1.0 / (m[c.x] + m[c.y]) * vc[3 * k + j];
        }
    }
    int iter;
    for (iter = 0; iter < rigid_maxiter; iter++) {
        double max_res = 0.0;
        for (int k = 0; k < nc; k++) {
            const int2 c = A.cij[c0 + k];
            res[k] = A.d2[c0 + k];
            for (int j = 0; j < 3; j++)
                res[k] -= (xp[3 * c.x + j] - xp[3 * c.y + j]) * (xp[3 * c.x + j] - xp[3 * c.y + j]);
            if (fabs(res[k]) > max_res) max_res = fabs(res[k]);
        }
        if (max_res < A.tol) break;
        for (int k = 0; k < nc; k++) {
            const int2 c = A.cij[c0 + k];
            const double lambda = 0.5 * res[k] /
                                  ((xp[3 * c.x] - xp[3 * c.y]) * vc[3 * k] +
                                   (xp[3 * c.x + 1] - xp[3 * c.y + 1]) * vc[3 * k + 1] +
                                   (xp[3 * c.x + 2] - xp[3 * c.y + 2]) * vc[3 * k + 2]);
            for (int j = 0; j < 3; j++) {
                const double w = lambda * wvc[3 * k + j];
                xp[3 * c.x + j] += w * m[c.y];
                xp[3 * c.y + j] -= w * m[c.x];
            }
        }
    }
    atomicMax(&A.stat[0], iter);
    if (iter == rigid_maxiter) atomicAdd(&A.stat[1], 1);
    store_group<RES>(A, p0, np, xp, shifts);
}

// P-SHAKE, src/rigid.c:336-475: FP64 iterations over mixed constraint directions, the
// float mixing matrix refined as the reference does.
template <int MP, int MC, bool RES>
__global__ void __launch_bounds__(128) rigid_pshake(RigidArgs A) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.nrig) return;
    if (RES && A.abort != nullptr && *(const volatile unsigned long long*)A.abort != 0) return;
    if (RES && A.fuse && r == 0) {     // completed steps, accepted pairs (integrate_cells' job)
        A.done[0] += 1ull;
        A.done[1] += *A.pairs;
    }
    const int p0 = A.roff[r], np = A.roff[r + 1] - p0;
    const int c0 = A.coff[r], nc = A.coff[r + 1] - c0;
    if (np > MP || nc > MC || (!RES && __float_as_int(A.x[p0].w) < 0)) return;
    float* a = A.a + A.aoff[r];
    double xp[3 * MP], xo[3 * MP], m[MP], vc[3 * MC * MP];
    int shifts[3 * MP];
    load_group<RES>(A, p0, np, xp, xo, m, shifts);
    const int rowlen = 3 * np;
    for (int k = 0; k < nc * rowlen; k++) vc[k] = 0.0;
    for (int k = 0; k < nc; k++) {
        const int2 c = A.cij[c0 + k];
        double dv[3];
        for (int j = 0; j < 3; j++) dv[j] = (xo[3 * c.x + j] - xo[3 * c.y + j]) / (m[c.x] + m[c.y]);
        for (int i = 0; i < nc; i++) {
            const float aki = a[k * nc + i];
            if (aki != 0.0f)
                for (int j = 0; j < 3; j++) {
                    vc[i * rowlen + c.x * 3 + j] += aki * dv[j] * m[c.y];
                    vc[i * rowlen + c.y * 3 + j] += -aki * dv[j] * m[c.x];
                }
        }
    }
    int iter;
    for (iter = 0; iter < rigid_maxiter; iter++) {
        double max_res = 0.0;
        for (int k = 0; k < nc; k++) {
            const int2 c = A.cij[c0 + k];
            double res = A.d2[c0 + k];
            for (int j = 0; j < 3; j++)
                res -= (xp[3 * c.x + j] - xp[3 * c.y + j]) * (xp[3 * c.x + j] - xp[3 * c.y + j]);
            if (fabs(res) > max_res) max_res = fabs(res);
            const double* vk = vc + k * rowlen;
            const double lambda = 0.5 * res /
                                  ((xp[3 * c.x + 0] - xp[3 * c.y + 0]) * (vk[3 * c.x + 0] - vk[3 * c.y + 0]) +
                                   (xp[3 * c.x + 1] - xp[3 * c.y + 1]) * (vk[3 * c.x + 1] - vk[3 * c.y + 1]) +
                                   (xp[3 * c.x + 2] - xp[3 * c.y + 2]) * (vk[3 * c.x + 2] - vk[3 * c.y + 2]));
            for (int j = 0; j < rowlen; j++) xp[j] += lambda * vk[j];
        }
        if (max_res < A.tol) break;
    }
    atomicMax(&A.stat[0], iter);
    if (iter == rigid_maxiter) atomicAdd(&A.stat[1], 1);

    // Matrix refinement, src/rigid.c:433-474.
    if (nc > 1 && (A.a_update || iter > rigid_pshake_refine)) {
        float a_new[MC * MC], tmp[MC * MC];
        float max_alpha = 0.0f;
        for (int i = 0; i < nc; i++) {
            const int2 c = A.cij[c0 + i];
            float dx[3];
            for (int j = 0; j < 3; j++) dx[j] = (float)(xp[3 * c.x + j] - xp[3 * c.y + j]);
            const double* vi = vc + i * rowlen;
            const float w = (float)(-1.0 / ((double)dx[0] * (vi[3 * c.x + 0] - vi[3 * c.y + 0]) +
                                            (double)dx[1] * (vi[3 * c.x + 1] - vi[3 * c.y + 1]) +
                                            (double)dx[2] * (vi[3 * c.x + 2] - vi[3 * c.y + 2])));
            for (int j = i + 1; j < nc; j++) {
                const double* vj = vc + j * rowlen;
                a_new[i + j * nc] = (float)((double)w * ((double)dx[0] * (vj[3 * c.x + 0] - vj[3 * c.y + 0]) +
                                                         (double)dx[1] * (vj[3 * c.x + 1] - vj[3 * c.y + 1]) +
                                                         (double)dx[2] * (vj[3 * c.x + 2] - vj[3 * c.y + 2])));
                a_new[j + i * nc] = a_new[i + j * nc];
                max_alpha = fmaxf(max_alpha, fabsf(a_new[i + j * nc]));
            }
            a_new[i + i * nc] = 1.0f;
        }
        if (max_alpha > rigid_pshake_maxalpha) {
            const float w = (float)(0.1 / (double)max_alpha);
            for (int i = 0; i < nc * nc; i++) a_new[i] *= w;
            for (int i = 0; i < nc; i++) a_new[i * nc + i] = 1.0f;
        }
        for (int i = 0; i < nc * nc; i++) tmp[i] = 0.0f;
        for (int j = 0; j < nc; j++)
            for (int k = 0; k < nc; k++)
                for (int i = 0; i < nc; i++) tmp[j * nc + i] += a[k * nc + i] * a_new[j * nc + k];
        for (int i = 0; i < nc * nc; i++) a[i] = tmp[i];
    }
    store_group<RES>(A, p0, np, xp, shifts);
}

// ---- small groups (water: 3 particles, 3 constraints): the same iterations with every
// per-group array in registers.  Particle indices come from the constraint list at run
// time; each access compares them against the unrolled positions, so no array is indexed
// dynamically and none spills to local memory.  The arithmetic and its order are those of
// the kernels above.

template <int MP>
__device__ __forceinline__ void reg_get3(const double (&a)[MP][3], int p, double o[3]) {
    o[0] = a[0][0];
    o[1] = a[0][1];
    o[2] = a[0][2];
#pragma unroll
    for (int q = 1; q < MP; q++)
        if (p == q) {
            o[0] = a[q][0];
            o[1] = a[q][1];
            o[2] = a[q][2];
        }
}

template <int MP>
__device__ __forceinline__ double reg_get(const double (&a)[MP], int p) {
    double o = a[0];
#pragma unroll
    for (int q = 1; q < MP; q++)
        if (p == q) o = a[q];
    return o;
}

template <int MP, bool RES>
__device__ __forceinline__ void load_group_reg(const RigidArgs& A, int p0, int np, double (&xp)[MP][3],
                                               double (&xo)[MP][3], double (&m)[MP], int (&shifts)[MP][3]) {
    int loc0[3] = {0, 0, 0};
    if (RES) slot_loc(A, A.slot_of[A.id0 + A.rpid[p0]], loc0);
#pragma unroll
    for (int k = 0; k < MP; k++) {
        xp[k][0] = xp[k][1] = xp[k][2] = 0.0;
        xo[k][0] = xo[k][1] = xo[k][2] = 0.0;
        m[k] = 0.0;
        shifts[k][0] = shifts[k][1] = shifts[k][2] = 0;
        if (k >= np) continue;
        float4 x, v;
        int sh[3];
        if (RES) {
            const int slot = A.slot_of[A.id0 + A.rpid[p0 + k]];
            x = A.rxq[slot];
            v = A.rv[slot];
            if (A.fuse) {   // symplectic Euler, as integrate_cells: v += f w, x += dt v
                const float w = (float)((double)A.dtf * A.imass[__float_as_int(x.w)]);
                const float f0 = (float)((double)(long long)A.force[3 * (size_t)slot + 0] * (1.0 / 16777216.0));
                const float f1 = (float)((double)(long long)A.force[3 * (size_t)slot + 1] * (1.0 / 16777216.0));
                const float f2 = (float)((double)(long long)A.force[3 * (size_t)slot + 2] * (1.0 / 16777216.0));
                v.x = __fadd_rn(v.x, __fmul_rn(f0, w));
                v.y = __fadd_rn(v.y, __fmul_rn(f1, w));
                v.z = __fadd_rn(v.z, __fmul_rn(f2, w));
                x.x = __fadd_rn(x.x, __fmul_rn(A.dtf, v.x));
                x.y = __fadd_rn(x.y, __fmul_rn(A.dtf, v.y));
                x.z = __fadd_rn(x.z, __fmul_rn(A.dtf, v.z));
                A.rxq[slot] = x;
                A.rv[slot] = v;
                if (!isfinite(x.x + x.y + x.z + v.x + v.y + v.z)) atomicOr(A.status, 64ull);
            }
            int loc[3];
            slot_loc(A, slot, loc);
#pragma unroll
            for (int j = 0; j < 3; j++) sh[j] = shift_dim(loc[j], loc0[j]);
        } else {
            x = A.x[p0 + k];
            v = A.v[p0 + k];
            const int code = __float_as_int(x.w);
            sh[0] = code % 3 - 1;
            sh[1] = (code / 3) % 3 - 1;
            sh[2] = code / 9 - 1;
        }
        const double h[3] = {A.h0, A.h1, A.h2};
        const float xv[3] = {x.x, x.y, x.z}, vv[3] = {v.x, v.y, v.z};
#pragma unroll
        for (int j = 0; j < 3; j++) {
            shifts[k][j] = sh[j];
            xp[k][j] = (double)xv[j] + h[j] * (double)sh[j];
            xo[k][j] = xp[k][j] - A.dt * (double)vv[j];
        }
        m[k] = A.mass[p0 + k];
    }
}

template <int MP, bool RES>
__device__ __forceinline__ void store_group_reg(const RigidArgs& A, int p0, int np, const double (&xp)[MP][3],
                                                const int (&shifts)[MP][3]) {
    const double h[3] = {A.h0, A.h1, A.h2};
    const double idt = 1.0 / A.dt;
#pragma unroll
    for (int k = 0; k < MP; k++) {
        if (k >= np) continue;
        if (!RES) {
#pragma unroll
            for (int j = 0; j < 3; j++) A.xp[3 * (size_t)p0 + 3 * k + j] = xp[k][j];
            continue;
        }
        const int slot = A.slot_of[A.id0 + A.rpid[p0 + k]];
        float4 x = A.rxq[slot], v = A.rv[slot];
        float xs[3] = {x.x, x.y, x.z}, vs[3] = {v.x, v.y, v.z};
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const double xn = xp[k][j] - h[j] * shifts[k][j];
            vs[j] = (float)((double)vs[j] + idt * (xn - (double)xs[j]));
            xs[j] = (float)xn;
        }
        A.rxq[slot] = make_float4(xs[0], xs[1], xs[2], x.w);
        A.rv[slot] = make_float4(vs[0], vs[1], vs[2], v.w);
    }
}

template <int MP, int MC, bool RES>
__global__ void __launch_bounds__(64) rigid_shake_reg(RigidArgs A) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.nrig) return;
    if (RES && A.abort != nullptr && *(const volatile unsigned long long*)A.abort != 0) return;
    if (RES && A.fuse && r == 0) {     // completed steps, accepted pairs (integrate_cells' job)
        A.done[0] += 1ull;
        A.done[1] += *A.pairs;
    }
    const int p0 = A.roff[r], np = A.roff[r + 1] - p0;
    const int c0 = A.coff[r], nc = A.coff[r + 1] - c0;
    if (np > MP || nc > MC || (!RES && __float_as_int(A.x[p0].w) < 0)) return;
    double xp[MP][3], xo[MP][3], m[MP], vc[MC][3], wvc[MC][3], res[MC];
    int shifts[MP][3], cx[MC], cy[MC];
    load_group_reg<MP, RES>(A, p0, np, xp, xo, m, shifts);
#pragma unroll
    for (int k = 0; k < MC; k++) {
        cx[k] = cy[k] = 0;
        if (k >= nc) continue;
        const int2 c = A.cij[c0 + k];
        cx[k] = c.x;
        cy[k] = c.y;
        double a[3], b[3];
        reg_get3<MP>(xo, c.x, a);
        reg_get3<MP>(xo, c.y, b);
        const double mx = reg_get<MP>(m, c.x), my = reg_get<MP>(m, c.y);
#pragma unroll
        for (int j = 0; j < 3; j++) {
            vc[k][j] = a[j] - b[j];
            wvc[k][j] = 1.0 / (mx + my) * vc[k][j];
        }
    }
    int iter;
    for (iter = 0; iter < rigid_maxiter; iter++) {
        double max_res = 0.0;
#pragma unroll
        for (int k = 0; k < MC; k++) {
            if (k >= nc) continue;
            double a[3], b[3];
            reg_get3<MP>(xp, cx[k], a);
            reg_get3<MP>(xp, cy[k], b);
            res[k] = A.d2[c0 + k];
#pragma unroll
            for (int j = 0; j < 3; j++) res[k] -= (a[j] - b[j]) * (a[j] - b[j]);
            if (fabs(res[k]) > max_res) max_res = fabs(res[k]);
        }
        if (max_res < A.tol) break;
#pragma unroll
        for (int k = 0; k < MC; k++) {
            if (k >= nc) continue;
            double a[3], b[3];
            reg_get3<MP>(xp, cx[k], a);
            reg_get3<MP>(xp, cy[k], b);
            const double lambda =
                0.5 * res[k] / ((a[0] - b[0]) * vc[k][0] + (a[1] - b[1]) * vc[k][1] + (a[2] - b[2]) * vc[k][2]);
            const double mx = reg_get<MP>(m, cx[k]), my = reg_get<MP>(m, cy[k]);
#pragma unroll
            for (int q = 0; q < MP; q++) {
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    const double w = lambda * wvc[k][j];
                    if (q == cx[k]) xp[q][j] += w * my;
                    if (q == cy[k]) xp[q][j] -= w * mx;
                }
            }
        }
    }
    atomicMax(&A.stat[0], iter);
    if (iter == rigid_maxiter) atomicAdd(&A.stat[1], 1);
    store_group_reg<MP, RES>(A, p0, np, xp, shifts);
}

template <int MP, int MC, bool RES>
__global__ void __launch_bounds__(64) rigid_pshake_reg(RigidArgs A) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.nrig) return;
    if (RES && A.abort != nullptr && *(const volatile unsigned long long*)A.abort != 0) return;
    if (RES && A.fuse && r == 0) {     // completed steps, accepted pairs (integrate_cells' job)
        A.done[0] += 1ull;
        A.done[1] += *A.pairs;
    }
    const int p0 = A.roff[r], np = A.roff[r + 1] - p0;
    const int c0 = A.coff[r], nc = A.coff[r + 1] - c0;
    if (np > MP || nc > MC || (!RES && __float_as_int(A.x[p0].w) < 0)) return;
    float* a = A.a + A.aoff[r];
    double xp[MP][3], xo[MP][3], m[MP], vc[MC][MP][3];
    int shifts[MP][3], cx[MC], cy[MC];
    load_group_reg<MP, RES>(A, p0, np, xp, xo, m, shifts);
#pragma unroll
    for (int i = 0; i < MC; i++)
#pragma unroll
        for (int q = 0; q < MP; q++) vc[i][q][0] = vc[i][q][1] = vc[i][q][2] = 0.0;
#pragma unroll
    for (int k = 0; k < MC; k++) {
        cx[k] = cy[k] = 0;
        if (k >= nc) continue;
        const int2 c = A.cij[c0 + k];
        cx[k] = c.x;
        cy[k] = c.y;
        double ox[3], oy[3], dv[3];
        reg_get3<MP>(xo, c.x, ox);
        reg_get3<MP>(xo, c.y, oy);
        const double mx = reg_get<MP>(m, c.x), my = reg_get<MP>(m, c.y);
#pragma unroll
        for (int j = 0; j < 3; j++) dv[j] = (ox[j] - oy[j]) / (mx + my);
#pragma unroll
        for (int i = 0; i < MC; i++) {
            if (i >= nc) continue;
            const float aki = a[k * nc + i];
            if (aki != 0.0f)
#pragma unroll
                for (int q = 0; q < MP; q++)
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        if (q == c.x) vc[i][q][j] += aki * dv[j] * my;
                        if (q == c.y) vc[i][q][j] += -aki * dv[j] * mx;
                    }
        }
    }
    int iter;
    for (iter = 0; iter < rigid_maxiter; iter++) {
        double max_res = 0.0;
#pragma unroll
        for (int k = 0; k < MC; k++) {
            if (k >= nc) continue;
            double a1[3], b1[3], va[3], vb[3];
            reg_get3<MP>(xp, cx[k], a1);
            reg_get3<MP>(xp, cy[k], b1);
            reg_get3<MP>(vc[k], cx[k], va);
            reg_get3<MP>(vc[k], cy[k], vb);
            double res = A.d2[c0 + k];
#pragma unroll
            for (int j = 0; j < 3; j++) res -= (a1[j] - b1[j]) * (a1[j] - b1[j]);
            if (fabs(res) > max_res) max_res = fabs(res);
            const double lambda = 0.5 * res /
                                  ((a1[0] - b1[0]) * (va[0] - vb[0]) + (a1[1] - b1[1]) * (va[1] - vb[1]) +
                                   (a1[2] - b1[2]) * (va[2] - vb[2]));
#pragma unroll
            for (int q = 0; q < MP; q++)
#pragma unroll
                for (int j = 0; j < 3; j++)
                    if (q < np) xp[q][j] += lambda * vc[k][q][j];
        }
        if (max_res < A.tol) break;
    }
    atomicMax(&A.stat[0], iter);
    if (iter == rigid_maxiter) atomicAdd(&A.stat[1], 1);

    // Matrix refinement, src/rigid.c:433-474.
    if (nc > 1 && (A.a_update || iter > rigid_pshake_refine)) {
        float a_new[MC][MC], tmp[MC][MC];
        float max_alpha = 0.0f;
#pragma unroll
        for (int i = 0; i < MC; i++) {
            if (i >= nc) continue;
            double pa[3], pb[3], va[3], vb[3];
            reg_get3<MP>(xp, cx[i], pa);
            reg_get3<MP>(xp, cy[i], pb);
            float dx[3];
#pragma unroll
            for (int j = 0; j < 3; j++) dx[j] = (float)(pa[j] - pb[j]);
            reg_get3<MP>(vc[i], cx[i], va);
            reg_get3<MP>(vc[i], cy[i], vb);
            const float w = (float)(-1.0 / ((double)dx[0] * (va[0] - vb[0]) + (double)dx[1] * (va[1] - vb[1]) +
                                            (double)dx[2] * (va[2] - vb[2])));
#pragma unroll
            for (int j = 0; j < MC; j++) {
                if (j <= i || j >= nc) continue;
                double ja[3], jb[3];
                reg_get3<MP>(vc[j], cx[i], ja);
                reg_get3<MP>(vc[j], cy[i], jb);
                a_new[j][i] = (float)((double)w * ((double)dx[0] * (ja[0] - jb[0]) + (double)dx[1] * (ja[1] - jb[1]) +
                                                   (double)dx[2] * (ja[2] - jb[2])));
                a_new[i][j] = a_new[j][i];
                max_alpha = fmaxf(max_alpha, fabsf(a_new[j][i]));
            }
            a_new[i][i] = 1.0f;
        }
        if (max_alpha > rigid_pshake_maxalpha) {
            const float w = (float)(0.1 / (double)max_alpha);
#pragma unroll
            for (int i = 0; i < MC; i++)
#pragma unroll
                for (int j = 0; j < MC; j++)
                    if (i < nc && j < nc) a_new[i][j] *= w;
#pragma unroll
            for (int i = 0; i < MC; i++)
                if (i < nc) a_new[i][i] = 1.0f;
        }
#pragma unroll
        for (int j = 0; j < MC; j++)
#pragma unroll
            for (int i = 0; i < MC; i++) tmp[j][i] = 0.0f;
#pragma unroll
        for (int j = 0; j < MC; j++) {
            if (j >= nc) continue;
#pragma unroll
            for (int k = 0; k < MC; k++) {
                if (k >= nc) continue;
#pragma unroll
                for (int i = 0; i < MC; i++)
                    if (i < nc) tmp[j][i] += a[k * nc + i] * a_new[j][k];
            }
        }
#pragma unroll
        for (int j = 0; j < MC; j++)
#pragma unroll
            for (int i = 0; i < MC; i++)
                if (j < nc && i < nc) a[j * nc + i] = tmp[j][i];
    }
    store_group_reg<MP, RES>(A, p0, np, xp, shifts);
}

struct RigidDev {
    int device = 0;
    int gen = -1, nrig = 0, nslots = 0, ncon = 0, namat = 0, maxp = 0, maxc = 0;
    cudaStream_t own_stream = nullptr;
    int *d_roff = nullptr, *d_coff = nullptr, *d_aoff = nullptr, *d_stat = nullptr, *d_rpid = nullptr;
    int2* d_cij = nullptr;
    double *d_d2 = nullptr, *d_mass = nullptr, *d_xp = nullptr;
    float* d_a = nullptr;
    float4 *d_x = nullptr, *d_v = nullptr;
    float4 *h_x = nullptr, *h_v = nullptr;
    double* h_xp = nullptr;
    int* h_stat = nullptr;
    std::vector<int> roff;
    std::vector<unsigned char> skip;     // groups not all present this evaluation
};

int rigid_fail(cudaError_t err, int line, const char* func) {
    errs_register(engine_err_cuda, cudaGetErrorString(err), line, func, __FILE__);
    engine_err = engine_err_cuda;
    return engine_err_cuda;
}

#define CU(call)                                                             \
    do {                                                                     \
        cudaError_t err_ = (call);                                           \
        if (err_ != cudaSuccess) return rigid_fail(err_, __LINE__, __func__); \
    } while (0)

void free_buffers(RigidDev* rd) {
    void* dev[] = {rd->d_roff, rd->d_coff, rd->d_aoff, rd->d_stat, rd->d_cij, rd->d_d2,
                   rd->d_mass, rd->d_xp, rd->d_a, rd->d_x, rd->d_v, rd->d_rpid};
    for (void* p : dev) cudaFree(p);
    void* host[] = {rd->h_x, rd->h_v, rd->h_xp, rd->h_stat};
    for (void* p : host) cudaFreeHost(p);
    rd->d_roff = rd->d_coff = rd->d_aoff = rd->d_stat = rd->d_rpid = nullptr;
    rd->d_cij = nullptr;
    rd->d_d2 = rd->d_mass = rd->d_xp = nullptr;
    rd->d_a = nullptr;
    rd->d_x = rd->d_v = nullptr;
    rd->h_x = rd->h_v = nullptr;
    rd->h_xp = nullptr;
    rd->h_stat = nullptr;
}

template <typename T>
int upload(T** d, const std::vector<T>& h) {
    CU(cudaMalloc(reinterpret_cast<void**>(d), sizeof(T) * (h.size() + 1)));
    if (!h.empty()) CU(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return 0;
}

// (Re)builds the static description of the groups after engine_rigid_add changed them.
int build(struct engine* e, RigidDev* rd) {
    free_buffers(rd);
    std::vector<int> roff(1, 0), coff(1, 0), aoff(1, 0), rpid;
    std::vector<int2> cij;
    std::vector<double> d2, mass;
    std::vector<float> amat;
    rd->maxp = rd->maxc = 0;
    for (int g = 0; g < e->nr_rigids; g++) {
        const struct rigid* r = &e->rigids[g];
        for (int k = 0; k < r->nr_parts; k++) {
            const int id = r->parts[k];
            const struct part* p = (id >= 0 && id < e->s.size_parts) ? e->s.partlist[id] : nullptr;
            mass.push_back(p ? e->types[p->type].mass : 1.0);
            rpid.push_back(id);
        }
        for (int k = 0; k < r->nr_constr; k++) {
            cij.push_back(make_int2(r->constr[k].i, r->constr[k].j));
            d2.push_back(r->constr[k].d2);
        }
        amat.insert(amat.end(), r->a, r->a + r->nr_constr * r->nr_constr);
        roff.push_back(roff.back() + r->nr_parts);
        coff.push_back(coff.back() + r->nr_constr);
        aoff.push_back(aoff.back() + r->nr_constr * r->nr_constr);
        rd->maxp = std::max(rd->maxp, r->nr_parts);
        rd->maxc = std::max(rd->maxc, r->nr_constr);
    }
    rd->nrig = e->nr_rigids;
    rd->nslots = roff.back();
    rd->ncon = coff.back();
    rd->namat = aoff.back();
    rd->roff = roff;
    rd->skip.assign(rd->nrig + 1, 0);
    if (upload(&rd->d_roff, roff) || upload(&rd->d_coff, coff) || upload(&rd->d_aoff, aoff) ||
        upload(&rd->d_cij, cij) || upload(&rd->d_d2, d2) || upload(&rd->d_mass, mass) || upload(&rd->d_a, amat) ||
        upload(&rd->d_rpid, rpid))
        return engine_err_cuda;
    const size_t ns = (size_t)rd->nslots + 1;
    CU(cudaMalloc(&rd->d_x, sizeof(float4) * ns));
    CU(cudaMalloc(&rd->d_v, sizeof(float4) * ns));
    CU(cudaMalloc(&rd->d_xp, sizeof(double) * 3 * ns));
    CU(cudaMalloc(&rd->d_stat, sizeof(int) * 2));
    CU(cudaMallocHost(&rd->h_x, sizeof(float4) * ns));
    CU(cudaMallocHost(&rd->h_v, sizeof(float4) * ns));
    CU(cudaMallocHost(&rd->h_xp, sizeof(double) * 3 * ns));
    CU(cudaMallocHost(&rd->h_stat, sizeof(int) * 2));
    rd->h_stat[0] = rd->h_stat[1] = 0;
    rd->gen = e->rigids_gen;
    return 0;
}

// Periodic cell offset of particle cell c relative to the group's first cell c0, per
// dimension -1, 0 or +1 (src/rigid.c:133-141).
inline int shift_of(const struct cell* c, const struct cell* c0, int j) {
    int s = c->loc[j] - c0->loc[j];
    if (s > 1) s = -1;
    else if (s < -1) s = 1;
    return s;
}

float bits_float(int v) {
    float f;
    std::memcpy(&f, &v, sizeof(f));
    return f;
}

template <int MP, int MC, bool RES>
void launch(bool pshake, const RigidArgs& A, cudaStream_t s) {
    const int grid = (A.nrig + 63) / 64;     // 64 groups per block: every SM gets work
    if (pshake)
        rigid_pshake<MP, MC, RES><<<grid, 64, 0, s>>>(A);
    else
        rigid_shake<MP, MC, RES><<<grid, 64, 0, s>>>(A);
}

template <int MP, int MC, bool RES>
void launch_reg(bool pshake, const RigidArgs& A, cudaStream_t s) {
    const int grid = (A.nrig + 63) / 64;
    if (pshake)
        rigid_pshake_reg<MP, MC, RES><<<grid, 64, 0, s>>>(A);
    else
        rigid_shake_reg<MP, MC, RES><<<grid, 64, 0, s>>>(A);
}

template <bool RES>
void launch_sized(const RigidDev* rd, bool pshake, const RigidArgs& A, cudaStream_t s) {
    if (rd->maxp <= 3 && rd->maxc <= 3)
        launch_reg<3, 3, RES>(pshake, A, s);
    else if (rd->maxp <= 4 && rd->maxc <= 6)
        launch_reg<4, 6, RES>(pshake, A, s);
    else
        launch<rigid_maxparts, rigid_maxconstr, RES>(pshake, A, s);
}

}  // namespace

extern "C" int rigid_device_free(struct engine* e) {
    if (e == nullptr || e->cuda_rigid == nullptr) return 0;
    RigidDev* rd = static_cast<RigidDev*>(e->cuda_rigid);
    cudaSetDevice(rd->device);
    free_buffers(rd);
    if (rd->own_stream) cudaStreamDestroy(rd->own_stream);
    delete rd;
    e->cuda_rigid = nullptr;
    return 0;
}

extern "C" int engine_rigid_eval(struct engine* e) {
    if (e == nullptr) return engine_err_null;
    if (e->nr_rigids == 0) return 0;
    if (e->dt == 0.0) {
        errs_register(engine_err_rigid, "Rigid constraints need a non-zero time step.", __LINE__, __func__, __FILE__);
        return engine_err = engine_err_rigid;
    }
    RigidDev* rd = static_cast<RigidDev*>(e->cuda_rigid);
    if (rd == nullptr) {
        rd = new RigidDev();
        rd->device = e->device;
        e->cuda_rigid = rd;
    }
    CU(cudaSetDevice(rd->device));
    if (rd->gen != e->rigids_gen || rd->nrig != e->nr_rigids) {
        const int rc = build(e, rd);
        if (rc < 0) return rc;
    }
    cudaStream_t stream = static_cast<cudaStream_t>(nb_engine_stream(e));
    if (stream == nullptr) {
        if (rd->own_stream == nullptr) CU(cudaStreamCreateWithFlags(&rd->own_stream, cudaStreamNonBlocking));
        stream = rd->own_stream;
    }
    struct space* s = &e->s;
    const bool pshake = !(e->flags & engine_flag_shake);

    // Pack: cell-relative positions, velocities and shift codes of every group's particles
    // (host threads over ranges of groups).
    HostPool::get().run(rd->nrig, 1024, [&](int, int gb, int ge) {
    for (int g = gb; g < ge; g++) {
        const struct rigid* r = &e->rigids[g];
        const int p0 = rd->roff[g];
        bool local = true;
        for (int k = 0; k < r->nr_parts; k++) {
            const int id = r->parts[k];
            if (id < 0 || id >= s->size_parts || s->partlist[id] == nullptr) local = false;
        }
        rd->skip[g] = !local;
        if (!local) {                       // src/rigid.c:119-125: skip groups not all present
            rd->h_x[p0] = make_float4(0.f, 0.f, 0.f, bits_float(-1));
            continue;
        }
        const struct cell* cfirst = s->celllist[r->parts[0]];
        for (int k = 0; k < r->nr_parts; k++) {
            const int id = r->parts[k];
            const struct part* p = s->partlist[id];
            const struct cell* c = s->celllist[id];
            const int code = (shift_of(c, cfirst, 0) + 1) + 3 * (shift_of(c, cfirst, 1) + 1) +
                             9 * (shift_of(c, cfirst, 2) + 1);
            rd->h_x[p0 + k] = make_float4(p->x[0], p->x[1], p->x[2], bits_float(code));
            rd->h_v[p0 + k] = make_float4(p->v[0], p->v[1], p->v[2], 0.f);
        }
    }
    });
    const size_t ns = (size_t)rd->nslots;
    CU(cudaMemcpyAsync(rd->d_x, rd->h_x, sizeof(float4) * ns, cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(rd->d_v, rd->h_v, sizeof(float4) * ns, cudaMemcpyHostToDevice, stream));
    CU(cudaMemsetAsync(rd->d_stat, 0, sizeof(int) * 2, stream));

    RigidArgs A;
    A.nrig = rd->nrig;
    A.roff = rd->d_roff;
    A.coff = rd->d_coff;
    A.aoff = rd->d_aoff;
    A.cij = rd->d_cij;
    A.d2 = rd->d_d2;
    A.mass = rd->d_mass;
    A.x = rd->d_x;
    A.v = rd->d_v;
    A.a = rd->d_a;
    A.xp = rd->d_xp;
    A.stat = rd->d_stat;
    A.h0 = s->h[0];
    A.h1 = s->h[1];
    A.h2 = s->h[2];
    A.dt = e->dt;
    A.tol = e->tol_rigid;
    A.a_update = e->time < engine_pshake_steps;
    launch_sized<false>(rd, pshake, A, stream);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(rd->h_xp, rd->d_xp, sizeof(double) * 3 * ns, cudaMemcpyDeviceToHost, stream));
    CU(cudaMemcpyAsync(rd->h_stat, rd->d_stat, sizeof(int) * 2, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));

    // Corrections, src/rigid.c:236-262 (SHAKE) and src/rigid.c:486-511 (P-SHAKE).
    const double idt = 1.0 / e->dt;
    HostPool::get().run(rd->nrig, 1024, [&](int, int gb, int ge) {
    for (int g = gb; g < ge; g++) {
        const struct rigid* r = &e->rigids[g];
        const int p0 = rd->roff[g];
        if (rd->skip[g]) continue;
        const struct cell* cfirst = s->celllist[r->parts[0]];
        for (int k = 0; k < r->nr_parts; k++) {
            const int id = r->parts[k];
            struct part* p = s->partlist[id];
            const struct cell* c = s->celllist[id];
            const double m = e->types[p->type].mass;
            for (int j = 0; j < 3; j++) {
                const double xn = rd->h_xp[3 * (size_t)(p0 + k) + j] - s->h[j] * shift_of(c, cfirst, j);
                if (pshake) p->f[j] += idt * idt * (xn - p->x[j]) * m;
                p->v[j] += idt * (xn - p->x[j]);
                p->x[j] = xn;
            }
        }
    }
    });
    return 0;
}

extern "C" int engine_rigid_stats(struct engine* e, int* max_iter, int* unconverged) {
    if (e == nullptr) return engine_err_null;
    const RigidDev* rd = static_cast<const RigidDev*>(e->cuda_rigid);
    if (max_iter) *max_iter = rd && rd->h_stat ? rd->h_stat[0] : 0;
    if (unconverged) *unconverged = rd && rd->h_stat ? rd->h_stat[1] : 0;
    return 0;
}

extern "C" int engine_rigid_getmatrices(struct engine* e) {
    if (e == nullptr) return engine_err_null;
    RigidDev* rd = static_cast<RigidDev*>(e->cuda_rigid);
    if (rd == nullptr || rd->gen != e->rigids_gen) return 0;     // the host copies are current
    CU(cudaSetDevice(rd->device));
    std::vector<float> amat((size_t)rd->namat + 1);
    CU(cudaDeviceSynchronize());
    CU(cudaMemcpy(amat.data(), rd->d_a, sizeof(float) * rd->namat, cudaMemcpyDeviceToHost));
    size_t off = 0;
    for (int g = 0; g < e->nr_rigids; g++) {
        struct rigid* r = &e->rigids[g];
        const size_t n = (size_t)r->nr_constr * r->nr_constr;
        std::memcpy(r->a, amat.data() + off, sizeof(float) * n);
        off += n;
    }
    return 0;
}

// Rigid constraints of a device-resident step: the groups' particles are read and
// corrected in place in the device cells (see nb_resident.cuh) on `stream`; the iteration
// statistics of the step stay on the device until rigid_resident_stats.  Capturable in a
// CUDA graph: no host work, no allocation after the first call.
extern "C" int rigid_eval_resident(struct engine* e, const struct rigid_resident_view* view, void* stream_v) {
    if (e == nullptr || view == nullptr) return engine_err_null;
    if (e->nr_rigids == 0) return 0;
    RigidDev* rd = static_cast<RigidDev*>(e->cuda_rigid);
    if (rd == nullptr) {
        rd = new RigidDev();
        rd->device = e->device;
        e->cuda_rigid = rd;
    }
    CU(cudaSetDevice(rd->device));
    if (rd->gen != e->rigids_gen || rd->nrig != e->nr_rigids) {
        const int rc = build(e, rd);
        if (rc < 0) return rc;
    }
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    struct space* s = &e->s;
    RigidArgs A = {};
    A.nrig = rd->nrig;
    A.roff = rd->d_roff;
    A.coff = rd->d_coff;
    A.aoff = rd->d_aoff;
    A.cij = rd->d_cij;
    A.d2 = rd->d_d2;
    A.mass = rd->d_mass;
    A.a = rd->d_a;
    A.stat = rd->d_stat;
    A.h0 = s->h[0];
    A.h1 = s->h[1];
    A.h2 = s->h[2];
    A.dt = e->dt;
    A.tol = e->tol_rigid;
    A.a_update = e->time < engine_pshake_steps;
    A.rpid = rd->d_rpid;
    A.slot_of = view->slot_of;
    A.id0 = view->id0;
    A.rxq = static_cast<float4*>(view->xq);
    A.rv = static_cast<float4*>(view->v);
    A.capc = view->capc;
    A.cell0 = view->cell0;
    A.cd0 = s->cdim[0];
    A.cd1 = s->cdim[1];
    A.cd2 = s->cdim[2];
    A.abort = view->abort;
    A.fuse = view->fuse;
    A.force = view->force;
    A.imass = view->imass;
    A.dtf = view->dtf;
    A.status = view->status;
    A.done = view->done;
    A.pairs = view->pairs;
    CU(cudaMemsetAsync(rd->d_stat, 0, sizeof(int) * 2, stream));
    launch_sized<true>(rd, !(e->flags & engine_flag_shake), A, stream);
    CU(cudaGetLastError());
    return 0;
}

// Iteration statistics of the last resident step (device counters to the host copy).
extern "C" int rigid_resident_stats(struct engine* e, void* stream_v, int wait) {
    if (e == nullptr || e->cuda_rigid == nullptr) return 0;
    RigidDev* rd = static_cast<RigidDev*>(e->cuda_rigid);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    CU(cudaMemcpyAsync(rd->h_stat, rd->d_stat, sizeof(int) * 2, cudaMemcpyDeviceToHost, stream));
    if (wait) CU(cudaStreamSynchronize(stream));
    return 0;
}
