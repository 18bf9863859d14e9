/* ORACLE -- test infrastructure only.  Nothing in the product links against, loads or calls
 * this file; tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it as the
 * checker.
 *
 * A CPU restatement of the reference mdcore nonbonded evaluation, in plain C, on the same
 * single-precision inputs the reference and the GPU engine see (cell-local float
 * coordinates, float potential tables):
 *
 *   - cell grid and task list: src/space.c:530-783 (space_init) with the shift/flip rule of
 *     src/space.c:80-114 (space_getsid);
 *   - pair set: every (i, j) of a pair task and every j < i of a self task whose float r2,
 *     computed as src/runner_dopair.c:625-631 does (pix = x_i - shift, dx = pix - x_j,
 *     r2 = (dx0^2 + dx1^2) + dx2^2), is <= cutoff^2 with a potential for the two types
 *     (src/runner_dopair.c:640-642, 954-955).  The cut is the float cutoff squared in float
 *     for pair tasks (src/runner_dopair.c:578-579) and the float of the double square for
 *     self tasks (src/runner_dopair.c:896).  For cubic cells the sorted sweep of the
 *     reference is a pruned walk over exactly this set, so the oracle enumerates it by brute
 *     force.  (For non-cubic cells the reference's sweep bound, the norm of the cell shift
 *     instead of its projection on the sort axis, src/runner_dopair.c:593-597, skips some
 *     pairs of this set; the engine uses the projection there and keeps them);
 *   - exclusions: excluded pairs are removed from the set (src/exclusion.c:81-295 subtracts
 *     them after the sweep, which is the same sum) and counted;
 *   - potential evaluation: the interval index is computed in float exactly as
 *     src/potential_eval.h:67-81 does, so the same chunk of the float table is used; the
 *     polynomial, the distance, the force and all sums are then evaluated in double
 *     (src/potential_eval.h:84-103 restated in FP64);
 *   - sort keys: src/runner_dosort.c:140-153, ordered by descending distance with ties in
 *     storage order;
 *   - bonded terms in double on the same float cell-relative positions: bonds
 *     (src/bond.c:81-250), angles (src/angle.c:81-300) and dihedrals (src/dihedral.c:81-380),
 *     each position taken near the cell of the second particle as the reference does, the
 *     table interval picked from a float copy of the distance or cosine; angle and
 *     dihedral gradients are written here from the vector form of d cos/dx (pinned against
 *     the reference's own bond_eval/angle_eval/dihedral_eval outputs in
 *     tests/golden/bonded.npz);
 *   - explicit electrostatics (the engine_setexplepot extension; the reference stores ep,
 *     src/engine.c:1029-1053, but no runner evaluates it): with table ep, every pair within
 *     the cutoff that is not excluded also contributes q_i q_j ep(r) to energy and force,
 *     and a pair whose types have no potential is in the set when ep is given.
 *
 * Compile with -ffp-contract=off: the float steps must round like the reference build.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define CELLID(cd, i, j, k) ((((i) * (cd)[1] + (j)) * (cd)[2]) + (k))

struct ocell {
    double origin[3];
    int start, count;
};

/* Shift and flip of src/space.c:80-114: returns the sort direction, swaps *a and *b when the
 * shift points into the negative half-space. */
static int getsid(const double dim[3], const struct ocell *cells, int *a, int *b, float shift[3]) {
    int idx = 0;
    for (int k = 0; k < 3; k++) {
        shift[k] = cells[*b].origin[k] - cells[*a].origin[k];
        if (shift[k] * 2 > dim[k])
            shift[k] -= dim[k];
        else if (shift[k] * 2 < -dim[k])
            shift[k] += dim[k];
    }
    for (int k = 0; k < 3; k++) idx = 3 * idx + ((shift[k] < 0) ? 0 : ((shift[k] > 0) ? 2 : 1));
    if (idx < 13) {
        int t = *a; *a = *b; *b = t;
        for (int k = 0; k < 3; k++) shift[k] = -shift[k];
        return idx;
    }
    return 26 - idx;
}

static int excl_cmp(const void *x, const void *y) {
    const long long a = *(const long long *)x, b = *(const long long *)y;
    return (a > b) - (a < b);
}

static int is_excluded(const long long *keys, int n, int i, int j) {
    long long key = (i < j) ? ((long long)i << 32) | (unsigned)j : ((long long)j << 32) | (unsigned)i;
    return bsearch(&key, keys, n, sizeof(long long), excl_cmp) != NULL;
}

/* Interval index in float (src/potential_eval.h:74-78), polynomial in double. */
static void eval_fp64(const float *coef, const float *alpha, int nmax, float r2f, double r, double *e, double *f) {
    float rf = sqrtf(r2f);
    int ind = (int)fmaxf(0.0f, alpha[0] + rf * (alpha[1] + rf * alpha[2]));
    if (ind > nmax) ind = nmax;
    const float *c = &coef[8 * ind];
    double x = (r - (double)c[0]) * (double)c[1];
    double ee = (double)c[2] * x + (double)c[3];
    double eff = (double)c[2];
    for (int k = 4; k < 8; k++) {
        eff = eff * x + ee;
        ee = ee * x + (double)c[k];
    }
    *e = ee;
    *f = eff * (double)c[1] / r;
}

/* Nonbonded forces (by particle id, FP64), energy, virial, the sums over pairs of |e_ij|
 * and |r_ij . F_ij| (the scales of the rounding errors of energy and virial: the net values
 * may cancel to far less) and counts.
 *   xrel[3N] float cell-local positions, cell[N] cell index, type[N]
 *   coef: tables concatenated; alpha[4*npots]; coff[npots] float offset of each table;
 *   potn[npots]; potidx[mt*mt] table index or -1.
 * Returns 0, or -1 on bad input. */
int oracle_nonbond(int N, const float *xrel, const int *cell, const int *type,
                   const double *origin, const double *dim, const int *cdim, double cutoff,
                   unsigned period, int mt, const int *potidx, const float *coef, const float *alpha,
                   const int *coff, const int *potn, int nexcl, const int *excl,
                   double *f_out, double *epot_out, double *epot_abs_out, double *virial_out,
                   double *virial_abs_out, long long *npairs_out, long long *nexcl_out, const double *q,
                   int ep) {
    const int ncells = cdim[0] * cdim[1] * cdim[2];
    double h[3];
    int span[3];
    for (int k = 0; k < 3; k++) {
        h[k] = dim[k] / cdim[k];
        span[k] = ceil(cutoff * (1.0 / h[k]));
    }
    struct ocell *cells = calloc(ncells, sizeof(struct ocell));
    int *order = malloc(sizeof(int) * (N + 1));
    long long *ekeys = malloc(sizeof(long long) * (nexcl + 1));
    if (!cells || !order || !ekeys) return -1;
    for (int i = 0; i < cdim[0]; i++)
        for (int j = 0; j < cdim[1]; j++)
            for (int k = 0; k < cdim[2]; k++) {
                struct ocell *c = &cells[CELLID(cdim, i, j, k)];
                c->origin[0] = origin[0] + i * h[0];
                c->origin[1] = origin[1] + j * h[1];
                c->origin[2] = origin[2] + k * h[2];
            }
    for (int p = 0; p < N; p++) {
        if (cell[p] < 0 || cell[p] >= ncells) return -1;
        cells[cell[p]].count++;
    }
    for (int c = 0, s = 0; c < ncells; c++) { cells[c].start = s; s += cells[c].count; cells[c].count = 0; }
    for (int p = 0; p < N; p++) { struct ocell *c = &cells[cell[p]]; order[c->start + c->count++] = p; }
    for (int k = 0; k < nexcl; k++) {
        int a = excl[2 * k], b = excl[2 * k + 1];
        ekeys[k] = (a < b) ? ((long long)a << 32) | (unsigned)b : ((long long)b << 32) | (unsigned)a;
    }
    qsort(ekeys, nexcl, sizeof(long long), excl_cmp);

    const float cutf = (float)cutoff;
    const float cut2_pair = cutf * cutf;
    const float cut2_self = (float)(cutoff * cutoff);
    double epot = 0.0, epot_abs = 0.0, vir = 0.0, vir_abs = 0.0;
    long long npairs = 0, nex = 0;
    memset(f_out, 0, sizeof(double) * 3 * N);

    for (int i = 0; i < cdim[0]; i++)
        for (int j = 0; j < cdim[1]; j++)
            for (int k = 0; k < cdim[2]; k++) {
                int id1 = CELLID(cdim, i, j, k), d[3], nb[3];
                for (d[0] = -span[0]; d[0] <= span[0]; d[0]++) {
                    nb[0] = i + d[0];
                    if (nb[0] < 0 || nb[0] >= cdim[0]) {
                        if (!(period & 1)) continue;
                        nb[0] = (nb[0] + cdim[0]) % cdim[0];
                    }
                    for (d[1] = -span[1]; d[1] <= span[1]; d[1]++) {
                        nb[1] = j + d[1];
                        if (nb[1] < 0 || nb[1] >= cdim[1]) {
                            if (!(period & 2)) continue;
                            nb[1] = (nb[1] + cdim[1]) % cdim[1];
                        }
                        for (d[2] = -span[2]; d[2] <= span[2]; d[2]++) {
                            double lh[3];
                            for (int q = 0; q < 3; q++) lh[q] = h[q] * fmax(abs(d[q]) - 1, 0);
                            if (lh[0] * lh[0] + lh[1] * lh[1] + lh[2] * lh[2] > cutoff * cutoff) continue;
                            nb[2] = k + d[2];
                            if (nb[2] < 0 || nb[2] >= cdim[2]) {
                                if (!(period & 4)) continue;
                                nb[2] = (nb[2] + cdim[2]) % cdim[2];
                            }
                            int id2 = CELLID(cdim, nb[0], nb[1], nb[2]);
                            int self = (id1 == id2);
                            if (!(id1 < id2 || (self && d[0] == 0 && d[1] == 0 && d[2] == 0))) continue;
                            int a = id1, b = id2;
                            float shift[3];
                            getsid(dim, cells, &a, &b, shift);
                            if (self) shift[0] = shift[1] = shift[2] = 0.0f;
                            const struct ocell *ca = &cells[a], *cb = &cells[b];
                            const float cut2 = self ? cut2_self : cut2_pair;
                            for (int ii = 0; ii < ca->count; ii++) {
                                int pi = order[ca->start + ii];
                                const float *xi = &xrel[3 * pi];
                                float pix[3] = {xi[0] - shift[0], xi[1] - shift[1], xi[2] - shift[2]};
                                int jend = self ? ii : cb->count;
                                for (int jj = 0; jj < jend; jj++) {
                                    int pj = order[cb->start + jj];
                                    const float *xj = &xrel[3 * pj];
                                    float dxf[3] = {pix[0] - xj[0], pix[1] - xj[1], pix[2] - xj[2]};
                                    float r2f = dxf[0] * dxf[0] + dxf[1] * dxf[1] + dxf[2] * dxf[2];
                                    int pot = potidx[type[pi] * mt + type[pj]];
                                    if ((pot < 0 && ep < 0) || r2f > cut2) continue;
                                    if (nexcl > 0 && is_excluded(ekeys, nexcl, pi, pj)) { nex++; continue; }
                                    double dx[3], r2 = 0.0;
                                    for (int q = 0; q < 3; q++) {
                                        dx[q] = ((double)xi[q] - (double)shift[q]) - (double)xj[q];
                                        r2 += dx[q] * dx[q];
                                    }
                                    double r = sqrt(r2), e = 0.0, fs = 0.0;
                                    if (pot >= 0)
                                        eval_fp64(coef + coff[pot], alpha + 4 * pot, potn[pot], r2f, r, &e, &fs);
                                    if (ep >= 0) {
                                        double ee, fe, qq = q[pi] * q[pj];
                                        eval_fp64(coef + coff[ep], alpha + 4 * ep, potn[ep], r2f, r, &ee, &fe);
                                        e += qq * ee;
                                        fs += qq * fe;
                                    }
                                    for (int q = 0; q < 3; q++) {
                                        double w = fs * dx[q];
                                        f_out[3 * pi + q] -= w;
                                        f_out[3 * pj + q] += w;
                                    }
                                    epot += e;
                                    epot_abs += fabs(e);
                                    vir += fs * r2;
                                    vir_abs += fabs(fs * r2);
                                    npairs++;
                                }
                            }
                        }
                    }
                }
            }
    *epot_out = epot;
    if (epot_abs_out) *epot_abs_out = epot_abs;
    *virial_out = -vir;
    if (virial_abs_out) *virial_abs_out = vir_abs;
    *npairs_out = npairs;
    *nexcl_out = nex;
    free(cells);
    free(order);
    free(ekeys);
    return 0;
}

/* Bonds (src/bond.c:81-250): for each bond (i, j) with table `tab`, the position of i shifted
 * by the periodic offset of the two cells (held to -1..1), the distance, r^2 held to
 * [a^2, b^2] (ab2), the table's energy and force, in double (the interval index from the
 * float r^2 as the reference computes it).  Forces added into f_out (by id), energy into
 * *e_out. */
int oracle_bonds(int nb, const int *bij, const float *xrel, const int *cell, const int *cdim, const double *dim,
                 const float *coef, const float *alpha, int potn, const double *ab2, double *f_out,
                 double *e_out) {
    double h[3];
    for (int k = 0; k < 3; k++) h[k] = dim[k] / cdim[k];
    double epot = 0.0;
    for (int b = 0; b < nb; b++) {
        const int i = bij[2 * b], j = bij[2 * b + 1];
        int li[3], lj[3];
        li[0] = cell[i] / (cdim[1] * cdim[2]); li[1] = (cell[i] / cdim[2]) % cdim[1]; li[2] = cell[i] % cdim[2];
        lj[0] = cell[j] / (cdim[1] * cdim[2]); lj[1] = (cell[j] / cdim[2]) % cdim[1]; lj[2] = cell[j] % cdim[2];
        double dx[3], r2 = 0.0;
        float dxf[3];
        for (int k = 0; k < 3; k++) {
            int sh = li[k] - lj[k];
            if (sh > 1) sh = -1;
            else if (sh < -1) sh = 1;
            float pix = (float)((double)xrel[3 * i + k] + h[k] * sh);
            dxf[k] = pix - xrel[3 * j + k];
            dx[k] = ((double)xrel[3 * i + k] + h[k] * sh) - (double)xrel[3 * j + k];
            r2 += dx[k] * dx[k];
        }
        float r2f = dxf[0] * dxf[0] + dxf[1] * dxf[1] + dxf[2] * dxf[2];
        if (r2f < ab2[0] || r2f > ab2[1]) r2f = (float)fmax(ab2[0], fmin(ab2[1], (double)r2f));
        if (r2 < ab2[0] || r2 > ab2[1]) r2 = fmax(ab2[0], fmin(ab2[1], r2));
        double e, fs;
        eval_fp64(coef, alpha, potn, r2f, sqrt(r2), &e, &fs);
        for (int k = 0; k < 3; k++) {
            f_out[3 * i + k] -= fs * dx[k];
            f_out[3 * j + k] += fs * dx[k];
        }
        epot += e;
    }
    *e_out = epot;
    return 0;
}

/* The table read at r itself (src/potential_eval.h:122-148, potential_eval_r): interval
 * index from the float rf as the reference computes it, polynomial in double at r; e and
 * dE/dr. */
static void eval_fp64_r(const float *coef, const float *alpha, int nmax, float rf, double r, double *e, double *f) {
    int ind = (int)fmaxf(0.0f, alpha[0] + rf * (alpha[1] + rf * alpha[2]));
    if (ind > nmax) ind = nmax;
    const float *c = &coef[8 * ind];
    double x = (r - (double)c[0]) * (double)c[1];
    double ee = (double)c[2] * x + (double)c[3];
    double eff = (double)c[2];
    for (int k = 4; k < 8; k++) {
        eff = eff * x + ee;
        ee = ee * x + (double)c[k];
    }
    *e = ee;
    *f = eff * (double)c[1];
}

/* Position of particle p near the cell of particle q (src/angle.c:141-158,
 * src/dihedral.c:146-171): its cell-relative position plus the cell edge times the cells'
 * offset, held to -1..1 per dimension; in double (xd) and rounded to float as the
 * reference stores it (xf). */
static void near_cell(int p, int q, const float *xrel, const int *cell, const int *cdim, const double *h,
                      double xd[3], float xf[3]) {
    int lp[3], lq[3];
    lp[0] = cell[p] / (cdim[1] * cdim[2]); lp[1] = (cell[p] / cdim[2]) % cdim[1]; lp[2] = cell[p] % cdim[2];
    lq[0] = cell[q] / (cdim[1] * cdim[2]); lq[1] = (cell[q] / cdim[2]) % cdim[1]; lq[2] = cell[q] % cdim[2];
    for (int k = 0; k < 3; k++) {
        int sh = lp[k] - lq[k];
        if (sh > 1) sh = -1;
        else if (sh < -1) sh = 1;
        xd[k] = (double)xrel[3 * p + k] + h[k] * sh;
        xf[k] = (float)xd[k];
    }
}

static double dotd(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static float dotf(const float *a, const float *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void crossd(const double *a, const double *b, double *o) {
    o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; o[2] = a[0] * b[1] - a[1] * b[0];
}
static void crossf(const float *a, const float *b, float *o) {
    o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; o[2] = a[0] * b[1] - a[1] * b[0];
}

/* A cosine held to [-1, 1] and then to the table's range [ab[0], ab[1]]
 * (src/angle.c:168, 183-187; src/dihedral.c:234, 254-260); the float copy picks the
 * interval. */
static void eval_cos(const float *coef, const float *alpha, int n, const double *ab, double c, float cf,
                     double *e, double *f) {
    c = fmax(-1.0, fmin(1.0, c));
    cf = fmaxf(-1.0f, fminf(1.0f, cf));
    if (c < ab[0] || c > ab[1]) c = fmax(ab[0], fmin(ab[1], c));
    if (cf < ab[0] || cf > ab[1]) cf = (float)fmax(ab[0], fmin(ab[1], (double)cf));
    eval_fp64_r(coef, alpha, n, cf, c, e, f);
}

/* Angles (src/angle.c:81-300) in double: for each angle (i, j, k, table t) of aijk[4 * na],
 * u = x_i - x_j and w = x_k - x_j near j's cell, cos = u.w / (|u| |w|), the table (coef at
 * coff[t], alpha[4 t], potn[t], range ab[2 t]) read at cos, and the forces
 * -dE/dcos * dcos/dx with dcos/dx_i = (w/|w| - cos u/|u|)/|u|, dcos/dx_k = (u/|u| - cos w/|w|)/|w|,
 * dcos/dx_j = -(the two).  Forces added into f_out (by id), energy into *e_out. */
int oracle_angles(int na, const int *aijk, const float *xrel, const int *cell, const int *cdim, const double *dim,
                  const float *coef, const int *coff, const float *alpha, const int *potn, const double *ab,
                  double *f_out, double *e_out) {
    double h[3], epot = 0.0;
    for (int k = 0; k < 3; k++) h[k] = dim[k] / cdim[k];
    for (int a = 0; a < na; a++) {
        const int i = aijk[4 * a], j = aijk[4 * a + 1], kk = aijk[4 * a + 2], t = aijk[4 * a + 3];
        double xi[3], xj[3], xk[3], u[3], w[3];
        float fi[3], fj[3], fk[3], uf[3], wf[3];
        near_cell(i, j, xrel, cell, cdim, h, xi, fi);
        near_cell(j, j, xrel, cell, cdim, h, xj, fj);
        near_cell(kk, j, xrel, cell, cdim, h, xk, fk);
        for (int k = 0; k < 3; k++) {
            u[k] = xi[k] - xj[k]; w[k] = xk[k] - xj[k];
            uf[k] = fi[k] - fj[k]; wf[k] = fk[k] - fj[k];
        }
        const double iu = 1.0 / sqrt(dotd(u, u)), iw = 1.0 / sqrt(dotd(w, w));
        const double c = fmax(-1.0, fmin(1.0, dotd(u, w) * iu * iw));
        const float cf = dotf(uf, wf) * (1.0f / sqrtf(dotf(uf, uf))) * (1.0f / sqrtf(dotf(wf, wf)));
        double e, fs;
        eval_cos(coef + coff[t], alpha + 4 * t, potn[t], ab + 2 * t, c, cf, &e, &fs);
        for (int k = 0; k < 3; k++) {
            const double gi = (w[k] * iw - c * u[k] * iu) * iu, gk = (u[k] * iu - c * w[k] * iw) * iw;
            f_out[3 * i + k] -= fs * gi;
            f_out[3 * kk + k] -= fs * gk;
            f_out[3 * j + k] += fs * (gi + gk);
        }
        epot += e;
    }
    *e_out = epot;
    return 0;
}

/* Dihedrals (src/dihedral.c:81-380) in double: for each dihedral (i, j, k, l, table t) of
 * dijkl[5 * nd], b1 = x_j - x_i, b2 = x_k - x_j, b3 = x_l - x_k near j's cell, normals
 * n1 = b1 x b2, n2 = b2 x b3, cos = n1.n2 / (|n1| |n2|), the table read at cos, and the
 * forces -dE/dcos * dcos/dx from g1 = (n2/|n2| - cos n1/|n1|)/|n1|,
 * g2 = (n1/|n1| - cos n2/|n2|)/|n2|: dcos/db1 = b2 x g1, dcos/db3 = g2 x b2,
 * dcos/db2 = g1 x b1 + b3 x g2. */
int oracle_dihedrals(int nd, const int *dijkl, const float *xrel, const int *cell, const int *cdim,
                     const double *dim, const float *coef, const int *coff, const float *alpha, const int *potn,
                     const double *ab, double *f_out, double *e_out) {
    double h[3], epot = 0.0;
    for (int k = 0; k < 3; k++) h[k] = dim[k] / cdim[k];
    for (int d = 0; d < nd; d++) {
        const int i = dijkl[5 * d], j = dijkl[5 * d + 1], kk = dijkl[5 * d + 2], l = dijkl[5 * d + 3];
        const int t = dijkl[5 * d + 4];
        double x[4][3], b1[3], b2[3], b3[3], n1[3], n2[3];
        float xf[4][3], b1f[3], b2f[3], b3f[3], n1f[3], n2f[3];
        near_cell(i, j, xrel, cell, cdim, h, x[0], xf[0]);
        near_cell(j, j, xrel, cell, cdim, h, x[1], xf[1]);
        near_cell(kk, j, xrel, cell, cdim, h, x[2], xf[2]);
        near_cell(l, j, xrel, cell, cdim, h, x[3], xf[3]);
        for (int k = 0; k < 3; k++) {
            b1[k] = x[1][k] - x[0][k]; b2[k] = x[2][k] - x[1][k]; b3[k] = x[3][k] - x[2][k];
            b1f[k] = xf[1][k] - xf[0][k]; b2f[k] = xf[2][k] - xf[1][k]; b3f[k] = xf[3][k] - xf[2][k];
        }
        crossd(b1, b2, n1); crossd(b2, b3, n2);
        crossf(b1f, b2f, n1f); crossf(b2f, b3f, n2f);
        const double i1 = 1.0 / sqrt(dotd(n1, n1)), i2 = 1.0 / sqrt(dotd(n2, n2));
        const double c = fmax(-1.0, fmin(1.0, dotd(n1, n2) * i1 * i2));
        const float cf = dotf(n1f, n2f) * (1.0f / sqrtf(dotf(n1f, n1f))) * (1.0f / sqrtf(dotf(n2f, n2f)));
        double e, fs, g1[3], g2[3], db1[3], db2[3], db3[3], t1[3], t2[3];
        eval_cos(coef + coff[t], alpha + 4 * t, potn[t], ab + 2 * t, c, cf, &e, &fs);
        for (int k = 0; k < 3; k++) {
            g1[k] = (n2[k] * i2 - c * n1[k] * i1) * i1;
            g2[k] = (n1[k] * i1 - c * n2[k] * i2) * i2;
        }
        crossd(b2, g1, db1); crossd(g2, b2, db3); crossd(g1, b1, t1); crossd(b3, g2, t2);
        for (int k = 0; k < 3; k++) {
            db2[k] = t1[k] + t2[k];
            const double di = -db1[k], dj = db1[k] - db2[k], dk = db2[k] - db3[k], dl = db3[k];
            f_out[3 * i + k] -= fs * di;
            f_out[3 * j + k] -= fs * dj;
            f_out[3 * kk + k] -= fs * dk;
            f_out[3 * l + k] -= fs * dl;
        }
        epot += e;
    }
    *e_out = epot;
    return 0;
}

/* Sort keys of one cell along direction sid (src/runner_dosort.c:118-153): key =
 * (k << 16) | (unsigned)(dscale*(bias + x.n)), dscale = 32767/(2 bias), bias = |h|; ordered
 * by descending distance, ties in storage order. */
int oracle_sortkeys(int count, const float *xrel, const double *h, int sid, unsigned *keys) {
    int idx = 26 - sid;
    int dv[3] = {idx / 9 - 1, (idx / 3) % 3 - 1, idx % 3 - 1};
    double len = sqrt((double)(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]));
    float n[3];
    for (int k = 0; k < 3; k++) n[k] = (float)(dv[k] / len);
    float bias = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    float dscale = (float)32767 / (2 * bias);
    for (int k = 0; k < count; k++) {
        const float *x = &xrel[3 * k];
        keys[k] = ((unsigned)k << 16) | (unsigned)(dscale * (bias + x[0] * n[0] + x[1] * n[1] + x[2] * n[2]));
    }
    /* insertion sort, descending by distance, stable */
    for (int a = 1; a < count; a++) {
        unsigned v = keys[a];
        int b = a - 1;
        while (b >= 0 && (keys[b] & 0xffff) < (v & 0xffff)) {
            keys[b + 1] = keys[b];
            b--;
        }
        keys[b + 1] = v;
    }
    return 0;
}

/* Rigid constraints of one evaluation (src/engine_rigid.c:352-583), FP64: SHAKE
 * (src/rigid.c:81-277) when pshake == 0, P-SHAKE (src/rigid.c:279-523) otherwise.
 *   Particles by id: x[3N], v[3N], f[3N] cell-relative float state (updated in place),
 *   cell[N] cell index, loc[3*ncells] cell grid coordinates, h[3] cell edge, mass[N].
 *   Groups: roff[ng+1] into parts[] (particle ids), coff[ng+1] into ci/cj (group-local
 *   indices) and d2; a[] the float P-SHAKE matrices (nc*nc per group, in group order),
 *   refined in place when pshake and (a_update or more than 10 iterations).
 *   iters[ng] receives each group's iteration count.
 * Mixed precision follows the reference's P-SHAKE exactly (double iterations, float
 * matrices); SHAKE is restated entirely in double (the reference's single build keeps
 * lambda, the gradients and the tolerance in float). */
#define O_MAXP 10
#define O_MAXC 30
#define O_MAXITER 100

static int oshift(const int *loc, int c, int c0, int j) {
    int s = loc[3 * c + j] - loc[3 * c0 + j];
    if (s > 1) s = -1;
    else if (s < -1) s = 1;
    return s;
}

int oracle_rigid(int ng, const int *roff, const int *parts, const int *coff, const int *ci, const int *cj,
                 const double *d2, float *a, const int *cell, const int *loc, const double *h,
                 const double *mass, float *x, float *v, float *f, double dt, double tol, int pshake,
                 int a_update, int *iters) {
    double idt = 1.0 / dt;
    int aoff = 0;
    for (int g = 0; g < ng; g++) {
        int np = roff[g + 1] - roff[g], nc = coff[g + 1] - coff[g];
        const int *pid = parts + roff[g];
        const int *gi = ci + coff[g], *gj = cj + coff[g];
        const double *gd2 = d2 + coff[g];
        float *ga = a + aoff;
        aoff += nc * nc;
        if (np > O_MAXP || nc > O_MAXC) return -1;
        double xp[3 * O_MAXP], xo[3 * O_MAXP], m[O_MAXP];
        int c0 = cell[pid[0]], iter;
        for (int k = 0; k < np; k++) {
            int id = pid[k];
            for (int j = 0; j < 3; j++) {
                xp[3 * k + j] = (double)x[3 * id + j] + h[j] * (double)oshift(loc, cell[id], c0, j);
                xo[3 * k + j] = xp[3 * k + j] - dt * (double)v[3 * id + j];
            }
            m[k] = mass[id];
        }
        if (!pshake) {
            double vc[3 * O_MAXC], wvc[3 * O_MAXC], res[O_MAXC];
            for (int k = 0; k < nc; k++)
                for (int j = 0; j < 3; j++) {
                    vc[3 * k + j] = xo[3 * gi[k] + j] - xo[3 * gj[k] + j];
                    wvc[3 * k + j] = 1.0 / (m[gi[k]] + m[gj[k]]) * vc[3 * k + j];
                }
            for (iter = 0; iter < O_MAXITER; iter++) {
                double max_res = 0.0;
                for (int k = 0; k < nc; k++) {
                    res[k] = gd2[k];
                    for (int j = 0; j < 3; j++)
                        res[k] -= (xp[3 * gi[k] + j] - xp[3 * gj[k] + j]) * (xp[3 * gi[k] + j] - xp[3 * gj[k] + j]);
                    if (fabs(res[k]) > max_res) max_res = fabs(res[k]);
                }
                if (max_res < tol) break;
                for (int k = 0; k < nc; k++) {
                    int p = gi[k], q = gj[k];
                    double lambda = 0.5 * res[k] / ((xp[3 * p] - xp[3 * q]) * vc[3 * k] +
                                                    (xp[3 * p + 1] - xp[3 * q + 1]) * vc[3 * k + 1] +
                                                    (xp[3 * p + 2] - xp[3 * q + 2]) * vc[3 * k + 2]);
                    for (int j = 0; j < 3; j++) {
                        double w = lambda * wvc[3 * k + j];
                        xp[3 * p + j] += w * m[q];
                        xp[3 * q + j] -= w * m[p];
                    }
                }
            }
        } else {
            static double vc[3 * O_MAXC * O_MAXP];
            int row = 3 * np;
            memset(vc, 0, sizeof(double) * nc * row);
            for (int k = 0; k < nc; k++) {
                int p = gi[k], q = gj[k];
                double dv[3];
                for (int j = 0; j < 3; j++) dv[j] = (xo[3 * p + j] - xo[3 * q + j]) / (m[p] + m[q]);
                for (int i = 0; i < nc; i++)
                    if (ga[k * nc + i] != 0.0f)
                        for (int j = 0; j < 3; j++) {
                            vc[i * row + p * 3 + j] += ga[k * nc + i] * dv[j] * m[q];
                            vc[i * row + q * 3 + j] += -ga[k * nc + i] * dv[j] * m[p];
                        }
            }
            for (iter = 0; iter < O_MAXITER; iter++) {
                double max_res = 0.0;
                for (int k = 0; k < nc; k++) {
                    int p = gi[k], q = gj[k];
                    const double *vk = vc + k * row;
                    double res = gd2[k];
                    for (int j = 0; j < 3; j++) res -= (xp[3 * p + j] - xp[3 * q + j]) * (xp[3 * p + j] - xp[3 * q + j]);
                    if (fabs(res) > max_res) max_res = fabs(res);
                    double lambda = 0.5 * res / ((xp[3 * p] - xp[3 * q]) * (vk[3 * p] - vk[3 * q]) +
                                                 (xp[3 * p + 1] - xp[3 * q + 1]) * (vk[3 * p + 1] - vk[3 * q + 1]) +
                                                 (xp[3 * p + 2] - xp[3 * q + 2]) * (vk[3 * p + 2] - vk[3 * q + 2]));
                    for (int j = 0; j < row; j++) xp[j] += lambda * vk[j];
                }
                if (max_res < tol) break;
            }
            if (nc > 1 && (a_update || iter > 10)) {
                float an[O_MAXC * O_MAXC], tmp[O_MAXC * O_MAXC], maxa = 0.0f;
                for (int i = 0; i < nc; i++) {
                    int p = gi[i], q = gj[i];
                    const double *vi = vc + i * row;
                    float dx[3];
                    for (int j = 0; j < 3; j++) dx[j] = (float)(xp[3 * p + j] - xp[3 * q + j]);
                    float w = -1.0 / (dx[0] * (vi[3 * p] - vi[3 * q]) + dx[1] * (vi[3 * p + 1] - vi[3 * q + 1]) +
                                      dx[2] * (vi[3 * p + 2] - vi[3 * q + 2]));
                    for (int j = i + 1; j < nc; j++) {
                        const double *vj = vc + j * row;
                        an[i + j * nc] = w * (dx[0] * (vj[3 * p] - vj[3 * q]) + dx[1] * (vj[3 * p + 1] - vj[3 * q + 1]) +
                                              dx[2] * (vj[3 * p + 2] - vj[3 * q + 2]));
                        an[j + i * nc] = an[i + j * nc];
                        maxa = fmaxf(maxa, fabsf(an[i + j * nc]));
                    }
                    an[i + i * nc] = 1.0f;
                }
                if (maxa > 0.1f) {
                    float w = 0.1 / maxa;
                    for (int i = 0; i < nc * nc; i++) an[i] *= w;
                    for (int i = 0; i < nc; i++) an[i * nc + i] = 1.0f;
                }
                memset(tmp, 0, sizeof(float) * nc * nc);
                for (int j = 0; j < nc; j++)
                    for (int k = 0; k < nc; k++)
                        for (int i = 0; i < nc; i++) tmp[j * nc + i] += ga[k * nc + i] * an[j * nc + k];
                memcpy(ga, tmp, sizeof(float) * nc * nc);
            }
        }
        iters[g] = iter;
        for (int k = 0; k < np; k++) {
            int id = pid[k];
            for (int j = 0; j < 3; j++) {
                double xn = xp[3 * k + j] - h[j] * oshift(loc, cell[id], c0, j);
                if (pshake) f[3 * id + j] += idt * idt * (xn - x[3 * id + j]) * m[k];
                v[3 * id + j] += idt * (xn - x[3 * id + j]);
                x[3 * id + j] = xn;
            }
        }
    }
    return 0;
}
