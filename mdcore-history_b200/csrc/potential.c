/* Interpolated pair-potential tables (host side).
 *
 * The device sweep evaluates mdcore's piecewise quintic tables, so the tables must be the
 * same floats the reference builds: this file restates the reference table constructor
 * (src/potential.c:963-1194 potential_init, :1401-1520 potential_getcoeffs, :1211-1374
 * potential_getfp/_fixend, :1537-1600 potential_getalpha) keeping its arithmetic -- which
 * operations run in float and which in double, and their order -- so that, compiled
 * without FMA contraction, every coefficient is bit-identical to the reference
 * single-precision build.  One defect of the reference is not reproduced: its
 * potential_getcoeffs declares the per-node arrays one element short
 * (src/potential.c:1404) and writes past them; here they hold n+1 nodes.
 *
 * Table layout (struct potential, src/potential.h:57-74): alpha[0..2] map r to an interval
 * index ind = (int)max(0, alpha0 + r*(alpha1 + r*alpha2)); chunk `ind` of 8 floats is
 * {centre, 1/halfwidth, c5, c4, c3, c2, c1, c0} of a quintic in x = (r-centre)/halfwidth.
 * Chunk 0 is a linear continuation of chunk 1 below r = a.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include "mdcore_b200.h"

int potential_err = potential_err_ok;

static const char *pot_msg[] = {
    "Nothing bad happened.",
    "An unexpected NULL pointer was encountered.",
    "A call to malloc failed, probably due to insufficient memory.",
    "The requested value was out of bounds.",
    "Not yet implemented.",
    "Maximum number of intervals reached before tolerance satisfied."
};
#define pot_error(id) (potential_err = errs_register((id), pot_msg[-(id)], __LINE__, __func__, __FILE__))

/* ------------------------------------------------------------------ shared constants */

/* Chebyshev-Gauss-Lobatto abscissae and weights 1/sqrt(1-x^2) for the derivative fit, and
 * the cosines cos(j*k*pi/N) (stored in float, as the reference does) for the projection. */
static double fit_x[potential_N], fit_w[potential_N];
static float proj_cos[7 * potential_N];
static int consts_ready = 0;

static void init_consts(void) {
    if (consts_ready) return;
    for (int k = 1; k < potential_N - 1; k++) {
        fit_x[k] = cos(k * M_PI / (potential_N - 1));
        fit_w[k] = 1.0 / sqrt(1.0 - fit_x[k] * fit_x[k]);
    }
    fit_x[0] = 1.0; fit_x[potential_N - 1] = -1.0;
    fit_w[0] = 0.0; fit_w[potential_N - 1] = 0.0;
    for (int k = 0; k < 7; k++)
        for (int j = 0; j < potential_N; j++)
            proj_cos[k * potential_N + j] = cos(j * k * M_PI / potential_N);
    consts_ready = 1;
}

/* Inner products of the cubic Hermite basis functions under the Chebyshev weight, the
 * coefficients of the normal equations for the end derivatives (same constants as the
 * reference, src/potential.c:1216-1226). */
static const double H_L0L1 = 0.1125317885884428;
static const double H_L1L1 = 0.03215579530433858;
static const double H_L0R1 = -0.04823369227661384;
static const double H_L1R1 = -0.02143719641629633;
static const double H_R0R1 = -0.1125317885884429;
static const double H_R1R1 = 0.03215579530433859;
static const double H_L1R0 = 0.04823369227661384;
static const double H_CL1[4] = {0.25, -0.25, -0.25, 0.25};
static const double H_CR1[4] = {-0.25, -0.25, 0.25, 0.25};

/* Least-squares optimal first derivatives at the n+1 nodes: a tridiagonal system solved by
 * forward elimination.  With fixed ends the end rows pin fp[0]=fpa, fp[n]=fpb. */
static int fit_derivatives(double (*f)(double), int fixed, double fpa, double fpb, int n,
                           const float *x, double *fp) {
    if (n < 1) return pot_error(potential_err_bounds);
    double *fx = malloc(sizeof(double) * (n + 1));
    double *hx = malloc(sizeof(double) * (n + 1));
    double *lo = malloc(sizeof(double) * (n + 1));
    double *di = malloc(sizeof(double) * (n + 1));
    double *up = malloc(sizeof(double) * (n + 1));
    double *rhs = malloc(sizeof(double) * (n + 1));
    double *vl = malloc(sizeof(double) * (n + 1));
    double *vr = malloc(sizeof(double) * (n + 1));
    if (!fx || !hx || !lo || !di || !up || !rhs || !vl || !vr) {
        free(fx); free(hx); free(lo); free(di); free(up); free(rhs); free(vl); free(vr);
        return pot_error(potential_err_malloc);
    }
    for (int i = 0; i <= n; i++) fx[i] = f(x[i]);
    for (int i = 0; i < n; i++) hx[i] = x[i + 1] - x[i];

    /* Projections of f onto the two derivative basis functions of each interval. */
    for (int i = 0; i < n; i++) {
        double m = 0.5 * (x[i] + x[i + 1]);
        double h = 0.5 * (x[i + 1] - x[i]);
        double sl = 0.0, sr = 0.0;
        for (int k = 1; k < potential_N - 1; k++) {
            double xk = fit_x[k];
            double v = f(m + h * xk);
            sl += fit_w[k] * (v * (H_CL1[0] + xk * (H_CL1[1] + xk * (H_CL1[2] + xk * H_CL1[3]))));
            sr += fit_w[k] * (v * (H_CR1[0] + xk * (H_CR1[1] + xk * (H_CR1[2] + xk * H_CR1[3]))));
        }
        vl[i] = sl / (potential_N - 2);
        vr[i] = sr / (potential_N - 2);
    }

    if (fixed) {
        di[0] = 1.0; up[0] = 0.0; rhs[0] = fpa;
    } else {
        di[0] = H_L1L1 * hx[0];
        up[0] = H_L1R1 * hx[0];
        rhs[0] = 2 * (vl[0] - fx[0] * H_L0L1 - fx[1] * H_L1R0);
    }
    for (int i = 1; i < n; i++) {
        lo[i] = H_L1R1 * hx[i - 1];
        di[i] = H_R1R1 * hx[i - 1] + H_L1L1 * hx[i];
        up[i] = H_L1R1 * hx[i];
        rhs[i] = 2 * (vr[i - 1] - fx[i - 1] * H_L0R1 - fx[i] * H_R0R1) +
                 2 * (vl[i] - fx[i] * H_L0L1 - fx[i + 1] * H_L1R0);
    }
    if (fixed) {
        lo[n] = 0.0; di[n] = 1.0; rhs[n] = fpb;
    } else {
        lo[n] = H_L1R1 * hx[n - 1];
        di[n] = H_R1R1 * hx[n - 1];
        rhs[n] = 2 * (vr[n - 1] - fx[n - 1] * H_L0R1 - fx[n] * H_R0R1);
    }
    for (int i = 1; i <= n; i++) {
        double m = lo[i] / di[i - 1];
        di[i] = di[i] - m * up[i - 1];
        rhs[i] = rhs[i] - m * rhs[i - 1];
    }
    fp[n] = rhs[n] / di[n];
    for (int i = n - 1; i >= 0; i--) fp[i] = (rhs[i] - up[i] * fp[i + 1]) / di[i];

    free(fx); free(hx); free(lo); free(di); free(up); free(rhs); free(vl); free(vr);
    return potential_err_ok;
}

/* Quintic coefficients of f on the n intervals between the float nodes xi[0..n]: Hermite
 * cubic from end values and derivatives, plus the degree-4 and degree-5 Chebyshev
 * corrections that leave end values and slopes unchanged.  *err receives the largest
 * per-interval error relative to max(|f|, 1). */
static int interval_coeffs(double (*f)(double), double (*fp)(double), const float *xi, int n,
                           float *c, float *err) {
    double cheb[7], cee[6], fx[potential_N];
    double *fnode = malloc(sizeof(double) * (n + 1));
    double *dnode = malloc(sizeof(double) * (n + 1));
    if (fnode == NULL || dnode == NULL) {
        free(fnode); free(dnode);
        return pot_error(potential_err_malloc);
    }
    init_consts();
    for (int k = 0; k <= n; k++) fnode[k] = f(xi[k]);
    if (fp == NULL) {
        if (fit_derivatives(f, 0, 0.0, 0.0, n, xi, dnode) < 0) { free(fnode); free(dnode); return potential_err; }
    } else {
        if (fit_derivatives(f, 1, fp(xi[0]), fp(xi[n]), n, xi, dnode) < 0) { free(fnode); free(dnode); return potential_err; }
    }

    *err = 0.0f;
    for (int i = 0; i < n; i++) {
        float *ci = &c[i * potential_chunk];
        float mf = (xi[i] + xi[i + 1]) / 2;
        float hf = (xi[i + 1] - xi[i]) / 2;
        double m = mf, h = hf;
        double fa = fnode[i], fb = fnode[i + 1];
        double dfa = dnode[i] * h, dfb = dnode[i + 1] * h;

        /* Chebyshev coefficients 0..6 of f on the interval. */
        for (int k = 0; k < potential_N; k++) fx[k] = f(m + h * cos(k * M_PI / potential_N));
        for (int j = 0; j < 7; j++) {
            double s = (fa + (1 - 2 * (j % 2)) * fb) / 2;
            for (int k = 1; k < potential_N; k++) s += fx[k] * proj_cos[j * potential_N + k];
            cheb[j] = s * (2.0 / potential_N);
        }

        /* Cubic Hermite interpolant in the Chebyshev basis. */
        cee[0] = (4 * (fa + fb) + dfa - dfb) / 4;
        cee[1] = -(9 * (fa - fb) + dfa + dfb) / 16;
        cee[2] = (dfb - dfa) / 8;
        cee[3] = (fa - fb + dfa + dfb) / 16;
        cee[4] = 0.0;
        cee[5] = 0.0;
        /* Degree-4 and degree-5 corrections towards the projection. */
        double w4 = (6 * (cee[0] - cheb[0]) - 4 * (cee[2] - cheb[2]) - cheb[4]) / (36 + 16 + 1);
        cee[0] += -6 * w4;
        cee[2] += 4 * w4;
        cee[4] = -w4;
        double w5 = (2 * (cee[1] - cheb[1]) - 3 * (cee[3] - cheb[3]) - cheb[5]) / (4 + 9 + 1);
        cee[1] += -2 * w5;
        cee[3] += 3 * w5;
        cee[5] = -w5;

        /* Monomials in x on [-1,1], highest degree first after {centre, 1/halfwidth}. */
        ci[7] = cee[0] / 2 - cee[2] + cee[4];
        ci[6] = cee[1] - 3 * cee[3] + 5 * cee[5];
        ci[5] = 2 * cee[2] - 8 * cee[4];
        ci[4] = 4 * cee[3] - 20 * cee[5];
        ci[3] = 8 * cee[4];
        ci[2] = 16 * cee[5];
        ci[1] = 1.0 / h;
        ci[0] = m;

        /* Local error on the projection nodes, relative to max(|f|, 1). */
        double fmaxabs = 0.0, eloc = 0.0;
        for (int k = 1; k < potential_N; k++) {
            fmaxabs = fmax(fabs(fx[k]), fmaxabs);
            double x = proj_cos[potential_N + k];
            double d = fabs(fx[k] - ci[7] - x * (ci[6] + x * (ci[5] + x * (ci[4] + x * (ci[3] + x * ci[2])))));
            eloc = fmax(d, eloc);
        }
        eloc /= fmax(fmaxabs, 1.0);
        *err = fmax(eloc, *err);
    }
    free(fnode);
    free(dnode);
    return potential_err_ok;
}

/* The node-density parameter alpha of the quadratic node transform: a golden-section
 * search for the alpha that minimises max |f6(x)| * (node spacing)^6 on 100 points. */
double potential_getalpha(double (*f6p)(double), double a, double b) {
    double xs[potential_N], f6[potential_N], amax = 0.0;
    const double g = 2.0 / (1 + sqrt(5));
    double al[4], fa[4];
    for (int i = 0; i < potential_N; i++) {
        xs[i] = ((double)i + 1) / (potential_N + 1);
        f6[i] = f6p(a + (b - a) * xs[i]);
        amax = fmax(amax, fabs(f6[i]));
    }
    if (amax == 0.0) return 1.0;

    al[0] = 0; al[3] = 2;
    al[1] = al[3] - 2 * g;
    al[2] = al[0] + 2 * g;
    for (int i = 0; i < 4; i++) {
        fa[i] = 0.0;
        for (int j = 0; j < potential_N; j++) {
            double t = fabs(pow(al[i] + 2 * (1 - al[i]) * xs[j], -6) * f6[j]);
            if (t > fa[i]) fa[i] = t;
        }
    }
    while (al[3] - al[0] > 1.0e-4) {
        int i;
        if (fa[1] < fa[2]) {
            al[3] = al[2]; fa[3] = fa[2];
            al[2] = al[1]; fa[2] = fa[1];
            al[1] = al[3] - (al[3] - al[0]) * g;
            i = 1;
        } else {
            al[0] = al[1]; fa[0] = fa[1];
            al[1] = al[2]; fa[1] = fa[2];
            al[2] = al[0] + (al[3] - al[0]) * g;
            i = 2;
        }
        fa[i] = 0.0;
        for (int j = 0; j < potential_N; j++) {
            double t = fabs(pow(al[i] + 2 * (1 - al[i]) * xs[j], -6) * f6[j]);
            if (t > fa[i]) fa[i] = t;
        }
    }
    return (al[0] + al[3]) / 2;
}

/* Nodes xi[0..n] of an n-interval table: the inverse of the quadratic transform
 * i = n*(alpha0 + x*(alpha1 + x*alpha2)), found by Newton steps from a uniform guess. */
static float *make_nodes(const struct potential *p, float a, float b, int n) {
    const float mtol = 10 * FLT_EPSILON;
    float *xi = malloc(sizeof(float) * (n + 1));
    if (xi == NULL) return NULL;
    xi[0] = a;
    xi[n] = b;
    for (int i = 1; i < n; i++) {
        xi[i] = a + (b - a) * i / n;
        while (1) {
            float t = p->alpha[0] + xi[i] * (p->alpha[1] + xi[i] * p->alpha[2]);
            double e = i - n * t;
            float slope = n * (p->alpha[1] + 2 * xi[i] * p->alpha[2]);
            xi[i] += e / slope;
            if (fabs(e) < n * mtol) break;
        }
    }
    return xi;
}

/* Builds the n-interval table into a fresh 64-byte aligned array (chunk 0 left for the
 * linear continuation). */
static int build_table(const struct potential *p, double (*f)(double), double (*fp)(double),
                       float a, float b, int n, float **c_out, float *err) {
    float *xi = make_nodes(p, a, b, n);
    float *c = NULL;
    if (xi == NULL) return pot_error(potential_err_malloc);
    if (posix_memalign((void **)&c, potential_align, sizeof(float) * (n + 1) * potential_chunk) != 0) {
        free(xi);
        return pot_error(potential_err_malloc);
    }
    memset(c, 0, sizeof(float) * potential_chunk);
    if (interval_coeffs(f, fp, xi, n, &c[potential_chunk], err) < 0) {
        free(xi);
        free(c);
        return pot_error(potential_err_null);
    }
    free(xi);
    *c_out = c;
    return potential_err_ok;
}

/* Chunk 0: first-order Taylor continuation of chunk 1 at r = a, written in chunk 1's
 * monomial form with x = (r - a)/a. */
static void linear_continuation(struct potential *p, float a) {
    double coeffs[potential_degree], eff[potential_degree];
    float *c = p->c;
    c[0] = a;
    c[1] = (a == 0) ? 1.0 : 1.0 / a;
    for (int k = 0; k < potential_degree; k++) {
        coeffs[k] = c[2 * potential_chunk - 1 - k];
        eff[k] = 0.0;
    }
    for (int i = 0; i < potential_degree; i++)
        for (int k = potential_degree - 1; k >= i; k--) {
            eff[i] = coeffs[k] + (-1.0) * eff[i];
            coeffs[k] *= (k - i) * c[potential_chunk + 1] * a;
        }
    c[potential_chunk - 1] = eff[0];
    c[potential_chunk - 2] = eff[1];
    c[potential_chunk - 3] = 0.5 * eff[2];
    for (int k = 3; k <= potential_degree; k++) c[potential_chunk - 1 - k] = 0.0;
}

/* Shifts alpha0/alpha1 so that r = b maps just below n+1 in float arithmetic. */
static void correct_edges(struct potential *p, float a, float b) {
    float bee = copysignf(sqrtf(b * b), b);
    float aye = copysignf(sqrtf(a * a), a);
    float fbee = fabsf(bee);
    double err_b = (p->n + 1) - (p->alpha[0] + bee * (p->alpha[1] + bee * p->alpha[2])) -
                   FLT_EPSILON * (fabsf(p->alpha[0]) + fbee * (fabsf(p->alpha[1]) + fbee * fabsf(p->alpha[2])));
    p->alpha[0] += (err_b * aye) / (aye - bee);
    p->alpha[1] += (-err_b) / (aye - bee);
}

int potential_init(struct potential *p, double (*f)(double), double (*fp)(double),
                   double (*f6p)(double), float a, float b, float tol) {
    int lo = potential_ivalsa, hi = potential_ivalsb;
    float err_lo, err_hi, err_mid;
    float *c_lo = NULL, *c_hi = NULL, *c_mid = NULL;

    if (p == NULL || f == NULL) return pot_error(potential_err_null);
    p->a = a;
    p->b = b;
    p->flags = potential_flag_none;

    /* Quadratic node transform with the optimal density parameter. */
    double alpha = (f6p != NULL) ? potential_getalpha(f6p, a, b) : 1.0;
    double w = 1.0 / (a - b);
    w *= w;
    p->alpha[0] = a * a * w - alpha * b * a * w;
    p->alpha[1] = -2 * a * w + alpha * (a + b) * w;
    p->alpha[2] = w - alpha * w;
    p->alpha[3] = 0.0;

    /* One interval may already do. */
    if (build_table(p, f, fp, a, b, lo, &c_lo, &err_lo) < 0) return potential_err;
    if (err_lo < tol) {
        p->n = lo;
        p->c = c_lo;
        p->alpha[0] *= p->n; p->alpha[1] *= p->n; p->alpha[2] *= p->n;
        p->alpha[0] += 1;
        linear_continuation(p, a);
        correct_edges(p, a, b);
        return potential_err_ok;
    }

    /* Double the interval count until the tolerance is met ... */
    while (1) {
        if (build_table(p, f, fp, a, b, hi, &c_hi, &err_hi) < 0) { free(c_lo); return potential_err; }
        if (err_hi < tol) break;
        if (2 * hi > potential_ivalsmax) {
            free(c_lo);
            free(c_hi);
            return pot_error(potential_err_ivalsmax);
        }
        free(c_lo);
        c_lo = c_hi;
        err_lo = err_hi;
        lo = hi;
        hi *= 2;
    }
    /* ... then bisect for the smallest count that meets it. */
    while (hi - lo > 1) {
        int mid = 0.5 * (hi + lo);
        if (build_table(p, f, fp, a, b, mid, &c_mid, &err_mid) != 0) {
            free(c_lo);
            free(c_hi);
            return pot_error(potential_err_null);
        }
        if (err_mid > tol) {
            free(c_lo);
            c_lo = c_mid;
            err_lo = err_mid;
            lo = mid;
        } else {
            free(c_hi);
            c_hi = c_mid;
            err_hi = err_mid;
            hi = mid;
        }
    }
    (void)err_lo;
    free(c_lo);

    p->n = hi;
    p->c = c_hi;
    p->alpha[0] *= p->n; p->alpha[1] *= p->n; p->alpha[2] *= p->n;
    p->alpha[0] += 1.0;
    correct_edges(p, a, b);
    linear_continuation(p, a);
    return potential_err_ok;
}

void potential_clear(struct potential *p) {
    if (p == NULL) return;
    p->flags = potential_flag_none;
    free(p->c);
    p->c = NULL;
}

/* Scalar evaluation, as src/potential_eval.h:67-104: e = U(r), f = U'(r)/r. */
void potential_eval(struct potential *p, float r2, float *e, float *f) {
    float r = sqrtf(r2);
    int ind = (int)fmaxf(0.0f, p->alpha[0] + r * (p->alpha[1] + r * p->alpha[2]));
    const float *c = &p->c[ind * potential_chunk];
    float x = (r - c[0]) * c[1];
    float ee = c[2] * x + c[3];
    float eff = c[2];
    for (int k = 4; k < potential_chunk; k++) {
        eff = eff * x + ee;
        ee = ee * x + c[k];
    }
    *e = ee;
    *f = eff * c[1] / r;
}

/* ------------------------------------------------------------------ analytic forms
 * U(r), U'(r) and U''''''(r) of the 12-6 Lennard-Jones, shifted Coulomb and Ewald
 * real-space terms (src/potential.c:114-265, :517-914).  Coulomb carries the reference's
 * prefactor 1/(4 pi); callers fold their unit conversion into q. */

static double lj(double r, double A, double B) {
    double ir = 1.0 / r, ir2 = ir * ir, ir6 = ir2 * ir2 * ir2, ir12 = ir6 * ir6;
    return (A * ir12 - B * ir6);
}
static double lj_p(double r, double A, double B) {
    double ir = 1.0 / r, ir2 = ir * ir, ir4 = ir2 * ir2, ir12 = ir4 * ir4 * ir4;
    return 6.0 * ir * (-2.0 * A * ir12 + B * ir4 * ir2);
}
static double lj_6p(double r, double A, double B) {
    double r2 = r * r, ir2 = 1.0 / r2, ir6 = ir2 * ir2 * ir2, ir12 = ir6 * ir6;
    return 10080.0 * ir12 * (884.0 * A * ir6 - 33.0 * B);
}
static double ewald(double r, double kappa) {
    return potential_escale * erfc(kappa * r) / r;
}
static double ewald_p(double r, double kappa) {
    const double isqrtpi = 0.56418958354775628695;
    double r2 = r * r, ir = 1.0 / r, ir2 = ir * ir;
    return potential_escale * (-2.0 * exp(-kappa * kappa * r2) * kappa * ir * isqrtpi - erfc(kappa * r) * ir2);
}
static double ewald_6p(double r, double kappa) {
    const double isqrtpi = 0.56418958354775628695;
    double r2 = r * r, ir2 = 1.0 / r2, r4 = r2 * r2, ir4 = ir2 * ir2, ir6 = ir2 * ir4;
    double k2 = kappa * kappa;
    double t6 = erfc(kappa * r);
    double t23 = exp(-k2 * r2);
    return potential_escale * (720.0 * t6 / r * ir6 +
        (1440.0 * ir6 + (960.0 * ir4 + (384.0 * ir2 + (144.0 + (-128.0 * r2 + 64.0 * k2 * r4) * k2) * k2) * k2) * k2) *
        kappa * isqrtpi * t23);
}
static double smooth_switch(double r, double A, double B) {
    if (r < A) return 1.0;
    if (r > B) return 0.0;
    double B2 = B * B, A2 = A * A, r2 = r * r;
    double B2mr2 = B2 - r2, B2mA2 = B2 - A2;
    return B2mr2 * B2mr2 * (B2 + 2 * r2 - 3 * A2) / (B2mA2 * B2mA2 * B2mA2);
}
static double smooth_switch_p(double r, double A, double B) {
    if (A < r && r < B) {
        double B2 = B * B, A2 = A * A, r2 = r * r;
        double B2mr2 = B2 - r2, B2mA2 = B2 - A2;
        double r2_p = 2 * r, B2mr2_p = -r2_p;
        return (2 * B2mr2_p * B2mr2 * (B2 + 2 * r2 - 3 * A2) + B2mr2 * B2mr2 * 2 * r2_p) / (B2mA2 * B2mA2 * B2mA2);
    }
    return 0.0;
}

/* Parameters of the potential being built (the constructor callbacks take r only). */
static struct { double A, B, q, kappa, b, s; } P;

static double f_lj(double r) { return lj(r, P.A, P.B); }
static double fp_lj(double r) { return lj_p(r, P.A, P.B); }
static double f6_lj(double r) { return lj_6p(r, P.A, P.B); }

static double f_coul(double r) { return potential_escale * P.q * (1.0 / r - 1.0 / P.b); }
static double fp_coul(double r) { return -potential_escale * P.q / (r * r); }
static double f6_coul(double r) {
    double r2 = r * r, r4 = r2 * r2, r7 = r * r2 * r4;
    return 720.0 * potential_escale * P.q / r7;
}

static double f_ljcoul(double r) { return lj(r, P.A, P.B) + potential_escale * P.q * (1.0 / r - 1.0 / P.b); }
static double fp_ljcoul(double r) { return lj_p(r, P.A, P.B) - potential_escale * P.q / (r * r); }
static double f6_ljcoul(double r) {
    double r2 = r * r, r4 = r2 * r2, r7 = r * r2 * r4;
    return lj_6p(r, P.A, P.B) + 720.0 * potential_escale * P.q / r7;
}

static double f_ew(double r) { return P.q * ewald(r, P.kappa); }
static double fp_ew(double r) { return P.q * ewald_p(r, P.kappa); }
static double f6_ew(double r) { return P.q * ewald_6p(r, P.kappa); }

static double f_ljew(double r) { return lj(r, P.A, P.B) + P.q * ewald(r, P.kappa); }
static double fp_ljew(double r) { return lj_p(r, P.A, P.B) + P.q * ewald_p(r, P.kappa); }
static double f6_ljew(double r) { return lj_6p(r, P.A, P.B) + P.q * ewald_6p(r, P.kappa); }

static double f_ljsw(double r) { return lj(r, P.A, P.B) * smooth_switch(r, P.s, P.b); }
static double fp_ljsw(double r) {
    return lj_p(r, P.A, P.B) * smooth_switch(r, P.s, P.b) + lj(r, P.A, P.B) * smooth_switch_p(r, P.s, P.b);
}
static double f6_ljsw(double r) { return lj_6p(r, P.A, P.B); }

static struct potential *create(double (*f)(double), double (*fp)(double), double (*f6)(double),
                                double a, double b, double tol, unsigned int flags) {
    struct potential *p = NULL;
    if (posix_memalign((void **)&p, 16, sizeof(struct potential)) != 0) {
        pot_error(potential_err_malloc);
        return NULL;
    }
    if (potential_init(p, f, fp, f6, a, b, tol) < 0) {
        free(p);
        return NULL;
    }
    p->flags = flags;
    return p;
}

struct potential *potential_create_LJ126(double a, double b, double A, double B, double tol) {
    P.A = A; P.B = B;
    return create(f_lj, fp_lj, f6_lj, a, b, tol, potential_flag_LJ126);
}
struct potential *potential_create_LJ126_switch(double a, double b, double A, double B, double s, double tol) {
    P.A = A; P.B = B; P.s = s; P.b = b;
    return create(f_ljsw, fp_ljsw, f6_ljsw, a, b, tol, potential_flag_LJ126);
}
/* LJ with the switch plus the Ewald real-space term: the switch acts on the LJ part only
 * (src/potential.c:607-676). */
static double f_ljewsw(double r) { return lj(r, P.A, P.B) * smooth_switch(r, P.s, P.b) + P.q * ewald(r, P.kappa); }
static double fp_ljewsw(double r) {
    return lj_p(r, P.A, P.B) * smooth_switch(r, P.s, P.b) + lj(r, P.A, P.B) * smooth_switch_p(r, P.s, P.b) +
           P.q * ewald_p(r, P.kappa);
}
static double f6_ljewsw(double r) { return lj_6p(r, P.A, P.B) + P.q * ewald_6p(r, P.kappa); }

struct potential *potential_create_LJ126_Ewald_switch(double a, double b, double A, double B, double q, double kappa,
                                                      double s, double tol) {
    P.A = A; P.B = B; P.q = q; P.kappa = kappa; P.s = s; P.b = b;
    return create(f_ljewsw, fp_ljewsw, f6_ljewsw, a, b, tol, potential_flag_LJ126 | potential_flag_Ewald);
}

/* The analytic 12-6 Lennard-Jones and Ewald real-space values, for callers that bound a
 * table's inner radius by the potential's size (the parameter-file readers). */
double nb_lj126(double r, double A, double B) { return lj(r, A, B); }
double nb_ewald(double r, double kappa) { return ewald(r, kappa); }

static struct { double K, r0; } H;
static double f_harm(double r) { return H.K * (r - H.r0) * (r - H.r0); }
static double f6_harm(double r) {
    (void)r;
    return 0.0;
}

struct potential *potential_create_harmonic(double a, double b, double K, double r0, double tol) {
    H.K = K;
    H.r0 = r0;
    return create(f_harm, NULL, f6_harm, a, b, tol, potential_flag_none);
}

/* Harmonic angle K (theta - theta0)^2 as a table over r = cos(theta) on [cos b, cos a],
 * the angle range held to [0, pi] (src/potential.c:414-482). */
static struct { double K, theta0; } HA;
static double f_hangle(double r) {
    const double theta = acos(fmin(1.0, fmax(-1.0, r)));
    return HA.K * (theta - HA.theta0) * (theta - HA.theta0);
}

struct potential *potential_create_harmonic_angle(double a, double b, double K, double theta0, double tol) {
    if (a < 0.0) a = 0.0;
    if (b > M_PI) b = M_PI;
    HA.K = K;
    HA.theta0 = theta0;
    return create(f_hangle, NULL, NULL, cos(b), cos(a), tol, potential_flag_none);
}

/* Harmonic dihedral K (1 + cos(n phi - delta)) as a table over r = cos(phi) on [-1, 1]
 * (src/potential.c:325-411).  With phi = acos(r): cos(n phi) = T_n(r) and
 * sin(n phi) = U_{n-1}(r) sqrt(1 - r^2), the Chebyshev polynomials of the first and second
 * kind from their three-term recurrences; delta = 0 and delta = pi exactly take the
 * cos-only forms, and |r| >= 1 drops the sine term. */
static struct { double K, delta; int n; } HD;
static double f_hdihedral(double r) {
    double t0 = 1.0, t1 = r, u0 = 1.0, u1 = 2 * r;      /* T_k, T_{k+1}; U_k, U_{k+1} */
    for (int k = 2; k <= HD.n; k++) {
        const double t2 = 2 * r * t1 - t0, u2 = 2 * r * u1 - u0;
        t0 = t1; t1 = t2;
        u0 = u1; u1 = u2;
    }
    /* now t1 = T_n and u0 = U_{n-1} (for n = 1: T_1 = r, U_0 = 1) */
    const double tn = HD.n == 0 ? 1.0 : t1, un1 = HD.n == 0 ? 0.0 : u0;
    if (HD.delta == 0.0) return HD.K * (1.0 + tn);
    if (HD.delta == M_PI) return HD.K * (1.0 - tn);
    if (fabs(r) < 1.0) return HD.K * (1.0 + tn * cos(HD.delta) + un1 * sqrt(1.0 - r * r) * sin(HD.delta));
    return HD.K * (1.0 + tn * cos(HD.delta));
}

struct potential *potential_create_harmonic_dihedral(double K, int n, double delta, double tol) {
    HD.K = K;
    HD.n = n;
    HD.delta = delta;
    return create(f_hdihedral, NULL, NULL, -1.0, 1.0, tol, potential_flag_none);
}

struct potential *potential_create_Coulomb(double a, double b, double q, double tol) {
    P.q = q; P.b = b;
    return create(f_coul, fp_coul, f6_coul, a, b, tol, potential_flag_Coulomb);
}
struct potential *potential_create_LJ126_Coulomb(double a, double b, double A, double B, double q, double tol) {
    P.A = A; P.B = B; P.q = q; P.b = b;
    return create(f_ljcoul, fp_ljcoul, f6_ljcoul, a, b, tol, potential_flag_LJ126 | potential_flag_Coulomb);
}
struct potential *potential_create_Ewald(double a, double b, double q, double kappa, double tol) {
    P.q = q; P.kappa = kappa;
    return create(f_ew, fp_ew, f6_ew, a, b, tol, potential_flag_Ewald);
}
struct potential *potential_create_LJ126_Ewald(double a, double b, double A, double B, double q, double kappa, double tol) {
    P.A = A; P.B = B; P.q = q; P.kappa = kappa;
    return create(f_ljew, fp_ljew, f6_ljew, a, b, tol, potential_flag_LJ126 | potential_flag_Ewald);
}
