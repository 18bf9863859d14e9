/* Test/bench infrastructure (not product code): the binary "system file" that describes
 * one synthetic nonbonded workload, read by the reference driver (oracle/ref_driver.c) and
 * written by tests/sysfile.py.  Little-endian, no padding surprises: every record is made
 * of 4- and 8-byte fields in the order below.
 *
 *   char    magic[8]           "MDB2SYS1"
 *   int32   N, ntypes, npots, nexcl, flags, period
 *   double  origin[3], dim[3], L[3], cutoff
 *   ntypes x { double mass, charge }
 *   npots  x { int32 kind, ti, tj, pad; double a, b, tol, p[4] }
 *   double  x[3*N]
 *   int32   type[N]
 *   int32   excl[2*nexcl]
 *
 * Potential kinds map onto the reference's potential_create_* calls
 * (src/potential.c:517-914):
 *   1 LJ126(A=p0,B=p1)            2 LJ126_Coulomb(A=p0,B=p1,q=p2)
 *   3 Coulomb(q=p0)               4 Ewald(q=p0,kappa=p1)
 *   5 LJ126_Ewald(A=p0,B=p1,q=p2,kappa=p3)
 *   6 pair counter: a one-interval table whose energy is exactly 1.0f and force 0,
 *     so the summed nonbonded energy equals the number of accepted pairs.
 */
#ifndef MDB2_SYSFILE_H
#define MDB2_SYSFILE_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

struct sys_pot {
    int kind, ti, tj, pad;
    double a, b, tol, p[4];
};

struct sys_desc {
    int N, ntypes, npots, nexcl, flags, period;
    double origin[3], dim[3], L[3], cutoff;
    double *mass, *charge;
    struct sys_pot *pots;
    double *x;
    int *type;
    int *excl;
};

static int sys_read(const char *fname, struct sys_desc *s) {
    FILE *f = fopen(fname, "rb");
    char magic[8];
    int k, hdr[6];
    double d[10];
    if (f == NULL) return -1;
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "MDB2SYS1", 8) != 0) { fclose(f); return -2; }
    if (fread(hdr, sizeof(int), 6, f) != 6) { fclose(f); return -3; }
    s->N = hdr[0]; s->ntypes = hdr[1]; s->npots = hdr[2]; s->nexcl = hdr[3];
    s->flags = hdr[4]; s->period = hdr[5];
    if (fread(d, sizeof(double), 10, f) != 10) { fclose(f); return -3; }
    for (k = 0; k < 3; k++) { s->origin[k] = d[k]; s->dim[k] = d[3 + k]; s->L[k] = d[6 + k]; }
    s->cutoff = d[9];
    s->mass = malloc(sizeof(double) * (s->ntypes + 1));
    s->charge = malloc(sizeof(double) * (s->ntypes + 1));
    for (k = 0; k < s->ntypes; k++) {
        double mc[2];
        if (fread(mc, sizeof(double), 2, f) != 2) { fclose(f); return -4; }
        s->mass[k] = mc[0]; s->charge[k] = mc[1];
    }
    s->pots = malloc(sizeof(struct sys_pot) * (s->npots + 1));
    if (s->npots > 0 && fread(s->pots, sizeof(struct sys_pot), s->npots, f) != (size_t)s->npots) { fclose(f); return -5; }
    s->x = malloc(sizeof(double) * 3 * (s->N + 1));
    s->type = malloc(sizeof(int) * (s->N + 1));
    s->excl = malloc(sizeof(int) * 2 * (s->nexcl + 1));
    if (fread(s->x, sizeof(double), 3 * (size_t)s->N, f) != 3 * (size_t)s->N) { fclose(f); return -6; }
    if (fread(s->type, sizeof(int), s->N, f) != (size_t)s->N) { fclose(f); return -7; }
    if (s->nexcl > 0 && fread(s->excl, sizeof(int), 2 * (size_t)s->nexcl, f) != 2 * (size_t)s->nexcl) { fclose(f); return -8; }
    fclose(f);
    return 0;
}

#endif
