/* Test/bench infrastructure (not product code).
 *
 * Driver for the reference mdcore CPU library (built by oracle/Makefile.ref into
 * oracle/_ref/).  It only uses the reference's public engine API, the way the reference's
 * own example drivers do (examples/argon/argon.c, examples/bulk/bulk.c):
 * engine_init, engine_addtype, potential_create_*, engine_addpot, engine_load,
 * engine_exclusion_add/_shrink, engine_start, engine_step.
 *
 *   ref_driver forces <sysfile> <outfile> <nr_runners>
 *       One engine_step with dt = 0 (positions do not move, src/engine.c:1975-1979), then
 *       dumps forces, energies, cell assignment, sort lists and the float potential tables.
 *   ref_driver rigid <sysfile> <rigidfile> <outfile> <nevals>
 *       Loads the system with velocities, adds the rigid constraints (engine_rigid_add),
 *       sets dt, then calls engine_rigid_eval nevals times (src/engine_rigid.c:352-583:
 *       SHAKE with engine_flag_shake, P-SHAKE otherwise) and dumps, after each call, the
 *       cell-relative positions, velocities and forces by particle id and every group's
 *       P-SHAKE matrix.  Rigid file (little-endian): "MDB2RIG1", int32 ncon, shake, pad,
 *       double dt, double v[3N], ncon x {int32 i, j; double d}.
 *   ref_driver mdbench <sysfile> <rigidfile> <nr_runners> <warmup> <steps>
 *       Loads the system with velocities and rigid constraints, sets dt from the rigid file,
 *       starts nr_runners runners and times full engine_step calls (sort + sweep +
 *       exclusions + integration + P-SHAKE, src/engine.c:2070-2240); one JSON line.
 *   ref_driver bonded <sysfile> <bondedfile> <outfile>
 *       Loads the system (no runners), adds the bonded potentials and terms of the bonded
 *       file (engine_bond_addpot/engine_bond_add, engine_angle_addpot/engine_angle_add,
 *       engine_dihedral_addpot/engine_dihedral_add with potential_create_harmonic,
 *       _harmonic_angle and _harmonic_dihedral), then calls the reference's bond_eval,
 *       angle_eval and dihedral_eval (src/bond.c:81, src/angle.c:81, src/dihedral.c:81)
 *       once each on zeroed forces and dumps each one's forces and energy, the
 *       cell-relative positions and cells, and every bonded table.  Bonded file
 *       (little-endian): "MDB2BND1", int32 nbondpot, nangpot, ndihpot, nbond, nang, ndih;
 *       nbondpot x {int32 ti, tj; double a, b, K, r0, tol}; nangpot x {double a, b, K,
 *       theta0, tol}; ndihpot x {int32 n, pad; double K, delta, tol}; nbond x {int32 i, j};
 *       nang x {int32 i, j, k, pid}; ndih x {int32 i, j, k, l, pid}.
 *   ref_driver bench <sysfile> <nr_runners> <warmup> <steps>
 *       Times engine_step (dt = 0: sort + pair/self sweep + exclusion subtraction +
 *       bookkeeping, src/engine.c:2070-2240) with clock_gettime and prints one JSON line.
 *
 * The pair-counter potential (sysfile kind 6) is a hand-made one-interval table:
 * alpha = {1,0,0} selects interval 1 for every r, its coefficients are all zero except the
 * constant term 1.0f, so potential_eval (src/potential_eval.h:67-104) returns e = 1.0f and
 * f = 0 exactly and the nonbonded energy sums to the number of accepted pairs.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <time.h>
#include <pthread.h>
#include <omp.h>
#include "cycle.h"
#include "mdcore.h"
#include "sysfile.h"

static struct potential *make_counter(void) {
    struct potential *p = NULL;
    float *c = NULL;
    if (posix_memalign((void **)&p, 16, sizeof(struct potential)) != 0) return NULL;
    if (posix_memalign((void **)&c, 64, sizeof(float) * 2 * potential_chunk) != 0) return NULL;
    memset(c, 0, sizeof(float) * 2 * potential_chunk);
    c[potential_chunk + 1] = 1.0f;                  /* x = r */
    c[2 * potential_chunk - 1] = 1.0f;              /* constant term */
    p->alpha[0] = 1.0f; p->alpha[1] = 0.0f; p->alpha[2] = 0.0f; p->alpha[3] = 0.0f;
    p->c = c; p->a = 0.0; p->b = DBL_MAX; p->flags = potential_flag_none; p->n = 1;
    return p;
}

static struct potential *make_pot(const struct sys_pot *sp) {
    switch (sp->kind) {
        case 1: return potential_create_LJ126(sp->a, sp->b, sp->p[0], sp->p[1], sp->tol);
        case 2: return potential_create_LJ126_Coulomb(sp->a, sp->b, sp->p[0], sp->p[1], sp->p[2], sp->tol);
        case 3: return potential_create_Coulomb(sp->a, sp->b, sp->p[0], sp->tol);
        case 4: return potential_create_Ewald(sp->a, sp->b, sp->p[0], sp->p[1], sp->tol);
        case 5: return potential_create_LJ126_Ewald(sp->a, sp->b, sp->p[0], sp->p[1], sp->p[2], sp->p[3], sp->tol);
        case 6: return make_counter();
    }
    return NULL;
}

static int build_v(struct engine *e, struct sys_desc *sd, struct potential ***pots_out, int runners, double *v,
                   unsigned int extra_flags, int start) {
    int k;
    struct potential **pots = malloc(sizeof(struct potential *) * (sd->npots + 1));
    if (engine_init(e, sd->origin, sd->dim, sd->L, sd->cutoff, sd->period, sd->ntypes,
                    sd->flags | extra_flags) != 0) {
        fprintf(stderr, "ref_driver: engine_init failed (%i)\n", engine_err);
        errs_dump(stderr);
        return -1;
    }
    for (k = 0; k < sd->ntypes; k++)
        if (engine_addtype(e, sd->mass[k], sd->charge[k], NULL, NULL) < 0) { errs_dump(stderr); return -1; }
    for (k = 0; k < sd->npots; k++) {
        if ((pots[k] = make_pot(&sd->pots[k])) == NULL) {
            fprintf(stderr, "ref_driver: potential %i (kind %i) failed (%i)\n", k, sd->pots[k].kind, potential_err);
            errs_dump(stderr);
            return -1;
        }
        if (engine_addpot(e, pots[k], sd->pots[k].ti, sd->pots[k].tj) < 0) { errs_dump(stderr); return -1; }
    }
    if (engine_load(e, sd->x, v, sd->type, NULL, NULL, NULL, NULL, sd->N) < 0) {
        fprintf(stderr, "ref_driver: engine_load failed (%i)\n", engine_err);
        errs_dump(stderr);
        return -1;
    }
    for (k = 0; k < sd->nexcl; k++)
        if (engine_exclusion_add(e, sd->excl[2 * k], sd->excl[2 * k + 1]) < 0) { errs_dump(stderr); return -1; }
    if (sd->nexcl > 0 && engine_exclusion_shrink(e) < 0) { errs_dump(stderr); return -1; }
    e->time = 0;
    e->dt = 0.0;
    if (start && engine_start(e, runners, runners) < 0) {
        fprintf(stderr, "ref_driver: engine_start failed (%i)\n", engine_err);
        errs_dump(stderr);
        return -1;
    }
    *pots_out = pots;
    return 0;
}

static int build(struct engine *e, struct sys_desc *sd, struct potential ***pots_out, int runners) {
    return build_v(e, sd, pots_out, runners, NULL, 0, 1);
}

static int do_rigid(const char *sysf, const char *rigf, const char *outf, int nevals) {
    struct sys_desc sd;
    static struct engine e;
    struct potential **pots;
    char magic[8];
    int hdr[3], k, id, ev;
    double dt;
    FILE *f, *out;
    if (sys_read(sysf, &sd) != 0) { fprintf(stderr, "ref_driver: bad system file %s\n", sysf); return 1; }
    f = fopen(rigf, "rb");
    if (f == NULL || fread(magic, 1, 8, f) != 8 || memcmp(magic, "MDB2RIG1", 8) != 0 ||
        fread(hdr, sizeof(int), 3, f) != 3 || fread(&dt, sizeof(double), 1, f) != 1) {
        fprintf(stderr, "ref_driver: bad rigid file %s\n", rigf);
        return 1;
    }
    double *v = malloc(sizeof(double) * 3 * sd.N);
    if (fread(v, sizeof(double), 3 * (size_t)sd.N, f) != 3 * (size_t)sd.N) return 1;
    if (build_v(&e, &sd, &pots, 1, v, hdr[1] ? engine_flag_shake : 0, 0) != 0) return 1;
    for (k = 0; k < hdr[0]; k++) {
        int ij[2];
        double d;
        if (fread(ij, sizeof(int), 2, f) != 2 || fread(&d, sizeof(double), 1, f) != 1) return 1;
        if (engine_rigid_add(&e, ij[0], ij[1], d) < 0) { errs_dump(stderr); return 1; }
    }
    fclose(f);
    e.dt = dt;
    e.time = 0;
    out = fopen(outf, "wb");
    if (out == NULL) return 1;
    fwrite(&sd.N, sizeof(int), 1, out);
    fwrite(&e.nr_rigids, sizeof(int), 1, out);
    fwrite(&nevals, sizeof(int), 1, out);
    for (ev = 0; ev < nevals; ev++) {
        if (engine_rigid_eval(&e) != 0) { errs_dump(stderr); return 1; }
        for (id = 0; id < sd.N; id++) fwrite(e.s.partlist[id]->x, sizeof(float), 3, out);
        for (id = 0; id < sd.N; id++) fwrite(e.s.partlist[id]->v, sizeof(float), 3, out);
        for (id = 0; id < sd.N; id++) fwrite(e.s.partlist[id]->f, sizeof(float), 3, out);
        for (k = 0; k < e.nr_rigids; k++) {
            struct rigid *r = &e.rigids[k];
            fwrite(&r->nr_parts, sizeof(int), 1, out);
            fwrite(r->parts, sizeof(int), r->nr_parts, out);
            fwrite(&r->nr_constr, sizeof(int), 1, out);
            for (int c = 0; c < r->nr_constr; c++) {
                fwrite(&r->constr[c].i, sizeof(int), 1, out);
                fwrite(&r->constr[c].j, sizeof(int), 1, out);
                fwrite(&r->constr[c].d2, sizeof(double), 1, out);
            }
            fwrite(r->a, sizeof(float), (size_t)r->nr_constr * r->nr_constr, out);
        }
    }
    for (id = 0; id < sd.N; id++) {
        int c = (int)(e.s.celllist[id] - e.s.cells);
        fwrite(&c, sizeof(int), 1, out);
    }
    fclose(out);
    return 0;
}

static double now_s(void);

static int do_mdbench(const char *sysf, const char *rigf, int runners, int warmup, int steps) {
    struct sys_desc sd;
    static struct engine e;
    struct potential **pots;
    char magic[8];
    int hdr[3], k;
    double dt, t0, t1;
    FILE *f;
    if (sys_read(sysf, &sd) != 0) { fprintf(stderr, "ref_driver: bad system file %s\n", sysf); return 1; }
    f = fopen(rigf, "rb");
    if (f == NULL || fread(magic, 1, 8, f) != 8 || memcmp(magic, "MDB2RIG1", 8) != 0 ||
        fread(hdr, sizeof(int), 3, f) != 3 || fread(&dt, sizeof(double), 1, f) != 1) {
        fprintf(stderr, "ref_driver: bad rigid file %s\n", rigf);
        return 1;
    }
    double *v = malloc(sizeof(double) * 3 * sd.N);
    if (fread(v, sizeof(double), 3 * (size_t)sd.N, f) != 3 * (size_t)sd.N) return 1;
    omp_set_num_threads(runners);
    if (build_v(&e, &sd, &pots, runners, v, hdr[1] ? engine_flag_shake : 0, 0) != 0) return 1;
    for (k = 0; k < hdr[0]; k++) {
        int ij[2];
        double d;
        if (fread(ij, sizeof(int), 2, f) != 2 || fread(&d, sizeof(double), 1, f) != 1) return 1;
        if (engine_rigid_add(&e, ij[0], ij[1], d) < 0) { errs_dump(stderr); return 1; }
    }
    fclose(f);
    if (engine_start(&e, runners, runners) < 0) { errs_dump(stderr); return 1; }
    e.dt = dt;
    for (k = 0; k < warmup; k++)
        if (engine_step(&e) != 0) { errs_dump(stderr); return 1; }
    t0 = now_s();
    for (k = 0; k < steps; k++)
        if (engine_step(&e) != 0) { errs_dump(stderr); return 1; }
    t1 = now_s();
    printf("{\"ms_per_step\": %.6f, \"steps\": %i, \"runners\": %i, \"epot\": %.17g}\n",
           1e3 * (t1 - t0) / steps, steps, runners, e.s.epot);
    return 0;
}

static int do_forces(const char *sysf, const char *outf, int runners) {
    struct sys_desc sd;
    static struct engine e;
    struct potential **pots;
    int k, id, cid, hdr[4];
    double en[3];
    FILE *out;
    if (sys_read(sysf, &sd) != 0) { fprintf(stderr, "ref_driver: bad system file %s\n", sysf); return 1; }
    if (build(&e, &sd, &pots, runners) != 0) return 1;
    if (engine_step(&e) != 0) { errs_dump(stderr); return 1; }
    out = fopen(outf, "wb");
    if (out == NULL) return 1;
    hdr[0] = sd.N; hdr[1] = sd.npots; hdr[2] = e.s.nr_cells; hdr[3] = e.nr_exclusions;
    fwrite(hdr, sizeof(int), 4, out);
    en[0] = e.s.epot; en[1] = e.s.epot_nonbond; en[2] = e.s.epot_exclusion;
    fwrite(en, sizeof(double), 3, out);
    /* Forces, cell-relative float positions and cell index, by particle id. */
    for (id = 0; id < sd.N; id++) {
        double f[3];
        struct part *p = e.s.partlist[id];
        for (k = 0; k < 3; k++) f[k] = p->f[k];
        fwrite(f, sizeof(double), 3, out);
    }
    for (id = 0; id < sd.N; id++) fwrite(e.s.partlist[id]->x, sizeof(float), 3, out);
    for (id = 0; id < sd.N; id++) {
        int c = (int)(e.s.celllist[id] - e.s.cells);
        fwrite(&c, sizeof(int), 1, out);
    }
    /* Per cell: count, sort-task flags, particle ids in cell order, 13*count sort keys. */
    for (cid = 0; cid < e.s.nr_cells; cid++) {
        struct cell *c = &e.s.cells[cid];
        int cf[2];
        cf[0] = c->count; cf[1] = c->sort ? (int)c->sort->flags : 0;
        fwrite(cf, sizeof(int), 2, out);
        for (k = 0; k < c->count; k++) fwrite(&c->parts[k].id, sizeof(int), 1, out);
        fwrite(c->sortlist, sizeof(unsigned int), 13 * (size_t)c->count, out);
    }
    /* Float tables. */
    for (k = 0; k < sd.npots; k++) {
        struct potential *p = pots[k];
        int n = p->n;
        fwrite(&n, sizeof(int), 1, out);
        fwrite(p->alpha, sizeof(float), 4, out);
        fwrite(p->c, sizeof(float), (size_t)(n + 1) * potential_chunk, out);
    }
    fclose(out);
    return 0;
}

static void zero_forces(struct engine *e, int N) {
    int id;
    for (id = 0; id < N; id++) e->s.partlist[id]->f[0] = e->s.partlist[id]->f[1] = e->s.partlist[id]->f[2] = 0.0f;
}

static void dump_forces(struct engine *e, int N, FILE *out) {
    int id;
    for (id = 0; id < N; id++) fwrite(e->s.partlist[id]->f, sizeof(float), 3, out);
}

static void dump_table(const struct potential *p, FILE *out) {
    int n = p->n;
    double ab[2];
    fwrite(&n, sizeof(int), 1, out);
    fwrite(p->alpha, sizeof(float), 4, out);
    fwrite(p->c, sizeof(float), (size_t)(n + 1) * potential_chunk, out);
    ab[0] = p->a; ab[1] = p->b;
    fwrite(ab, sizeof(double), 2, out);
}

static int do_bonded(const char *sysf, const char *bndf, const char *outf) {
    struct sys_desc sd;
    static struct engine e;
    struct potential **pots, **bp, **ap, **dp;
    char magic[8];
    int hdr[6], k, id;
    double en[3] = {0.0, 0.0, 0.0};
    FILE *f, *out;
    if (sys_read(sysf, &sd) != 0) { fprintf(stderr, "ref_driver: bad system file %s\n", sysf); return 1; }
    if (build_v(&e, &sd, &pots, 1, NULL, 0, 0) != 0) return 1;
    f = fopen(bndf, "rb");
    if (f == NULL || fread(magic, 1, 8, f) != 8 || memcmp(magic, "MDB2BND1", 8) != 0 ||
        fread(hdr, sizeof(int), 6, f) != 6) {
        fprintf(stderr, "ref_driver: bad bonded file %s\n", bndf);
        return 1;
    }
    bp = malloc(sizeof(struct potential *) * (hdr[0] + 1));
    ap = malloc(sizeof(struct potential *) * (hdr[1] + 1));
    dp = malloc(sizeof(struct potential *) * (hdr[2] + 1));
    for (k = 0; k < hdr[0]; k++) {
        int t[2];
        double d[5];
        if (fread(t, sizeof(int), 2, f) != 2 || fread(d, sizeof(double), 5, f) != 5) return 1;
        if ((bp[k] = potential_create_harmonic(d[0], d[1], d[2], d[3], d[4])) == NULL) { errs_dump(stderr); return 1; }
        if (engine_bond_addpot(&e, bp[k], t[0], t[1]) < 0) { errs_dump(stderr); return 1; }
    }
    for (k = 0; k < hdr[1]; k++) {
        double d[5];
        if (fread(d, sizeof(double), 5, f) != 5) return 1;
        if ((ap[k] = potential_create_harmonic_angle(d[0], d[1], d[2], d[3], d[4])) == NULL) { errs_dump(stderr); return 1; }
        if (engine_angle_addpot(&e, ap[k]) != k) { errs_dump(stderr); return 1; }
    }
    for (k = 0; k < hdr[2]; k++) {
        int t[2];
        double d[3];
        if (fread(t, sizeof(int), 2, f) != 2 || fread(d, sizeof(double), 3, f) != 3) return 1;
        if ((dp[k] = potential_create_harmonic_dihedral(d[0], t[0], d[1], d[2])) == NULL) { errs_dump(stderr); return 1; }
        if (engine_dihedral_addpot(&e, dp[k]) != k) { errs_dump(stderr); return 1; }
    }
    for (k = 0; k < hdr[3]; k++) {
        int t[2];
        if (fread(t, sizeof(int), 2, f) != 2) return 1;
        if (engine_bond_add(&e, t[0], t[1]) < 0) { errs_dump(stderr); return 1; }
    }
    for (k = 0; k < hdr[4]; k++) {
        int t[4];
        if (fread(t, sizeof(int), 4, f) != 4) return 1;
        if (engine_angle_add(&e, t[0], t[1], t[2], t[3]) < 0) { errs_dump(stderr); return 1; }
    }
    for (k = 0; k < hdr[5]; k++) {
        int t[5];
        if (fread(t, sizeof(int), 5, f) != 5) return 1;
        if (engine_dihedral_add(&e, t[0], t[1], t[2], t[3], t[4]) < 0) { errs_dump(stderr); return 1; }
    }
    fclose(f);
    out = fopen(outf, "wb");
    if (out == NULL) return 1;
    fwrite("MDB2BOU1", 1, 8, out);
    {
        int oh[4];
        oh[0] = sd.N; oh[1] = hdr[0]; oh[2] = hdr[1]; oh[3] = hdr[2];
        fwrite(oh, sizeof(int), 4, out);
    }
    zero_forces(&e, sd.N);
    if (bond_eval(e.bonds, e.nr_bonds, &e, &en[0]) < 0) { errs_dump(stderr); return 1; }
    dump_forces(&e, sd.N, out);
    zero_forces(&e, sd.N);
    if (angle_eval(e.angles, e.nr_angles, &e, &en[1]) < 0) { errs_dump(stderr); return 1; }
    dump_forces(&e, sd.N, out);
    zero_forces(&e, sd.N);
    if (dihedral_eval(e.dihedrals, e.nr_dihedrals, &e, &en[2]) < 0) { errs_dump(stderr); return 1; }
    dump_forces(&e, sd.N, out);
    fwrite(en, sizeof(double), 3, out);
    for (id = 0; id < sd.N; id++) fwrite(e.s.partlist[id]->x, sizeof(float), 3, out);
    for (id = 0; id < sd.N; id++) {
        int c = (int)(e.s.celllist[id] - e.s.cells);
        fwrite(&c, sizeof(int), 1, out);
    }
    for (k = 0; k < hdr[0]; k++) dump_table(bp[k], out);
    for (k = 0; k < hdr[1]; k++) dump_table(ap[k], out);
    for (k = 0; k < hdr[2]; k++) dump_table(dp[k], out);
    fclose(out);
    return 0;
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static int do_bench(const char *sysf, int runners, int warmup, int steps) {
    struct sys_desc sd;
    static struct engine e;
    struct potential **pots;
    int k;
    double t0, t1, tmin = 1e30;
    if (sys_read(sysf, &sd) != 0) { fprintf(stderr, "ref_driver: bad system file %s\n", sysf); return 1; }
    omp_set_num_threads(runners);
    if (build(&e, &sd, &pots, runners) != 0) return 1;
    for (k = 0; k < warmup; k++)
        if (engine_step(&e) != 0) { errs_dump(stderr); return 1; }
    t0 = now_s();
    for (k = 0; k < steps; k++) {
        double ts = now_s();
        if (engine_step(&e) != 0) { errs_dump(stderr); return 1; }
        ts = now_s() - ts;
        if (ts < tmin) tmin = ts;
    }
    t1 = now_s();
    printf("{\"ms_per_step\": %.6f, \"ms_min\": %.6f, \"steps\": %i, \"runners\": %i, "
           "\"epot\": %.17g, \"nr_tasks\": %i, \"nr_cells\": %i}\n",
           1e3 * (t1 - t0) / steps, 1e3 * tmin, steps, runners, e.s.epot, e.s.nr_tasks, e.s.nr_cells);
    return 0;
}

int main(int argc, char *argv[]) {
    if (argc >= 5 && strcmp(argv[1], "forces") == 0)
        return do_forces(argv[2], argv[3], atoi(argv[4]));
    if (argc >= 7 && strcmp(argv[1], "mdbench") == 0)
        return do_mdbench(argv[2], argv[3], atoi(argv[4]), atoi(argv[5]), atoi(argv[6]));
    if (argc >= 6 && strcmp(argv[1], "rigid") == 0)
        return do_rigid(argv[2], argv[3], argv[4], atoi(argv[5]));
    if (argc >= 5 && strcmp(argv[1], "bonded") == 0)
        return do_bonded(argv[2], argv[3], argv[4]);
    if (argc >= 6 && strcmp(argv[1], "bench") == 0)
        return do_bench(argv[2], atoi(argv[3]), atoi(argv[4]), atoi(argv[5]));
    fprintf(stderr, "usage: ref_driver forces <sys> <out> <runners> | bench <sys> <runners> <warmup> <steps>\n");
    return 2;
}
