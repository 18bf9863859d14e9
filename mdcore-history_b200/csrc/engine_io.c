/* Topology and parameter readers of the engine API (src/engine_io.c:82-1618, the tokenizer
 * src/reader.c:52-608):
 *
 *   engine_read_psf    a PSF topology (atoms, bonds, angles, dihedrals, impropers) and the
 *                      PDB coordinates of the same atoms (src/engine_io.c:1234-1618);
 *   engine_read_cpf    a CHARMM parameter file (src/engine_io.c:630-1232);
 *   engine_read_xplor  an XPLOR parameter file (src/engine_io.c:82-628).
 *
 * What they build is the reference's, decision for decision, so that an engine loaded from
 * the same files holds the same types, bonds, constraints, angle and dihedral potentials
 * and pair tables: a PSF atom's type is its atom type name joined with its charge string
 * (one engine type per such pair), positions are read in Angstrom and wrapped into the
 * box; a bond over a type whose name starts with 'H' becomes a rigid constraint when
 * rigidH is set (the bond is removed), other bond lines give harmonic bond tables for the
 * matching type pairs; an angle line gives its table to every matching angle; a dihedral
 * line gives its table to the matching dihedrals that have none yet (the first matching
 * line wins, 'X' matches any type); an improper line likewise to the impropers; the
 * nonbonded lines set each type's epsilon and Rmin, from which every type pair with
 * parameters gets a table: LJ (with the switch for CHARMM files), LJ + shifted Coulomb
 * (kappa = 0) or LJ + Ewald real space (kappa > 0), from an inner radius found by halving
 * [Rmin/2, Rmin] until the potential there is at most engine_maxKcutoff times its size at
 * Rmin; type pairs whose parameters (and charges, with electrostatics) equal an earlier
 * pair's share that pair's table.
 *
 * The files are read through their descriptors in one piece and split into tokens by
 * this file's own reader: whitespace separates tokens, a comment runs from a comment
 * character to the end of the line. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#include <unistd.h>

#include "internal.h"

#define engine_maxKcutoff 2   /* src/engine.h:82 */

/* ------------------------------------------------------------------ tokens */

struct toks {
    char *buf;
    size_t n, i;
    const char *comm;    /* characters that start a comment (to the end of the line) */
};

static int toks_open(struct toks *t, int fd, const char *comm) {
    size_t cap = 1 << 16;
    t->buf = malloc(cap);
    t->n = t->i = 0;
    t->comm = comm;
    if (t->buf == NULL) return -1;
    for (;;) {
        if (t->n == cap) {
            char *nb = realloc(t->buf, cap *= 2);
            if (nb == NULL) return -1;
            t->buf = nb;
        }
        ssize_t got = read(fd, t->buf + t->n, cap - t->n);
        if (got < 0) return -1;
        if (got == 0) break;
        t->n += (size_t)got;
    }
    return 0;
}

static void toks_close(struct toks *t) {
    free(t->buf);
    t->buf = NULL;
}

static int is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v'; }
static int is_comm(const struct toks *t, char c) { return t->comm != NULL && c != 0 && strchr(t->comm, c) != NULL; }

/* Skips whitespace and comments. */
static void toks_skip(struct toks *t) {
    while (t->i < t->n) {
        const char c = t->buf[t->i];
        if (is_ws(c)) {
            t->i++;
        } else if (is_comm(t, c)) {
            while (t->i < t->n && t->buf[t->i] != '\n') t->i++;
        } else {
            break;
        }
    }
}

/* The next token into out (at most cap-1 characters); its length, or -1 at the end. */
static int toks_next(struct toks *t, char *out, int cap) {
    toks_skip(t);
    if (t->i >= t->n) return -1;
    int len = 0;
    while (t->i < t->n && !is_ws(t->buf[t->i]) && !is_comm(t, t->buf[t->i])) {
        if (len < cap - 1) out[len++] = t->buf[t->i];
        t->i++;
    }
    out[len] = 0;
    return len;
}

/* Skips to the start of the next line. */
static void toks_skipline(struct toks *t) {
    while (t->i < t->n && t->buf[t->i] != '\n') t->i++;
    if (t->i < t->n) t->i++;
}

/* The comment that follows on this line (after blanks and the comment character). */
static int toks_comment(struct toks *t, char *out, int cap) {
    while (t->i < t->n && (t->buf[t->i] == ' ' || t->buf[t->i] == '\t')) t->i++;
    int len = 0;
    if (t->i < t->n && is_comm(t, t->buf[t->i])) {
        t->i++;
        while (t->i < t->n && t->buf[t->i] != '\n' && t->buf[t->i] != '\r') {
            if (len < cap - 1) out[len++] = t->buf[t->i];
            t->i++;
        }
    }
    out[len] = 0;
    return len;
}

static int tok_long(struct toks *t, long *v) {
    char b[100], *end;
    if (toks_next(t, b, sizeof(b)) < 0) return -1;
    *v = strtol(b, &end, 0);
    return *end == 0 ? 0 : -2;
}

static int tok_double(struct toks *t, double *v) {
    char b[100], *end;
    if (toks_next(t, b, sizeof(b)) < 0) return -1;
    *v = strtod(b, &end);
    return *end == 0 ? 0 : -2;
}

static int io_error(int code) {
    engine_err = code;
    errs_register(code, "Error while reading a topology or parameter file.", __LINE__, __func__, __FILE__);
    return code;
}

/* ------------------------------------------------------------------ type lookups */

int engine_gettype(struct engine *e, char *name) {
    if (e == NULL || name == NULL) return engine_err = engine_err_null;
    for (int k = 0; k < e->nr_types; k++)
        if (strcmp(e->types[k].name, name) == 0) return k;
    return engine_err_range;
}

int engine_gettype2(struct engine *e, char *name2) {
    if (e == NULL || name2 == NULL) return engine_err = engine_err_null;
    for (int k = 0; k < e->nr_types; k++)
        if (strcmp(e->types[k].name2, name2) == 0) return k;
    return engine_err_range;
}

static const char *type_of(struct engine *e, int id) { return e->types[e->s.partlist[id]->type].name; }

/* ------------------------------------------------------------------ PSF + PDB */

/* Reads a count and the comment after it, which must start with `tag`. */
static int psf_section(struct toks *t, const char *tag, long *n) {
    char c[100];
    if (tok_long(t, n) != 0) return engine_err_psf;
    toks_comment(t, c, sizeof(c));
    return strncmp(c, tag, strlen(tag)) == 0 ? 0 : engine_err_psf;
}

int engine_read_psf(struct engine *e, int psf, int pdb) {
    if (e == NULL) return io_error(engine_err_null);
    struct toks t;
    char b[100], type[100], name2[200];
    if (toks_open(&t, psf, "!") < 0) return io_error(engine_err_reader);
    int rc = 0;
    int *typeids = NULL, *resids = NULL;
    long n = 0;
    if (toks_next(&t, b, sizeof(b)) < 0 || strcmp(b, "PSF") != 0) { rc = engine_err_psf; goto out; }
    /* the title: a count, then the rest of that line and the title lines */
    if (tok_long(&t, &n) != 0) { rc = engine_err_psf; goto out; }
    for (long k = 0; k <= n; k++) toks_skipline(&t);
    if ((rc = psf_section(&t, "NATOM", &n)) < 0) goto out;
    typeids = malloc(sizeof(int) * (n > 0 ? n : 1));
    resids = malloc(sizeof(int) * (n > 0 ? n : 1));
    if (typeids == NULL || resids == NULL) { rc = engine_err_malloc; goto out; }
    const long natoms = n;
    for (long k = 0; k < natoms; k++) {
        long resid;
        double q, m;
        /* id, segment, residue id, residue name, atom name, type, charge, mass, 0 */
        if (toks_next(&t, b, sizeof(b)) < 0 || toks_next(&t, b, sizeof(b)) < 0) { rc = engine_err_reader; goto out; }
        if (tok_long(&t, &resid) != 0) { rc = engine_err_psf; goto out; }
        if (toks_next(&t, b, sizeof(b)) < 0 || toks_next(&t, b, sizeof(b)) < 0) { rc = engine_err_reader; goto out; }
        if (toks_next(&t, type, sizeof(type)) < 0) { rc = engine_err_reader; goto out; }
        char qs[100], *end;
        if (toks_next(&t, qs, sizeof(qs)) < 0) { rc = engine_err_reader; goto out; }
        q = strtod(qs, &end);
        if (*end != 0) { rc = engine_err_psf; goto out; }
        snprintf(name2, sizeof(name2), "%s%s", type, qs);
        if (tok_double(&t, &m) != 0) { rc = engine_err_psf; goto out; }
        resids[k] = (int)resid;
        int id = engine_gettype2(e, name2);
        if (id == engine_err_range) id = engine_addtype(e, m, q, type, name2);
        if (id < 0) { rc = engine_err; goto out; }
        typeids[k] = id;
        if (toks_next(&t, b, sizeof(b)) < 0) { rc = engine_err_reader; goto out; }
    }
    /* bonds, angles, dihedrals, impropers: 1-based atom numbers */
    static const struct { const char *tag; int arity, pid; } secs[4] = {
        {"NBOND", 2, 0}, {"NTHETA", 3, -1}, {"NPHI", 4, -1}, {"NIMP", 4, -2}};
    for (int sct = 0; sct < 4; sct++) {
        if ((rc = psf_section(&t, secs[sct].tag, &n)) < 0) goto out;
        for (long k = 0; k < n; k++) {
            long a[4];
            for (int q = 0; q < secs[sct].arity; q++)
                if (tok_long(&t, &a[q]) != 0) { rc = engine_err_psf; goto out; }
            int r;
            if (secs[sct].arity == 2) r = engine_bond_add(e, (int)a[0] - 1, (int)a[1] - 1);
            else if (secs[sct].arity == 3) r = engine_angle_add(e, (int)a[0] - 1, (int)a[1] - 1, (int)a[2] - 1, -1);
            else r = engine_dihedral_add(e, (int)a[0] - 1, (int)a[1] - 1, (int)a[2] - 1, (int)a[3] - 1, secs[sct].pid);
            if (r < 0) { rc = engine_err; goto out; }
        }
    }
    toks_close(&t);

    /* PDB: REMARK lines, ATOM records (serial, name, two more fields, x, y, z in Angstrom;
     * the k-th ATOM is atom k of the PSF), END */
    if (toks_open(&t, pdb, NULL) < 0) { rc = engine_err_reader; goto out_noclose; }
    struct part p;
    memset(&p, 0, sizeof(p));
    long pid = 0;
    for (;;) {
        if (toks_next(&t, b, sizeof(b)) < 0) { rc = engine_err_reader; goto out; }
        if (strncmp(b, "REMARK", 6) == 0) {
            toks_skipline(&t);
        } else if (strncmp(b, "ATOM", 4) == 0) {
            pid += 1;
            if (pid > natoms) { rc = engine_err_pdb; goto out; }
            for (int q = 0; q < 4; q++)
                if (toks_next(&t, b, sizeof(b)) < 0) { rc = engine_err_reader; goto out; }
            double x[3];
            for (int k = 0; k < 3; k++) {
                double v;
                if (tok_double(&t, &v) != 0) { rc = engine_err_pdb; goto out; }
                x[k] = fmod(e->s.dim[k] - e->s.origin[k] + 0.1 * v, e->s.dim[k]) + e->s.origin[k];
            }
            p.id = (int)pid - 1;
            p.vid = resids[pid - 1];
            p.q = (float)e->types[typeids[pid - 1]].charge;
            p.flags = part_flag_none;
            p.type = (short)typeids[pid - 1];
            if (space_addpart(&e->s, &p, x) < 0) { rc = engine_err_space; goto out; }
            toks_skipline(&t);
        } else if (strncmp(b, "END", 3) == 0) {
            break;
        } else {
            rc = engine_err_pdb;
            goto out;
        }
    }
out:
    toks_close(&t);
out_noclose:
    free(typeids);
    free(resids);
    return rc < 0 ? io_error(rc) : engine_err_ok;
}

/* ------------------------------------------------------------------ parameter lines */

/* A bond line: rigid constraints for bonds over an 'H' type (rigidH), else a harmonic
 * bond table K (r - r0)^2 (kcal/mol/A^2 -> kJ/mol/nm^2, A -> nm) on [r0/2, 3 r0/2] for
 * every matching type pair. */
static int bond_line(struct engine *e, const char *t1, const char *t2, double K, double r0, double tol, int rigidH,
                     int *ind1, int *ind2) {
    if (rigidH && (t1[0] == 'H' || t2[0] == 'H')) {
        for (int k = 0; k < e->nr_bonds; k++) {
            const char *a = type_of(e, e->bonds[k].i), *b = type_of(e, e->bonds[k].j);
            if ((strcmp(a, t1) == 0 && strcmp(b, t2) == 0) || (strcmp(a, t2) == 0 && strcmp(b, t1) == 0)) {
                if (engine_rigid_add(e, e->bonds[k].i, e->bonds[k].j, 0.1 * r0) < 0) return engine_err;
                e->nr_bonds -= 1;
                e->bonds[k] = e->bonds[e->nr_bonds];
                k -= 1;
            }
        }
        return 0;
    }
    int n1 = 0, n2 = 0;
    const int same = strcmp(t1, t2) == 0;
    for (int k = 0; k < e->nr_types; k++) {
        if (strcmp(t1, e->types[k].name) == 0) ind1[n1++] = k;
        else if (!same && strcmp(t2, e->types[k].name) == 0) ind2[n2++] = k;
    }
    if (n1 == 0 || (!same && n2 == 0)) return 0;
    struct potential *p = potential_create_harmonic(0.05 * r0, 0.15 * r0, 418.4 * K, 0.1 * r0, tol);
    if (p == NULL) return engine_err_potential;
    for (int a = 0; a < n1; a++)
        for (int b = same ? a : 0; b < (same ? n1 : n2); b++)
            if (engine_bond_addpot(e, p, ind1[a], same ? ind1[b] : ind2[b]) < 0) return engine_err;
    return 0;
}

/* An angle line: a harmonic angle table K (theta - theta0)^2 (degrees, kcal/mol/rad^2) on
 * theta0 +- halfwidth degrees for every angle over the three types (either direction). */
static int angle_line(struct engine *e, const char *t1, const char *t2, const char *t3, double K, double r0,
                      double halfwidth, double tol) {
    int potid = -1;
    for (int k = 0; k < e->nr_angles; k++) {
        const char *a = type_of(e, e->angles[k].i), *b = type_of(e, e->angles[k].j), *c = type_of(e, e->angles[k].k);
        if (strcmp(b, t2) != 0) continue;
        if (!((strcmp(a, t1) == 0 && strcmp(c, t3) == 0) || (strcmp(a, t3) == 0 && strcmp(c, t1) == 0))) continue;
        if (potid < 0) {
            struct potential *p = potential_create_harmonic_angle(M_PI / 180 * (r0 - halfwidth),
                                                                  M_PI / 180 * (r0 + halfwidth), 4.184 * K,
                                                                  M_PI / 180 * r0, tol);
            if (p == NULL) return engine_err_potential;
            if ((potid = engine_angle_addpot(e, p)) < 0) return engine_err;
        }
        e->angles[k].pid = potid;
    }
    return 0;
}

/* Does dihedral k (i, j, k, l) match the four types, forwards or backwards ('X': any)? */
static int dihedral_matches(struct engine *e, const struct dihedral *d, char t[4][100], const int wc[4]) {
    const char *n[4] = {type_of(e, d->i), type_of(e, d->j), type_of(e, d->k), type_of(e, d->l)};
    int fwd = 1, bwd = 1;
    for (int q = 0; q < 4; q++) {
        fwd = fwd && (wc[q] || strcmp(n[q], t[q]) == 0);
        bwd = bwd && (wc[3 - q] || strcmp(n[q], t[3 - q]) == 0);
    }
    return fwd || bwd;
}

/* A dihedral line (K, n, delta) for the proper dihedrals still without a table (pid -1), or
 * an improper line (K, theta0: a harmonic angle table on theta0 +- 45 degrees) for the
 * impropers still without one (pid -2). */
static int dihedral_line(struct engine *e, char t[4][100], double K, int n, double r0, double tol, int improper) {
    int wc[4];
    for (int q = 0; q < 4; q++) wc[q] = strcmp(t[q], "X") == 0;
    const int want = improper ? -2 : -1;
    int potid = -1;
    for (int k = 0; k < e->nr_dihedrals; k++) {
        if (e->dihedrals[k].pid != want || !dihedral_matches(e, &e->dihedrals[k], t, wc)) continue;
        if (potid < 0) {
            struct potential *p =
                improper ? potential_create_harmonic_angle(M_PI / 180 * (r0 - 45), M_PI / 180 * (r0 + 45), 4.184 * K,
                                                           M_PI / 180 * r0, tol)
                         : potential_create_harmonic_dihedral(4.184 * K, n, M_PI / 180 * r0, tol);
            if (p == NULL) return engine_err_potential;
            if ((potid = engine_dihedral_addpot(e, p)) < 0) return engine_err;
        }
        e->dihedrals[k].pid = potid;
    }
    return 0;
}

/* Do any of the line's types (not wildcards) exist in the engine? */
static int any_type(struct engine *e, char t[][100], int nt, int wildcards) {
    for (int q = 0; q < nt; q++)
        if (!(wildcards && strcmp(t[q], "X") == 0) && engine_gettype(e, t[q]) >= 0) return 1;
    return 0;
}

/* The largest r in [rmin/2, rmin] (halving to 1e-5) at which |V| is still at least
 * engine_maxKcutoff |V(rmin)|: the inner end of a pair table. */
static double inner_radius(double r0, double A, double B, double q, double kappa) {
    double al = r0 / 2, ar = r0;
    double v0 = nb_lj126(r0, A, B);
    if (kappa == 0.0) v0 += potential_escale * q / r0;
    else if (kappa > 0.0) v0 += q * nb_ewald(r0, kappa);
    const double Kr0 = fabs(v0);
    while (ar - al > 1e-5) {
        const double am = 0.5 * (al + ar);
        double vm = nb_lj126(am, A, B);
        if (kappa == 0.0) vm += potential_escale * q / am;
        else if (kappa > 0.0) vm += q * nb_ewald(am, kappa);
        if (fabs(vm) < engine_maxKcutoff * Kr0) ar = am;
        else al = am;
    }
    return al;
}

/* The pair tables of every type pair with parameters (cpf: the CHARMM forms with the LJ
 * switch at switchlen). */
static int pair_tables(struct engine *e, double kappa, double tol, double switchlen, int cpf) {
    for (int j = 0; j < e->nr_types; j++)
        for (int k = j; k < e->nr_types; k++) {
            const struct part_type *tj = &e->types[j], *tk = &e->types[k];
            if ((tj->eps == 0.0 || tk->eps == 0.0) && (kappa < 0.0 || tj->charge == 0.0 || tk->charge == 0.0))
                continue;
            /* an earlier pair with the same parameters (and charges) lends its table */
            int jj, kk;
            for (jj = 0; jj < j; jj++) {
                const struct part_type *u = &e->types[jj];
                if (u->eps == tj->eps && u->rmin == tj->rmin && (kappa < 0.0 || u->charge == tj->charge)) break;
            }
            for (kk = 0; kk < k; kk++) {
                const struct part_type *u = &e->types[kk];
                if (u->eps == tk->eps && u->rmin == tk->rmin && (kappa < 0.0 || u->charge == tk->charge)) break;
            }
            if (jj < j && kk < k) {
                struct potential *lent = e->p[jj * e->max_type + kk];
                if (lent != NULL && engine_addpot(e, lent, j, k) < 0) return engine_err;
                continue;
            }
            const double K = sqrt(tj->eps * tk->eps);
            const double r0 = tj->rmin + tk->rmin, r2 = r0 * r0, r6 = r2 * r2 * r2;
            const double A = K * r6 * r6, B = 2 * K * r6, q = tj->charge * tk->charge;
            struct potential *p = NULL;
            if (K == 0.0 && q != 0.0 && kappa >= 0.0) {
                p = kappa > 0.0 ? potential_create_Ewald(0.1, e->s.cutoff, q, kappa, tol)
                                : potential_create_Coulomb(0.1, e->s.cutoff, q, tol);
                if (p == NULL) return engine_err_potential;
            }
            const double al = inner_radius(r0, A, B, q, kappa);
            if (kappa < 0.0)
                p = cpf ? potential_create_LJ126_switch(al, e->s.cutoff, A, B, switchlen, tol)
                        : potential_create_LJ126(al, e->s.cutoff, A, B, tol);
            else if (kappa == 0.0)
                p = potential_create_LJ126_Coulomb(al, e->s.cutoff, A, B, q, tol);
            else
                p = cpf ? potential_create_LJ126_Ewald_switch(al, e->s.cutoff, A, B, q, kappa, switchlen, tol)
                        : potential_create_LJ126_Ewald(al, e->s.cutoff, A, B, q, kappa, tol);
            if (p == NULL) return engine_err_potential;
            if (engine_addpot(e, p, j, k) < 0) return engine_err;
        }
    return 0;
}

/* ------------------------------------------------------------------ CHARMM parameters */

int engine_read_cpf(struct engine *e, int cpf, double kappa, double tol, int rigidH, double switchlen) {
    if (e == NULL) return io_error(engine_err_null);
    struct toks t;
    if (toks_open(&t, cpf, "!") < 0) return io_error(engine_err_reader);
    int *ind1 = malloc(sizeof(int) * (e->nr_types + 1)), *ind2 = malloc(sizeof(int) * (e->nr_types + 1));
    char ty[4][100], b[100];
    int rc = 0;
    if (ind1 == NULL || ind2 == NULL) { rc = engine_err_malloc; goto out; }
    /* title lines start with '*' */
    while (t.i < t.n && t.buf[t.i] == '*') toks_skipline(&t);
    if (toks_next(&t, b, sizeof(b)) < 0 || strncmp(b, "BOND", 4) != 0) { rc = engine_err_cpf; goto out; }
    for (;;) {                                   /* BONDS: type type K r0 */
        double K, r0;
        if (toks_next(&t, ty[0], 100) < 0) { rc = engine_err_reader; goto out; }
        if (strncmp(ty[0], "ANGL", 4) == 0) break;
        if (toks_next(&t, ty[1], 100) < 0) { rc = engine_err_reader; goto out; }
        if (tok_double(&t, &K) != 0 || tok_double(&t, &r0) != 0) { rc = engine_err_cpf; goto out; }
        if ((rc = bond_line(e, ty[0], ty[1], K, r0, tol, rigidH, ind1, ind2)) < 0) goto out;
        toks_skipline(&t);
    }
    toks_skipline(&t);
    for (;;) {                                   /* ANGLES: type type type K theta0 [UB terms] */
        double K, r0;
        if (toks_next(&t, ty[0], 100) < 0) { rc = engine_err_reader; goto out; }
        if (strncmp(ty[0], "DIHE", 4) == 0) break;
        if (toks_next(&t, ty[1], 100) < 0 || toks_next(&t, ty[2], 100) < 0) { rc = engine_err_reader; goto out; }
        if (!any_type(e, ty, 3, 0)) { toks_skipline(&t); continue; }
        if (tok_double(&t, &K) != 0 || tok_double(&t, &r0) != 0) { rc = engine_err_cpf; goto out; }
        if ((rc = angle_line(e, ty[0], ty[1], ty[2], K, r0, 40.0, tol)) < 0) goto out;
        toks_skipline(&t);
    }
    toks_skipline(&t);
    for (int sect = 0; sect < 2; sect++) {      /* DIHEDRALS: 4 types K n delta; IMPROPER: 4 types K 0 psi0 */
        for (;;) {
            double K, r0;
            long nn = 0;
            if (toks_next(&t, ty[0], 100) < 0) { rc = engine_err_reader; goto out; }
            if (strncmp(ty[0], sect == 0 ? "IMPR" : "NONB", 4) == 0) break;
            for (int q = 1; q < 4; q++)
                if (toks_next(&t, ty[q], 100) < 0) { rc = engine_err_reader; goto out; }
            if (!any_type(e, ty, 4, 1)) { toks_skipline(&t); continue; }
            if (tok_double(&t, &K) != 0) { rc = engine_err_cpf; goto out; }
            if (sect == 0) {
                if (tok_long(&t, &nn) != 0) { rc = engine_err_cpf; goto out; }
            } else if (toks_next(&t, b, sizeof(b)) < 0) {
                rc = engine_err_reader;
                goto out;
            }
            if (tok_double(&t, &r0) != 0) { rc = engine_err_cpf; goto out; }
            if ((rc = dihedral_line(e, ty, K, (int)nn, r0, sect == 0 ? 1e-2 : tol, sect == 1)) < 0) goto out;
            toks_skipline(&t);
        }
        toks_skipline(&t);
    }
    for (;;) {                                   /* NONBONDED: type ignored epsilon Rmin/2 [1-4 terms] */
        double K, r0;
        if (toks_next(&t, ty[0], 100) < 0) { rc = engine_err_reader; goto out; }
        if (strncmp(ty[0], "HBOND", 5) == 0) break;
        if (toks_next(&t, b, sizeof(b)) < 0) { rc = engine_err_reader; goto out; }
        if (tok_double(&t, &K) != 0 || tok_double(&t, &r0) != 0) { rc = engine_err_cpf; goto out; }
        for (int k = 0; k < e->nr_types; k++)
            if (strcmp(e->types[k].name, ty[0]) == 0) {
                e->types[k].eps = 4.184 * K;
                e->types[k].rmin = 0.1 * r0;
            }
        toks_skipline(&t);
    }
    toks_close(&t);
    rc = pair_tables(e, kappa, tol, switchlen, 1);
    free(ind1);
    free(ind2);
    return rc < 0 ? io_error(rc) : engine_err_ok;
out:
    toks_close(&t);
    free(ind1);
    free(ind2);
    return io_error(rc < 0 ? rc : engine_err_cpf);
}

/* ------------------------------------------------------------------ XPLOR parameters */

int engine_read_xplor(struct engine *e, int xplor, double kappa, double tol, int rigidH) {
    if (e == NULL) return io_error(engine_err_null);
    struct toks t;
    if (toks_open(&t, xplor, "!{") < 0) return io_error(engine_err_reader);
    int *ind1 = malloc(sizeof(int) * (e->nr_types + 1)), *ind2 = malloc(sizeof(int) * (e->nr_types + 1));
    char ty[4][100], b[100];
    int rc = 0;
    if (ind1 == NULL || ind2 == NULL) { rc = engine_err_malloc; goto out; }
    /* one statement per line, keyword first (any case); other lines are ignored */
    while (toks_next(&t, b, sizeof(b)) >= 0) {
        double K, r0;
        long nn = 0;
        if (strncasecmp(b, "BOND", 4) == 0) {
            if (toks_next(&t, ty[0], 100) < 0 || toks_next(&t, ty[1], 100) < 0) { rc = engine_err_reader; goto out; }
            if (tok_double(&t, &K) != 0 || tok_double(&t, &r0) != 0) { rc = engine_err_cpf; goto out; }
            if ((rc = bond_line(e, ty[0], ty[1], K, r0, tol, rigidH, ind1, ind2)) < 0) goto out;
        } else if (strncasecmp(b, "ANGL", 4) == 0) {
            for (int q = 0; q < 3; q++)
                if (toks_next(&t, ty[q], 100) < 0) { rc = engine_err_reader; goto out; }
            if (!any_type(e, ty, 3, 0)) { toks_skipline(&t); continue; }
            if (tok_double(&t, &K) != 0 || tok_double(&t, &r0) != 0) { rc = engine_err_cpf; goto out; }
            if ((rc = angle_line(e, ty[0], ty[1], ty[2], K, r0, 45.0, tol)) < 0) goto out;
        } else if (strncasecmp(b, "DIHE", 4) == 0 || strncasecmp(b, "IMPR", 4) == 0) {
            const int improper = strncasecmp(b, "IMPR", 4) == 0;
            for (int q = 0; q < 4; q++)
                if (toks_next(&t, ty[q], 100) < 0) { rc = engine_err_reader; goto out; }
            if (!any_type(e, ty, 4, 1)) { toks_skipline(&t); continue; }
            if (tok_double(&t, &K) != 0) { rc = engine_err_cpf; goto out; }
            if (!improper) {
                if (tok_long(&t, &nn) != 0) { rc = engine_err_cpf; goto out; }
            } else if (toks_next(&t, b, sizeof(b)) < 0) {
                rc = engine_err_reader;
                goto out;
            }
            if (tok_double(&t, &r0) != 0) { rc = engine_err_cpf; goto out; }
            if ((rc = dihedral_line(e, ty, K, (int)nn, r0, tol, improper)) < 0) goto out;
        } else if (strncasecmp(b, "NONB", 4) == 0) {
            if (toks_next(&t, ty[0], 100) < 0) { rc = engine_err_reader; goto out; }
            if (tok_double(&t, &K) != 0 || tok_double(&t, &r0) != 0) { rc = engine_err_cpf; goto out; }
            for (int k = 0; k < e->nr_types; k++)
                if (strcmp(e->types[k].name, ty[0]) == 0) {
                    e->types[k].eps = 4.184 * K;
                    e->types[k].rmin = 0.05 * r0;
                }
        }
        toks_skipline(&t);
    }
    toks_close(&t);
    rc = pair_tables(e, kappa, tol, 0.0, 0);
    free(ind1);
    free(ind2);
    return rc < 0 ? io_error(rc) : engine_err_ok;
out:
    toks_close(&t);
    free(ind1);
    free(ind2);
    return io_error(rc < 0 ? rc : engine_err_cpf);
}
