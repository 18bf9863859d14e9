/* Engine API (host side): set-up, particle load/unload, exclusions, the time step.
 *
 * Stands in for the parts of src/engine.c, src/engine_bonded.c and src/engine_rigid.c that
 * the nonbonded path needs.  All force evaluation runs on the GPU through
 * engine_nonbond_cuda (nonbond.cu); there is no CPU force path.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <time.h>
#include "mdcore_b200.h"
#include "internal.h"
#include "cycle.h"

int engine_err = engine_err_ok;

static const char *engine_msg[] = {
    "Nothing bad happened.",
    "An unexpected NULL pointer was encountered.",
    "A call to malloc failed, probably due to insufficient memory.",
    "An error occured when calling a space function.",
    "A call to a pthread routine failed.",
    "An error occured when calling a runner function.",
    "One or more values were outside of the allowed range.",
    "An error occured while calling a cell function.",
    "The computational domain is too small for the requested operation.",
    "mdcore was not compiled with MPI.",
    "An error occured while calling an MPI function.",
    "An error occured when calling a bond function.",
    "An error occured when calling an angle function.",
    "An error occured when calling a reader function.",
    "An error occured while interpreting the PSF file.",
    "An error occured while interpreting the PDB file.",
    "An error occured while interpreting the CPF file.",
    "An error occured when calling a potential function.",
    "An error occured when calling an exclusion function.",
    "An error occured while computing the bonded sets.",
    "An error occured when calling a dihedral funtion.",
    "An error occured when calling a CUDA funtion.",
    "mdcore was not compiled with CUDA support.",
    "CUDA support is only available in single-precision.",
    "Max. number of parts per cell exceeded.",
    "An error occured when calling a queue funtion.",
    "An error occured when evaluating a rigid constraint.",
    "Cell cutoff size doesn't work with METIS",
    "METIS library undefined",
    "Dependencies could not be computed.",
    "Not yet implemented."
};
#define engine_error(id) (engine_err = errs_register((id), engine_msg[-(id)], __LINE__, __func__, __FILE__))

/* Flags this engine implements (others are refused with engine_err_nyi). */
#define ENGINE_FLAGS_SUPPORTED                                                                 \
    (engine_flag_static | engine_flag_localparts | engine_flag_cuda | engine_flag_verlet |     \
     engine_flag_verlet_pairwise | engine_flag_affinity | engine_flag_prefetch |               \
     engine_flag_verlet_pseudo | engine_flag_unsorted | engine_flag_shake | engine_flag_nullpart |   \
     engine_flag_explepot)

size_t engine_sizeof(void) { return sizeof(struct engine); }

int engine_init(struct engine *e, const double *origin, const double *dim, double *L,
                double cutoff, unsigned int period, int max_type, unsigned int flags) {
    if (e == NULL || origin == NULL || dim == NULL || L == NULL) return engine_error(engine_err_null);
    if (flags & ~ENGINE_FLAGS_SUPPORTED) return engine_error(engine_err_nyi);
    memset(e, 0, sizeof(struct engine));
    if (space_init(&e->s, origin, dim, L, cutoff, period) < 0) return engine_error(engine_err_space);
    /* Flag implications of src/engine.c:2458-2463. */
    if (flags & engine_flag_verlet_pseudo) flags |= engine_flag_verlet_pairwise;
    if (flags & engine_flag_verlet_pairwise) flags |= engine_flag_verlet;
    e->flags = flags;
    e->time = 0;
    e->dt = 0.0;
    e->device = 0;
    if (flags & engine_flag_nullpart) max_type += 1;
    e->max_type = max_type;
    e->nr_types = 0;
    e->types = calloc(max_type, sizeof(struct part_type));
    e->p = calloc((size_t)max_type * max_type, sizeof(struct potential *));
    e->exclusions_size = 100;
    e->exclusions = malloc(sizeof(struct exclusion) * e->exclusions_size);
    e->rigids_size = 100;
    e->rigids = malloc(sizeof(struct rigid) * e->rigids_size);
    if (e->types == NULL || e->p == NULL || e->exclusions == NULL || e->rigids == NULL)
        return engine_error(engine_err_malloc);
    e->tol_rigid = 1e-6;
    if (flags & engine_flag_nullpart) {
        /* Type 0 is the interaction-free NULL type (src/engine.c:2517-2533). */
        strcpy(e->types[0].name, "NULL");
        strcpy(e->types[0].name2, "NULL");
        e->nr_types = 1;
    }
    return engine_err_ok;
}

int engine_addtype(struct engine *e, double mass, double charge, char *name, char *name2) {
    if (e == NULL) return engine_error(engine_err_null);
    if (e->nr_types >= e->max_type) return engine_error(engine_err_range);
    struct part_type *t = &e->types[e->nr_types];
    t->id = e->nr_types;
    t->mass = mass;
    t->imass = 1.0 / mass;
    t->charge = charge;
    strncpy(t->name, name ? name : "X", sizeof(t->name) - 1);
    strncpy(t->name2, name2 ? name2 : "X", sizeof(t->name2) - 1);
    return e->nr_types++;
}

int engine_addpot(struct engine *e, struct potential *p, int i, int j) {
    if (e == NULL) return engine_error(engine_err_null);
    if (i < 0 || i >= e->max_type || j < 0 || j >= e->max_type) return engine_error(engine_err_range);
    e->p[i * e->max_type + j] = p;
    if (i != j) e->p[j * e->max_type + i] = p;
    return engine_err_ok;
}

int engine_load(struct engine *e, double *x, double *v, int *type, int *pid, int *vid,
                double *q, unsigned int *flags, int N) {
    struct part p;
    if (e == NULL || x == NULL || type == NULL) return engine_error(engine_err_null);
    memset(&p, 0, sizeof(p));
    for (int j = 0; j < N; j++) {
        if (type[j] < 0 || type[j] >= e->max_type) return engine_error(engine_err_range);
        p.type = type[j];
        p.id = pid ? pid[j] : j;
        p.vid = vid ? vid[j] : 0;
        p.flags = flags ? flags[j] : part_flag_none;
        for (int k = 0; k < 3; k++) {
            p.v[k] = v ? v[3 * j + k] : 0.0;
            p.f[k] = 0.0f;
        }
        p.q = q ? q[j] : 0.0;
        if (space_addpart(&e->s, &p, &x[3 * j]) < 0) return engine_error(engine_err_space);
    }
    return engine_err_ok;
}

int engine_unload(struct engine *e, double *x, double *v, int *type, int *pid, int *vid,
                  double *q, unsigned int *flags, double *epot, int N) {
    if (e == NULL) return engine_error(engine_err_null);
    struct space *s = &e->s;
    int total = 0;
    for (int c = 0; c < s->nr_cells; c++) total += s->cells[c].count;
    if (total > N) return engine_error(engine_err_range);
    int count = 0;
    double ep = 0.0;
    for (int c = 0; c < s->nr_cells; c++) {
        struct cell *cl = &s->cells[c];
        ep += cl->epot;
        for (int k = 0; k < cl->count; k++, count++) {
            struct part *p = &cl->parts[k];
            if (x)
                for (int j = 0; j < 3; j++) x[3 * count + j] = cl->origin[j] + p->x[j];
            if (v)
                for (int j = 0; j < 3; j++) v[3 * count + j] = p->v[j];
            if (type) type[count] = p->type;
            if (pid) pid[count] = p->id;
            if (vid) vid[count] = p->vid;
            if (q) q[count] = p->q;
            if (flags) flags[count] = p->flags;
        }
    }
    if (epot) *epot += ep;
    return count;
}

int engine_getforces(struct engine *e, double *f, int N) {
    if (e == NULL || f == NULL) return engine_error(engine_err_null);
    struct space *s = &e->s;
    for (int id = 0; id < N; id++) {
        if (id >= s->size_parts || s->partlist[id] == NULL) {
            f[3 * id] = f[3 * id + 1] = f[3 * id + 2] = 0.0;
            continue;
        }
        for (int k = 0; k < 3; k++) f[3 * id + k] = s->partlist[id]->f[k];
    }
    return engine_err_ok;
}

int engine_getcells(struct engine *e, int *cell, int N) {
    if (e == NULL || cell == NULL) return engine_error(engine_err_null);
    struct space *s = &e->s;
    for (int id = 0; id < N; id++)
        cell[id] = (id < s->size_parts && s->celllist[id]) ? (int)(s->celllist[id] - s->cells) : -1;
    return engine_err_ok;
}

int engine_nonbond_stats(struct engine *e, struct nb_stats *out) {
    if (e == NULL || out == NULL) return engine_error(engine_err_null);
    *out = e->stats;
    return engine_err_ok;
}

/* ---------------------------------------------------------------- exclusions */

int engine_exclusion_add(struct engine *e, int i, int j) {
    if (e == NULL) return engine_error(engine_err_null);
    if (e->nr_exclusions == e->exclusions_size) {
        int nsize = e->exclusions_size * 2;
        struct exclusion *ne = realloc(e->exclusions, sizeof(struct exclusion) * nsize);
        if (ne == NULL) return engine_error(engine_err_malloc);
        e->exclusions = ne;
        e->exclusions_size = nsize;
    }
    struct exclusion *x = &e->exclusions[e->nr_exclusions++];
    x->i = i < j ? i : j;
    x->j = i < j ? j : i;
    return engine_err_ok;
}

static int excl_cmp(const void *a, const void *b) {
    const struct exclusion *x = a, *y = b;
    if (x->i != y->i) return x->i < y->i ? -1 : 1;
    if (x->j != y->j) return x->j < y->j ? -1 : 1;
    return 0;
}

/* Sort by (i, j) and drop duplicates, as src/engine_bonded.c:1301-1390. */
int engine_exclusion_shrink(struct engine *e) {
    if (e == NULL) return engine_error(engine_err_null);
    if (e->nr_exclusions == 0) return engine_err_ok;
    qsort(e->exclusions, e->nr_exclusions, sizeof(struct exclusion), excl_cmp);
    int j = 0;
    for (int k = 1; k < e->nr_exclusions; k++)
        if (e->exclusions[k].i != e->exclusions[j].i || e->exclusions[k].j != e->exclusions[j].j)
            e->exclusions[++j] = e->exclusions[k];
    e->nr_exclusions = j + 1;
    return engine_err_ok;
}

/* ---------------------------------------------------------------- rigid constraints */

/* Sets the P-SHAKE matrix of group r to the identity (src/engine_rigid.c:212-215). */
static void rigid_reset_matrix(struct rigid *r) {
    memset(r->a, 0, sizeof(float) * r->nr_constr * r->nr_constr);
    for (int k = 0; k < r->nr_constr; k++) r->a[k + k * r->nr_constr] = 1.0f;
}

/* src/engine_rigid.c:78-229: a distance constraint between particles pid and pjd joins
 * them into one rigid group -- a new group, an existing group of either particle, or the
 * merger of two groups.  Constraint ends are group-local indices. */
int engine_rigid_add(struct engine *e, int pid, int pjd, double d) {
    if (e == NULL) return engine_error(engine_err_null);
    if (pid < 0 || pjd < 0 || pid == pjd) return engine_error(engine_err_range);
    int need = (pid > pjd ? pid : pjd) + 1;
    if (need < e->s.size_parts) need = e->s.size_parts;
    if (e->part2rigid == NULL || need > e->part2rigid_size) {
        int *np = realloc(e->part2rigid, sizeof(int) * need);
        if (np == NULL) return engine_error(engine_err_malloc);
        for (int k = e->part2rigid ? e->part2rigid_size : 0; k < need; k++) np[k] = -1;
        e->part2rigid = np;
        e->part2rigid_size = need;
    }
    int rid = e->part2rigid[pid], rjd = e->part2rigid[pjd];
    struct rigid *r;
    if (rid < 0 && rjd < 0) {
        if (e->nr_rigids == e->rigids_size) {
            int nsize = e->rigids_size + e->rigids_size / 2 + 1;
            struct rigid *nr = realloc(e->rigids, sizeof(struct rigid) * nsize);
            if (nr == NULL) return engine_error(engine_err_malloc);
            e->rigids = nr;
            e->rigids_size = nsize;
        }
        r = &e->rigids[e->nr_rigids];
        r->nr_parts = 2;
        r->nr_constr = 1;
        r->parts[0] = pid;
        r->parts[1] = pjd;
        r->constr[0].i = 0;
        r->constr[0].j = 1;
        r->constr[0].d2 = d * d;
        e->part2rigid[pid] = e->part2rigid[pjd] = e->nr_rigids++;
    } else if (rid >= 0 && rjd >= 0 && rid != rjd) {
        /* Merge group rjd into rid, then add the constraint between the two. */
        r = &e->rigids[rid];
        struct rigid *o = &e->rigids[rjd];
        if (r->nr_parts + o->nr_parts > rigid_maxparts || r->nr_constr + o->nr_constr + 1 > rigid_maxconstr)
            return engine_error(engine_err_range);
        int ind = 0, jnd = 0;
        while (r->parts[ind] != pid) ind++;
        while (o->parts[jnd] != pjd) jnd++;
        for (int k = 0; k < o->nr_constr; k++) {
            r->constr[r->nr_constr + k] = o->constr[k];
            r->constr[r->nr_constr + k].i += r->nr_parts;
            r->constr[r->nr_constr + k].j += r->nr_parts;
        }
        for (int k = 0; k < o->nr_parts; k++) {
            r->parts[r->nr_parts + k] = o->parts[k];
            e->part2rigid[o->parts[k]] = rid;
        }
        r->nr_constr += o->nr_constr;
        jnd += r->nr_parts;
        r->nr_parts += o->nr_parts;
        r->constr[r->nr_constr].i = ind;
        r->constr[r->nr_constr].j = jnd;
        r->constr[r->nr_constr].d2 = d * d;
        r->nr_constr++;
        /* The last group takes the place of the merged one. */
        e->nr_rigids--;
        if (rjd < e->nr_rigids) {
            e->rigids[rjd] = e->rigids[e->nr_rigids];
            for (int k = 0; k < e->rigids[rjd].nr_parts; k++) e->part2rigid[e->rigids[rjd].parts[k]] = rjd;
            if (rid == e->nr_rigids) r = &e->rigids[rjd];
        }
    } else {
        /* One or both particles already in the same group. */
        r = &e->rigids[rid >= 0 ? rid : rjd];
        const int g = (int)(r - e->rigids);
        int ind = -1, jnd = -1;
        for (int k = 0; k < r->nr_parts; k++) {
            if (r->parts[k] == pid) ind = k;
            else if (r->parts[k] == pjd) jnd = k;
        }
        if (r->nr_constr >= rigid_maxconstr || ((ind < 0 || jnd < 0) && r->nr_parts >= rigid_maxparts))
            return engine_error(engine_err_range);
        if (ind < 0) {
            ind = r->nr_parts++;
            r->parts[ind] = pid;
            e->part2rigid[pid] = g;
        } else if (jnd < 0) {
            jnd = r->nr_parts++;
            r->parts[jnd] = pjd;
            e->part2rigid[pjd] = g;
        }
        r->constr[r->nr_constr].i = ind;
        r->constr[r->nr_constr].j = jnd;
        r->constr[r->nr_constr].d2 = d * d;
        r->nr_constr++;
    }
    rigid_reset_matrix(r);
    e->nr_constr++;
    e->rigids_gen++;
    return engine_err_ok;
}

int engine_rigid_get(struct engine *e, int g, struct rigid *out) {
    if (e == NULL) return engine_error(engine_err_null);
    if (out == NULL) return e->nr_rigids;
    if (g < 0 || g >= e->nr_rigids) return engine_error(engine_err_range);
    *out = e->rigids[g];
    return e->nr_rigids;
}

int engine_getparts(struct engine *e, float *x, float *v, float *f, int *cell, int N) {
    if (e == NULL) return engine_error(engine_err_null);
    struct space *s = &e->s;
    for (int id = 0; id < N; id++) {
        const struct part *p = (id < s->size_parts) ? s->partlist[id] : NULL;
        for (int k = 0; k < 3; k++) {
            if (x) x[3 * id + k] = p ? p->x[k] : 0.0f;
            if (v) v[3 * id + k] = p ? p->v[k] : 0.0f;
            if (f) f[3 * id + k] = p ? p->f[k] : 0.0f;
        }
        if (cell) cell[id] = p ? (int)(s->celllist[id] - s->cells) : -1;
    }
    return engine_err_ok;
}

/* ---------------------------------------------------------------- running */

int engine_start(struct engine *e, int nr_runners, int nr_queues) {
    (void)nr_queues;
    if (e == NULL) return engine_error(engine_err_null);
    e->nr_runners = nr_runners;
    if (engine_cuda_load(e) < 0) return engine_error(engine_err_cuda);
    return engine_err_ok;
}

/* Symplectic Euler update v += f/m dt, x += v dt, as src/engine.c:1945-2052; particles
 * that leave their cell are moved at the start of the next step.  Host threads over
 * ranges of cells. */
static void advance_cells(void *ctx, int part, int begin, int end) {
    struct engine *e = ctx;
    struct space *s = &e->s;
    float dt = e->dt;
    (void)part;
    for (int c = begin; c < end; c++) {
        struct cell *cl = &s->cells[c];
        for (int k = 0; k < cl->count; k++) {
            struct part *p = &cl->parts[k];
            float w = dt * e->types[p->type].imass;
            for (int j = 0; j < 3; j++) {
                p->v[j] += p->f[j] * w;
                p->x[j] += dt * p->v[j];
            }
        }
    }
}

int engine_advance(struct engine *e) {
    if (e == NULL) return engine_error(engine_err_null);
    struct space *s = &e->s;
    int grain = 8192 / (s->nr_parts / (s->nr_cells > 0 ? s->nr_cells : 1) + 1);
    nb_parallel_for(s->nr_cells, grain < 16 ? 16 : grain, advance_cells, e);
    return engine_err_ok;
}

/* One time step on the device with the host's particles as input and output: upload,
 * re-binning, forces, integration and constraints as device launches, download
 * (engine_cuda_step).  The same trajectory as engine_step_host, bit for bit. */
int engine_step(struct engine *e) {
    if (e == NULL) return engine_error(engine_err_null);
    struct timespec w0, w1;
    clock_gettime(CLOCK_MONOTONIC, &w0);
    const ticks tic = getticks();
    if (engine_cuda_step(e) < 0) return engine_error(engine_err_cuda);
    const ticks toc = getticks();
    clock_gettime(CLOCK_MONOTONIC, &w1);
    /* the step's phases (host milliseconds) in ticks at the rate this step ran */
    const double ms = (w1.tv_sec - w0.tv_sec) * 1e3 + (w1.tv_nsec - w0.tv_nsec) * 1e-6;
    e->timers[engine_timer_step] += toc - tic;
    if (ms > 0.0) {
        const double tpms = (double)(toc - tic) / ms;
        e->timers[engine_timer_cuda_load] += (ticks)(e->stats.ms_pack * tpms);
        e->timers[engine_timer_cuda_dopairs] += (ticks)(e->stats.ms_device * tpms);
        e->timers[engine_timer_cuda_unload] += (ticks)(e->stats.ms_unpack * tpms);
    }
    return engine_err_ok;
}

/* src/engine.c:167-183: every timer back to 0. */
int engine_timers_reset(struct engine *e) {
    if (e == NULL) return engine_error(engine_err_null);
    for (int k = 0; k < engine_timer_last; k++) e->timers[k] = 0;
    return engine_err_ok;
}

/* src/engine_rigid.c:266-345 splits the rigid groups into local, semi-local and remote
 * ones for the MPI ranks; one process holds every group here, so there is nothing to
 * split. */
int engine_rigid_sort(struct engine *e) {
    if (e == NULL) return engine_error(engine_err_null);
    return engine_err_ok;
}

/* src/engine_rigid.c:231-250: the rigid groups in a random order (rand(): each group
 * swapped with a random one); part2rigid follows, and the device copy of the groups is
 * rebuilt at the next step.  The constraints' results do not depend on the order. */
int engine_rigid_unsort(struct engine *e) {
    if (e == NULL) return engine_error(engine_err_null);
    const int n = e->nr_rigids;
    if (n < 2) return engine_err_ok;
    const double scale = (double)n / RAND_MAX;
    for (int k = 0; k < n; k++) {
        int j = (int)(rand() * scale);
        if (j >= n) j = n - 1;
        if (j != k) {
            const struct rigid t = e->rigids[j];
            e->rigids[j] = e->rigids[k];
            e->rigids[k] = t;
        }
    }
    for (int g = 0; g < n; g++)
        for (int k = 0; k < e->rigids[g].nr_parts; k++) e->part2rigid[e->rigids[g].parts[k]] = g;
    e->rigids_gen++;
    return engine_err_ok;
}

/* engine_step with re-binning and integration on the host threads and the force
 * evaluation and constraints through host buffers. */
int engine_step_host(struct engine *e) {
    if (e == NULL) return engine_error(engine_err_null);
    /* bonds, angles and dihedrals: device steps only */
    if (e->nr_bonds > 0 || e->nr_angles > 0 || e->nr_dihedrals > 0) return engine_error(engine_err_nyi);
    struct space *s = &e->s;
    e->time += 1;
    if (space_shuffle(s) < 0) return engine_error(engine_err_space);
    /* space_prepare's zeroing and the force evaluation in one pass over the particles */
    if (engine_nonbond_cuda_fresh(e) < 0) return engine_error(engine_err_cuda);
    s->epot += s->epot_nonbond;
    if (engine_advance(e) < 0) return engine_error(engine_err);
    /* Resolve the rigid constraints (src/engine.c:2196-2231). */
    if (e->nr_rigids > 0 && engine_rigid_eval(e) < 0) return engine_error(engine_err_rigid);
    return engine_err_ok;
}

int engine_finalize(struct engine *e) {
    if (e == NULL) return engine_error(engine_err_null);
    nb_device_free(e);
    rigid_device_free(e);
    for (int c = 0; c < e->s.nr_cells; c++) free(e->s.cells[c].parts);
    free(e->s.cells);
    free(e->s.cid_real);                 /* cid_marked is the same array */
    free(e->s.tasks);
    free(e->s.partlist);
    free(e->s.celllist);
    free(e->types);
    free(e->p);
    free(e->exclusions);
    free(e->rigids);
    free(e->part2rigid);
    free(e->bonds);
    free(e->p_bond);
    free(e->angles);
    free(e->p_angle);
    free(e->dihedrals);
    free(e->p_dihedral);
    memset(e, 0, sizeof(struct engine));
    return engine_err_ok;
}

int engine_setexplepot(struct engine *e, struct potential *ep) {
    if (e == NULL) return engine_error(engine_err_null);
    if (ep != NULL) {
        e->flags |= engine_flag_explepot;
        e->ep = ep;
    } else {
        e->flags &= ~engine_flag_explepot;
        e->ep = NULL;
    }
    return engine_err_ok;
}

int engine_bond_addpot(struct engine *e, struct potential *p, int i, int j) {
    if (e == NULL) return engine_error(engine_err_null);
    if (i < 0 || i >= e->max_type || j < 0 || j >= e->max_type) return engine_error(engine_err_range);
    if (e->p_bond == NULL) {
        e->p_bond = calloc((size_t)e->max_type * e->max_type, sizeof(struct potential *));
        if (e->p_bond == NULL) return engine_error(engine_err_malloc);
    }
    e->p_bond[i * e->max_type + j] = p;
    if (i != j) e->p_bond[j * e->max_type + i] = p;
    e->bonds_gen++;
    return engine_err_ok;
}

int engine_bond_add(struct engine *e, int i, int j) {
    if (e == NULL) return engine_error(engine_err_null);
    if (e->nr_bonds == e->bonds_size) {
        int nsize = e->bonds_size ? 2 * e->bonds_size : 100;
        struct bond *nb = realloc(e->bonds, sizeof(struct bond) * nsize);
        if (nb == NULL) return engine_error(engine_err_malloc);
        e->bonds = nb;
        e->bonds_size = nsize;
    }
    e->bonds[e->nr_bonds].i = i;
    e->bonds[e->nr_bonds].j = j;
    e->nr_bonds += 1;
    e->bonds_gen++;
    return engine_err_ok;
}

/* Grows an array of `size` elements of `elem` bytes holding `used` to at least used + 1. */
static int grow(void **arr, int *size, int used, size_t elem, int first) {
    if (used < *size) return 0;
    const int nsize = *size ? 2 * *size : first;
    void *na = realloc(*arr, elem * (size_t)nsize);
    if (na == NULL) return -1;
    *arr = na;
    *size = nsize;
    return 0;
}

int engine_angle_addpot(struct engine *e, struct potential *p) {
    if (e == NULL || p == NULL) return engine_error(engine_err_null);
    if (grow((void **)&e->p_angle, &e->anglepots_size, e->nr_anglepots, sizeof(struct potential *), 100) < 0)
        return engine_error(engine_err_malloc);
    e->p_angle[e->nr_anglepots] = p;
    e->bonds_gen++;
    return e->nr_anglepots++;
}

int engine_angle_add(struct engine *e, int i, int j, int k, int pid) {
    if (e == NULL) return engine_error(engine_err_null);
    if (grow((void **)&e->angles, &e->angles_size, e->nr_angles, sizeof(struct angle), 100) < 0)
        return engine_error(engine_err_malloc);
    struct angle *a = &e->angles[e->nr_angles++];
    a->i = i;
    a->j = j;
    a->k = k;
    a->pid = pid;
    e->bonds_gen++;
    return engine_err_ok;
}

int engine_dihedral_addpot(struct engine *e, struct potential *p) {
    if (e == NULL || p == NULL) return engine_error(engine_err_null);
    if (grow((void **)&e->p_dihedral, &e->dihedralpots_size, e->nr_dihedralpots, sizeof(struct potential *),
             100) < 0)
        return engine_error(engine_err_malloc);
    e->p_dihedral[e->nr_dihedralpots] = p;
    e->bonds_gen++;
    return e->nr_dihedralpots++;
}

int engine_dihedral_add(struct engine *e, int i, int j, int k, int l, int pid) {
    if (e == NULL) return engine_error(engine_err_null);
    if (grow((void **)&e->dihedrals, &e->dihedrals_size, e->nr_dihedrals, sizeof(struct dihedral), 100) < 0)
        return engine_error(engine_err_malloc);
    struct dihedral *d = &e->dihedrals[e->nr_dihedrals++];
    d->i = i;
    d->j = j;
    d->k = k;
    d->l = l;
    d->pid = pid;
    e->bonds_gen++;
    return engine_err_ok;
}

int engine_energies(struct engine *e, double *out) {
    if (e == NULL || out == NULL) return engine_error(engine_err_null);
    const struct space *s = &e->s;
    out[0] = s->epot;
    out[1] = s->epot_nonbond;
    out[2] = s->epot_bond;
    out[3] = s->epot_angle;
    out[4] = s->epot_dihedral;
    out[5] = s->epot_exclusion;
    return engine_err_ok;
}

int engine_set_dt(struct engine *e, double dt) {
    if (e == NULL) return engine_error(engine_err_null);
    e->dt = dt;
    return engine_err_ok;
}

/* Zeroes forces and energies before a stand-alone force evaluation (what space_prepare,
 * src/space.c:186-219, does at the start of a step). */
int engine_zero_forces(struct engine *e) {
    if (e == NULL) return engine_error(engine_err_null);
    struct space *s = &e->s;
    s->epot = s->epot_nonbond = s->epot_bond = s->epot_angle = s->epot_dihedral = s->epot_exclusion = 0.0;
    nb_zero_cells(s);
    return engine_err_ok;
}
