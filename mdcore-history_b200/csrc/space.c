/* Cell grid, particle binning and cell-pair task list (host side).
 *
 * Stands in for src/space.c:530-783 (space_init), :80-114 (space_getsid) and :382-434
 * (space_addpart) of the reference.  The grid, the cell-local float coordinates and the
 * (self, pair+sort-direction) task list are the same as the reference's, because the
 * device sweep must see the same cells, shifts and sort directions to reproduce its
 * pair set bit for bit.  The task dependency graph and the pthreads runner machinery of
 * the reference are not built: the device runs sort and sweep as two launches.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "mdcore_b200.h"
#include "internal.h"

int space_err = space_err_ok;

static const char *space_msg[] = {
    "Nothing bad happened.",
    "An unexpected NULL pointer was encountered.",
    "A call to malloc failed, probably due to insufficient memory.",
    "An error occured when calling a cell function.",
    "A call to a pthread routine failed.",
    "One or more values were outside of the allowed range.",
    "Too many pairs associated with a single particle in Verlet list.",
    "Task list too short.",
    "An error occured when calling a task function."
};
#define space_error(id) (space_err = errs_register((id), space_msg[-(id)], __LINE__, __func__, __FILE__))

/* Sort direction of a canonical (flipped) direction index: directions with index >= 13
 * point into the positive half-space and map to sid = 26 - index; the 13 directions with
 * index < 13 are their negatives (the cells get swapped).  This is the mapping of
 * cell_sortlistID / cell_flip, src/cell.c:56-101. */
static inline int sid_of_index(int idx) { return (idx < 13) ? idx : 26 - idx; }
static inline int flip_of_index(int idx) { return idx < 13; }

void sort_axis(int sid, float n[3]) {
    /* The unit vector along the direction with index 26 - sid. */
    int idx = 26 - sid;
    int d[3] = {idx / 9 - 1, (idx / 3) % 3 - 1, idx % 3 - 1};
    double len = sqrt((double)(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
    for (int k = 0; k < 3; k++) n[k] = (float)(d[k] / len);
}

int space_getsid(struct space *s, struct cell **ci, struct cell **cj, float *shift) {
    float lshift[3];
    if (shift == NULL) shift = lshift;
    for (int k = 0; k < 3; k++) {
        shift[k] = (*cj)->origin[k] - (*ci)->origin[k];
        if (shift[k] * 2 > s->dim[k])
            shift[k] -= s->dim[k];
        else if (shift[k] * 2 < -s->dim[k])
            shift[k] += s->dim[k];
    }
    int idx = 0;
    for (int k = 0; k < 3; k++) idx = 3 * idx + ((shift[k] < 0) ? 0 : ((shift[k] > 0) ? 2 : 1));
    if (flip_of_index(idx)) {
        struct cell *t = *ci;
        *ci = *cj;
        *cj = t;
        shift[0] = -shift[0];
        shift[1] = -shift[1];
        shift[2] = -shift[2];
    }
    return sid_of_index(idx);
}

static int add_task(struct space *s, int type, int sid, int i, int j) {
    if (s->nr_tasks >= s->tasks_size) {
        int nsize = s->tasks_size * 2 + 64;
        struct task *t = realloc(s->tasks, sizeof(struct task) * nsize);
        if (t == NULL) return space_error(space_err_malloc);
        s->tasks = t;
        s->tasks_size = nsize;
    }
    struct task *t = &s->tasks[s->nr_tasks++];
    t->type = (short)type;
    t->subtype = 0;
    t->flags = sid;
    t->i = i;
    t->j = j;
    return 0;
}

int space_init(struct space *s, const double *origin, const double *dim, double *L,
               double cutoff, unsigned int period) {
    if (s == NULL || origin == NULL || dim == NULL || L == NULL) return space_error(space_err_null);
    memset(s, 0, sizeof(struct space));
    for (int k = 0; k < 3; k++) {
        s->origin[k] = origin[k];
        s->dim[k] = dim[k];
        s->cdim[k] = floor(dim[k] / L[k]);
        if (s->cdim[k] < 1) return space_error(space_err_range);
    }
    s->cutoff = cutoff;
    s->cutoff2 = cutoff * cutoff;
    s->period = period;
    s->nr_cells = s->cdim[0] * s->cdim[1] * s->cdim[2];
    s->cells = calloc(s->nr_cells, sizeof(struct cell));
    if (s->cells == NULL) return space_error(space_err_malloc);
    /* every cell is real (and marked): one process holds the whole space, no ghosts */
    s->cid_real = malloc(sizeof(int) * s->nr_cells);
    if (s->cid_real == NULL) return space_error(space_err_malloc);
    for (int c = 0; c < s->nr_cells; c++) s->cid_real[c] = c;
    s->cid_marked = s->cid_real;
    s->cid_ghost = NULL;
    s->nr_real = s->nr_marked = s->nr_cells;
    s->nr_ghost = 0;
    for (int k = 0; k < 3; k++) {
        s->h[k] = s->dim[k] / s->cdim[k];
        s->ih[k] = 1.0 / s->h[k];
    }
    int l[3];
    for (l[0] = 0; l[0] < s->cdim[0]; l[0]++)
        for (l[1] = 0; l[1] < s->cdim[1]; l[1]++)
            for (l[2] = 0; l[2] < s->cdim[2]; l[2]++) {
                int cid = space_cellid(s, l[0], l[1], l[2]);
                struct cell *c = &s->cells[cid];
                c->id = cid;
                for (int k = 0; k < 3; k++) {
                    c->loc[k] = l[k];
                    c->origin[k] = origin[k] + l[k] * s->h[k];
                    c->dim[k] = s->h[k];
                }
                c->size = 0;
                c->count = 0;
                c->parts = NULL;
            }

    for (int k = 0; k < 3; k++) s->span[k] = ceil(cutoff * s->ih[k]);
    /* A periodic dimension narrower than 2*span+1 cells would pair a cell with the same
     * neighbour through both images; the reference then emits duplicate tasks. */
    for (int k = 0; k < 3; k++)
        if ((period & (1u << k)) && s->cdim[k] < 2 * s->span[k] + 1) return space_error(space_err_range);

    /* Self and pair tasks: every cell against every neighbour within the cutoff, each
     * unordered pair once (lower cell id first), cells flipped into the canonical
     * half-space by space_getsid. */
    s->tasks_size = s->nr_cells * 16;
    s->tasks = malloc(sizeof(struct task) * s->tasks_size);
    if (s->tasks == NULL) return space_error(space_err_malloc);
    s->nr_tasks = 0;
    for (int i = 0; i < s->cdim[0]; i++)
        for (int j = 0; j < s->cdim[1]; j++)
            for (int k = 0; k < s->cdim[2]; k++) {
                int id1 = space_cellid(s, i, j, k);
                int d[3], nb[3];
                for (d[0] = -s->span[0]; d[0] <= s->span[0]; d[0]++) {
                    nb[0] = i + d[0];
                    if (nb[0] < 0 || nb[0] >= s->cdim[0]) {
                        if (!(period & space_periodic_x)) continue;
                        nb[0] = (nb[0] + s->cdim[0]) % s->cdim[0];
                    }
                    for (d[1] = -s->span[1]; d[1] <= s->span[1]; d[1]++) {
                        nb[1] = j + d[1];
                        if (nb[1] < 0 || nb[1] >= s->cdim[1]) {
                            if (!(period & space_periodic_y)) continue;
                            nb[1] = (nb[1] + s->cdim[1]) % s->cdim[1];
                        }
                        for (d[2] = -s->span[2]; d[2] <= s->span[2]; d[2]++) {
                            double lh[3];
                            for (int q = 0; q < 3; q++) lh[q] = s->h[q] * fmax(abs(d[q]) - 1, 0);
                            if (lh[0] * lh[0] + lh[1] * lh[1] + lh[2] * lh[2] > s->cutoff2) continue;
                            nb[2] = k + d[2];
                            if (nb[2] < 0 || nb[2] >= s->cdim[2]) {
                                if (!(period & space_periodic_z)) continue;
                                nb[2] = (nb[2] + s->cdim[2]) % s->cdim[2];
                            }
                            int id2 = space_cellid(s, nb[0], nb[1], nb[2]);
                            struct cell *ci = &s->cells[id1], *cj = &s->cells[id2];
                            int sid = space_getsid(s, &ci, &cj, NULL);
                            if (id1 < id2 || (id1 == id2 && d[0] == 0 && d[1] == 0 && d[2] == 0)) {
                                int ci_id = (int)(ci - s->cells), cj_id = (int)(cj - s->cells);
                                if (add_task(s, (id1 == id2) ? task_type_self : task_type_pair, sid,
                                             ci_id, cj_id) < 0)
                                    return space_err;
                            }
                        }
                    }
                }
            }
    /* Sort directions each cell has to provide. */
    for (int t = 0; t < s->nr_tasks; t++)
        if (s->tasks[t].type == task_type_pair) {
            s->cells[s->tasks[t].i].sortmask |= 1u << s->tasks[t].flags;
            s->cells[s->tasks[t].j].sortmask |= 1u << s->tasks[t].flags;
        }

    s->size_parts = 0;
    s->nr_parts = 0;
    s->partlist = NULL;
    s->celllist = NULL;
    s->verlet_rebuild = 1;
    s->maxdx = 0.0f;
    return space_err_ok;
}

/* Append p to cell c, growing its buffer. */
struct part *cell_add(struct cell *c, const struct part *p) {
    if (c->count == c->size) {
        int nsize = c->size ? c->size * 2 : 16;
        struct part *np = NULL;
        if (posix_memalign((void **)&np, 64, sizeof(struct part) * nsize) != 0) return NULL;
        if (c->count) memcpy(np, c->parts, sizeof(struct part) * c->count);
        free(c->parts);
        c->parts = np;
        c->size = nsize;
    }
    c->parts[c->count] = *p;
    return &c->parts[c->count++];
}

int space_addpart(struct space *s, struct part *p, double *x) {
    int ind[3];
    if (s == NULL || p == NULL || x == NULL) return space_error(space_err_null);
    if (p->id < 0) return space_error(space_err_range);
    if (p->id >= s->size_parts) {
        int nsize = p->id + 1 > 2 * s->size_parts ? p->id + 1 : 2 * s->size_parts;
        struct part **pl = realloc(s->partlist, sizeof(struct part *) * nsize);
        struct cell **cl = realloc(s->celllist, sizeof(struct cell *) * nsize);
        if (pl == NULL || cl == NULL) return space_error(space_err_malloc);
        for (int k = s->size_parts; k < nsize; k++) { pl[k] = NULL; cl[k] = NULL; }
        s->partlist = pl;
        s->celllist = cl;
        s->size_parts = nsize;
    }
    /* Cell index by truncation of the double-precision scaled offset, and the position
     * stored relative to the cell origin in single precision (src/space.c:410-423). */
    for (int k = 0; k < 3; k++) ind[k] = (x[k] - s->origin[k]) * s->ih[k];
    for (int k = 0; k < 3; k++)
        if (ind[k] < 0 || ind[k] >= s->cdim[k]) return space_error(space_err_range);
    struct cell *c = &s->cells[space_cellid(s, ind[0], ind[1], ind[2])];
    for (int k = 0; k < 3; k++) p->x[k] = x[k] - c->origin[k];
    if (cell_add(c, p) == NULL) return space_error(space_err_malloc);
    if (s->partlist[p->id] == NULL) s->nr_parts++;
    s->celllist[p->id] = c;
    space_relink(s, c);
    return space_err_ok;
}

/* Refresh partlist entries of all particles of cell c (after its buffer moved). */
void space_relink(struct space *s, struct cell *c) {
    for (int k = 0; k < c->count; k++) {
        s->partlist[c->parts[k].id] = &c->parts[k];
        s->celllist[c->parts[k].id] = c;
    }
}

/* Particles that left their cell move into the neighbour cell (periodic wrap), as
 * src/space.c:235-291 does after each integration step, in a fixed order that does not
 * depend on threads: every cell keeps its remaining particles in their order, then
 * appends the arrivals from its 26 neighbours by direction index (dx+1)*9 + (dy+1)*3 +
 * (dz+1) of the move, each neighbour's leavers in their order.  (The reference's order
 * depends on which runner thread takes its cell mutex first.)  The device-resident steps
 * re-bin by the same rule, so host and device steps keep the same particle order.
 * Two parallel passes: leavers out of every cell, then arrivals into every cell with the
 * partlist/celllist entries of the cells that changed. */
struct shuffle_mover {
    struct part p;
    int dir;
};

struct shuffle_ctx {
    struct space *s;
    struct shuffle_mover **lists;   /* per host thread */
    int *count, *size;
    int *first, *nmove, *owner;     /* per cell: its leavers in lists[owner][first ..] */
    unsigned char *touched;
    int fail;
};

static void shuffle_scan(void *vctx, int part, int begin, int end) {
    struct shuffle_ctx *ctx = vctx;
    struct space *s = ctx->s;
    float h[3];
    for (int k = 0; k < 3; k++) h[k] = s->h[k];
    for (int cid = begin; cid < end; cid++) {
        struct cell *c = &s->cells[cid];
        int keep = 0;
        ctx->first[cid] = ctx->count[part];
        ctx->owner[cid] = part;
        for (int pid = 0; pid < c->count; pid++) {
            const struct part *p = &c->parts[pid];
            int delta[3];
            for (int k = 0; k < 3; k++) delta[k] = (p->x[k] >= h[k]) - (p->x[k] < 0.0f);
            if (delta[0] || delta[1] || delta[2]) {
                if (ctx->count[part] == ctx->size[part]) {
                    int nsize = ctx->size[part] * 2 + 64;
                    struct shuffle_mover *nl = realloc(ctx->lists[part], sizeof(struct shuffle_mover) * nsize);
                    if (nl == NULL) {
                        ctx->fail = 1;
                        return;
                    }
                    ctx->lists[part] = nl;
                    ctx->size[part] = nsize;
                }
                struct shuffle_mover *m = &ctx->lists[part][ctx->count[part]++];
                m->p = *p;
                for (int k = 0; k < 3; k++) m->p.x[k] -= delta[k] * h[k];
                m->dir = (delta[0] + 1) * 9 + (delta[1] + 1) * 3 + (delta[2] + 1);
            } else {
                if (keep < pid) c->parts[keep] = *p;
                keep += 1;
            }
        }
        ctx->nmove[cid] = ctx->count[part] - ctx->first[cid];
        if (keep < c->count) ctx->touched[cid] = 1;
        c->count = keep;
    }
}

static void shuffle_gather(void *vctx, int part, int begin, int end) {
    struct shuffle_ctx *ctx = vctx;
    struct space *s = ctx->s;
    (void)part;
    for (int cid = begin; cid < end && !ctx->fail; cid++) {
        struct cell *c = &s->cells[cid];
        for (int d = 0; d < 27; d++) {
            if (d == 13) continue;
            /* a particle that moved by delta(d) comes from the neighbour at -delta(d) */
            const int delta[3] = {d / 9 - 1, (d / 3) % 3 - 1, d % 3 - 1};
            int nl[3];
            for (int k = 0; k < 3; k++) nl[k] = (c->loc[k] - delta[k] + s->cdim[k]) % s->cdim[k];
            const int src = space_cellid(s, nl[0], nl[1], nl[2]);
            const struct shuffle_mover *m = ctx->lists[ctx->owner[src]] + ctx->first[src];
            for (int k = 0; k < ctx->nmove[src]; k++) {
                if (m[k].dir != d) continue;
                if (cell_add(c, &m[k].p) == NULL) {
                    ctx->fail = 1;
                    return;
                }
                ctx->touched[cid] = 1;
            }
        }
        if (ctx->touched[cid]) space_relink(s, c);
    }
}

int space_shuffle(struct space *s) {
    const int parts = nb_host_parts();
    const int nc = s->nr_cells > 0 ? s->nr_cells : 1;
    struct shuffle_ctx ctx;
    ctx.s = s;
    ctx.fail = 0;
    ctx.lists = calloc(parts, sizeof(struct shuffle_mover *));
    ctx.count = calloc(parts, sizeof(int));
    ctx.size = calloc(parts, sizeof(int));
    ctx.first = calloc(nc, sizeof(int));
    ctx.nmove = calloc(nc, sizeof(int));
    ctx.owner = calloc(nc, sizeof(int));
    ctx.touched = calloc(nc, 1);
    int rc = 0, moved = 0;
    if (ctx.lists == NULL || ctx.count == NULL || ctx.size == NULL || ctx.first == NULL || ctx.nmove == NULL ||
        ctx.owner == NULL || ctx.touched == NULL) {
        rc = space_error(space_err_malloc);
    } else {
        const int avg = s->nr_parts / nc + 1;
        const int grain = 8192 / avg < 16 ? 16 : 8192 / avg;
        nb_parallel_for(s->nr_cells, grain, shuffle_scan, &ctx);
        for (int q = 0; q < parts; q++) moved = moved || ctx.count[q] > 0;
        if (!ctx.fail && moved) nb_parallel_for(s->nr_cells, grain, shuffle_gather, &ctx);
        if (ctx.fail) rc = space_error(space_err_malloc);
        for (int q = 0; q < parts; q++) free(ctx.lists[q]);
    }
    free(ctx.lists); free(ctx.count); free(ctx.size); free(ctx.first); free(ctx.nmove); free(ctx.owner);
    free(ctx.touched);
    return rc < 0 ? rc : moved;
}

/* Sort-key scale and sweep bound, computed with the reference's float arithmetic
 * (src/runner_dosort.c:118-119, src/runner_dopair.c:580-583): bias = |h|, dscale =
 * 32767/(2 bias), dmaxdist = 2 + dscale*(cutoff + maxdx_i + maxdx_j) with maxdx = 0. */
void nb_sweep_scales(const struct space *s, float *bias, float *dscale, int *dmaxdist) {
    float b = sqrt(s->h[0] * s->h[0] + s->h[1] * s->h[1] + s->h[2] * s->h[2]);
    float ds = (float)32767 / (2 * b);
    float cutoff = s->cutoff;
    float maxdx = 0.0f;
    *bias = b;
    *dscale = ds;
    *dmaxdist = 2 + ds * (cutoff + maxdx + maxdx);
}

/* Shift of cell j relative to cell i of task t and its discretised norm
 * (src/runner_dopair.c:586-597).  The sweep takes dnshift as the distance of cell j from
 * cell i along the task's sort axis.  For cubic cells the shift lies on that axis and its
 * norm, which the reference uses, is that distance; for other cells the norm exceeds it and
 * the reference's sweep skips pairs inside the cutoff, so the projection on the axis is
 * used there (a lower bound, like the truncation to an integer). */
int nb_task_shift(struct space *s, int t, float dscale, float shift[3], int *dnshift, int *ci_out,
                  int *cj_out) {
    struct task *tk = &s->tasks[t];
    struct cell *ci = &s->cells[tk->i], *cj = &s->cells[tk->j];
    int sid = space_getsid(s, &ci, &cj, shift);
    float nshift = sqrt(shift[0] * shift[0] + shift[1] * shift[1] + shift[2] * shift[2]);
    if (!(s->h[0] == s->h[1] && s->h[1] == s->h[2])) {
        float n[3];
        sort_axis(sid, n);
        nshift = shift[0] * n[0] + shift[1] * n[1] + shift[2] * n[2];
        if (nshift < 0.0f) nshift = 0.0f;
    }
    *dnshift = dscale * nshift;
    *ci_out = (int)(ci - s->cells);
    *cj_out = (int)(cj - s->cells);
    return sid;
}

/* src/space.c:186-219: a space made ready for one time step -- the swap and stall
 * counters and the energies reset, every cell's energy and every particle's force zeroed
 * (there are no task waits to re-arm: no CPU runners). */
int space_prepare(struct space *s) {
    if (s == NULL) return space_error(space_err_null);
    s->nr_swaps = 0;
    s->nr_stalls = 0;
    s->epot = s->epot_nonbond = s->epot_bond = s->epot_angle = s->epot_dihedral = s->epot_exclusion = 0.0;
    nb_zero_cells(s);
    return space_err_ok;
}

/* src/space.c:447-466: the position of particle id (local id), its cell's origin plus the
 * cell-relative position. */
int space_getpos(struct space *s, int id, double *x) {
    if (s == NULL || x == NULL) return space_error(space_err_null);
    if (id < 0 || id >= s->nr_parts || s->partlist[id] == NULL) return space_error(space_err_range);
    for (int k = 0; k < 3; k++) x[k] = (double)s->partlist[id]->x[k] + s->celllist[id]->origin[k];
    return space_err_ok;
}
