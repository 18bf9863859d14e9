/* Declarations shared by the host sources of libmdcore_b200 (not part of the public ABI). */
#ifndef MDCORE_B200_INTERNAL_H
#define MDCORE_B200_INTERNAL_H

#include "mdcore_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define space_cellid(s, i, j, k) ((((i) * (s)->cdim[1] + (j)) * (s)->cdim[2]) + (k))

/* Unit vector of sort direction sid (the values of cell_shift, src/cell.c:84-98). */
void sort_axis(int sid, float n[3]);
struct part *cell_add(struct cell *c, const struct part *p);
void space_relink(struct space *s, struct cell *c);
int space_shuffle(struct space *s);

void nb_sweep_scales(const struct space *s, float *bias, float *dscale, int *dmaxdist);
int nb_task_shift(struct space *s, int t, float dscale, float shift[3], int *dnshift, int *ci_out,
                  int *cj_out);

/* Analytic 12-6 Lennard-Jones A/r^12 - B/r^6 and Ewald real-space erfc(kappa r)/r (with the
 * 1/(4 pi) prefactor) values (potential.c). */
double nb_lj126(double r, double A, double B);
double nb_ewald(double r, double kappa);

/* Device side (nonbond.cu, rigid.cu). */
int nb_device_free(struct engine *e);
int rigid_device_free(struct engine *e);
/* Zeroes forces and energies of every cell of s (host threads over ranges of cells). */
void nb_zero_cells(struct space *s);
/* Calls fn(ctx, part, begin, end) over contiguous ranges of [0, n) of at least `grain`
 * items on the engine's host threads and returns when all are done; nb_host_parts() is
 * the largest number of ranges (parts are numbered from 0). */
void nb_parallel_for(int n, int grain, void (*fn)(void *ctx, int part, int begin, int end), void *ctx);
int nb_host_parts(void);
/* Rigid constraints inside a device-resident step (rigid.cu): where the engine's
 * particles live on the device. */
struct rigid_resident_view {
    const int *slot_of;     /* global particle id -> device slot */
    int id0;                /* the engine's first global id */
    void *xq, *v;           /* float4 device cells: position (w = type), velocity */
    int capc, cell0;        /* slots per cell, the engine's first global cell */
    const unsigned long long *abort;   /* nonzero: the step was aborted, launch nothing */
    /* fuse != 0: every particle of the engine is in a rigid group, and the constraint
     * kernel also runs the update (v += f dt/m, x += dt v) of each group's particles and
     * counts the completed step (done += {1, *pairs}); else all of these are unused. */
    int fuse;
    const unsigned long long *force;   /* fixed-point forces by slot */
    const double *imass;               /* 1/mass by type */
    float dtf;                         /* the time step as the update uses it */
    unsigned long long *status, *done;
    const unsigned long long *pairs;
};
int rigid_eval_resident(struct engine *e, const struct rigid_resident_view *view, void *stream);
/* Copies the iteration statistics of the last resident step to the host copy (wait = 0:
 * only enqueues the copy on `stream`). */
int rigid_resident_stats(struct engine *e, void *stream, int wait);
/* Launch stream of the engine's device state (NULL before engine_cuda_load). */
void *nb_engine_stream(struct engine *e);

#ifdef __cplusplus
}
#endif

#endif
