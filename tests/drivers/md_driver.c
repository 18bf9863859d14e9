/* A molecular-dynamics driver written against the mdcore engine API the way the
 * reference's example programs use it (examples/argon/argon.c): set up an engine, a
 * Lennard-Jones table and one particle type, insert particles with space_addpart, remove
 * the net momentum through e.s.cells[].parts[], set e.time and e.dt by hand, start the
 * engine and call engine_step, reading e.s.epot and rescaling the velocities in the cells
 * between steps.  The same source is compiled unchanged against the reference library
 * (whose src/mdcore.h the include resolves to) and against libmdcore_b200 (include/mdcore.h).
 *
 *   md_driver [runners] [steps] [particles]
 *
 * Prints one line per step: "step <time> <epot> <ekin> <temperature> <swaps> <stalls>
 * <ticks of engine_step>". */
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cycle.h"
#include "mdcore.h"

#ifndef ENGINE_FLAGS
#define ENGINE_FLAGS engine_flag_none
#endif

static int fail(const char *what, int code) {
    printf("md_driver: %s failed (%d).\n", what, code);
    errs_dump(stdout);
    return 1;
}

int main(int argc, char *argv[]) {
    const double origin[3] = {0.0, 0.0, 0.0};
    double dim[3] = {10.0, 10.0, 10.0};
    double L[3] = {1.0, 1.0, 1.0};
    const double cutoff = 1.0, mass = 39.948, kB = 0.0083144626, T_target = 100.0;
    const int runners = argc > 1 ? atoi(argv[1]) : 1;
    const int nsteps = argc > 2 ? atoi(argv[2]) : 20;
    const int nparts = argc > 3 ? atoi(argv[3]) : 32000;
    struct engine e;
    struct part p;
    struct potential *pot;
    double x[3], vsum[3] = {0.0, 0.0, 0.0};

    if (engine_init(&e, origin, dim, L, cutoff, space_periodic_full, 2, ENGINE_FLAGS) != 0)
        return fail("engine_init", engine_err);
    printf("cells %d %d %d of %.6f %.6f %.6f nm, %d tasks\n", e.s.cdim[0], e.s.cdim[1], e.s.cdim[2], e.s.h[0],
           e.s.h[1], e.s.h[2], e.s.nr_tasks);

    /* argon: 12-6 Lennard-Jones on [0.275, 1.0] nm, table tolerance 1e-3 */
    pot = potential_create_LJ126(0.275, 1.0, 9.5075e-06, 6.1545e-03, 1.0e-3);
    if (pot == NULL) return fail("potential_create_LJ126", potential_err);
    printf("table intervals %d\n", pot->n);

    memset(&p, 0, sizeof(p));
    p.type = engine_addtype(&e, mass, 0.0, "Ar", "Ar");
    if (p.type < 0) return fail("engine_addtype", engine_err);
    if (engine_addpot(&e, pot, p.type, p.type) < 0) return fail("engine_addpot", engine_err);

    /* a simple cubic arrangement filled in order, each particle moving in a random
     * direction at 0.3 nm/ps */
    srand(6178);
    p.flags = part_flag_none;
    const int side = (int)ceil(cbrt((double)nparts));
    const double h = dim[0] / side;
    for (int id = 0; id < nparts; id++) {
        const int i = id / (side * side), j = (id / side) % side, k = id % side;
        x[0] = 0.05 + i * h;
        x[1] = 0.05 + j * h;
        x[2] = 0.05 + k * h;
        double w = 0.0;
        for (int d = 0; d < 3; d++) {
            p.v[d] = (float)((double)rand() / RAND_MAX - 0.5);
            w += (double)p.v[d] * p.v[d];
        }
        w = 0.3 / sqrt(w);
        for (int d = 0; d < 3; d++) {
            p.v[d] = (float)(p.v[d] * w);
            vsum[d] += p.v[d];
        }
        p.id = id;
        p.vid = id;
        if (space_addpart(&e.s, &p, x) != 0) return fail("space_addpart", space_err);
    }
    for (int c = 0; c < e.s.nr_cells; c++)
        for (int q = 0; q < e.s.cells[c].count; q++)
            for (int d = 0; d < 3; d++) e.s.cells[c].parts[q].v[d] -= vsum[d] / nparts;
    printf("particles %d\n", e.s.nr_parts);

    e.time = 0;
    e.dt = 0.005;
    if (engine_start(&e, runners, runners) != 0) return fail("engine_start", engine_err);

    for (int step = 0; step < nsteps; step++) {
        const ticks tic = getticks();
        if (engine_step(&e) != 0) return fail("engine_step", engine_err);
        const ticks toc = getticks();
        double ekin = 0.0;
        for (int c = 0; c < e.s.nr_cells; c++)
            for (int q = 0; q < e.s.cells[c].count; q++) {
                const float *v = e.s.cells[c].parts[q].v;
                ekin += 0.5 * mass * ((double)v[0] * v[0] + (double)v[1] * v[1] + (double)v[2] * v[2]);
            }
        const double temp = ekin / (1.5 * kB * nparts);
        printf("step %d %.12e %.12e %.6f %d %d %.0f\n", e.time, e.s.epot, ekin, temp, e.s.nr_swaps, e.s.nr_stalls,
               elapsed(toc, tic));
        fflush(stdout);
        /* weak velocity rescaling towards the target temperature */
        const double w = sqrt(1.0 + 0.1 * (T_target / temp - 1.0));
        for (int c = 0; c < e.s.nr_cells; c++)
            for (int q = 0; q < e.s.cells[c].count; q++)
                for (int d = 0; d < 3; d++) e.s.cells[c].parts[q].v[d] *= w;
    }
    return 0;
}
