/* Loads a system from a PSF topology, a PDB file and a CHARMM or XPLOR parameter file
 * through the engine API (engine_read_psf, engine_read_cpf / engine_read_xplor), the way
 * the reference's JAC example does (examples/jac/jac.c: the readers, then exclusions for
 * bonds, angle ends, dihedral ends and constrained pairs), and prints what the engine
 * holds: types, bonds, constraints, angles, dihedrals, every bonded and pair table (by
 * type names), and the particles.  With a step count it then starts the engine and prints
 * the energies after each engine_step.  The same source is compiled against the reference
 * library and against libmdcore_b200; the two outputs are compared line by line.
 *
 *   topo_driver <psf> <pdb> <param> cpf|xplor <kappa> <tol> <rigidH> <switchlen>
 *               <box nm> <cutoff nm> <steps> <dt ps>
 */
#include <fcntl.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "cycle.h"
#include "mdcore.h"

#ifndef ENGINE_FLAGS
#define ENGINE_FLAGS engine_flag_none
#endif

static int fail(const char *what) {
    printf("topo_driver: %s failed (%d)\n", what, engine_err);
    errs_dump(stdout);
    return 1;
}

/* A table as its size, range, interval transform and an FNV-1a hash of the bits of its
 * coefficients (equal hashes: bit-identical tables). */
static void table(const char *tag, const struct potential *p) {
    if (p == NULL) {
        printf("%s none\n", tag);
        return;
    }
    unsigned long long h = 1469598103934665603ull;
    const unsigned char *c = (const unsigned char *)p->c;
    for (size_t k = 0; k < sizeof(float) * 8 * (size_t)(p->n + 1); k++) h = (h ^ c[k]) * 1099511628211ull;
    printf("%s n %d a %.17g b %.17g alpha %a %a %a %a c %016llx\n", tag, p->n, p->a, p->b, (double)p->alpha[0],
           (double)p->alpha[1], (double)p->alpha[2], (double)p->alpha[3], h);
}

static const char *tname(struct engine *e, int id) { return e->types[e->s.partlist[id]->type].name2; }

int main(int argc, char *argv[]) {
    if (argc < 13) {
        printf("usage: topo_driver psf pdb param cpf|xplor kappa tol rigidH switchlen box cutoff steps dt\n");
        return 2;
    }
    const double kappa = atof(argv[5]), tol = atof(argv[6]), switchlen = atof(argv[8]);
    const int rigidH = atoi(argv[7]), nsteps = atoi(argv[11]);
    const double box = atof(argv[9]), cutoff = atof(argv[10]);
    double origin[3] = {0.0, 0.0, 0.0}, dim[3] = {box, box, box}, L[3] = {cutoff, cutoff, cutoff};
    struct engine e;
    if (engine_init(&e, origin, dim, L, cutoff, space_periodic_full, 100, ENGINE_FLAGS) != 0) return fail("engine_init");
    const int psf = open(argv[1], O_RDONLY), pdb = open(argv[2], O_RDONLY), par = open(argv[3], O_RDONLY);
    if (psf < 0 || pdb < 0 || par < 0) return fail("open");
    if (engine_read_psf(&e, psf, pdb) < 0) return fail("engine_read_psf");
    if (strcmp(argv[4], "cpf") == 0) {
        if (engine_read_cpf(&e, par, kappa, tol, rigidH, switchlen) < 0) return fail("engine_read_cpf");
    } else if (engine_read_xplor(&e, par, kappa, tol, rigidH) < 0) {
        return fail("engine_read_xplor");
    }
    close(psf);
    close(pdb);
    close(par);

    for (int k = 0; k < e.nr_types; k++)
        printf("type %s %s mass %.17g charge %.17g eps %.17g rmin %.17g\n", e.types[k].name, e.types[k].name2,
               e.types[k].mass, e.types[k].charge, e.types[k].eps, e.types[k].rmin);
    for (int k = 0; k < e.nr_bonds; k++) {
        char tag[256];
        snprintf(tag, sizeof(tag), "bond %d %d %s %s", e.bonds[k].i, e.bonds[k].j, tname(&e, e.bonds[k].i),
                 tname(&e, e.bonds[k].j));
        table(tag, e.p_bond == NULL ? NULL
                                    : e.p_bond[e.s.partlist[e.bonds[k].i]->type * e.max_type +
                                               e.s.partlist[e.bonds[k].j]->type]);
    }
    for (int g = 0; g < e.nr_rigids; g++)
        for (int c = 0; c < e.rigids[g].nr_constr; c++)
            printf("constraint %d %d d2 %.17g\n", e.rigids[g].parts[e.rigids[g].constr[c].i],
                   e.rigids[g].parts[e.rigids[g].constr[c].j], e.rigids[g].constr[c].d2);
    for (int k = 0; k < e.nr_angles; k++) {
        char tag[256];
        snprintf(tag, sizeof(tag), "angle %d %d %d pid %d", e.angles[k].i, e.angles[k].j, e.angles[k].k,
                 e.angles[k].pid);
        table(tag, e.angles[k].pid >= 0 ? e.p_angle[e.angles[k].pid] : NULL);
    }
    for (int k = 0; k < e.nr_dihedrals; k++) {
        char tag[256];
        snprintf(tag, sizeof(tag), "dihedral %d %d %d %d pid %d", e.dihedrals[k].i, e.dihedrals[k].j,
                 e.dihedrals[k].k, e.dihedrals[k].l, e.dihedrals[k].pid);
        table(tag, e.dihedrals[k].pid >= 0 ? e.p_dihedral[e.dihedrals[k].pid] : NULL);
    }
    for (int j = 0; j < e.nr_types; j++)
        for (int k = j; k < e.nr_types; k++) {
            char tag[256];
            snprintf(tag, sizeof(tag), "pair %s %s", e.types[j].name2, e.types[k].name2);
            table(tag, e.p[j * e.max_type + k]);
        }
    for (int id = 0; id < e.s.nr_parts; id++) {
        const struct part *p = e.s.partlist[id];
        printf("part %d %s vid %d q %.9g x %.9g %.9g %.9g\n", id, e.types[p->type].name2, p->vid, (double)p->q,
               (double)p->x[0], (double)p->x[1], (double)p->x[2]);
    }
    if (nsteps <= 0) return 0;

    /* exclusions as examples/jac/jac.c adds them, then the steps */
    for (int k = 0; k < e.nr_bonds; k++)
        if (engine_exclusion_add(&e, e.bonds[k].i, e.bonds[k].j) < 0) return fail("engine_exclusion_add");
    for (int k = 0; k < e.nr_angles; k++)
        if (engine_exclusion_add(&e, e.angles[k].i, e.angles[k].k) < 0) return fail("engine_exclusion_add");
    for (int k = 0; k < e.nr_dihedrals; k++)
        if (engine_exclusion_add(&e, e.dihedrals[k].i, e.dihedrals[k].l) < 0) return fail("engine_exclusion_add");
    for (int g = 0; g < e.nr_rigids; g++)
        for (int c = 0; c < e.rigids[g].nr_constr; c++)
            if (engine_exclusion_add(&e, e.rigids[g].parts[e.rigids[g].constr[c].i],
                                     e.rigids[g].parts[e.rigids[g].constr[c].j]) < 0)
                return fail("engine_exclusion_add");
    if (engine_exclusion_shrink(&e) < 0) return fail("engine_exclusion_shrink");
    printf("exclusions %d\n", e.nr_exclusions);
    e.dt = atof(argv[12]);
    e.time = 0;
    if (engine_start(&e, 8, 8) != 0) return fail("engine_start");
    for (int step = 0; step < nsteps; step++) {
        if (engine_step(&e) != 0) return fail("engine_step");
        printf("energy %d epot %.12e\n", e.time, e.s.epot);
    }
    return 0;
}
