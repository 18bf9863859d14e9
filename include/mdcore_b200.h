/*
 * mdcore_b200.h -- C ABI of the B200-native mdcore nonbonded engine.
 *
 * A driver written against the reference mdcore engine API compiles against this header
 * and links against libmdcore_b200.so instead of libmdcore_single.  Every declaration below
 * cites the reference declaration it stands in for (file:line in the mdcore sources).
 * Semantics follow the reference: functions return 0 (or a non-negative id/count) on
 * success and a negative error code on failure, after pushing an entry on the error stack
 * (errs_dump prints and clears it).
 *
 * Precision model: positions are single precision relative to their cell's origin, as in
 * the reference FPTYPE_SINGLE build.  Pair forces are computed in FP32 and accumulated on
 * the device in 64-bit fixed point (scale 2^24 per kJ/mol/nm); energies and virials are
 * accumulated in FP64.  Nonbonded forces are therefore independent of the order in which
 * cell-pair tasks run.
 *
 * Exclusions are honoured inside the pair sweep (excluded pairs are skipped) instead of
 * being subtracted afterwards as src/exclusion.c:81-295 does; the total potential energy
 * s.epot is the same quantity, s.epot_exclusion stays 0 and s.epot_nonbond already holds
 * the net nonbonded energy.
 */
#ifndef MDCORE_B200_H
#define MDCORE_B200_H

#include <stdio.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- error stack
 * Replaces src/errs.h:21-41 (errs_register / errs_dump / errs_clear). */
#define errs_maxstack 100
int errs_register(int id, const char *msg, int line, const char *func, const char *file);
int errs_dump(FILE *out);
void errs_clear(void);

/* ---------------------------------------------------------------- error codes
 * Same values as src/engine.h:22-52, src/potential.h:21-27, src/space.h:21-30. */
#define engine_err_ok          0
#define engine_err_null       -1
#define engine_err_malloc     -2
#define engine_err_space      -3
#define engine_err_pthread    -4
#define engine_err_runner     -5
#define engine_err_range      -6
#define engine_err_cell       -7
#define engine_err_domain     -8
#define engine_err_nompi      -9
#define engine_err_mpi       -10
#define engine_err_bond      -11
#define engine_err_angle     -12
#define engine_err_reader    -13
#define engine_err_psf       -14
#define engine_err_pdb       -15
#define engine_err_cpf       -16
#define engine_err_potential -17
#define engine_err_exclusion -18
#define engine_err_sets      -19
#define engine_err_dihedral  -20
#define engine_err_cuda      -21
#define engine_err_nocuda    -22
#define engine_err_cudasp    -23
#define engine_err_maxparts  -24
#define engine_err_queue     -25
#define engine_err_rigid     -26
#define engine_err_cutoff    -27
#define engine_err_nometis   -28
#define engine_err_deps      -29
#define engine_err_nyi       -30

#define potential_err_ok        0
#define potential_err_null     -1
#define potential_err_malloc   -2
#define potential_err_bounds   -3
#define potential_err_nyi      -4
#define potential_err_ivalsmax -5

#define space_err_ok        0
#define space_err_null     -1
#define space_err_malloc   -2
#define space_err_cell     -3
#define space_err_pthread  -4
#define space_err_range    -5
#define space_err_maxpairs -6
#define space_err_nrtasks  -7
#define space_err_task     -8

extern int engine_err;     /* src/engine.h:117 */
extern int potential_err;  /* src/potential.h:48 */
extern int space_err;      /* src/space.h:60 */

/* ---------------------------------------------------------------- engine flags
 * Same bits as src/engine.h:56-72.  Honoured: none, cuda, unsorted (sweep without the
 * projection cut), verlet (implied by verlet_pairwise, which verlet_pseudo implies, as in
 * src/engine.c:2458-2461: in the device-resident steps particles are re-binned and sorted
 * only when twice the largest displacement since the last rebuild exceeds the skin
 * min(h) - cutoff or it exceeds cutoff/4, src/engine.c:193-315, and the sweep bound carries
 * both cells' displacements, src/runner_dopair.c:583; engine_step and the host-buffer
 * evaluations re-sort every call), affinity (ignored), shake.  Others make engine_init fail
 * with engine_err_nyi. */
#define engine_flag_none             0
#define engine_flag_static           1
#define engine_flag_localparts       2
#define engine_flag_cuda             4
#define engine_flag_explepot         8
#define engine_flag_verlet          16
#define engine_flag_verlet_pairwise 32
#define engine_flag_affinity        64
#define engine_flag_prefetch       128
#define engine_flag_verlet_pseudo  256
#define engine_flag_unsorted       512
#define engine_flag_shake         1024
#define engine_flag_mpi           2048
#define engine_flag_parbonded     4096
#define engine_flag_async         8192
#define engine_flag_dpd          16384
#define engine_flag_nullpart     32768

/* Periodicity bits, src/space.h:33-42. */
#define space_periodic_none  0
#define space_periodic_x     1
#define space_periodic_y     2
#define space_periodic_z     4
#define space_periodic_full  7

/* ---------------------------------------------------------------- particles
 * Same 64-byte layout as struct part, src/part.h:46-69 (FPTYPE = float). */
#define part_flag_none   0
#define part_flag_frozen 1
#define part_flag_ghost  2

struct part {
    float x[4] __attribute__((aligned(16)));
    float v[4] __attribute__((aligned(16)));
    float f[4] __attribute__((aligned(16)));
    float q;
    int id, vid;
    short int type;
    unsigned short int flags;
} __attribute__((aligned(64)));

/* src/bond.h:31-36: a bond between particles i and j (ids). */
struct bond {
    int i, j;
};

/* src/angle.h:31-39: the angle i-j-k (ids, j the vertex) with angle potential pid. */
struct angle {
    int i, j, k;
    int pid;
};

/* src/dihedral.h:31-39: the dihedral i-j-k-l (ids) with dihedral potential pid. */
struct dihedral {
    int i, j, k, l;
    int pid;
};

/* src/part.h:73-88 */
struct part_type {
    int id;
    double mass, imass, charge;
    double eps, rmin;
    char name[64], name2[64];
};

/* ---------------------------------------------------------------- potentials
 * struct potential and constants as in src/potential.h:30-74: a piecewise quintic
 * interpolant on n intervals; interval 0 is a linear continuation for r < a.  The table
 * holds (n+1) chunks of 8 floats {centre, 1/halfwidth, c5, c4, c3, c2, c1, c0}. */
#define potential_degree   5
#define potential_chunk    (potential_degree + 3)
#define potential_ivalsa   1
#define potential_ivalsb   10
#define potential_N        100
#define potential_align    64
#define potential_ivalsmax 320
#define potential_escale   (0.079577471545947667882)

#define potential_flag_none    0
#define potential_flag_LJ126   1
#define potential_flag_Ewald   2
#define potential_flag_Coulomb 4

struct potential {
    float alpha[4];
    float *c;
    double a, b;
    unsigned int flags;
    int n;
};

/* Table construction, src/potential.c:963-1194 (potential_init) and the creators at
 * src/potential.c:517-914.  Tables are bit-identical to the reference single-precision
 * build compiled without FMA contraction. */
int potential_init(struct potential *p, double (*f)(double), double (*fp)(double),
                   double (*f6p)(double), float a, float b, float tol);
double potential_getalpha(double (*f6p)(double), double a, double b);
struct potential *potential_create_LJ126(double a, double b, double A, double B, double tol);
struct potential *potential_create_LJ126_switch(double a, double b, double A, double B, double s, double tol);
struct potential *potential_create_LJ126_Ewald(double a, double b, double A, double B, double q, double kappa, double tol);
struct potential *potential_create_LJ126_Coulomb(double a, double b, double A, double B, double q, double tol);
/* src/potential.c:651-676: the LJ term switched off between s and b, plus the Ewald
 * real-space term. */
struct potential *potential_create_LJ126_Ewald_switch(double a, double b, double A, double B, double q, double kappa,
                                                      double s, double tol);
struct potential *potential_create_Ewald(double a, double b, double q, double kappa, double tol);
struct potential *potential_create_Coulomb(double a, double b, double q, double tol);
/* src/potential.c:301-322: harmonic bond K (r - r0)^2 on [a, b]. */
struct potential *potential_create_harmonic(double a, double b, double K, double r0, double tol);
/* src/potential.c:448-482: harmonic angle K (theta - theta0)^2 for theta in [a, b] (held to
 * [0, pi]), tabulated over cos(theta) on [cos b, cos a]. */
struct potential *potential_create_harmonic_angle(double a, double b, double K, double theta0, double tol);
/* src/potential.c:382-411: harmonic dihedral K (1 + cos(n phi - delta)), tabulated over
 * cos(phi) on [-1, 1]. */
struct potential *potential_create_harmonic_dihedral(double K, int n, double delta, double tol);
void potential_clear(struct potential *p);
/* Scalar host evaluation, src/potential_eval.h:67-104. */
void potential_eval(struct potential *p, float r2, float *e, float *f);

/* ---------------------------------------------------------------- cells, tasks, space
 * src/cell.h:58-118, src/task.h:47-88, src/space.h:65-142 (the fields drivers read). */
struct cell {
    unsigned int flags;
    int id;
    int loc[3];
    double origin[3];
    double dim[3];
    int size, count;
    struct part *parts;
    double epot;
    unsigned int sortmask;   /* sort directions this cell's pair tasks need */
};

enum { task_type_none = 0, task_type_self, task_type_pair, task_type_sort };

struct task {
    short int type, subtype;
    int flags;               /* sort direction (sid) of a pair task */
    int i, j;                /* cell indices, already flipped as by space_getsid */
};

struct space {
    double dim[3];
    double origin[3];
    int cdim[3];
    int span[3];
    double h[3], ih[3];
    double cutoff, cutoff2;
    unsigned int period;
    int nr_cells;
    struct cell *cells;
    int nr_tasks, tasks_size;
    struct task *tasks;
    struct part **partlist;
    struct cell **celllist;
    int nr_parts, size_parts;
    int verlet_rebuild;
    float maxdx;
    double epot, epot_nonbond, epot_bond, epot_angle, epot_dihedral, epot_exclusion;
    double ekin;
    /* Queue statistics of the reference's CPU runners (src/space.h:118, reset per step by
     * space_prepare): there are no CPU runner queues here, so both stay 0. */
    int nr_swaps, nr_stalls;
    /* src/space.h:92-93: the real, ghost and marked cells by index.  There are no ghost
     * cells here (one process holds the whole space): every cell is real and marked. */
    int *cid_real, *cid_ghost, *cid_marked;
    int nr_real, nr_ghost, nr_marked;
};

/* src/space.c:530-783 and src/space.c:80-114. */
int space_init(struct space *s, const double *origin, const double *dim, double *L,
               double cutoff, unsigned int period);
int space_getsid(struct space *s, struct cell **ci, struct cell **cj, float *shift);
int space_addpart(struct space *s, struct part *p, double *x);
/* src/space.c:307-364 (space_shuffle_local): every particle that left its cell moves to
 * the cell it is now in (periodic wrap), partlist/celllist relinked (host threads). */
int space_shuffle(struct space *s);
/* src/space.c:186-219: swap/stall counters and energies reset, cell energies and particle
 * forces zeroed. */
int space_prepare(struct space *s);
/* src/space.c:447-466: global position of particle id (cell origin + relative position);
 * space_err_range for an id past nr_parts. */
int space_getpos(struct space *s, int id, double *x);

/* ---------------------------------------------------------------- exclusions, rigids
 * src/exclusion.h:34-41 and src/rigid.h:31-52. */
struct exclusion { int i, j; };
/* Rigid groups, src/rigid.h:27-59 (same fields in the same order): up to rigid_maxparts
 * particles (by id) and rigid_maxconstr distance constraints between group-local indices
 * i, j with squared length d2; a is the P-SHAKE constraint mixing matrix (identity when a
 * constraint is added, refined on the device during the first engine_pshake_steps steps
 * and whenever a group needs more than rigid_pshake_refine iterations). */
#define rigid_maxparts        10
#define rigid_maxconstr       (3 * rigid_maxparts)
#define rigid_maxiter         100
#define rigid_pshake_refine   10
#define rigid_pshake_maxalpha 0.1f
#define engine_pshake_steps   20
struct rigid {
    int nr_parts;
    int parts[rigid_maxparts];
    int nr_constr;
    struct { int i, j; double d2; } constr[rigid_maxconstr];
    float a[rigid_maxconstr * rigid_maxconstr];
};

/* ---------------------------------------------------------------- the engine
 * Field-compatible prefix of struct engine, src/engine.h:169-302: drivers may read and
 * write flags, s, time, dt, max_type, nr_types, types, p, nr_exclusions, tol_rigid. */
struct nb_stats {
    int64_t pairs;          /* unordered pairs with r2 <= rc^2, potential set, not excluded */
    int64_t excluded;       /* excluded pairs that would otherwise have been counted */
    int64_t candidates;     /* pairs examined by the sorted sweep (inside the projection cut) */
    double epot;            /* FP64 nonbonded energy of the last force evaluation */
    double virial;          /* FP64 sum over pairs of r_ij . F_ij */
    int status;             /* device status word of the last launch (0 = ok) */
    float ms_kernels;       /* device time of the last force evaluation (CUDA events) */
    float ms_pack;          /* host: packing the cells into the staging buffers */
    float ms_device;        /* host wall time from the first copy to the last copy's completion */
    float ms_unpack;        /* host: adding the forces into the cells */
};

/* src/engine.h:92-112: the phases engine_step times, in CPU ticks (cycle.h getticks).
 * Here: step = the whole engine_step; cuda_load / cuda_dopairs / cuda_unload = packing and
 * upload, the device step with its copies, rebuilding the cells; nonbond, advance and rigid
 * are parts of the device step and stay 0; the others belong to paths not built here. */
enum {
    engine_timer_step = 0,
    engine_timer_prepare,
    engine_timer_verlet,
    engine_timer_exchange1,
    engine_timer_nonbond,
    engine_timer_bonded,
    engine_timer_bonded_sort,
    engine_timer_bonds,
    engine_timer_angles,
    engine_timer_dihedrals,
    engine_timer_exclusions,
    engine_timer_advance,
    engine_timer_rigid,
    engine_timer_exchange2,
    engine_timer_shuffle,
    engine_timer_cuda_load,
    engine_timer_cuda_unload,
    engine_timer_cuda_dopairs,
    engine_timer_last
};

struct engine {
    unsigned int flags;
    struct space s;
    int time;
    double dt;
    int max_type;
    int nr_types;
    struct part_type *types;
    struct potential **p;
    struct exclusion *exclusions;
    int nr_exclusions, exclusions_size;
    struct rigid *rigids;
    int *part2rigid;
    int nr_rigids, rigids_size, nr_constr;
    double tol_rigid;
    int nr_runners;
    int device;
    void *cuda;             /* device state, owned by the engine */
    struct nb_stats stats;
    void *cuda_rigid;       /* device state of the rigid groups, owned by the engine */
    int part2rigid_size;    /* entries of part2rigid */
    int rigids_gen;         /* bumped by every engine_rigid_add */
    struct potential *ep;   /* explicit electrostatics (engine_setexplepot), or NULL */
    struct bond *bonds;     /* engine_bond_add */
    int nr_bonds, bonds_size;
    struct potential **p_bond;   /* max_type x max_type bond potentials (engine_bond_addpot) */
    int bonds_gen;          /* bumped by every change of the bonds, angles or dihedrals */
    struct angle *angles;   /* engine_angle_add */
    int nr_angles, angles_size, nr_anglepots, anglepots_size;
    struct potential **p_angle;      /* angle potentials by index (engine_angle_addpot) */
    struct dihedral *dihedrals;      /* engine_dihedral_add */
    int nr_dihedrals, dihedrals_size, nr_dihedralpots, dihedralpots_size;
    struct potential **p_dihedral;   /* dihedral potentials by index (engine_dihedral_addpot) */
    unsigned long long timers[engine_timer_last];   /* src/engine.h:293, CPU ticks per phase */
};

/* src/engine.c:2439-2591 */
int engine_init(struct engine *e, const double *origin, const double *dim, double *L,
                double cutoff, unsigned int period, int max_type, unsigned int flags);
/* src/engine.c:1543-1567 */
int engine_addtype(struct engine *e, double mass, double charge, char *name, char *name2);
/* src/engine.c:1584-1600 */
int engine_addpot(struct engine *e, struct potential *p, int i, int j);
/* src/engine.c:1345-1392 */
int engine_load(struct engine *e, double *x, double *v, int *type, int *pid, int *vid,
                double *q, unsigned int *flags, int N);
/* src/engine.c:1076-1145 */
int engine_unload(struct engine *e, double *x, double *v, int *type, int *pid, int *vid,
                  double *q, unsigned int *flags, double *epot, int N);
/* src/engine_bonded.c:1400-1440 and :1301-1390 */
int engine_exclusion_add(struct engine *e, int i, int j);
int engine_exclusion_shrink(struct engine *e);
/* Type lookups by name and by name2 (src/engine.c:1473-1530): the index of the first type
 * with that name, engine_err_range when there is none. */
int engine_gettype(struct engine *e, char *name);
int engine_gettype2(struct engine *e, char *name2);
/* Topology and parameter readers (src/engine_io.c): engine_read_psf adds the atoms of a
 * PSF file (one type per atom type and charge, named type + charge string in name2), its
 * bonds, angles, dihedrals and impropers (angles and dihedrals without a potential yet:
 * pid -1, impropers -2), and places them at the positions of the PDB file's ATOM records
 * (Angstrom, wrapped into the box); engine_read_cpf (CHARMM) and engine_read_xplor (XPLOR)
 * read a parameter file and add the bond, angle, dihedral and improper potentials of the
 * matching terms, rigid constraints for bonds over a type whose name starts with 'H'
 * (rigidH), and a pair table for every type pair with parameters: kappa < 0 LJ (with the
 * switch at switchlen for CHARMM), kappa = 0 LJ + shifted Coulomb, kappa > 0 LJ + Ewald
 * real space (switched LJ for CHARMM).  Files are given as open descriptors and read to
 * their end. */
int engine_read_psf(struct engine *e, int psf, int pdb);
int engine_read_cpf(struct engine *e, int cpf, double kappa, double tol, int rigidH, double switchlen);
int engine_read_xplor(struct engine *e, int xplor, double kappa, double tol, int rigidH);
/* src/engine_rigid.c:78-229 */
int engine_rigid_add(struct engine *e, int pid, int pjd, double d);
/* src/engine.c:1029-1053.  Sets the explicit electrostatic potential (engine_flag_explepot)
 * or clears it (ep = NULL).  The reference stores ep but no runner reads it; here every
 * pair within the cutoff that is not excluded also interacts through q_i q_j ep(r) with the
 * particles' charges (engine_load's q), in addition to its type pair's potential, if any:
 * a pair whose types have no potential still interacts through ep.  ep is normally
 * potential_create_Coulomb(a, b, 1, tol) (prefactor 1/(4 pi) as the reference's tables),
 * so that q in units of e * sqrt(4 pi * 138.935458) gives kJ/mol.  Call before
 * engine_start. */
int engine_setexplepot(struct engine *e, struct potential *ep);
/* src/engine_bonded.c:2086-2102: the bond potential of type pair (i, j) (symmetric). */
int engine_bond_addpot(struct engine *e, struct potential *p, int i, int j);
/* src/engine_bonded.c:1447-1475: a bond between particles i and j.  Bonds are evaluated
 * as bond_eval does (src/bond.c:81-250: the potential of the two particles' types, the
 * distance from the cell-relative positions and the cells' periodic offset, r^2 held to
 * the table's range [a^2, b^2]) by engine_step (the device step) and the device-resident
 * steps, into the same fixed-point forces as the nonbonded sweep; their energy goes to
 * e->s.epot_bond.  engine_step_host returns engine_err_nyi for an engine with bonds. */
int engine_bond_add(struct engine *e, int i, int j);
/* Extension: the potential energies of the last step or force evaluation, out[6] = e->s.epot,
 * epot_nonbond, epot_bond, epot_angle, epot_dihedral, epot_exclusion (engine_unload's epot
 * sums the cells' nonbonded energies only, as the reference's does). */
int engine_energies(struct engine *e, double *out);
/* src/engine_bonded.c:2151-2177: adds an angle potential; returns its index. */
int engine_angle_addpot(struct engine *e, struct potential *p);
/* src/engine_bonded.c:1258-1290: the angle i-j-k with angle potential pid.  Evaluated as
 * angle_eval does (src/angle.c:81-300: positions relative to j's cell, the cells' periodic
 * offsets held to -1..1, cos(theta) held to [-1, 1] and then to the table's range, the
 * table read at cos(theta), force = -dE/dcos * dcos/dx) on the device by engine_step and
 * the device-resident steps; energy to e->s.epot_angle. */
int engine_angle_add(struct engine *e, int i, int j, int k, int pid);
/* src/engine_bonded.c:2114-2140: adds a dihedral potential; returns its index. */
int engine_dihedral_addpot(struct engine *e, struct potential *p);
/* src/engine_bonded.c:1210-1243: the dihedral i-j-k-l with dihedral potential pid.
 * Evaluated as dihedral_eval does (src/dihedral.c:81-380: cos(phi) of the planes i-j-k and
 * j-k-l, held to [-1, 1] and then to the table's range) on the device by engine_step and
 * the device-resident steps; energy to e->s.epot_dihedral.  engine_step_host returns
 * engine_err_nyi for an engine with angles or dihedrals. */
int engine_dihedral_add(struct engine *e, int i, int j, int k, int l, int pid);
/* src/engine.c:1674-1826 */
int engine_start(struct engine *e, int nr_runners, int nr_queues);
/* src/engine.c:2070-2240.  One time step (re-binning, forces, symplectic Euler, rigid
 * constraints) run on the device with the host cells as input and output: the particles
 * go up, one device-resident step runs (engine_cuda_resident_*), particles (in the
 * device's cell order), forces, energies and statistics come back. */
int engine_step(struct engine *e);
/* engine_step with re-binning and integration on the host threads and the force evaluation
 * (engine_nonbond_cuda_fresh) and the constraints (engine_rigid_eval) through host buffers.
 * Same positions, velocities and energies as engine_step, bit for bit. */
int engine_step_host(struct engine *e);
/* The device part of engine_step (no error stack entry of its own). */
int engine_cuda_step(struct engine *e);
/* src/engine.c:1945-2052 */
int engine_advance(struct engine *e);
/* src/engine.c:2338-2430 */
int engine_finalize(struct engine *e);
/* src/engine.c:167-183: all of e->timers back to 0. */
int engine_timers_reset(struct engine *e);

/* ---------------------------------------------------------------- GPU entry points
 * The two functions src/engine.c calls when engine_flag_cuda is set, plus the device
 * selection and particle load/unload helpers of src/runner_cuda.cu / src/engine_cuda.cu. */
/* src/runner_cuda.cu:2931-3545: upload tables, cell geometry, task list. */
int engine_cuda_load(struct engine *e);
/* src/runner_cuda.cu:2287-2628: one nonbonded force evaluation; packs the cells' particles,
 * copies them to the device, sorts, sweeps, and copies forces and energy back into
 * the cells (f += nonbonded force; cell epot and s.epot_nonbond updated). */
int engine_nonbond_cuda(struct engine *e);
/* src/runner_cuda.cu:2641-2825 */
int engine_cuda_load_parts(struct engine *e);
int engine_cuda_unload_parts(struct engine *e);
/* src/engine_cuda.cu:109-167 */
int engine_cuda_setdevice(struct engine *e, int id);
int engine_cuda_setdevices(struct engine *e, int nr_devices, int *ids);

/* ---------------------------------------------------------------- extensions
 * No counterpart in the reference. */

/* sizeof(struct engine), for foreign-function callers that allocate it themselves. */
size_t engine_sizeof(void);
/* Forces by particle id (N x 3 doubles), as accumulated by the last step. */
int engine_getforces(struct engine *e, double *f, int N);
/* Cell index of each particle by id. */
int engine_getcells(struct engine *e, int *cell, int N);
/* Counters and FP64 sums of the last nonbonded evaluation. */
int engine_nonbond_stats(struct engine *e, struct nb_stats *out);
/* The sorted key lists the device built in the last evaluation for cell cid
 * (13 x count entries, sid-major, same key format as src/runner_dosort.c:148-149). */
int engine_cuda_getsort(struct engine *e, int cid, unsigned int *keys, int size);
/* Device-resident force evaluation: positions already on the device (uploaded by
 * engine_cuda_load_parts), forces left on the device.  Used to time the kernels alone. */
int engine_nonbond_cuda_resident(struct engine *e);
/* Sets the time step (the field e->dt of a C driver). */
int engine_set_dt(struct engine *e, double dt);
/* Zeroes forces and energies ahead of a stand-alone engine_nonbond_cuda call. */
int engine_zero_forces(struct engine *e);
/* engine_zero_forces + engine_nonbond_cuda in one pass over the particles: the cells'
 * forces and energies become those of this evaluation (engine_step uses it). */
int engine_nonbond_cuda_fresh(struct engine *e);
/* Makes later launches use this cudaStream_t (e.g. the caller framework's stream). */
int engine_cuda_setstream(struct engine *e, void *stream);
/* Device time (ms) of the last evaluation: its launches from the first to the last (the
 * zeroing, sort and sweep; after resident steps the whole last step), and the sweep kernel
 * alone.  Events recorded on the launch stream, inside the CUDA graph when one is replayed,
 * so host launch latency is not counted. */
int engine_cuda_kernel_times(struct engine *e, float *total_ms, float *sweep_ms);
/* Measured FP32 FMA throughput of a device in TFLOP/s (a register-only FMA loop). */
int engine_cuda_fp32_peak(int device, float *tflops);
/* Allocation-free force evaluation.  No counterpart in the reference.  For callers that
 * cannot allocate device memory when they need forces (a fixed, pre-reserved device
 * budget; code between set-up and a stream capture): sort + persistent sweep on
 * caller-provided device buffers, with the only scratch (sort keys, queue head, a
 * layout-error word) in a static device array of at most 65,536 particle slots, shared by
 * all calls; calls that overlap on the GPU race on it.  The first call on a device looks
 * up that array's address and should come before any stream capture.  Inputs use the
 * device layout of engine_cuda_load_parts (cell-major slots, cell starts multiples of 4):
 * xq = float4 {x, y, z cell-local, type bits} and pid, both 16-byte aligned;
 * cstart[ncells], ccount[ncells]; maxcount = the largest cell count (a larger cell is
 * skipped and reported as status bit 2).  A cell whose start is not a multiple of 4 or
 * whose 4-rounded block leaves [0, nslots) makes the call do nothing but set status bit
 * 128.  Outputs (zeroed by the call, 8-byte aligned): force[3*nslots] int64 fixed point
 * 2^24/(kJ/mol/nm), cell_epot[ncells] int64 2^32/(kJ/mol), acc[8] {unused, virial*2^32
 * (negated), pairs, excluded, candidates, status}.  stream may be NULL (engine stream).
 * Tables, tasks and exclusions come from engine_cuda_load.  The call leaves the launch
 * state of the engine's own evaluations (grids, graphs) alone and restores the caller's
 * current device. */
int engine_nonbond_cuda_noalloc(struct engine *e, const void *xq, const int *pid, const int *cstart,
                                const int *ccount, int nslots, int maxcount, unsigned long long *force,
                                unsigned long long *cell_epot, unsigned long long *acc, void *stream);
/* ---- learned task-cost scheduler (no counterpart in the reference) ----
 * A small MLP (NB_MLP_IN -> 32 -> 32 -> 1) predicts each task's cost from the two cells'
 * particle counts, the fraction of i particles within the sort-axis reach of cell j, the
 * type mix and the neighbour class; it is trained on the GPU on clock64 task durations the
 * sweep records, and orders the device queue longest-first.  Forces do not depend on the
 * order (fixed-point accumulation). */
#define NB_MLP_IN 10
#define NB_MLP_HIDDEN 32
#define NB_MLP_NPARAM (NB_MLP_HIDDEN * NB_MLP_IN + NB_MLP_HIDDEN + NB_MLP_HIDDEN * NB_MLP_HIDDEN + \
                       NB_MLP_HIDDEN + NB_MLP_HIDDEN + 1)
/* Device kernels on caller buffers (X: n x NB_MLP_IN floats; weights: NB_MLP_NPARAM bf16). */
int nb_mlp_predict(const float *X, int n, const void *w_bf16, float *out, void *stream);
int nb_mlp_grad(const float *X, const float *target, const int *idx, int n, const void *w_bf16,
                float *grad, float *loss, void *stream);
int nb_mlp_adam(float *w_master, void *w_bf16, const float *grad, float *m, float *v, float lr,
                float beta1, float beta2, float eps, int step, void *stream);
int nb_mlp_round(const float *w_master, void *w_bf16, void *stream);
/* Engine-level use: record per-task durations over nsteps device-resident MD steps (when
 * engine_cuda_resident_begin holds the particles; the trajectory advances) or else nsteps
 * force evaluations of the uploaded particles, compute features (of the last step's
 * particles and keys), train, and apply an order (use_mlp = 0 restores the count-product
 * heuristic order; 1 = longest predicted first).  engine_sched_order orders with locality:
 * tiles of `tile` consecutive tasks of the cell-major task list (0: an automatic size of
 * about an eighth of the tasks per worker warp) in decreasing class of their summed cost
 * (source 0: count-product weights, 1: the network's predictions; a class per factor
 * 2^(1/4)), tiles of one class in cell-major order, each tile's tasks longest first. */
int engine_sched_record(struct engine *e, int nsteps);
int engine_sched_features(struct engine *e, float *features_out, int n);
int engine_sched_targets(struct engine *e, float *targets_out, int n);
int engine_sched_train(struct engine *e, int epochs, int batch, float lr, unsigned seed, float *loss_out);
int engine_sched_predict(struct engine *e, float *pred_out, int n);
int engine_sched_apply(struct engine *e, int use_mlp);
int engine_sched_order(struct engine *e, int source, int tile);
/* The current queue order (n = the task count). */
int engine_cuda_getorder(struct engine *e, int *order, int n);
/* Sweep kernel launch parameters: warps per block (0 = default) and plain = 1 for the
 * plain form (one block per task, IEEE sqrt/div) instead of the persistent queue. */
int engine_cuda_settune(struct engine *e, int warps, int plain);
/* Replaces the device task-queue order (a permutation of 0..ntasks-1). */
int engine_cuda_setorder(struct engine *e, const int *order, int n);
/* Per-task clock64 records of the persistent sweep: enable/disable, and read the last
 * launch's (start, end) pairs and SM ids when clocks/sms are non-NULL. */
int engine_cuda_taskclocks(struct engine *e, int enable, long long *clocks, int *sms, int n);
/* Number of device tasks (self + pair). */
int engine_cuda_ntasks(struct engine *e);

/* ---- rigid constraints on the device ----
 * src/engine_rigid.c:352-583: resolves every rigid group after the position update of a
 * step, SHAKE (src/rigid.c:81-277) when engine_flag_shake is set, P-SHAKE
 * (src/rigid.c:279-523) otherwise; engine_step calls it when the engine has rigid groups.
 * The iterations run on the GPU in FP64, one thread per group; positions, velocities (and
 * for P-SHAKE the constraint forces) of the cells are corrected as in the reference.  The
 * P-SHAKE matrices live on the device once the first evaluation has uploaded them. */
int engine_rigid_eval(struct engine *e);
/* src/engine_rigid.c:266-345: splits the groups for MPI ranks; a single process holds all
 * of them, so it only checks its argument. */
int engine_rigid_sort(struct engine *e);
/* src/engine_rigid.c:231-250: the groups in a random order (rand()); the device copy is
 * rebuilt at the next step and the results do not depend on the order. */
int engine_rigid_unsort(struct engine *e);
/* Largest iteration count of any group in the last engine_rigid_eval and the number of
 * groups that did not converge within rigid_maxiter iterations. */
int engine_rigid_stats(struct engine *e, int *max_iter, int *unconverged);
/* Copies the device's P-SHAKE matrices back into e->rigids[].a. */
int engine_rigid_getmatrices(struct engine *e);
/* Copies rigid group g into *out; returns the number of groups (out may be NULL). */
int engine_rigid_get(struct engine *e, int g, struct rigid *out);
/* Particle state by id: cell-relative float positions, velocities and forces (3 floats
 * each) and cell index; any pointer may be NULL. */
int engine_getparts(struct engine *e, float *x, float *v, float *f, int *cell, int N);
/* Sweep steps each lane holds before the warp reduce-scatter of the persistent sweep: 4
 * (default) or 8 (used at 640 threads per SM).  Same pair set. */
int engine_cuda_setwindow(struct engine *e, int window);
/* CUDA-graph replay of each evaluation's launches (zeroing, sort, queue compaction,
 * sweep): enable = 1 captures the launches on the second evaluation of a launch
 * configuration and replays the graph from then on; a new configuration (other slot
 * count, largest cell, buffers, launch shape) is captured anew. */
int engine_cuda_graph(struct engine *e, int enable);
/* Persistent sweep shape: lane layout 0 = one i particle per lane (32 per warp, the
 * default), 1 = a tile of 8 i particles x 4 j columns per warp; stages = 1 or 2 staging
 * buffers per worker warp (2: the next task's bulk copies land while the warp sweeps the
 * current one; not with occupancy 768); occupancy = resident threads per SM the kernel's
 * registers are sized for: 640 (96 registers, the default), 768 (80) or 1024 (64).  Same
 * pair set. */
int engine_cuda_setlayout(struct engine *e, int layout, int stages, int occupancy);
/* Times every persistent launch shape (2, 4, 8 worker warps per block x lane layout x
 * staging buffers x occupancy, window 4) on the resident particles (uploaded first if none
 * are) and keeps the fastest; returns the chosen shape and its median device time (sort +
 * sweep).  Results stay resident. */
int engine_cuda_autotune(struct engine *e, int reps, int *warps, int *layout, int *stages, int *occupancy,
                         float *ms);

/* ---- device-resident time steps (replace engine_step, src/engine.c:2070-2240, while
 * the particles stay on the device) ----
 * engine_cuda_resident_begin uploads every particle into fixed blocks of slots per cell
 * (the largest cell plus `margin` spare slots, rounded up to 4; margin < 0: 8).  engine_cuda_resident_steps runs nsteps time steps of
 * engine_step -- space_shuffle, the nonbonded forces, engine_advance, the rigid
 * constraints -- as device launches only (with engine_cuda_graph, one CUDA graph per
 * step); e->time advances, the host's particles do not.  A step in which a cell outgrows
 * its block (or more than 16 particles, doubled on each such event, leave one cell) is
 * aborted on the device together with the steps after it; the call then re-blocks the
 * particles of the last completed step with twice the spare room and runs the remaining
 * steps, at most 8 times per call, and returns engine_err_maxparts only when a cell
 * would exceed 1,024 particles (the device then still holds the last completed step).
 * engine_cuda_resident_sync rebuilds the host cells (the device's particles in the
 * device's order: positions, velocities, the last step's forces before the constraint
 * corrections; zero before the first resident step), cell and engine energies, stats and
 * the rigid iteration statistics; engine_cuda_resident_end syncs and frees the blocks.
 * Host and device re-binning keep the same particle order, so the trajectories are
 * engine_step's bit for bit, and engine_step may carry on after a sync. */
int engine_cuda_resident_begin(struct engine *e, int margin);
int engine_cuda_resident_steps(struct engine *e, int nsteps);
int engine_cuda_resident_sync(struct engine *e);
int engine_cuda_resident_end(struct engine *e);
/* Slots per cell, leavers per cell and step, completed resident steps, the accepted pairs
 * summed over them, and automatic re-blockings since engine_cuda_resident_begin; any
 * pointer may be NULL. */
int engine_cuda_resident_info(struct engine *e, int *capc, int *mcap, long long *steps, long long *pairs,
                              int *regrows);
/* Energy minimisation, no counterpart in the reference (its drivers start from relaxed or
 * lattice systems): with gamma > 0 the resident steps move every particle by gamma f,
 * held to at most dmax nm, and zero its velocity (steepest descent; the rigid constraints
 * still apply); gamma <= 0 restores the time step. */
int engine_cuda_minimize(struct engine *e, double gamma, double dmax);
/* Per-step energy log of the resident steps, no counterpart in the reference (its drivers
 * sum energies on the host every step): engine_cuda_energylog keeps a ring of the last
 * `cap` steps' records (0: off; setting it clears the log, and so does
 * engine_cuda_resident_begin); engine_cuda_energylog_read copies up to max records in step
 * order: out[4 k + 0..3] = resident step number (1 = the first step after
 * engine_cuda_resident_begin), potential energy (nonbonded + bonded), kinetic energy
 * sum m v^2 / 2 of the velocities after the step (FP64 sums in fixed point), and their sum,
 * in kJ/mol.  Returns the number of records.  The records sum over every engine of a
 * batch. */
int engine_cuda_energylog(struct engine *e, int cap);
int engine_cuda_energylog_read(struct engine *e, double *out, int max);
/* Force accumulation of the plain form (engine_cuda_settune(e, 0, 1)): 1 = FP32, each
 * task's partial forces added as floats with float atomics (order-dependent, the way of
 * the reference's GPU runner, src/runner_cuda.cu); 0 = 64-bit fixed point (the default,
 * order-independent).  The persistent sweeps always accumulate in fixed point. */
int engine_cuda_setaccum(struct engine *e, int fp32);
/* The failure path of the device waits, no counterpart in the reference: every wait of a
 * sweep on its staging copies (an mbarrier) polls at most `polls` times (<= 0: the default,
 * 2^22), after which the kernel records a copy timeout, waits once more for copies in
 * flight and returns; the evaluation then fails with engine_err_cuda and "Bulk copy into
 * shared memory timed out." in the error stack, and the device stays usable.
 * engine_cuda_copytimeout_test(e, 1) makes every such wait run out (nothing arrives on the
 * barriers and no copy is issued, so nothing is in flight), for testing that path; 0 turns
 * it off.
 * Both settings hold for every engine on the engine's device. */
int engine_cuda_setspin(struct engine *e, int polls);
/* With engine_flag_verlet: the rebuilds (re-binning and sort) the resident steps did since
 * the particles were uploaded; -1 without the flag or resident particles. */
int engine_cuda_verlet_rebuilds(struct engine *e, int *rebuilds);
int engine_cuda_copytimeout_test(struct engine *e, int enable);

/* ---- batches of engines (no counterpart in the reference) ----
 * One device state for many independent engines (replicas: the same potentials, cutoff
 * and flags; their own particles, boxes and cell sizes).  Each evaluation sorts every
 * engine's cells in one launch and sweeps the concatenated task list with one persistent
 * launch; forces, per-cell energies, energies and virials go back to each engine (its
 * cells and stats; pair counts of each engine's stats are -1), totals to
 * engine_batch_stats.  The engines keep their host data and must outlive the batch; they
 * need no device state of their own (engine_start is not required). */
struct engine_batch;
int engine_batch_create(struct engine **engines, int n, struct engine_batch **out);
int engine_batch_free(struct engine_batch *b);
/* engine_nonbond_cuda for every engine: upload, sort + sweep, download. */
int engine_batch_nonbond(struct engine_batch *b);
/* engine_nonbond_cuda_fresh for every engine. */
int engine_batch_nonbond_fresh(struct engine_batch *b);
/* engine_step for every engine: one device step of the whole batch, the engines' host
 * cells as input and output.  Large batches step in groups of engines (contiguous runs of
 * about equal particle counts, each with its own device blocks and stream) so that the
 * host packing and unpacking of one group overlap the device work of the others; the
 * result of every engine is the same as in one group. */
int engine_batch_step(struct engine_batch *b);
/* Groups of engine_batch_step: 0 = automatic (one per 2^18 particles, at most 4), else 1 to
 * 64 (never more than the engines).  A batch holding resident particles
 * (engine_batch_resident_begin) steps as one group. */
int engine_batch_setgroups(struct engine_batch *b, int groups);
/* engine_sched_order for a batch, from the count-product costs (each engine's tasks are
 * consecutive, so a tile stays inside one engine's box); tile = 0: automatic. */
int engine_batch_sched_order(struct engine_batch *b, int tile);
/* engine_step_host for every engine with the forces of one batch evaluation. */
int engine_batch_step_host(struct engine_batch *b);
int engine_batch_load_parts(struct engine_batch *b);
int engine_batch_resident(struct engine_batch *b);
int engine_batch_unload_parts(struct engine_batch *b);
int engine_batch_stats(struct engine_batch *b, struct nb_stats *out);
/* engine_zero_forces for every engine of the batch. */
int engine_batch_zero_forces(struct engine_batch *b);
int engine_batch_setstream(struct engine_batch *b, void *stream);
int engine_batch_kernel_times(struct engine_batch *b, float *total_ms, float *sweep_ms);
int engine_batch_settune(struct engine_batch *b, int warps, int plain);
int engine_batch_graph(struct engine_batch *b, int enable);
int engine_batch_autotune(struct engine_batch *b, int reps, int *warps, int *layout, int *stages, int *occupancy,
                          float *ms);
int engine_batch_setlayout(struct engine_batch *b, int layout, int stages, int occupancy);
int engine_batch_ntasks(struct engine_batch *b);
/* Device-resident steps of every engine of the batch (engine_cuda_resident_*): one
 * re-binning, sort, sweep, integration and constraint launch sequence for all engines. */
int engine_batch_resident_begin(struct engine_batch *b, int margin);
int engine_batch_resident_steps(struct engine_batch *b, int nsteps);
int engine_batch_resident_sync(struct engine_batch *b);
int engine_batch_resident_end(struct engine_batch *b);
int engine_batch_resident_info(struct engine_batch *b, int *capc, int *mcap, long long *steps, long long *pairs,
                               int *regrows);

#ifdef __cplusplus
}
#endif

#endif
