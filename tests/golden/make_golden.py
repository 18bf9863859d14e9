"""Generates the golden fixtures in this directory by running the reference mdcore CPU
library (built by oracle/Makefile.ref into oracle/_ref, single precision, no FMA
contraction) on small seeded systems.  Run from the repository root, in a container where
the reference sources are available:

    make -f oracle/Makefile.ref && python tests/golden/make_golden.py

Every fixture stores its own inputs (positions, types, exclusions, potential parameters),
so the tests never regenerate them from random streams.

Fixtures
  argon_1372.npz   jittered FCC LJ argon, 1,372 atoms, 4^3 cells, table tol 1e-4
  water_3000.npz   rigid SPC/E water, 1,000 molecules, 3^3 cells, 3,000 exclusions
  tables.npz       float tables of potential_create_* for a parameter sweep
  bonded.npz       bead chains (W.bonded_chains: 12 chains of 20 beads, bond angles 100-150
                   degrees) with harmonic bonds, angles and dihedrals: the reference's
                   bond_eval, angle_eval and dihedral_eval forces (FP32, by id) and energies,
                   each alone, the cell-relative positions and cells, and the bonded tables
  water_rigid.npz  the water_3000 system with its 3,000 distance constraints (O-H, O-H, H-H)
                   and Maxwell-Boltzmann velocities at 300 K: the reference's
                   engine_rigid_eval, P-SHAKE three times in a row (matrix refinement on)
                   and SHAKE (engine_flag_shake) once, positions/velocities/forces after
                   each call, the rigid groups and their P-SHAKE matrices
For each system: reference forces (FP32, by id), energies (total, sweep, exclusion
subtraction), the pair count of the reference sweep (one-interval counter tables),
cell assignment, cell-local float positions, the reference's sort key lists and tables.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "mdcore-history_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import workloads as W  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver_strict")


def run(sysm, tmp):
    sysf = os.path.join(tmp, "s.sys")
    outf = os.path.join(tmp, "s.out")
    W.write_sysfile(sysm, sysf)
    subprocess.run([DRIVER, "forces", sysf, outf, "4"], check=True)
    return W.read_refout(outf, sysm)


def system_fixture(sysm, fname, tmp):
    ref = run(sysm, tmp)
    cnt = run(sysm.counting(), tmp)
    # Sort keys of every cell, 13 x count, sid-major; the sort-task mask says which are set.
    masks = np.array([c[0] for c in ref["cells"]], np.int32)
    counts = np.array([len(c[1]) for c in ref["cells"]], np.int32)
    ids = np.concatenate([c[1] for c in ref["cells"]]).astype(np.int32)
    keys = np.concatenate([c[2].reshape(-1) for c in ref["cells"]]).astype(np.uint32)
    tabs = {}
    for k, (n, alpha, c) in enumerate(ref["tables"]):
        tabs[f"tab{k}_n"] = np.int32(n)
        tabs[f"tab{k}_alpha"] = alpha
        tabs[f"tab{k}_c"] = c
    pots = np.array([[p.kind, p.ti, p.tj, p.a, p.b, p.tol, *p.p] for p in sysm.pots], np.float64)
    np.savez_compressed(
        os.path.join(HERE, fname),
        name=sysm.name, x=sysm.x, type=sysm.type, excl=sysm.excl, origin=sysm.origin, dim=sysm.dim,
        L=sysm.L, cutoff=sysm.cutoff, masses=np.array(sysm.masses), charges=np.array(sysm.charges),
        pots=pots, dt=sysm.dt,
        f=ref["f"], epot=ref["epot"], epot_nonbond=ref["epot_nonbond"], epot_exclusion=ref["epot_exclusion"],
        pairs_swept=np.int64(round(cnt["epot_nonbond"])), excl_in_cut=np.int64(round(-cnt["epot_exclusion"])),
        cell=ref["cell"], xrel=ref["xrel"], sort_mask=masks, sort_count=counts, sort_ids=ids, sort_keys=keys,
        npots=len(sysm.pots), **tabs)
    print(fname, sysm.n, "pairs", cnt["epot_nonbond"], "excluded", -cnt["epot_exclusion"], "epot", ref["epot"])


# Table parameter sweep: (kind, a, b, tol, p0..p3), spanning the creators and tolerances the
# reference's examples use (examples/argon/argon.c, examples/bulk/bulk.c).
A_AR, B_AR = W.lj_AB(0.996, 0.3405)
A_W, B_W = W.lj_AB(0.650, 0.3166)
TABLE_CASES = [
    (W.KIND_LJ126, 0.25, 1.0, 1e-4, A_AR, B_AR, 0, 0),
    (W.KIND_LJ126, 0.275, 1.0, 1e-3, A_AR, B_AR, 0, 0),
    (W.KIND_LJ126, 0.3, 1.2, 1e-5, A_AR, B_AR, 0, 0),
    (W.KIND_LJ126_COULOMB, 0.25, 1.0, 1e-4, A_W, B_W, 0.8476 ** 2 * W.Q_SCALE, 0),
    (W.KIND_COULOMB, 0.05, 1.0, 1e-4, -0.8476 * 0.4238 * W.Q_SCALE, 0, 0, 0),
    (W.KIND_COULOMB, 0.1, 1.0, 1e-3, 0.4238 ** 2 * W.Q_SCALE, 0, 0, 0),
    (W.KIND_EWALD, 0.1, 1.0, 1e-3, -0.35921288, 3.0, 0, 0),
    (W.KIND_LJ126_EWALD, 0.25, 1.0, 1e-3, 2.637775819766153e-06, 2.619222661792581e-03, 7.1842576e-01, 3.0),
]


def read_rigidout(path, n):
    """Parses the output of `ref_driver rigid`."""
    raw = open(path, "rb").read()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype, count, off)
        off += a.nbytes
        return a

    N, nrig, nev = take("<i4", 3)
    assert N == n
    evals = []
    groups = None
    for _ in range(nev):
        x = take("<f4", 3 * N).reshape(N, 3)
        v = take("<f4", 3 * N).reshape(N, 3)
        f = take("<f4", 3 * N).reshape(N, 3)
        gs, mats = [], []
        for _ in range(nrig):
            np_ = int(take("<i4", 1)[0])
            parts = take("<i4", np_).copy()
            nc = int(take("<i4", 1)[0])
            con = []
            for _ in range(nc):
                i, j = take("<i4", 2)
                d2 = float(take("<f8", 1)[0])
                con.append((int(i), int(j), d2))
            mats.append(take("<f4", nc * nc).copy())
            gs.append((parts, con))
        groups = gs
        evals.append((x.copy(), v.copy(), f.copy(), np.concatenate(mats)))
    cell = take("<i4", N).copy()
    return groups, evals, cell


def rigid_fixture(tmp):
    sysm = W.with_rigid_water(W.water_spce(10), 300.0, seed=1)
    # Positions one free step ahead (x + dt v, as after the position update of a step):
    # the constraints are violated by ~dt |v| and the positions before the step
    # (x - dt v, which SHAKE reconstructs) satisfy them.
    sysm.x = W.wrap_positions(sysm.x + sysm.dt * sysm.v, sysm.dim)
    sysf = os.path.join(tmp, "w.sys")
    W.write_sysfile(sysm, sysf)
    out = {"x": sysm.x, "v": sysm.v, "rigid": sysm.rigid, "dt": sysm.dt}
    for shake, nev, tag in ((0, 3, "p"), (1, 1, "s")):
        rigf, outf = os.path.join(tmp, "w.rig"), os.path.join(tmp, "w.rout")
        W.write_rigidfile(sysm, rigf, shake=bool(shake))
        subprocess.run([DRIVER, "rigid", sysf, rigf, outf, str(nev)], check=True)
        groups, evals, cell = read_rigidout(outf, sysm.n)
        out[f"{tag}x"] = np.stack([e[0] for e in evals])
        out[f"{tag}v"] = np.stack([e[1] for e in evals])
        out[f"{tag}f"] = np.stack([e[2] for e in evals])
        out[f"{tag}a"] = np.stack([e[3] for e in evals])
        out["cell"] = cell
    out["roff"] = np.cumsum([0] + [len(g[0]) for g in groups]).astype(np.int32)
    out["parts"] = np.concatenate([g[0] for g in groups]).astype(np.int32)
    out["coff"] = np.cumsum([0] + [len(g[1]) for g in groups]).astype(np.int32)
    out["constr"] = np.array([c for g in groups for c in g[1]], np.float64)
    np.savez_compressed(os.path.join(HERE, "water_rigid.npz"), **out)
    print("rigid", len(groups), "groups; P-SHAKE x3, SHAKE x1")


def table_fixture(tmp):
    out = {}
    for k, (kind, a, b, tol, p0, p1, p2, p3) in enumerate(TABLE_CASES):
        # One-particle system carrying one potential; the driver dumps the table.
        sysm = W.System(name=f"tab{k}", origin=np.zeros(3), dim=np.full(3, 3.0), L=np.full(3, 1.0),
                        cutoff=1.0, masses=[1.0], charges=[0.0],
                        pots=[W.PotSpec(kind, 0, 0, a, b, tol, (p0, p1, p2, p3))],
                        x=np.array([[0.5, 0.5, 0.5]]), type=np.zeros(1, np.int32),
                        excl=np.zeros((0, 2), np.int32))
        ref = run(sysm, tmp)
        n, alpha, c = ref["tables"][0]
        out[f"case{k}"] = np.array([kind, a, b, tol, p0, p1, p2, p3], np.float64)
        out[f"case{k}_n"] = np.int32(n)
        out[f"case{k}_alpha"] = alpha
        out[f"case{k}_c"] = c
        print("table", k, "kind", kind, "n", n)
    np.savez_compressed(os.path.join(HERE, "tables.npz"), ncases=len(TABLE_CASES), **out)


def bonded_fixture(tmp):
    sysm = W.bonded_chains()
    sysf, bndf, outf = (os.path.join(tmp, n) for n in ("b.sys", "b.bnd", "b.out"))
    W.write_sysfile(sysm, sysf)
    W.write_bondedfile(sysm, bndf)
    subprocess.run([DRIVER, "bonded", sysf, bndf, outf], check=True)
    ref = W.read_bondedout(outf)
    out = dict(x=sysm.x, dim=sysm.dim, L=sysm.L, cutoff=np.float64(sysm.cutoff), type=sysm.type, excl=sysm.excl,
               mass=np.array(sysm.masses), lj=np.array([[p.a, p.b, p.tol, *p.p] for p in sysm.pots]),
               bonds=sysm.bonds, bond_pot=np.array([sysm.bond_pot.a, sysm.bond_pot.b, sysm.bond_pot.tol,
                                                    *sysm.bond_pot.p]),
               angles=sysm.angles, angle_pots=np.array(sysm.angle_pots, np.float64),
               dihedrals=sysm.dihedrals, dihedral_pots=np.array(sysm.dihedral_pots, np.float64))
    for key in ("f_bond", "f_angle", "f_dihedral", "xrel", "cell"):
        out[key] = ref[key]
    out["energies"] = np.array([ref["e_bond"], ref["e_angle"], ref["e_dihedral"]])
    for kind in ("bond", "angle", "dihedral"):
        for k, (n, alpha, c, a, b) in enumerate(ref[f"{kind}_tables"]):
            out[f"{kind}{k}_n"] = np.int32(n)
            out[f"{kind}{k}_alpha"] = alpha
            out[f"{kind}{k}_c"] = c
            out[f"{kind}{k}_ab"] = np.array([a, b])
    np.savez_compressed(os.path.join(HERE, "bonded.npz"), **out)
    print("bonded", sysm.n, "beads,", len(sysm.angles), "angles,", len(sysm.dihedrals), "dihedrals")


if __name__ == "__main__":
    if not os.path.exists(DRIVER):
        sys.exit("build the reference first: make -f oracle/Makefile.ref")
    with tempfile.TemporaryDirectory() as tmp:
        system_fixture(W.argon_fcc(7), "argon_1372.npz", tmp)
        system_fixture(W.water_spce(10), "water_3000.npz", tmp)
        table_fixture(tmp)
        rigid_fixture(tmp)
        bonded_fixture(tmp)
