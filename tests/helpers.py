"""Shared test helpers: golden fixtures as workloads.System objects, error metrics."""
import os

import numpy as np

import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(fname):
    """Returns (System, dict of reference outputs) for a fixture written by make_golden.py."""
    z = np.load(os.path.join(GOLDEN, fname))
    pots = [W.PotSpec(int(r[0]), int(r[1]), int(r[2]), float(r[3]), float(r[4]), float(r[5]),
                      tuple(float(v) for v in r[6:10])) for r in z["pots"]]
    sysm = W.System(name=str(z["name"]), origin=z["origin"], dim=z["dim"], L=z["L"], cutoff=float(z["cutoff"]),
                    masses=list(z["masses"]), charges=list(z["charges"]), pots=pots, x=z["x"],
                    type=z["type"].astype(np.int32), excl=z["excl"].astype(np.int32).reshape(-1, 2),
                    dt=float(z["dt"]))
    ref = {k: z[k] for k in z.files}
    ref["tables"] = [(int(z[f"tab{k}_n"]), z[f"tab{k}_alpha"], z[f"tab{k}_c"]) for k in range(int(z["npots"]))]
    return sysm, ref


def load_bonded_golden():
    """The bonded-chains fixture: (System with bonds, angles and dihedrals; dict of the
    reference's outputs with its tables as lists of (n, alpha, coef, a, b))."""
    z = np.load(os.path.join(GOLDEN, "bonded.npz"))
    lj = z["lj"]
    bp = z["bond_pot"]
    sysm = W.System(name="bonded-golden", origin=np.zeros(3), dim=z["dim"], L=z["L"], cutoff=float(z["cutoff"]),
                    masses=list(z["mass"]), charges=[0.0] * len(z["mass"]),
                    pots=[W.PotSpec(W.KIND_LJ126, 0, 0, float(r[0]), float(r[1]), float(r[2]),
                                    tuple(float(v) for v in r[3:7])) for r in lj],
                    x=z["x"], type=z["type"].astype(np.int32), excl=z["excl"].astype(np.int32).reshape(-1, 2),
                    bonds=z["bonds"].astype(np.int32),
                    bond_pot=W.PotSpec(W.KIND_HARMONIC, 0, 0, float(bp[0]), float(bp[1]), float(bp[2]),
                                       tuple(float(v) for v in bp[3:7])),
                    angles=z["angles"].astype(np.int32),
                    angle_pots=[tuple(float(v) for v in r) for r in z["angle_pots"]],
                    dihedrals=z["dihedrals"].astype(np.int32),
                    dihedral_pots=[(float(r[0]), int(r[1]), float(r[2]), float(r[3])) for r in z["dihedral_pots"]])
    ref = {k: z[k] for k in z.files}
    for kind in ("bond", "angle", "dihedral"):
        ref[f"{kind}_tables"] = []
        k = 0
        while f"{kind}{k}_n" in z.files:
            ab = z[f"{kind}{k}_ab"]
            ref[f"{kind}_tables"].append((int(z[f"{kind}{k}_n"]), z[f"{kind}{k}_alpha"], z[f"{kind}{k}_c"],
                                          float(ab[0]), float(ab[1])))
            k += 1
    return sysm, ref


def tables_of(sysm):
    """The library's tables of a system's potentials, in oracle order (type tables, then the
    explicit electrostatic potential's, if any)."""
    import mdcore_b200 as M
    specs = list(sysm.pots) + ([sysm.ep] if getattr(sysm, "ep", None) is not None else [])
    return [M.create_potential(p).contents.table() for p in specs]


def force_errors(f, f_ref):
    """Error metrics of forces f against f_ref (both N x 3, by particle id)."""
    d = np.linalg.norm(f - f_ref, axis=1)
    fn = np.linalg.norm(f_ref, axis=1)
    frms = np.sqrt((f_ref ** 2).sum(1).mean())
    rel = d / np.maximum(fn, 1e-30)
    return dict(global_rel=float(np.linalg.norm(f - f_ref) / np.linalg.norm(f_ref)),
                max_over_frms=float(d.max() / frms), rel_max=float(rel.max()),
                rel_p99=float(np.percentile(rel, 99)), rel_median=float(np.median(rel)),
                frac_over_1e5=float((rel > 1e-5).mean()))


def sort_cells_of(ref):
    """Yields (cell id, sort mask, particle ids, keys[13, count]) of a fixture."""
    off_i = off_k = 0
    for cid, (mask, cnt) in enumerate(zip(ref["sort_mask"], ref["sort_count"])):
        ids = ref["sort_ids"][off_i:off_i + cnt]
        keys = ref["sort_keys"][off_k:off_k + 13 * cnt].reshape(13, cnt)
        off_i += cnt
        off_k += 13 * cnt
        yield cid, int(mask), ids, keys


def load_rigid_golden():
    """The rigid-water fixture: (System with positions one free step ahead, velocities and
    constraints; fixture arrays; the reference's groups as oracle input with identity
    P-SHAKE matrices)."""
    import dataclasses
    sysm, _ = load_golden("water_3000.npz")
    z = np.load(os.path.join(GOLDEN, "water_rigid.npz"))
    sysm = dataclasses.replace(sysm, x=z["x"], v=z["v"], rigid=z["rigid"], dt=float(z["dt"]))
    roff, parts, coff, con = z["roff"], z["parts"], z["coff"], z["constr"]
    groups = []
    for g in range(len(roff) - 1):
        nc = int(coff[g + 1] - coff[g])
        groups.append(([int(p) for p in parts[roff[g]:roff[g + 1]]],
                       [(int(c[0]), int(c[1]), float(c[2])) for c in con[coff[g]:coff[g + 1]]],
                       np.eye(nc, dtype=np.float32)))
    return sysm, z, groups


def rigid_oracle_steps(sysm, groups, x, v, f, pshake, nevals, time0=0, tol=1e-6):
    """nevals oracle rigid evaluations from cell-relative state (x, v, f by id); returns the
    state after each evaluation and the final matrices."""
    import oracle as O
    b = O.bin_system(sysm)
    mass = np.asarray(sysm.masses, np.float64)[sysm.type]
    out = []
    for k in range(nevals):
        x, v, f, mats, it = O.rigid(groups, x, v, f, b["cell"], b["cdim"], b["h"], mass, sysm.dt, tol, pshake,
                                    (time0 + k) < 20)
        groups = [(g[0], g[1], m) for g, m in zip(groups, mats)]
        out.append((x, v, f, np.concatenate([m.reshape(-1) for m in mats]), it))
    return out
