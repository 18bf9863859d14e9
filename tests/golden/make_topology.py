"""Writes the synthetic topology fixtures under tests/golden/topo/ and, when the reference
CPU build (oracle/_ref) is present, the reference's view of them.

The system (seeded): three chains of five alanine-like residues (N, HN, CA, HA, CB, HB1-3,
C, O with CHARMM-style types NH1, H, CT1, HB, CT3, HA, C, O) in ~700 three-site waters
(OT, HT) in a 3.0 nm box.  Its files: small.psf (atoms, bonds, angles from every pair of
bonds sharing an atom, dihedrals from every bonded path of four, two impropers per inner
residue), small.pdb (Angstrom), small.cpf (a CHARMM parameter file: BONDS with H bonds
that rigidH turns into constraints, ANGLES with Urey-Bradley columns, DIHEDRALS with X
wildcards and a repeated type quadruple whose first line must win, IMPROPER with
wildcards, NONBONDED with 1-4 columns and two types of equal parameters and charge, lines
for types the system does not have) and small.xplor (the same parameters in XPLOR form).

With the reference build, tests/drivers/topo_driver.c compiled against it
(oracle/_ref/topo_driver_ref) loads the files through the reference's engine_read_psf and
engine_read_cpf / engine_read_xplor for each case in CASES and its output is stored
gzipped as tests/golden/topo/ref_<case>.txt.gz: types, bonds, constraints, angles,
dihedrals, table hashes, particles and, for the cases with steps, the energies of
engine_step.

    python tests/golden/make_topology.py
"""
import gzip
import math
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "topo")
ROOT = os.path.dirname(os.path.dirname(HERE))
BOX_NM = 3.0
CUTOFF = 0.9

# (case name, parameter file, format, kappa, tol, rigidH, switchlen, steps, dt)
CASES = [
    ("cpf_ewald", "small.cpf", "cpf", 3.0, 1e-4, 1, 0.7, 2, 0.001),
    ("cpf_lj", "small.cpf", "cpf", -1.0, 1e-4, 0, 0.7, 0, 0.001),
    ("cpf_coulomb", "small.cpf", "cpf", 0.0, 1e-4, 1, 0.7, 0, 0.001),
    ("xplor_ewald", "small.xplor", "xplor", 3.0, 1e-4, 1, 0.0, 2, 0.001),
    ("xplor_lj", "small.xplor", "xplor", -1.0, 1e-4, 0, 0.0, 0, 0.001),
]

# the driver's output lines (the reference also prints warnings, which are not kept)
TAGS = ("type", "bond", "constraint", "angle", "dihedral", "pair", "part", "exclusions", "energy")

MASS = {"NH1": 14.007, "H": 1.008, "CT1": 12.011, "HB": 1.008, "CT3": 12.011, "HA": 1.008, "C": 12.011,
        "O": 15.999, "OT": 15.9994, "HT": 1.008}
# residue atoms: name, type, charge, bonded-to (earlier atom of the residue)
RESIDUE = [("N", "NH1", -0.47, None), ("HN", "H", 0.31, "N"), ("CA", "CT1", 0.07, "N"), ("HA", "HB", 0.09, "CA"),
           ("CB", "CT3", -0.27, "CA"), ("HB1", "HA", 0.09, "CB"), ("HB2", "HA", 0.09, "CB"),
           ("HB3", "HA", 0.09, "CB"), ("C", "C", 0.51, "CA"), ("O", "O", -0.51, "C")]
BONDLEN = {frozenset(("NH1", "H")): 0.997, frozenset(("NH1", "CT1")): 1.43, frozenset(("CT1", "HB")): 1.08,
           frozenset(("CT1", "CT3")): 1.538, frozenset(("CT3", "HA")): 1.111, frozenset(("CT1", "C")): 1.49,
           frozenset(("C", "O")): 1.23, frozenset(("C", "NH1")): 1.345}


def build(seed=0, nchains=3, nres=5, nwater=700):
    rng = np.random.default_rng(seed)
    atoms, bonds = [], []           # atoms: (segment, resid, resname, name, type, charge, mass)
    pos = []
    for ch in range(nchains):
        start = rng.uniform(5.0, 25.0, 3)
        direction = rng.normal(size=3)
        direction /= np.linalg.norm(direction)
        prev_c = None
        for r in range(nres):
            idx = {}
            for name, typ, q, parent in RESIDUE:
                k = len(atoms)
                idx[name] = k
                # charges of the first residue's CA and CB differ: the same atom type with two
                # charges gives two engine types
                qq = q + (0.14 if (r == 0 and name in ("CA", "CB")) else 0.0)
                atoms.append((f"P{ch + 1}", r + 1 + ch * nres, "ALA", name, typ, qq, MASS[typ]))
                if parent is None:
                    if prev_c is None:
                        p = start
                    else:
                        p = pos[prev_c] + direction * 1.345
                    if prev_c is not None:
                        bonds.append((prev_c, k))
                else:
                    pk = idx[parent]
                    d = rng.normal(size=3)
                    d /= np.linalg.norm(d)
                    if name in ("CA", "C"):
                        d = 0.7 * direction + 0.3 * d
                        d /= np.linalg.norm(d)
                    p = pos[pk] + d * BONDLEN[frozenset((typ, atoms[pk][4]))]
                    bonds.append((pk, k))
                pos.append(np.array(p, dtype=float))
            prev_c = idx["C"]
            direction = direction + 0.3 * rng.normal(size=3)
            direction /= np.linalg.norm(direction)
    nsolute = len(atoms)
    # waters on a jittered grid away from the solute
    n = int(math.ceil((nwater * 4) ** (1 / 3)))
    grid = (np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3) + 0.5) * (BOX_NM * 10 / n)
    grid = grid[rng.permutation(len(grid))]
    solute = np.array(pos)
    placed = 0
    hh = 0.9572 * math.sin(math.radians(104.52) / 2)
    hz = 0.9572 * math.cos(math.radians(104.52) / 2)
    for site in grid:
        if placed == nwater:
            break
        d = solute - site
        d -= np.round(d / (BOX_NM * 10)) * BOX_NM * 10
        if np.min(np.linalg.norm(d, axis=1)) < 3.0:
            continue
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        o = site + rng.normal(0, 0.05, 3)
        h1 = o + q @ np.array([hh, 0, hz])
        h2 = o + q @ np.array([-hh, 0, hz])
        res = 100 + placed
        k = len(atoms)
        for name, typ, qq, p in (("OH2", "OT", -0.834, o), ("H1", "HT", 0.417, h1), ("H2", "HT", 0.417, h2)):
            atoms.append(("W", res, "TIP3", name, typ, qq, MASS[typ]))
            pos.append(p)
        bonds += [(k, k + 1), (k, k + 2), (k + 1, k + 2)]
        placed += 1
    pos = np.array(pos) % (BOX_NM * 10)
    # angles: every pair of bonds sharing an atom (waters: the H-O-H angle only)
    nbr = [[] for _ in atoms]
    for i, j in bonds:
        nbr[i].append(j)
        nbr[j].append(i)
    angles = []
    for j in range(len(atoms)):
        nb = sorted(nbr[j])
        for a in range(len(nb)):
            for b in range(a + 1, len(nb)):
                if atoms[j][4] == "HT":
                    continue
                angles.append((nb[a], j, nb[b]))
    dihedrals = []
    for j, k in bonds:
        if j >= nsolute:
            continue
        for i in nbr[j]:
            for l in nbr[k]:
                if i != k and l != j and i != l:
                    dihedrals.append((i, j, k, l))
    impropers = []
    for r in range(1, nchains * nres):
        if (r % nres) == 0:
            continue
        base = r * len(RESIDUE)
        n_, hn, ca, c, o = base + 0, base + 1, base + 2, base + 8, base + 9
        prev_c = base - len(RESIDUE) + 8
        impropers.append((n_, hn, ca, prev_c))          # NH1 H CT1 C
        impropers.append((o, c, ca, n_ - len(RESIDUE)))  # O C CT1 NH1 (the previous residue's N)
    return atoms, pos, bonds, angles, dihedrals, impropers


def write_psf(path, atoms, bonds, angles, dihedrals, impropers):
    with open(path, "w") as f:
        f.write("PSF\n\n       1 !NTITLE\n REMARKS synthetic alanine chains in water\n\n")
        f.write(f"{len(atoms):8d} !NATOM\n")
        for k, (seg, resid, resname, name, typ, q, m) in enumerate(atoms):
            f.write(f"{k + 1:8d} {seg:<4s} {resid:<4d} {resname:<4s} {name:<4s} {typ:<4s} {q:10.6f} {m:13.4f}"
                    f"           0\n")

        def block(items, tag, per):
            f.write(f"\n{len(items):8d} !{tag}\n")
            flat = [v + 1 for it in items for v in it]
            width = len(items[0]) if items else 1
            for s in range(0, len(flat), per * width):
                f.write("".join(f"{v:8d}" for v in flat[s:s + per * width]) + "\n")

        block(bonds, "NBOND: bonds", 4)
        block(angles, "NTHETA: angles", 3)
        block(dihedrals, "NPHI: dihedrals", 2)
        block(impropers, "NIMPHI: impropers", 2)
        f.write("\n       0 !NDON: donors\n\n")


def write_pdb(path, atoms, pos):
    with open(path, "w") as f:
        f.write("REMARK synthetic alanine chains in water\n")
        for k, ((seg, resid, resname, name, typ, q, m), x) in enumerate(zip(atoms, pos)):
            f.write(f"ATOM {k + 1:6d} {name:<4s} {resname:<4s} {resid:5d} {x[0]:9.3f} {x[1]:9.3f} {x[2]:9.3f}"
                    f"  1.00  0.00      {seg}\n")
        f.write("END\n")


BOND_PARAMS = [("NH1", "H", 440.0, 0.997), ("NH1", "CT1", 320.0, 1.430), ("CT1", "HB", 330.0, 1.080),
               ("CT1", "CT3", 222.5, 1.538), ("CT3", "HA", 322.0, 1.111), ("CT1", "C", 250.0, 1.490),
               ("C", "O", 620.0, 1.230), ("C", "NH1", 370.0, 1.345), ("OT", "HT", 450.0, 0.9572),
               ("HT", "HT", 0.0, 1.5139), ("CT2", "CT2", 222.5, 1.530)]
ANGLE_PARAMS = [("H", "NH1", "CT1", 35.0, 117.0, None), ("H", "NH1", "C", 34.0, 123.0, None),
                ("NH1", "CT1", "HB", 48.0, 108.0, None), ("NH1", "CT1", "CT3", 70.0, 113.5, None),
                ("NH1", "CT1", "C", 50.0, 107.0, None), ("HB", "CT1", "CT3", 35.0, 111.0, None),
                ("HB", "CT1", "C", 50.0, 109.5, None), ("CT3", "CT1", "C", 52.0, 108.0, None),
                ("CT1", "CT3", "HA", 33.43, 110.1, (22.53, 2.179)), ("HA", "CT3", "HA", 35.5, 108.4, (5.40, 1.802)),
                ("CT1", "C", "O", 80.0, 121.0, None), ("CT1", "C", "NH1", 80.0, 116.5, None),
                ("O", "C", "NH1", 80.0, 122.5, None), ("C", "NH1", "CT1", 50.0, 120.0, None),
                ("HT", "OT", "HT", 55.0, 104.52, None), ("CT2", "CT2", "CT2", 58.35, 113.6, (11.16, 2.561))]
DIHEDRAL_PARAMS = [("H", "NH1", "CT1", "C", 0.10, 1, 0.0),        # a repeated quadruple: the first line wins
                   ("H", "NH1", "CT1", "C", 0.20, 2, 180.0),
                   ("X", "CT1", "CT3", "X", 0.20, 3, 0.0), ("X", "CT1", "NH1", "X", 0.25, 1, 180.0),
                   ("X", "C", "NH1", "X", 2.50, 2, 180.0), ("X", "CT1", "C", "X", 0.05, 6, 180.0),
                   ("O", "C", "NH1", "H", 2.50, 2, 180.0), ("X", "CT2", "CT2", "X", 0.19, 3, 0.0)]
IMPROPER_PARAMS = [("NH1", "X", "X", "C", 20.0, 0.0), ("O", "X", "X", "NH1", 120.0, 0.0)]
NONBONDED = [("C", 0.0, -0.110, 2.000, None), ("CT1", 0.0, -0.020, 2.275, (0.0, -0.01, 1.9)),
             ("CT3", 0.0, -0.080, 2.060, (0.0, -0.01, 1.9)), ("H", 0.0, -0.046, 0.2245, None),
             ("HA", 0.0, -0.022, 1.320, None), ("HB", 0.0, -0.022, 1.320, None),
             ("NH1", 0.0, -0.200, 1.850, (0.0, -0.20, 1.55)), ("O", 0.0, -0.120, 1.700, (0.0, -0.12, 1.40)),
             ("OT", 0.0, -0.1521, 1.7682, None), ("HT", 0.0, -0.046, 0.2245, None),
             ("CT2", 0.0, -0.055, 2.175, (0.0, -0.01, 1.9))]


def write_cpf(path):
    with open(path, "w") as f:
        f.write("* synthetic CHARMM-style parameters for the alanine-chain test system\n*\n\n! comment line\n")
        f.write("BONDS\n!V(bond) = Kb(b - b0)**2\n")
        for a, b, K, r0 in BOND_PARAMS:
            f.write(f"{a:<6s}{b:<6s}{K:10.3f}{r0:10.4f} ! {a}-{b}\n")
        f.write("\nANGLES\n")
        for a, b, c, K, t0, ub in ANGLE_PARAMS:
            f.write(f"{a:<6s}{b:<6s}{c:<6s}{K:9.3f}{t0:10.2f}" + (f"{ub[0]:9.2f}{ub[1]:9.3f}" if ub else "") + "\n")
        f.write("\nDIHEDRALS\n")
        for a, b, c, d, K, n, dl in DIHEDRAL_PARAMS:
            f.write(f"{a:<6s}{b:<6s}{c:<6s}{d:<6s}{K:9.4f}{n:3d}{dl:9.2f}\n")
        f.write("\nIMPROPER\n")
        for a, b, c, d, K, p0 in IMPROPER_PARAMS:
            f.write(f"{a:<6s}{b:<6s}{c:<6s}{d:<6s}{K:9.4f}{0:3d}{p0:9.2f}\n")
        f.write("\nNONBONDED nbxmod 5 atom cdiel shift vatom vdistance vswitch cutnb 14.0 ctofnb 12.0\n"
                "!atom  ignored  epsilon  Rmin/2\n")
        for t, ign, eps, rm, x14 in NONBONDED:
            f.write(f"{t:<6s}{ign:6.1f}{eps:10.4f}{rm:10.4f}" +
                    (f"{x14[0]:8.2f}{x14[1]:8.3f}{x14[2]:8.3f}" if x14 else "") + "\n")
        f.write("\nHBOND CUTHB 0.5\n\nEND\n")


def write_xplor(path):
    with open(path, "w") as f:
        f.write("remark synthetic XPLOR-style parameters { braces start a comment }\n\n")
        for a, b, K, r0 in BOND_PARAMS:
            f.write(f"BOND {a:<5s} {b:<5s} {K:9.3f} {r0:8.4f}\n")
        for a, b, c, K, t0, ub in ANGLE_PARAMS:
            f.write(f"ANGLe {a:<5s} {b:<5s} {c:<5s} {K:8.3f} {t0:8.2f}\n")
        for a, b, c, d, K, n, dl in DIHEDRAL_PARAMS:
            f.write(f"DIHEdral {a:<5s} {b:<5s} {c:<5s} {d:<5s} {K:8.4f} {n:2d} {dl:8.2f}\n")
        for a, b, c, d, K, p0 in IMPROPER_PARAMS:
            f.write(f"IMPRoper {a:<5s} {b:<5s} {c:<5s} {d:<5s} {K:8.4f} 0 {p0:8.2f}\n")
        for t, ign, eps, rm, x14 in NONBONDED:
            # XPLOR gives epsilon and sigma; the reader takes Rmin = sigma / 2 per type
            f.write(f"NONBonded {t:<5s} {eps:9.4f} {2 * rm:9.4f} ! sigma\n")
        f.write("\nend\n")


def main():
    os.makedirs(OUT, exist_ok=True)
    atoms, pos, bonds, angles, dihedrals, impropers = build()
    write_psf(os.path.join(OUT, "small.psf"), atoms, bonds, angles, dihedrals, impropers)
    write_pdb(os.path.join(OUT, "small.pdb"), atoms, pos)
    write_cpf(os.path.join(OUT, "small.cpf"))
    write_xplor(os.path.join(OUT, "small.xplor"))
    print(f"{len(atoms)} atoms, {len(bonds)} bonds, {len(angles)} angles, {len(dihedrals)} dihedrals, "
          f"{len(impropers)} impropers")
    exe = os.path.join(ROOT, "oracle", "_ref", "topo_driver_ref")
    if not os.path.exists(exe):
        print("reference build absent: no reference outputs written")
        return
    for name, par, fmt, kappa, tol, rigid, sw, steps, dt in CASES:
        args = [exe, os.path.join(OUT, "small.psf"), os.path.join(OUT, "small.pdb"), os.path.join(OUT, par), fmt,
                repr(kappa), repr(tol), str(rigid), repr(sw), repr(BOX_NM), repr(CUTOFF), str(steps), repr(dt)]
        r = subprocess.run(args, capture_output=True, text=True, env=dict(os.environ, OMP_NUM_THREADS="8"))
        if r.returncode != 0:
            print(r.stdout[-3000:], r.stderr[-3000:])
            sys.exit(f"reference driver failed on {name}")
        lines = [l for l in r.stdout.splitlines() if l.split(" ", 1)[0] in TAGS]
        with gzip.open(os.path.join(OUT, f"ref_{name}.txt.gz"), "wt") as f:
            f.write("\n".join(lines) + "\n")
        print(name, len(lines), "lines")


if __name__ == "__main__":
    main()
