"""Seeded synthetic workloads of the shapes the mdcore nonbonded path is measured on.

Each generator returns a ``System``: box, cutoff, particle types, per-type-pair potential
specifications (arguments of the reference's ``potential_create_*`` calls,
src/potential.c:517-914), positions in id order and exclusion pairs.  The same ``System``
drives this package's engine (``mdcore_b200.Engine.from_system``) and, serialised with
``write_sysfile``, the reference CPU driver used as oracle and baseline.

No public benchmark data is involved: these generators are the benchmark inputs.

Units: nm, kJ/mol, amu, ps.  The reference's Coulomb prefactor is 1/(4 pi)
(src/potential.h:40), so charges products are passed as q_i q_j * 4 pi * 138.935458
to obtain kJ/mol.
"""
from __future__ import annotations

import dataclasses
import math
import struct
from typing import List, Optional

import numpy as np

COULOMB_K = 138.935458                     # kJ mol^-1 nm e^-2
Q_SCALE = 4.0 * math.pi * COULOMB_K        # undoes potential_escale = 1/(4 pi)

# Potential kinds shared with oracle/sysfile.h.
KIND_LJ126, KIND_LJ126_COULOMB, KIND_COULOMB, KIND_EWALD, KIND_LJ126_EWALD, KIND_COUNTER = 1, 2, 3, 4, 5, 6
KIND_HARMONIC = 7                            # p = (K, r0): K (r - r0)^2


@dataclasses.dataclass
class PotSpec:
    kind: int
    ti: int
    tj: int
    a: float
    b: float
    tol: float
    p: tuple = (0.0, 0.0, 0.0, 0.0)


@dataclasses.dataclass
class System:
    name: str
    origin: np.ndarray            # (3,)
    dim: np.ndarray               # (3,)
    L: np.ndarray                 # (3,) requested cell edge
    cutoff: float
    masses: List[float]
    charges: List[float]
    pots: List[PotSpec]
    x: np.ndarray                 # (N,3) float64, inside [origin, origin+dim)
    type: np.ndarray              # (N,) int32
    excl: np.ndarray              # (M,2) int32
    dt: float = 0.002
    flags: int = 0
    period: int = 7
    v: Optional[np.ndarray] = None          # (N,3) velocities, nm/ps (None: at rest)
    rigid: Optional[np.ndarray] = None      # (M,3) rigid constraints: id i, id j, length d (nm)
    q: Optional[np.ndarray] = None          # (N,) per-particle charges (explicit electrostatics)
    ep: Optional[PotSpec] = None            # explicit electrostatic potential (engine_setexplepot)
    bonds: Optional[np.ndarray] = None      # (M,2) bonded particle ids
    bond_pot: Optional[PotSpec] = None      # the bond potential of every bonded type pair
    angles: Optional[np.ndarray] = None     # (M,4) ids i, j (vertex), k and angle potential index
    angle_pots: Optional[list] = None       # (a, b, K, theta0, tol) of potential_create_harmonic_angle
    dihedrals: Optional[np.ndarray] = None  # (M,5) ids i, j, k, l and dihedral potential index
    dihedral_pots: Optional[list] = None    # (K, n, delta, tol) of potential_create_harmonic_dihedral

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    def counting(self) -> "System":
        """Copy whose potentials are all pair counters (energy 1 per accepted pair)."""
        pots = [PotSpec(KIND_COUNTER, p.ti, p.tj, 0.0, 1.0, 1.0) for p in self.pots]
        return dataclasses.replace(self, pots=pots, name=self.name + "-count")


def lj_AB(eps: float, sigma: float):
    """A = 4 eps sigma^12, B = 4 eps sigma^6 for U = A/r^12 - B/r^6."""
    return 4.0 * eps * sigma ** 12, 4.0 * eps * sigma ** 6


def _wrap(x: np.ndarray, dim: np.ndarray) -> np.ndarray:
    x = np.mod(x, dim)
    # np.mod can return dim itself for tiny negative inputs; keep strictly inside.
    hi = np.nextafter(dim, 0.0)
    return np.minimum(x, hi)


def wrap_positions(x: np.ndarray, dim: np.ndarray) -> np.ndarray:
    """Positions wrapped into the periodic box [0, dim)."""
    return _wrap(np.asarray(x, np.float64), np.asarray(dim, np.float64))


def argon_fcc(ncell: int = 20, seed: int = 0, density: float = 21.0, jitter: float = 0.01,
              tol: float = 1e-4, cutoff: float = 1.0) -> System:
    """Plain LJ argon: 4*ncell^3 atoms on a jittered FCC lattice at `density` atoms/nm^3.

    ncell=20 gives the 32,000-atom system in an 11.5074 nm box (11^3 cells)."""
    n = 4 * ncell ** 3
    L = (n / density) ** (1.0 / 3.0)
    a = L / ncell
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]], dtype=np.float64)
    g = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell), indexing="ij"), -1)
    g = g.reshape(-1, 1, 3).astype(np.float64)
    x = ((g + basis[None, :, :]) * a + 0.25 * a).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    x = x + rng.normal(0.0, jitter, size=x.shape)
    dim = np.full(3, L)
    x = _wrap(x, dim)
    A, B = lj_AB(0.996, 0.3405)
    return System(
        name=f"argon-fcc-{n}", origin=np.zeros(3), dim=dim, L=np.full(3, cutoff), cutoff=cutoff,
        masses=[39.948], charges=[0.0],
        pots=[PotSpec(KIND_LJ126, 0, 0, 0.25, cutoff, tol, (A, B, 0.0, 0.0))],
        x=x, type=np.zeros(n, np.int32), excl=np.zeros((0, 2), np.int32), dt=0.005)


def _random_rotations(rng, m: int) -> np.ndarray:
    """m uniformly distributed rotation matrices (random unit quaternions)."""
    q = rng.normal(size=(m, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((m, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z); R[:, 0, 1] = 2 * (x * y - z * w); R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w); R[:, 1, 1] = 1 - 2 * (x * x + z * z); R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w); R[:, 2, 1] = 2 * (y * z + x * w); R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def water_spce(nside: int = 32, seed: int = 0, density: float = 33.4, jitter: float = 0.01,
               tol: float = 1e-4, cutoff: float = 1.0, coul_a: float = 0.05) -> System:
    """Rigid SPC/E water: nside^3 molecules on a jittered cubic grid, random orientations.

    nside=32 gives 32,768 molecules (98,304 atoms) in a 9.9365 nm box (9^3 cells).
    Particle ids are 3k (O), 3k+1, 3k+2 (H); the three intramolecular pairs are excluded.
    O-O: LJ (sigma 0.3166, eps 0.650) + shifted Coulomb; O-H, H-H: shifted Coulomb.

    The O-H and H-H tables start at coul_a = 0.05 nm, below the 0.1 nm O-H bond: the
    reference's table continuation below r = a drops the degree-5 term of the first
    interval (src/potential.c:1167-1185), so its tables jump by |c5| at r = a, and a bond
    sitting exactly at a lands on either side depending on how r^2 was rounded."""
    nmol = nside ** 3
    L = (nmol / density) ** (1.0 / 3.0)
    gsp = L / nside
    g = np.stack(np.meshgrid(np.arange(nside), np.arange(nside), np.arange(nside), indexing="ij"), -1)
    o = (g.reshape(-1, 3).astype(np.float64) + 0.5) * gsp
    rng = np.random.default_rng(seed)
    o = o + rng.normal(0.0, jitter, size=o.shape)
    theta = math.radians(109.47)
    d = 0.1
    local = np.array([[d, 0.0, 0.0], [d * math.cos(theta), d * math.sin(theta), 0.0]])
    R = _random_rotations(rng, nmol)
    h = o[:, None, :] + np.einsum("mij,hj->mhi", R, local)
    x = np.concatenate([o[:, None, :], h], axis=1).reshape(-1, 3)
    dim = np.full(3, L)
    x = _wrap(x, dim)
    typ = np.tile(np.array([0, 1, 1], np.int32), nmol)
    k = np.arange(nmol, dtype=np.int32) * 3
    excl = np.stack([np.stack([k, k + 1], 1), np.stack([k, k + 2], 1), np.stack([k + 1, k + 2], 1)], 1)
    excl = excl.reshape(-1, 2).astype(np.int32)
    qO, qH = -0.8476, 0.4238
    A, B = lj_AB(0.650, 0.3166)
    pots = [
        PotSpec(KIND_LJ126_COULOMB, 0, 0, 0.25, cutoff, tol, (A, B, qO * qO * Q_SCALE, 0.0)),
        PotSpec(KIND_COULOMB, 0, 1, coul_a, cutoff, tol, (qO * qH * Q_SCALE, 0.0, 0.0, 0.0)),
        PotSpec(KIND_COULOMB, 1, 1, coul_a, cutoff, tol, (qH * qH * Q_SCALE, 0.0, 0.0, 0.0)),
    ]
    return System(
        name=f"water-spce-{3 * nmol}", origin=np.zeros(3), dim=dim, L=np.full(3, cutoff), cutoff=cutoff,
        masses=[15.9994, 1.00794], charges=[qO, qH], pots=pots, x=x, type=typ, excl=excl, dt=0.002)


KB = 0.0083144626                         # kJ mol^-1 K^-1


def maxwell_velocities(sysm: System, temperature: float, seed: int = 1) -> np.ndarray:
    """Velocities (nm/ps) drawn from the Maxwell-Boltzmann distribution at `temperature`
    for every particle's mass, net momentum removed."""
    rng = np.random.default_rng(seed)
    m = np.asarray(sysm.masses, np.float64)[sysm.type]
    v = rng.normal(size=(sysm.n, 3)) * np.sqrt(KB * temperature / m)[:, None]
    v -= (m[:, None] * v).sum(0) / m.sum()
    return v


def with_rigid_water(sysm: System, temperature: float = 300.0, seed: int = 1) -> System:
    """The SPC/E system with its three distance constraints per molecule (O-H 0.1 nm twice,
    H-H 0.163298 nm, the geometry examples/bulk/bulk.c:308-310 holds with SHAKE), added in
    the order O-H1, O-H2, H1-H2, and Maxwell-Boltzmann velocities."""
    nmol = sysm.n // 3
    k = np.arange(nmol) * 3
    hh = 2.0 * 0.1 * math.sin(math.radians(109.47) / 2.0)
    rig = np.stack([np.stack([k, k + 1, np.full(nmol, 0.1)], 1), np.stack([k, k + 2, np.full(nmol, 0.1)], 1),
                    np.stack([k + 1, k + 2, np.full(nmol, hh)], 1)], 1).reshape(-1, 3)
    return dataclasses.replace(sysm, rigid=rig, v=maxwell_velocities(sysm, temperature, seed),
                               name=sysm.name + "-rigid")


def write_rigidfile(sysm: System, path: str, shake: bool) -> None:
    """Velocities and rigid constraints for the reference driver's rigid mode."""
    rig = np.zeros((0, 3)) if sysm.rigid is None else np.asarray(sysm.rigid)
    v = np.zeros((sysm.n, 3)) if sysm.v is None else np.asarray(sysm.v, np.float64)
    with open(path, "wb") as f:
        f.write(b"MDB2RIG1")
        f.write(struct.pack("<iii", len(rig), int(shake), 0))
        f.write(struct.pack("<d", sysm.dt))
        f.write(np.ascontiguousarray(v, "<f8").tobytes())
        for i, j, d in rig:
            f.write(struct.pack("<iid", int(i), int(j), float(d)))


def lb_mix(eps_i, sig_i, eps_j, sig_j):
    """Lorentz-Berthelot: sigma arithmetic mean, epsilon geometric mean."""
    return math.sqrt(eps_i * eps_j), 0.5 * (sig_i + sig_j)


def lj_slab(nx: int = 110, nz: int = 77, n_total: int = 1 << 20, seed: int = 0, box=(40.0, 40.0, 160.0),
            slab: float = 28.07, jitter: float = 0.02, frac_a: float = 0.8, tol: float = 1e-4,
            cutoff: float = 1.0) -> System:
    """Inhomogeneous LJ slab: a liquid slab of thickness `slab` at the box centre along z
    (jittered simple-cubic lattice, nx*nx*nz sites, ~21 atoms/nm^3 for the defaults) and a
    uniform vapour filling the rest of the box with the remaining n_total - nx*nx*nz atoms
    (~0.55 atoms/nm^3).  Two types mixed 80/20 at random (sigma 0.3405/0.30 nm,
    eps 0.996/0.80 kJ/mol, Lorentz-Berthelot cross term).  Defaults: 2^20 atoms in a
    40 x 40 x 160 nm box, 40 x 40 x 160 cells."""
    rng = np.random.default_rng(seed)
    Lx, Ly, Lz = box
    dx, dy, dz = Lx / nx, Ly / nx, slab / nz
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(nx), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    z0 = 0.5 * (Lz - slab)
    liq = (g + 0.5) * np.array([dx, dy, dz]) + np.array([0.0, 0.0, z0])
    liq = liq + rng.normal(0.0, jitter, size=liq.shape)
    nv = n_total - len(liq)
    vz = rng.uniform(0.0, Lz - slab, size=nv)
    vz = np.where(vz < z0, vz, vz + slab)
    vap = np.stack([rng.uniform(0.0, Lx, nv), rng.uniform(0.0, Ly, nv), vz], 1)
    x = np.concatenate([liq, vap])
    dim = np.array(box, dtype=np.float64)
    x = _wrap(x, dim)
    typ = (rng.uniform(size=n_total) >= frac_a).astype(np.int32)
    eps, sig = (0.996, 0.80), (0.3405, 0.30)
    pots = []
    for i in range(2):
        for j in range(i, 2):
            e_ij, s_ij = lb_mix(eps[i], sig[i], eps[j], sig[j])
            pots.append(PotSpec(KIND_LJ126, i, j, 0.25, cutoff, tol, (*lj_AB(e_ij, s_ij), 0.0, 0.0)))
    return System(name=f"lj-slab-{n_total}", origin=np.zeros(3), dim=dim, L=np.full(3, cutoff), cutoff=cutoff,
                  masses=[39.948, 39.948], charges=[0.0, 0.0], pots=pots, x=x, type=typ,
                  excl=np.zeros((0, 2), np.int32), dt=0.005)


def argon_replicas(nrep: int = 512, seed: int = 0, nmin: int = 500, nmax: int = 8000, rho=(18.0, 24.0),
                   jitter: float = 0.01, tol: float = 1e-4, cutoff: float = 1.0) -> List[System]:
    """An ensemble of independent LJ argon replicas of different sizes and densities, the
    workload of a replica batch: N log-uniform in [nmin, nmax], density uniform in `rho`
    atoms/nm^3, cubic box of edge (N/density)^(1/3) (drawn again if below three cutoffs),
    atoms on a random subset of a simple-cubic lattice, jittered.  Every replica carries
    the same LJ potential (argon, table from 0.25 nm to the cutoff)."""
    rng = np.random.default_rng(seed)
    A, B = lj_AB(0.996, 0.3405)
    out = []
    while len(out) < nrep:
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        dens = rng.uniform(*rho)
        L = (n / dens) ** (1.0 / 3.0)
        if L < 3.0 * cutoff:
            continue
        m = int(math.ceil(n ** (1.0 / 3.0)))
        sites = rng.choice(m ** 3, size=n, replace=False)
        g = np.stack(np.unravel_index(sites, (m, m, m)), 1).astype(np.float64)
        x = (g + 0.5) * (L / m) + rng.normal(0.0, jitter, size=(n, 3))
        dim = np.full(3, L)
        out.append(System(
            name=f"argon-replica-{len(out)}-{n}", origin=np.zeros(3), dim=dim, L=np.full(3, cutoff), cutoff=cutoff,
            masses=[39.948], charges=[0.0], pots=[PotSpec(KIND_LJ126, 0, 0, 0.25, cutoff, tol, (A, B, 0.0, 0.0))],
            x=_wrap(x, dim), type=np.zeros(n, np.int32), excl=np.zeros((0, 2), np.int32), dt=0.005))
    return out


def write_sysfile(sysm: System, path: str) -> None:
    """Serialise in the format of oracle/sysfile.h."""
    with open(path, "wb") as f:
        f.write(b"MDB2SYS1")
        f.write(struct.pack("<6i", sysm.n, len(sysm.masses), len(sysm.pots), len(sysm.excl),
                            sysm.flags, sysm.period))
        f.write(np.concatenate([sysm.origin, sysm.dim, sysm.L, [sysm.cutoff]]).astype("<f8").tobytes())
        for m, q in zip(sysm.masses, sysm.charges):
            f.write(struct.pack("<2d", m, q))
        for p in sysm.pots:
            f.write(struct.pack("<4i7d", p.kind, p.ti, p.tj, 0, p.a, p.b, p.tol, *p.p))
        f.write(np.ascontiguousarray(sysm.x, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(sysm.type, dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(sysm.excl, dtype="<i4").tobytes())


def read_refout(path: str, sysm: System):
    """Parse the output of `ref_driver forces` (oracle/ref_driver.c)."""
    buf = open(path, "rb").read()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(buf, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a

    N, npots, ncells, nexcl = take("<i4", 4)
    epot, epot_nb, epot_ex = take("<f8", 3)
    f = take("<f8", 3 * N).reshape(N, 3)
    xr = take("<f4", 3 * N).reshape(N, 3)
    cell = take("<i4", N)
    cells = []
    for _ in range(ncells):
        cnt, flags = take("<i4", 2)
        ids = take("<i4", cnt)
        keys = take("<u4", 13 * cnt).reshape(13, cnt)
        cells.append((int(flags), ids.copy(), keys.copy()))
    tables = []
    for _ in range(npots):
        (n,) = take("<i4", 1)
        alpha = take("<f4", 4)
        c = take("<f4", (n + 1) * 8)
        tables.append((int(n), alpha.copy(), c.copy()))
    return dict(N=int(N), nexcl=int(nexcl), epot=float(epot), epot_nonbond=float(epot_nb),
                epot_exclusion=float(epot_ex), f=f.copy(), xrel=xr.copy(), cell=cell.copy(),
                cells=cells, tables=tables)


QSCALE = math.sqrt(Q_SCALE)     # e -> per-particle charge unit of tables with prefactor 1/(4 pi)


def chains_water(nchains: int = 220, length: int = 100, nwater: int = 23400, box=(10.8, 10.8, 7.8), seed: int = 0,
                 cutoff: float = 1.2, tol: float = 1e-4, bond: float = 0.15, gap: float = 0.12,
                 bond_k: float = 2.0e5, clearance: float = 0.25, angles_dihedrals: bool = True,
                 h_sigma: float = 0.2) -> System:
    """Heterogeneous solvated-chain system: `nchains` linear bead chains of `length` beads
    (bond 0.15 nm, 20 LJ bead types with sigma U[0.25, 0.40] nm and epsilon U[0.1, 1.0]
    kJ/mol, Lorentz-Berthelot mixing, charges N(0, 0.3) e neutralised per chain) and up to
    `nwater` 3-site water molecules in the SPC/E geometry (O -0.8476 e, H +0.4238 e, O-O LJ
    sigma 0.3166 nm, epsilon 0.650, the three intramolecular distances constrained) on a
    jittered grid at 33.4 molecules/nm^3, waters whose oxygen is closer than `gap` to a bead
    left out (0.12 nm: the 23,400 waters of the named system fit; the close contacts this
    leaves make the unrelaxed system unfit for dynamics, 0.25 nm gives a calmer one).  Charges act through explicit electrostatics (ep: the shifted Coulomb table
    with unit charge, cutoff 1.2 nm); the type tables are LJ only (H: sigma h_sigma, epsilon 0.1).  1-2 and 1-3
    exclusions along the chains, the three intramolecular pairs of every water excluded;
    chain bonds harmonic, bond_k (r - 0.15 nm)^2 (bond_pot, a table on [0.05, 0.3] nm).
    With `angles_dihedrals`, every three consecutive beads also form a harmonic angle
    (CHAINS_ANGLE_POTS, one of two at random) and every four a dihedral (CHAINS_DIHEDRAL_POTS,
    one of three at random, drawn after everything else so the positions do not depend on it).
    Types: 0 O, 1 H, 2..21 beads.  Seeded.

    Chains grow together as self-avoiding random walks (every new bead at least `clearance`
    from the beads placed before it other than its two predecessors, bond angles >= 90
    degrees, up to 20 tries per bead)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    dim = np.array(box, np.float64)
    nbt = 20
    sig_b = rng.uniform(0.25, 0.40, nbt)
    eps_b = rng.uniform(0.1, 1.0, nbt)
    pos = np.zeros((nchains, length, 3))
    pos[:, 0] = rng.uniform(0, 1, (nchains, 3)) * dim
    prev = rng.normal(size=(nchains, 3))
    prev /= np.linalg.norm(prev, axis=1)[:, None]
    for t in range(1, length):
        placed = pos[:, :t].reshape(-1, 3) % dim
        tree = cKDTree(placed, boxsize=dim)
        todo = np.arange(nchains)
        cand = np.zeros((nchains, 3))
        for _try in range(20):
            u = rng.normal(size=(len(todo), 3))
            u /= np.linalg.norm(u, axis=1)[:, None]
            flip = (u * prev[todo]).sum(1) < 0.0
            u[flip] = -u[flip]
            p = (pos[todo, t - 1] + bond * u) % dim
            d, idx = tree.query(p, k=3)
            # neighbours that are the chain's own last two beads do not count
            own = (idx // t == todo[:, None]) & (idx % t >= t - 2)
            dmin = np.where(own, np.inf, d).min(1)
            ok = dmin >= clearance
            cand[todo[ok]] = p[ok]
            prev[todo[ok]] = u[ok]
            if _try == 19:
                cand[todo[~ok]] = p[~ok]
                prev[todo[~ok]] = u[~ok]
            todo = todo[~ok]
            if len(todo) == 0:
                break
        pos[:, t] = cand
    xb = pos.reshape(-1, 3) % dim
    tb = rng.integers(0, nbt, size=len(xb)).astype(np.int32) + 2
    qb = rng.normal(0.0, 0.3, size=(nchains, length))
    qb -= qb.mean(1, keepdims=True)
    qb = qb.reshape(-1)
    # --- water on a grid, away from the beads
    spacing = (1.0 / 33.4) ** (1.0 / 3.0)
    nsite = np.maximum(1, np.round(dim / spacing)).astype(int)
    sites = np.stack(np.meshgrid(*[np.arange(n) for n in nsite], indexing="ij"), -1).reshape(-1, 3)
    sites = (sites + 0.5) * (dim / nsite) + rng.normal(0.0, 0.01, (len(sites), 3))
    sites = sites % dim
    d, _ = cKDTree(xb, boxsize=dim).query(sites, k=1)
    sites = sites[d >= gap]
    sites = sites[rng.permutation(len(sites))[:nwater]]
    nw = len(sites)
    rot = _random_rotations(rng, nw)
    hh = 0.1 * math.sin(math.radians(109.47) / 2.0)
    hz = 0.1 * math.cos(math.radians(109.47) / 2.0)
    h1 = np.einsum("mij,j->mi", rot, np.array([hh, 0.0, hz]))
    h2 = np.einsum("mij,j->mi", rot, np.array([-hh, 0.0, hz]))
    xw = np.stack([sites, sites + h1, sites + h2], 1).reshape(-1, 3)
    tw = np.tile(np.array([0, 1, 1], np.int32), nw)
    qw = np.tile(np.array([-0.8476, 0.4238, 0.4238]), nw)
    x = np.concatenate([xw, xb])
    typ = np.concatenate([tw, tb]).astype(np.int32)
    q = np.concatenate([qw, qb]) * QSCALE
    nwa = 3 * nw
    # --- exclusions and constraints
    k = np.arange(nw) * 3
    ex = [np.stack([k, k + 1], 1), np.stack([k, k + 2], 1), np.stack([k + 1, k + 2], 1)]
    b0 = nwa + np.arange(nchains)[:, None] * length
    i1 = (b0 + np.arange(length - 1)[None, :]).reshape(-1)
    i2 = (b0 + np.arange(length - 2)[None, :]).reshape(-1)
    ex += [np.stack([i1, i1 + 1], 1), np.stack([i2, i2 + 2], 1)]
    hhd = 2.0 * 0.1 * math.sin(math.radians(109.47) / 2.0)
    rig = np.stack([np.stack([k, k + 1, np.full(nw, 0.1)], 1), np.stack([k, k + 2, np.full(nw, 0.1)], 1),
                    np.stack([k + 1, k + 2, np.full(nw, hhd)], 1)], 1).reshape(-1, 3)
    # --- potentials: LJ among O, H and the bead types (Lorentz-Berthelot).  SPC/E gives H
    # no LJ; with per-particle charges an H next to a negative bead would then meet no
    # repulsion at all, so H carries a small one (sigma `h_sigma`, epsilon 0.1 kJ/mol).
    # With sigma 0.1 nm the H-bead contacts are stiff enough that 2 fs steps heat the
    # system about twice as fast as with 0.2 nm (the drift of either falls as dt^2).
    sig = np.concatenate([[0.3166, h_sigma], sig_b])
    eps = np.concatenate([[0.650, 0.1], eps_b])
    lj_types = [0, 1] + list(range(2, 2 + nbt))
    pots = []
    for a_i, ti in enumerate(lj_types):
        for b_i in range(a_i, len(lj_types)):
            e_ij, s_ij = lb_mix(eps[a_i], sig[a_i], eps[b_i], sig[b_i])
            pots.append(PotSpec(KIND_LJ126, ti, lj_types[b_i], 0.2, cutoff, tol, (*lj_AB(e_ij, s_ij), 0.0, 0.0)))
    ep = PotSpec(KIND_COULOMB, 0, 0, 0.05, cutoff, tol, (1.0, 0.0, 0.0, 0.0))
    masses = [15.9994, 1.008] + list(rng.uniform(12.0, 44.0, nbt))
    bonds = np.stack([i1, i1 + 1], 1).astype(np.int32)
    bond_pot = PotSpec(KIND_HARMONIC, 2, 2, 0.05, 0.3, 1e-5, (bond_k, bond, 0.0, 0.0))
    angles = angle_pots = dihedrals = dihedral_pots = None
    if angles_dihedrals and length >= 3:
        angles = np.stack([i2, i2 + 1, i2 + 2, rng.integers(0, len(CHAINS_ANGLE_POTS), len(i2))], 1)
        angle_pots = list(CHAINS_ANGLE_POTS)
        if length >= 4:
            i3 = (b0 + np.arange(length - 3)[None, :]).reshape(-1)
            dihedrals = np.stack([i3, i3 + 1, i3 + 2, i3 + 3, rng.integers(0, len(CHAINS_DIHEDRAL_POTS), len(i3))], 1)
            dihedral_pots = list(CHAINS_DIHEDRAL_POTS)
    return System(name=f"chains-water-{len(x)}", origin=np.zeros(3), dim=dim, L=np.full(3, cutoff), cutoff=cutoff,
                  masses=masses, charges=[0.0] * len(masses), pots=pots, x=_wrap(x, dim), type=typ,
                  excl=np.concatenate(ex).astype(np.int32), dt=0.002, rigid=rig, q=q, ep=ep,
                  bonds=bonds, bond_pot=bond_pot,
                  angles=None if angles is None else angles.astype(np.int32), angle_pots=angle_pots,
                  dihedrals=None if dihedrals is None else dihedrals.astype(np.int32), dihedral_pots=dihedral_pots)


# Bonded potentials of the chains: harmonic angles (a, b, K, theta0, tol) and harmonic
# dihedrals (K, n, delta, tol).  The table builder (the reference's) needs an angle range
# that stops short of 180 degrees and a dihedral phase of 0 or pi: dE/dcos is unbounded at
# cos = -1 for an angle, and at cos = +-1 for a dihedral of any other phase, and no
# interval count meets the tolerance (potential_err_ivalsmax).  Angles of the random-walk
# chains beyond the range are held to it, as the reference holds them.
CHAINS_ANGLE_POTS = [
    (math.radians(60.0), math.radians(175.0), 120.0, math.radians(120.0), 1e-4),
    (math.radians(50.0), math.radians(170.0), 80.0, math.radians(110.0), 1e-4),
]
CHAINS_DIHEDRAL_POTS = [(5.0, 3, 0.0, 1e-4), (2.0, 1, math.pi, 1e-4), (1.5, 2, 0.0, 1e-4)]


def bonded_chains(nchains: int = 12, length: int = 20, box=(3.6, 3.6, 3.6), seed: int = 0, bond: float = 0.15,
                  theta=(100.0, 150.0), tol: float = 1e-4) -> System:
    """Bead chains with every bond angle in `theta` degrees (each bead placed from its three
    predecessors by bond length, bond angle and a uniform random torsion), bonds, angles and
    dihedrals as chains_water's, one LJ type (sigma 0.25 nm, epsilon 0.2 kJ/mol) and 1-2/1-3
    exclusions; no solvent.  Chains may overlap each other: meant for the bonded terms."""
    rng = np.random.default_rng(seed)
    dim = np.array(box, np.float64)
    pos = np.zeros((nchains, length, 3))
    pos[:, 0] = rng.uniform(0, 1, (nchains, 3)) * dim
    for c in range(nchains):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        pos[c, 1] = pos[c, 0] + bond * d
        for t in range(2, length):
            a = pos[c, t - 1] - pos[c, t - 2]
            a /= np.linalg.norm(a)
            ref = pos[c, t - 3] - pos[c, t - 2] if t >= 3 else rng.normal(size=3)
            n = np.cross(a, ref)
            n /= np.linalg.norm(n)
            m = np.cross(n, a)
            th = math.radians(rng.uniform(*theta))
            ph = rng.uniform(-math.pi, math.pi)
            # the new bond makes angle th with the previous one (bond angle at bead t-1)
            step = -math.cos(th) * a + math.sin(th) * (math.cos(ph) * m + math.sin(ph) * n)
            pos[c, t] = pos[c, t - 1] + bond * step
    x = _wrap(pos.reshape(-1, 3), dim)
    b0 = np.arange(nchains)[:, None] * length
    i1 = (b0 + np.arange(length - 1)[None, :]).reshape(-1)
    i2 = (b0 + np.arange(length - 2)[None, :]).reshape(-1)
    i3 = (b0 + np.arange(length - 3)[None, :]).reshape(-1)
    ex = np.concatenate([np.stack([i1, i1 + 1], 1), np.stack([i2, i2 + 2], 1)]).astype(np.int32)
    A, B = lj_AB(0.2, 0.25)
    return System(name=f"bonded-chains-{len(x)}", origin=np.zeros(3), dim=dim, L=np.full(3, 1.2), cutoff=1.2,
                  masses=[14.0], charges=[0.0], pots=[PotSpec(KIND_LJ126, 0, 0, 0.1, 1.2, tol, (A, B, 0.0, 0.0))],
                  x=x, type=np.zeros(len(x), np.int32), excl=ex, dt=0.002,
                  bonds=np.stack([i1, i1 + 1], 1).astype(np.int32),
                  bond_pot=PotSpec(KIND_HARMONIC, 0, 0, 0.05, 0.3, 1e-5, (2.0e5, bond, 0.0, 0.0)),
                  angles=np.stack([i2, i2 + 1, i2 + 2, rng.integers(0, 2, len(i2))], 1).astype(np.int32),
                  angle_pots=list(CHAINS_ANGLE_POTS),
                  dihedrals=np.stack([i3, i3 + 1, i3 + 2, i3 + 3, rng.integers(0, 3, len(i3))], 1).astype(np.int32),
                  dihedral_pots=list(CHAINS_DIHEDRAL_POTS))


def write_bondedfile(sysm: System, path: str) -> None:
    """The bonded terms of sysm in the format `ref_driver bonded` reads (oracle/ref_driver.c):
    the bond potential for every type pair that a bond joins."""
    bonds = np.zeros((0, 2), np.int32) if sysm.bonds is None else np.asarray(sysm.bonds, np.int32)
    pairs = sorted({(int(min(a, b)), int(max(a, b))) for a, b in np.asarray(sysm.type)[bonds]}) if len(bonds) else []
    angles = np.zeros((0, 4), np.int32) if sysm.angles is None else np.asarray(sysm.angles, np.int32)
    dihedrals = np.zeros((0, 5), np.int32) if sysm.dihedrals is None else np.asarray(sysm.dihedrals, np.int32)
    apots = sysm.angle_pots or []
    dpots = sysm.dihedral_pots or []
    with open(path, "wb") as f:
        f.write(b"MDB2BND1")
        f.write(struct.pack("<6i", len(pairs), len(apots), len(dpots), len(bonds), len(angles), len(dihedrals)))
        bp = sysm.bond_pot
        for ti, tj in pairs:
            f.write(struct.pack("<2i5d", ti, tj, bp.a, bp.b, bp.p[0], bp.p[1], bp.tol))
        for a, b, K, th0, tol in apots:
            f.write(struct.pack("<5d", a, b, K, th0, tol))
        for K, n, delta, tol in dpots:
            f.write(struct.pack("<2i3d", n, 0, K, delta, tol))
        f.write(np.ascontiguousarray(bonds, "<i4").tobytes())
        f.write(np.ascontiguousarray(angles, "<i4").tobytes())
        f.write(np.ascontiguousarray(dihedrals, "<i4").tobytes())


def read_bondedout(path: str):
    """Parse the output of `ref_driver bonded`: forces by id of the bonds, the angles and the
    dihedrals (float), their energies, cell-relative positions, cells and the tables
    (n, alpha, coef, a, b) of the bond, angle and dihedral potentials in that order."""
    buf = open(path, "rb").read()
    assert buf[:8] == b"MDB2BOU1"
    off = 8

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(buf, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a

    N, nb, na, nd = (int(v) for v in take("<i4", 4))
    fb = take("<f4", 3 * N).reshape(N, 3).copy()
    fa = take("<f4", 3 * N).reshape(N, 3).copy()
    fd = take("<f4", 3 * N).reshape(N, 3).copy()
    eb, ea, ed = (float(v) for v in take("<f8", 3))
    xr = take("<f4", 3 * N).reshape(N, 3).copy()
    cell = take("<i4", N).copy()
    tables = []
    for _ in range(nb + na + nd):
        (n,) = take("<i4", 1)
        alpha = take("<f4", 4).copy()
        c = take("<f4", (int(n) + 1) * 8).copy()
        a, b = take("<f8", 2)
        tables.append((int(n), alpha, c, float(a), float(b)))
    return dict(f_bond=fb, f_angle=fa, f_dihedral=fd, e_bond=eb, e_angle=ea, e_dihedral=ed, xrel=xr, cell=cell,
                bond_tables=tables[:nb], angle_tables=tables[nb:nb + na], dihedral_tables=tables[nb + na:])
