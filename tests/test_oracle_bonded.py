"""CPU tests of the bonded terms: the FP64 angle and dihedral oracle against the reference's
own angle_eval / dihedral_eval outputs (tests/golden/bonded.npz), the bond oracle against
bond_eval, and the library's angle and dihedral tables against the reference's, bit for bit.

Tolerances (the reference evaluates in FP32, the oracle in FP64 on the same float inputs):
  forces   ||dF|| / ||F|| <= 1e-5 and max_i |dF_i| <= 2e-5 F_rms
  energy   |dE| <= 1e-6 |E|
  tables   bit-exact (n, alpha, coefficients, range)
"""
import numpy as np
import pytest

import mdcore_b200 as M
import oracle as O
from helpers import force_errors, load_bonded_golden


@pytest.fixture(scope="module")
def golden():
    return load_bonded_golden()


def check(f, e, f_ref, e_ref):
    err = force_errors(f, f_ref.astype(np.float64))
    assert err["global_rel"] <= 1e-5, err
    assert err["max_over_frms"] <= 2e-5, err
    assert abs(e - e_ref) <= 1e-6 * abs(e_ref), (e, e_ref)


def test_angles_vs_reference(golden):
    sysm, ref = golden
    o = O.angles(sysm, ref["angle_tables"], xrel=ref["xrel"], cell=ref["cell"])
    check(o["f"], o["epot"], ref["f_angle"], float(ref["energies"][1]))


def test_dihedrals_vs_reference(golden):
    sysm, ref = golden
    o = O.dihedrals(sysm, ref["dihedral_tables"], xrel=ref["xrel"], cell=ref["cell"])
    check(o["f"], o["epot"], ref["f_dihedral"], float(ref["energies"][2]))


def test_bonds_vs_reference(golden):
    """Bonds at their rest length: forces near zero, compared against the bond force scale."""
    sysm, ref = golden
    n, alpha, c, a, b = ref["bond_tables"][0]
    o = O.bonds(sysm, (n, alpha, c), binned=dict(xrel=ref["xrel"], cell=ref["cell"],
                                                   cdim=np.floor(sysm.dim / sysm.L).astype(np.int32)))
    scale = np.abs(ref["f_angle"]).max()
    assert np.abs(o["f"] - ref["f_bond"]).max() <= 1e-5 * scale
    assert abs(o["epot"] - float(ref["energies"][0])) <= 1e-6 * abs(float(ref["energies"][1]))


def test_oracle_positions_are_the_reference_cells(golden):
    sysm, ref = golden
    b = O.bin_system(sysm)
    assert np.array_equal(b["cell"], ref["cell"]) and np.array_equal(b["xrel"], ref["xrel"])


def test_tables_bit_identical(golden):
    sysm, ref = golden
    mine = M.bonded_tables([M.create_angle_potential(*p) for p in sysm.angle_pots])
    mine += M.bonded_tables([M.create_dihedral_potential(*p) for p in sysm.dihedral_pots])
    theirs = ref["angle_tables"] + ref["dihedral_tables"]
    assert len(mine) == len(theirs)
    for m, r in zip(mine, theirs):
        assert m[0] == r[0]
        assert np.array_equal(m[1], r[1]) and np.array_equal(m[2], r[2])
        assert m[3] == r[3] and m[4] == r[4]


def test_angle_range_near_180_degrees_is_refused():
    """An angle range reaching 180 degrees has no table within tolerance (the reference's
    builder gives up too: potential_err_ivalsmax); the library returns NULL."""
    with pytest.raises(M.MdcoreError):
        M.create_angle_potential(np.radians(60.0), np.pi, 120.0, np.radians(120.0), 1e-4)
    M.lib().errs_clear()
