"""The CPU oracle's unrestricted (DF-UHF) path: known answers and finite differences.

The reference's UHF DF path (``src/scf/density_fitting.cpp:844,919``) has no
stored energies; the unrestricted oracle is pinned instead by properties that
hold for any correct implementation:

* a closed-shell singlet solved unrestricted reproduces the restricted
  energy and forces (the RHF path itself is pinned to the reference goldens);
* one electron (the H atom): the DF Coulomb and exchange terms cancel
  exactly, so the energy is the lowest generalised eigenvalue of the core
  Hamiltonian in the basis;
* analytic forces of an open-shell doublet (OH radical) match central finite
  differences of the energy.
"""

import numpy as np
import pytest
import scipy.linalg

from oracle import oracle
from vibeqc_b200 import basis as bas
from vibeqc_b200 import geometry

OH = [("O", (0.0, 0.0, 0.0)), ("H", (0.3, 0.2, 1.85))]


def test_spin_counts():
    assert oracle.spin_counts(9, 2) == (5, 4)
    assert oracle.spin_counts(8, 3) == (5, 3)
    assert oracle.spin_counts(10, 1) == (5, 5)
    with pytest.raises(ValueError):
        oracle.spin_counts(9, 1)
    with pytest.raises(ValueError):
        oracle.spin_counts(1, 4)


def test_closed_shell_singlet_equals_restricted():
    atoms = geometry.water_cluster(1, np.random.default_rng(3))
    r = oracle.df_rhf(atoms)
    u = oracle.df_uhf(atoms, multiplicity=1)
    assert u.converged
    assert abs(u.energy - r.energy) < 1e-10
    assert np.abs(u.forces - r.forces).max() < 1e-8


def test_hydrogen_atom_is_the_core_eigenvalue():
    atoms = [("H", (0.1, -0.2, 0.3))]
    u = oracle.df_uhf(atoms, multiplicity=2)
    z, xyz = oracle.molecule_arrays(atoms)
    orb = oracle.OracleBasis(bas.expand_shells(z.astype(int), "def2-svp"))
    s, t, v = oracle.int1e(orb, xyz, z)
    assert u.converged
    assert abs(u.energy - scipy.linalg.eigh(t + v, s, eigvals_only=True)[0]) < 1e-12
    assert np.abs(u.forces).max() < 1e-12


def test_open_shell_forces_match_finite_differences():
    ref = oracle.df_uhf(OH, multiplicity=2)
    assert ref.converged
    h = 1e-3
    for ia, ix in [(0, 0), (1, 2), (1, 1)]:
        es = []
        for sgn in (1.0, -1.0):
            atoms = [list(a) for a in OH]
            p = list(atoms[ia][1])
            p[ix] += sgn * h
            atoms[ia][1] = tuple(p)
            es.append(oracle.df_uhf([tuple(a) for a in atoms], multiplicity=2, forces=False).energy)
        assert -(es[0] - es[1]) / (2 * h) == pytest.approx(ref.forces[ia, ix], abs=1e-6)
