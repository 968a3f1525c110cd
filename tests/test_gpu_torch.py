"""Autograd through the native adjoint, checked by central finite differences.

Alkanes C_nH_{2n+2} (built as in the alkane workload).  The orbital basis is
def2-SVP (cc-pVDZ for carbon is not among the bundled records; def2-SVP has
the same H/C shell structure) and the auxiliary basis def2-TZVP (no carbon
JK-fit set is bundled).  Step 1e-3 Bohr; tolerance 2e-6 Eh/Bohr, far above the
O(h^2) truncation error and the 1e-10 Eh SCF convergence noise / h.
"""

import numpy as np
import pytest
import torch

from vibeqc_b200 import Calculator, geometry
from vibeqc_b200.torch import batched_energy, energy

pytestmark = pytest.mark.gpu

BASIS, AUX = "def2-svp", "def2-tzvp"


def _system(n, seed):
    atoms = geometry.alkane(n, seed)
    z = [a[0] for a in atoms]
    from vibeqc_b200.basis import atomic_number

    return atoms, [atomic_number(s) for s in z], torch.tensor([a[1] for a in atoms], dtype=torch.float64)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_energy_autograd_matches_finite_differences(precision):
    calc = Calculator(method="rhf", basis=BASIS, auxiliary_basis=AUX, device="cuda",
                      density_fitting="cuda", precision=precision)
    systems = [_system(n, 10 + n) for n in (2, 3, 4)]
    batch = calc.prepare_batch([s[0] for s in systems])
    coords = [s[2].cuda().requires_grad_(True) for s in systems]
    e = batched_energy(coords, [s[1] for s in systems], prepared_batch=batch)
    e.sum().backward()
    rng = np.random.default_rng(0)
    h = 1e-3
    for i, s in enumerate(systems):
        g = coords[i].grad.detach().cpu().numpy()
        assert np.abs(g.sum(axis=0)).max() < 1e-8  # translational invariance
        for _ in range(3):
            a, d = int(rng.integers(len(s[1]))), int(rng.integers(3))
            vals = []
            for sgn in (1.0, -1.0):
                xyz = [c.detach().cpu().numpy().copy() for c in coords]
                xyz[i][a, d] += sgn * h
                res = batch.execute(xyz, properties=("energy",), strict=True)
                vals.append(res.items[i].energy)
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(fd - g[a, d]) < 2e-6, (i, a, d, fd, g[a, d])
    batch.close()


def test_single_energy_backward_equals_minus_forces():
    calc = Calculator(method="rhf", basis=BASIS, auxiliary_basis=AUX, device="cuda",
                      density_fitting="cuda")
    atoms, z, xyz = _system(2, 3)
    c = xyz.cuda().requires_grad_(True)
    e = energy(c, z, calc)
    (g,) = torch.autograd.grad(e, c)
    res = calc.singlepoint(atoms)
    assert abs(float(e) - res.energy) < 1e-9
    assert np.abs(g.cpu().numpy() + res.forces).max() < 1e-9
    with pytest.raises(RuntimeError):  # second order is not available
        c2 = xyz.cuda().requires_grad_(True)
        e2 = energy(c2, z, calc)
        (g2,) = torch.autograd.grad(e2, c2, create_graph=True)
        g2.sum().backward()
