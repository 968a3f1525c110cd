"""The standalone DF gradient entry (reference generativeqc_system_df_gradient_cuda contract).

Random nonsymmetric full weights bar_a[mu][nu][P] and bar_m[P][Q] are
contracted through the C ABI (host arrays in, host gradient out) and compared
with the CPU oracle's contraction of the same weights, every element counted
once (include/generativeqc/generativeqc.h:1320-1333 of the reference).
Failing calls must leave the caller's gradient untouched.
"""

import numpy as np
import pytest

from oracle import oracle
from vibeqc_b200 import _lib, geometry
from vibeqc_b200.gradient import df_gradient_host
from vibeqc_b200.plan import make_molecule

pytestmark = pytest.mark.gpu

CASES = [
    (geometry.water_cluster(1, 11), "def2-svp", "cc-pvdz-jkfit"),
    (geometry.alkane(2, 5), "def2-svp", "def2-tzvp"),  # d orbital, f auxiliary shells
]


def _weights(mol, seed):
    orb = oracle.OracleBasis(mol.orbital_shells, True)
    aux = oracle.OracleBasis(mol.aux_shells, True)
    rng = np.random.default_rng(seed)
    n, x = orb.nfunc, aux.nfunc
    return orb, aux, rng.standard_normal((n, n, x)), rng.standard_normal((x, x))


@pytest.mark.parametrize("case", range(len(CASES)))
def test_nonsymmetric_weights_match_oracle(case):
    mol = make_molecule(*CASES[case])
    orb, aux, bar_a, bar_m = _weights(mol, 7 + case)
    ref3 = oracle.grad3c(orb, aux, mol.coordinates, bar_a)
    ref2 = oracle.grad2c(aux, mol.coordinates, bar_m)
    g, rec = df_gradient_host(mol, bar_a, bar_m)
    ref = ref3 + ref2
    scale = np.abs(ref).max()
    assert np.abs(g - ref).max() <= 1e-10 * scale, np.abs(g - ref).max() / scale
    assert rec["tiles"] == 1 and rec["device_to_host_bytes"] == g.size * 8
    # null channels mean zero
    g3, _ = df_gradient_host(mol, bar_a, None)
    g2, _ = df_gradient_host(mol, None, bar_m)
    assert np.abs(g3 - ref3).max() <= 1e-10 * np.abs(ref3).max()
    assert np.abs(g2 - ref2).max() <= 1e-10 * np.abs(ref2).max()


def test_tiled_weights_match_single_tile():
    mol = make_molecule(*CASES[1])
    orb, aux, bar_a, bar_m = _weights(mol, 3)
    whole, rec1 = df_gradient_host(mol, bar_a, bar_m)
    n = orb.nfunc
    tiled, rec = df_gradient_host(mol, bar_a, bar_m, maximum_tile_elements=n * n * 24)
    assert rec["tiles"] > 3 and rec1["tiles"] == 1
    assert rec["weight_tile_elements"] <= n * n * 24
    assert np.abs(tiled - whole).max() <= 1e-12 * np.abs(whole).max()
    # a byte bound that forces tiles gives the same answer too
    small, rec2 = df_gradient_host(mol, bar_a, bar_m,
                                   maximum_bytes=rec1["device_bytes"] // 3)
    assert rec2["tiles"] > 1 and rec2["device_bytes"] <= rec1["device_bytes"] // 3
    assert np.abs(small - whole).max() <= 1e-12 * np.abs(whole).max()


def test_failures_preserve_caller_output():
    mol = make_molecule(*CASES[0])
    orb, aux, bar_a, bar_m = _weights(mol, 5)
    natom = len(mol.atomic_numbers)
    out = np.full((natom, 3), 123.25)
    with pytest.raises(_lib.VqcError) as e:  # wrong weight count
        df_gradient_host(mol, bar_a[:, :, :-1], bar_m, out=out)
    assert e.value.status == 1
    with pytest.raises(_lib.VqcError) as e:  # budget below one auxiliary shell of weights
        df_gradient_host(mol, bar_a, None, maximum_bytes=4096, out=out)
    assert e.value.status == 7
    assert (out == 123.25).all()
    g, _ = df_gradient_host(mol, bar_a, bar_m, out=out)
    assert g.base is out or g is out
    assert not (out == 123.25).any()
