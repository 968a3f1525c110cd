"""Warm-start replay and checkpoint restarts of a prepared batch on the GPU.

A second execution at a displaced geometry starts from the first one's
converged densities (reference python/generativeqc/batch.py:123-130): it must
report the warm start, need fewer SCF iterations than a cold start, and reach
the cold start's energy and forces.  Frozen updates, clearing and checkpoint
restarts follow the reference's controls (batch.py:1312-1390).
"""

import numpy as np
import pytest

from vibeqc_b200 import Calculator, geometry

pytestmark = pytest.mark.gpu

SYSTEMS = [geometry.water_cluster(3, 5), geometry.water_cluster(4, 6)]


def _displaced(seed, scale=0.02):
    rng = np.random.default_rng(seed)
    out = []
    for atoms in SYSTEMS:
        xyz = np.array([p for _, p in atoms])
        out.append(xyz + scale * rng.standard_normal(xyz.shape))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_warm_start_replays_previous_density(precision):
    calc = Calculator(method="rhf", basis="def2-svp", auxiliary_basis="cc-pvdz-jkfit", device="cuda",
                      density_fitting="cuda", precision=precision)
    moved = _displaced(1)
    with calc.prepare_batch(SYSTEMS, warm_start=False) as cold_batch:
        cold = cold_batch.execute(moved, strict=True)
    with calc.prepare_batch(SYSTEMS) as batch:
        first = batch.execute(strict=True)
        assert not any(i.warm_start_used for i in first.items)
        warm = batch.execute(moved, strict=True)
        for w, c in zip(warm.items, cold.items):
            assert w.warm_start_used and not w.warm_start_fallback
            assert w.iterations < c.iterations, (w.iterations, c.iterations)
            assert abs(w.energy - c.energy) < 1e-9
            assert np.abs(w.forces - c.forces).max() < 1e-6
        # frozen updates: two replays start from the same snapshot
        batch.set_warm_start_updates(False)
        again = batch.execute(_displaced(2), strict=True)
        again2 = batch.execute(_displaced(2), strict=True)
        assert [i.iterations for i in again.items] == [i.iterations for i in again2.items]
        batch.clear_warm_starts()
        fresh = batch.execute(moved, strict=True)
        assert not any(i.warm_start_used for i in fresh.items)
        assert all(abs(f.energy - c.energy) < 1e-9 for f, c in zip(fresh.items, cold.items))


def test_checkpoint_restart_in_a_new_batch(tmp_path):
    calc = Calculator(method="rhf", basis="def2-svp", auxiliary_basis="cc-pvdz-jkfit", device="cuda",
                      density_fitting="cuda")
    with calc.prepare_batch(SYSTEMS) as batch:
        ref = batch.execute(strict=True)
        info = batch.save_checkpoint(tmp_path / "run.ckpt")
    assert info["seeds"] == len(SYSTEMS)
    with calc.prepare_batch(SYSTEMS) as restart:
        rep = restart.load_checkpoint(tmp_path / "run.ckpt")
        assert rep["seeded"] == [0, 1]
        res = restart.execute(strict=True)
    for r, a in zip(res.items, ref.items):
        assert r.warm_start_used
        assert r.iterations <= 3, r.iterations  # restarted at the converged density
        assert abs(r.energy - a.energy) < 1e-9
