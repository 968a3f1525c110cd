"""Autotuned schedules per chunk shape: pick, by timing on the GPU, how each
homogeneous chunk (N, X, n_occ) runs.

The reference picks its CUDA tile shapes and schedules from build-time tuning
manifests (``python/generativeqc_compiler/integral/df_tuning/policy.py``,
``manifest.py``); here the choices are runtime ones, measured per shape on
the device that will run them and stored in a table
(``vibeqc_b200/data/tuning.json``) that the calculator applies per chunk:

* ``whiten``: the mixed path's whitening B = A W on the int8 tensor cores
  (7-bit slices, ``"int8"``) or as FP64 GEMMs (``"fp64"``) -- both give
  FP64-accurate B; small shapes can favour the plain GEMMs;
* ``gram_waves``: the exchange Gram product splits its K range until about
  this many CTAs per SM exist (library knob ``VQC_TUNE_GRAM_WAVES``);
* ``sp2_steps``: purification steps per captured CUDA graph (more steps mean
  fewer host round trips, but converged molecules idle longer);
* ``sp2_gemm``: how the mixed path forms the purification product X^2 --
  batched FP64 GEMMs (``"fp64"``) or FP64-accurate sliced products on the
  int8 tensor cores (``"int8"``).

    python -m vibeqc_b200.tuning [--count 256] [--out path]

times every shape of the 256-cluster workload and writes the table.  Shapes
missing from a table use the nearest tuned N of the same precision, else the
defaults.
"""

from __future__ import annotations

import argparse
import json
import time
from dataclasses import asdict, dataclass
from pathlib import Path

TABLE_PATH = Path(__file__).resolve().parent / "data" / "tuning.json"
WHITEN_CHOICES = ("int8", "fp64")
GRAM_WAVES = (1, 2, 4, 8)
SP2_STEPS = (4, 8, 16)
SP2_GEMMS = ("fp64", "int8")


@dataclass(frozen=True)
class Schedule:
    whiten: str = "int8"
    gram_waves: int = 2
    sp2_steps: int = 8
    sp2_gemm: str = "fp64"

    def __post_init__(self):
        if self.whiten not in WHITEN_CHOICES:
            raise ValueError(f"whiten must be one of {WHITEN_CHOICES}")
        if not 1 <= int(self.gram_waves) <= 64:
            raise ValueError("gram_waves must be in 1..64")
        if int(self.sp2_steps) < 2 or int(self.sp2_steps) % 2:
            raise ValueError("sp2_steps must be an even number >= 2")
        if self.sp2_gemm not in SP2_GEMMS:
            raise ValueError(f"sp2_gemm must be one of {SP2_GEMMS}")


DEFAULT = Schedule()


def shape_key(nao: int, naux: int, nocc: int) -> str:
    return f"{int(nao)}/{int(naux)}/{int(nocc)}"


class TuningTable:
    """Schedules per chunk shape, with the timings that chose them."""

    def __init__(self, entries: dict | None = None, meta: dict | None = None):
        self.entries: dict[str, Schedule] = dict(entries or {})
        self.meta = dict(meta or {})
        self.timings: dict[str, dict] = {}

    @classmethod
    def load(cls, path: Path | str = TABLE_PATH) -> "TuningTable":
        path = Path(path)
        if not path.exists():
            return cls()
        doc = json.loads(path.read_text())
        if doc.get("schema") != "vibeqc_b200.tuning" or doc.get("version") != 1:
            raise ValueError(f"{path}: not a tuning table of this package")
        t = cls({k: Schedule(**v["schedule"]) for k, v in doc["shapes"].items()}, doc.get("meta"))
        t.timings = {k: v.get("timings_ms", {}) for k, v in doc["shapes"].items()}
        return t

    def save(self, path: Path | str = TABLE_PATH) -> None:
        shapes = {k: {"schedule": asdict(s), "timings_ms": self.timings.get(k, {})}
                  for k, s in sorted(self.entries.items(), key=lambda kv: [int(v) for v in kv[0].split("/")])}
        Path(path).write_text(json.dumps({"schema": "vibeqc_b200.tuning", "version": 1,
                                          "meta": self.meta, "shapes": shapes}, indent=1) + "\n")

    def lookup(self, nao: int, naux: int, nocc: int) -> Schedule:
        s = self.entries.get(shape_key(nao, naux, nocc))
        if s is not None:
            return s
        if not self.entries:
            return DEFAULT
        near = min(self.entries, key=lambda k: abs(int(k.split("/")[0]) - int(nao)))
        return self.entries[near]


_ACTIVE: list = [None]


def active_table() -> TuningTable:
    """The table the calculator applies (loaded once from TABLE_PATH)."""
    if _ACTIVE[0] is None:
        _ACTIVE[0] = TuningTable.load()
    return _ACTIVE[0]


def set_active_table(table: TuningTable | None) -> None:
    _ACTIVE[0] = table


def apply_library_knobs(schedule: Schedule) -> None:
    from . import _lib

    _lib.call("vqc_tune_set", _lib.TUNE_GRAM_WAVES, int(schedule.gram_waves))


# -- the tuner --------------------------------------------------------------

def _time(fn, reps: int = 3) -> float:
    import torch

    fn()  # warm-up (graph capture, allocator)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    return best


def tune_chunk(chunk, xyz) -> tuple[Schedule, dict]:
    """Time every candidate of every knob on one chunk (coordinate-wise)."""
    import torch

    from . import _lib
    from . import jk as jkmod
    from .scf import (_orthogonalizer, compute_integrals, factor_metric, purify_sp2,
                      whiten_in_place, whiten_tensor_cores)

    timings: dict = {}
    ints = compute_integrals(chunk.plan, xyz)
    mf = factor_metric(ints.metric)
    a0 = ints.a_packed
    work = torch.empty_like(a0)

    def whiten(kind):
        work.copy_(a0)
        if kind == "int8":
            whiten_tensor_cores(work, mf, ints.metric)
        else:
            whiten_in_place(work, mf)

    timings["whiten"] = {k: round(_time(lambda k=k: whiten(k), 2), 3) for k in WHITEN_CHOICES}
    whiten_best = min(timings["whiten"], key=timings["whiten"].get)
    del a0
    ints.a_packed = None
    # exchange Gram product over a mixed builder's split U
    jk = jkmod.MixedBuilder(work, chunk.nao, chunk.naux, chunk.nocc)
    del work
    gen = torch.Generator(device=xyz.device).manual_seed(5)
    c = torch.randn(chunk.nb, chunk.nao, chunk.nocc, dtype=torch.float64, device=xyz.device,
                    generator=gen) / chunk.nao ** 0.5
    d = 2.0 * c @ c.transpose(1, 2)
    jk.build(d, c)
    kout = torch.zeros(chunk.nb, chunk.nao, chunk.nao, dtype=torch.float64, device=xyz.device)
    st = torch.cuda.current_stream().cuda_stream

    def gram():
        _lib.call("vqc_tc_gram", jk.u_hi.data_ptr(), jk.u_lo.data_ptr(), chunk.nb, chunk.nao,
                  chunk.nocc * jk.ldq, kout.data_ptr(), jk.err.data_ptr(), st)

    timings["gram_waves"] = {}
    for w in GRAM_WAVES:
        _lib.call("vqc_tune_set", _lib.TUNE_GRAM_WAVES, w)
        timings["gram_waves"][str(w)] = round(_time(gram), 3)
    _lib.call("vqc_tune_set", _lib.TUNE_GRAM_WAVES, DEFAULT.gram_waves)
    waves_best = int(min(timings["gram_waves"], key=timings["gram_waves"].get))
    del jk
    # purification of the core Hamiltonian
    xo = _orthogonalizer(ints.s)
    fo = xo.transpose(1, 2) @ ints.h @ xo
    timings["sp2_steps"] = {}
    for n_steps in SP2_STEPS:
        graphs: dict = {}
        timings["sp2_steps"][str(n_steps)] = round(
            _time(lambda: purify_sp2(fo, chunk.nocc, graphs=graphs, steps=n_steps)), 3)
    steps_best = int(min(timings["sp2_steps"], key=timings["sp2_steps"].get))
    timings["sp2_gemm"] = {}
    for gemm in SP2_GEMMS:
        graphs = {}
        timings["sp2_gemm"][gemm] = round(
            _time(lambda: purify_sp2(fo, chunk.nocc, graphs=graphs, steps=steps_best, gemm=gemm)), 3)
    gemm_best = min(timings["sp2_gemm"], key=timings["sp2_gemm"].get)
    return Schedule(whiten_best, waves_best, steps_best, gemm_best), timings


def autotune(systems, basis: str, auxiliary_basis: str, precision: str = "mixed") -> TuningTable:
    """Tune every chunk shape of ``systems`` (the largest chunk of each shape)."""
    import torch

    from .calculator import Calculator

    calc = Calculator(method="rhf", basis=basis, auxiliary_basis=auxiliary_basis, device="cuda",
                      density_fitting="cuda", precision=precision)
    batch = calc.prepare_batch(systems, warm_start=False)
    coords = batch.upload_coordinates()
    best: dict = {}
    for chunk, xyz in zip(batch._chunks, coords):
        key = shape_key(chunk.nao, chunk.naux, chunk.nocc)
        if key not in best or chunk.nb > best[key][0].nb:
            best[key] = (chunk, xyz)
    table = TuningTable(meta={"device": torch.cuda.get_device_name(), "precision": precision,
                              "basis": basis, "auxiliary_basis": auxiliary_basis,
                              "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())})
    for key, (chunk, xyz) in sorted(best.items(), key=lambda kv: kv[1][0].nao):
        sched, timings = tune_chunk(chunk, xyz)
        table.entries[key] = sched
        table.timings[key] = timings
        print(f"{key} nb={chunk.nb}: {sched} {timings}", flush=True)
        torch.cuda.empty_cache()
    batch.close()
    return table


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=str(TABLE_PATH))
    args = ap.parse_args()
    from . import geometry

    systems = geometry.water_cluster_batch(args.count, 2, 16, args.seed)
    table = autotune(systems, "def2-svp", "cc-pvdz-jkfit")
    table.meta["workload"] = f"water_cluster_batch({args.count}, 2, 16, seed={args.seed})"
    table.save(args.out)
    print(f"wrote {args.out}")


if __name__ == "__main__":
    main()
