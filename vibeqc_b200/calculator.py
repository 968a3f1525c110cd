"""Drop-in ``Calculator`` / ``PreparedBatch`` for the DF-RHF CUDA path.

Same constructor keywords, methods and result records as the reference's
``python/generativeqc/calculator.py:157-186`` (``Calculator``), ``:1931``
(``prepare_batch``), ``:2128`` (``singlepoint``) and
``python/generativeqc/batch.py:58-121,799`` (``BatchItemResult``,
``BatchResult``, ``PreparedBatch.execute``).  Units are Bohr and Hartree;
forces are -dE/dR.  Only ``method="rhf"`` (closed-shell singlets) or ``method="uhf"`` (any
multiplicity) with ``density_fitting="cuda"`` (or ``"auto"``/``True``) on
``device="cuda"`` is served here; any other combination raises
``NotImplementedError`` naming the unsupported option.
"""

from __future__ import annotations

import threading
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np
import torch

from . import _lib, tuning
from .gradient import df_rhf_gradient, df_uhf_gradient
from .plan import make_molecule
from .scf import Chunk, compute_integrals, run_scf
from .uhf import run_scf_uhf

STATUS_SUCCESS = 0
STATUS_INVALID_ARGUMENT = 1
STATUS_NOT_CONVERGED = 4
STATUS_NUMERICAL_FAILURE = 5


@dataclass(frozen=True)
class Result:
    """Single-system output (reference ``_api_types.py:149-170``)."""

    energy: float
    forces: np.ndarray | None
    converged: bool
    iterations: int
    energy_change: float
    density_rms: float
    executed_backend: str
    basis_metadata: dict = field(default_factory=dict)
    precision: dict | None = None


@dataclass(frozen=True)
class BatchItemResult:
    index: int
    status: int
    status_message: str
    energy: float
    forces: np.ndarray | None
    converged: bool
    iterations: int
    energy_change: float
    density_rms: float
    executed_backend: str
    bucket_id: int
    warm_start_used: bool = False
    warm_start_fallback: bool = False
    basis_metadata: dict = field(default_factory=dict)
    precision: dict | None = None

    @property
    def succeeded(self) -> bool:
        return self.status == STATUS_SUCCESS


@dataclass(frozen=True)
class BatchResult:
    """Input-ordered results for a ragged batch; forces are never padded."""

    items: tuple[BatchItemResult, ...]

    @property
    def energies(self) -> np.ndarray:
        return np.asarray([i.energy if i.succeeded else np.nan for i in self.items], dtype=np.float64)

    @property
    def failure_indices(self) -> tuple[int, ...]:
        return tuple(i.index for i in self.items if not i.succeeded)

    @property
    def succeeded(self) -> bool:
        return not self.failure_indices

    def raise_for_failures(self) -> None:
        failures = [f"{i.index}: {i.status_message}" for i in self.items if not i.succeeded]
        if failures:
            raise RuntimeError("batched item failures: " + "; ".join(failures))


_PRECISIONS = {"fp64": "fp64", "mixed": "mixed", "auto": "fp64"}


class Calculator:
    """DF-RHF energy and analytic forces on one CUDA device (coordinates in Bohr)."""

    def __init__(
        self,
        method="rhf",
        basis=None,
        device: str = "cpu",
        device_id: int = 0,
        basis_representation: str | None = None,
        *,
        density_fitting="none",
        auxiliary_basis=None,
        density_fitting_relative_threshold: float = 1.0e-10,
        density_fitting_memory_budget_bytes: int = 0,
        max_iterations: int = 100,
        energy_tolerance: float = 1.0e-10,
        density_tolerance: float = 1.0e-8,
        diis_history: int = 8,
        precision: str = "fp64",
        **unsupported,
    ) -> None:
        if unsupported:
            raise NotImplementedError(f"options outside the DF-RHF CUDA path: {sorted(unsupported)}")
        if str(method).lower() not in ("rhf", "uhf"):
            raise NotImplementedError("only method='rhf' or 'uhf' is served by this engine")
        if density_fitting not in ("cuda", "auto", True):
            raise NotImplementedError("this engine serves density_fitting='cuda' (or 'auto'/True)")
        if device != "cuda":
            raise NotImplementedError("this engine runs on device='cuda' only")
        if basis is None or auxiliary_basis is None:
            raise ValueError("basis and auxiliary_basis are required")
        if basis_representation not in (None, "spherical", "cartesian"):
            raise ValueError("basis_representation must be 'spherical' or 'cartesian'")
        if precision not in _PRECISIONS:
            raise ValueError("precision must be 'fp64', 'mixed' or 'auto'")
        if not (0.0 <= density_fitting_relative_threshold < 1.0):
            raise ValueError("density_fitting_relative_threshold must be in [0, 1)")
        if max_iterations < 1 or diis_history < 1:
            raise ValueError("max_iterations and diis_history must be positive")
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device is visible")
        _lib.lib()  # fail loudly if the native library is missing
        self.method = str(method).lower()
        self.basis = basis
        self.auxiliary_basis = auxiliary_basis
        self.device = torch.device("cuda", device_id)
        self.spherical = basis_representation != "cartesian"
        self.relative_threshold = float(density_fitting_relative_threshold)
        self.memory_budget_bytes = int(density_fitting_memory_budget_bytes)
        self.max_iterations = int(max_iterations)
        self.energy_tolerance = float(energy_tolerance)
        self.density_tolerance = float(density_tolerance)
        self.diis_history = int(diis_history)
        self.precision = _PRECISIONS[precision]
        self._lock = threading.Lock()

    def singlepoint(self, atoms, *, charge: int = 0, multiplicity: int = 1,
                    properties: Iterable[str] | None = None) -> Result:
        with self._lock:
            batch = self.prepare_batch([list(atoms)], charges=[charge], multiplicities=[multiplicity])
            res = batch.execute(strict=True, properties=properties)
            batch.close()
        item = res.items[0]
        return Result(item.energy, item.forces, item.converged, item.iterations,
                      item.energy_change, item.density_rms, item.executed_backend,
                      item.basis_metadata, item.precision)

    def prepare_batch(self, systems: Sequence, *, charges: Sequence[int] | None = None,
                      multiplicities: Sequence[int] | None = None, warm_start: bool = True):
        return PreparedBatch(self, systems, charges=charges, multiplicities=multiplicities,
                             warm_start=warm_start)


class PreparedBatch:
    """Persistent plan over a ragged batch (not re-entrant; one caller at a time)."""

    def __init__(self, calculator: Calculator, systems, *, charges=None, multiplicities=None,
                 warm_start: bool = True):
        systems = [list(s) for s in systems]
        if not systems:
            raise ValueError("a batch needs at least one system")
        n = len(systems)
        charges = [0] * n if charges is None else list(charges)
        mults = [1] * n if multiplicities is None else list(multiplicities)
        if len(charges) != n or len(mults) != n:
            raise ValueError("charges and multiplicities must match the ragged batch size")
        self._calc = calculator
        self._closed = False
        # warm starts (reference python/generativeqc/batch.py:123-130,1376-1390):
        # the converged density of each item's last successful execution seeds
        # its next one; updates can be frozen for reproducible replays
        self._warm_start = bool(warm_start)
        self._warm_updates = True
        self._warm: list = [None] * len(systems)  # device (N, N) densities
        self._warm_origin: list = [None] * len(systems)  # "execution" or "checkpoint"
        self._source_coordinates: list = [None] * len(systems)  # where each density converged
        self.charges = tuple(int(q) for q in charges)
        self.multiplicities = tuple(int(m) for m in mults)
        self._molecules = []
        for atoms, q, m in zip(systems, charges, mults):
            mol = make_molecule(atoms, calculator.basis, calculator.auxiliary_basis, q, m)
            if calculator.method == "rhf" and (m != 1 or mol.nelectron % 2):
                raise NotImplementedError("RHF needs a closed-shell singlet (multiplicity 1, even electrons)")
            self._molecules.append(mol)
        self._unrestricted = calculator.method == "uhf"
        # homogeneous chunks: identical (nao, naux, n_alpha, n_beta), input order
        # kept inside a chunk
        groups: dict = {}
        from . import basis as bas

        for i, mol in enumerate(self._molecules):
            key = (bas.count_functions(mol.orbital_shells, calculator.spherical),
                   bas.count_functions(mol.aux_shells, calculator.spherical), mol.nalpha,
                   mol.nbeta)
            groups.setdefault(key, []).append(i)
        budget = calculator.memory_budget_bytes
        if budget <= 0:
            budget = int(0.6 * torch.cuda.get_device_properties(calculator.device).total_memory)
        self._chunks = []
        for (nao, naux, nocc, _nbeta), idx in sorted(groups.items()):
            prec = chunk_precision(calculator.precision, nao, nocc)
            per_mol = _device_bytes_per_molecule(nao, naux, prec, self._unrestricted)
            limit = max(1, budget // per_mol)
            for s in range(0, len(idx), limit):
                part = idx[s:s + limit]
                chunk = Chunk([self._molecules[i] for i in part], part, calculator.spherical)
                chunk.precision = prec
                self._chunks.append(chunk)
        self._natoms = [len(m.atomic_numbers) for m in self._molecules]
        self.atomic_numbers = tuple(tuple(int(z) for z in m.atomic_numbers) for m in self._molecules)

    @property
    def size(self) -> int:
        return len(self._molecules)

    def close(self) -> None:
        if not self._closed:
            for c in self._chunks:
                c.close()
            self._closed = True

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _coords_for(self, coordinates):
        if coordinates is None:
            return [m.coordinates for m in self._molecules]
        if len(coordinates) != len(self._molecules):
            raise ValueError("coordinates must give one array per system")
        out = []
        for i, c in enumerate(coordinates):
            if c is None:
                out.append(self._molecules[i].coordinates)
                continue
            arr = np.asarray(c, dtype=np.float64)
            if arr.shape != (self._natoms[i], 3):
                raise ValueError(f"system {i}: coordinates must have shape ({self._natoms[i]}, 3)")
            out.append(arr)
        return out

    # -- warm starts -------------------------------------------------------

    def set_warm_start_updates(self, enabled: bool) -> None:
        """Whether successful executions replace the retained densities.

        Disabling updates freezes the current snapshots (warm starts stay on),
        so every replay begins from the same densities.
        """
        self._warm_updates = bool(enabled)

    def clear_warm_starts(self) -> None:
        """Forget every retained density: the next execution starts cold."""
        self._warm = [None] * len(self._molecules)
        self._warm_origin = [None] * len(self._molecules)

    def warm_start_available(self, index: int) -> bool:
        return self._warm_start and self._warm[index] is not None

    def _chunk_warm(self, chunk):
        if not self._warm_start or all(self._warm[i] is None for i in chunk.indices):
            return None, None
        dev = self._calc.device
        n = chunk.nao
        shape = (chunk.nb, 2, n, n) if self._unrestricted else (chunk.nb, n, n)
        dens = torch.zeros(*shape, dtype=torch.float64, device=dev)
        mask = torch.zeros(chunk.nb, dtype=torch.bool, device=dev)
        for j, i in enumerate(chunk.indices):
            if self._warm[i] is not None:
                dens[j] = self._warm[i]
                mask[j] = True
        return dens, mask

    def _retain(self, chunk, density: torch.Tensor, converged, coords, skip=()) -> None:
        if not (self._warm_start and self._warm_updates):
            return
        for j, i in enumerate(chunk.indices):
            if bool(converged[j]) and i not in skip:
                self._warm[i] = density[j].detach().clone()
                self._warm_origin[i] = "execution"
                c = coords[i]
                self._source_coordinates[i] = (c.detach().cpu().numpy() if torch.is_tensor(c)
                                               else np.asarray(c, dtype=np.float64)).copy()

    def save_checkpoint(self, path, *, max_bytes: int = 256 << 20) -> dict:
        """Atomically write the retained densities (reference ``batch.py:1312``)."""
        from .checkpoint import save_checkpoint

        return save_checkpoint(self, path, max_bytes=max_bytes)

    def load_checkpoint(self, path, *, allow_warm: bool = False, strict: bool = True,
                        max_bytes: int = 256 << 20) -> dict:
        """Seed the next execution from a checkpoint (reference ``batch.py:1324``)."""
        from .checkpoint import load_checkpoint

        return load_checkpoint(self, path, allow_warm=allow_warm, strict=strict, max_bytes=max_bytes)

    def _run_chunk(self, chunk, xyz: torch.Tensor, want_forces: bool):
        """Integrals, SCF and (optionally) the gradient of one chunk, all on device."""
        calc = self._calc
        ints = compute_integrals(chunk.plan, xyz)
        warm_density, warm_mask = self._chunk_warm(chunk)
        schedule = tuning.active_table().lookup(chunk.nao, chunk.naux, chunk.nocc)
        driver = run_scf_uhf if self._unrestricted else run_scf
        out = driver(chunk, ints, xyz, precision=chunk.precision, schedule=schedule,
                      max_iterations=calc.max_iterations,
                      energy_tolerance=calc.energy_tolerance,
                      density_tolerance=calc.density_tolerance,
                      diis_history=calc.diis_history,
                      relative_threshold=calc.relative_threshold,
                      warm_density=warm_density, warm_mask=warm_mask)
        gradient = df_uhf_gradient if self._unrestricted else df_rhf_gradient
        grad = gradient(chunk, ints, out, xyz) if want_forces else None
        # keep only per-molecule results; the chunk's B tensor and factors go
        mf = out.pop("metric")
        slim = {k: out[k] for k in ("energy", "converged", "iterations", "energy_change",
                                    "density_rms", "density", "warm_used", "warm_fallback")}
        if self._unrestricted:
            # the retained warm-start state is the pair of spin densities
            slim["density"] = torch.stack(out["spin_densities"], dim=1)
        slim["metric_rank"] = mf.rank
        slim["metric_condition"] = mf.condition
        slim["metric_kind"] = mf.kind
        out.clear()
        del ints
        return slim, grad

    def upload_coordinates(self, coordinates=None) -> list:
        """Per-chunk device coordinate tensors (Bohr) for :meth:`execute_device`."""
        coords = self._coords_for(coordinates)
        return [
            torch.as_tensor(np.concatenate([coords[i] for i in c.indices], axis=0),
                            dtype=torch.float64).to(self._calc.device, non_blocking=True)
            for c in self._chunks
        ]

    def execute_device(self, xyz_chunks: list, *, want_forces: bool = True,
                       chunk_events: list | None = None) -> list:
        """Device-resident execution: inputs and outputs stay in HBM.

        Returns, per chunk, ``(scf_output_dict, gradient_or_None)`` with device
        tensors; no host copies are made.  With ``chunk_events`` (a list), a
        (shape, start event, end event) triple per chunk is appended for
        per-chunk device timing.
        """
        out = []
        with torch.cuda.device(self._calc.device):
            for c, x in zip(self._chunks, xyz_chunks):
                if chunk_events is not None:
                    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    s.record()
                out.append(self._run_chunk(c, x, want_forces))
                if chunk_events is not None:
                    e.record()
                    chunk_events.append(((c.nao, c.naux, c.nocc, c.nb), s, e))
        return out

    def execute_tensors(self, coordinates: list) -> tuple:
        """Energies and gradients for per-system coordinate tensors, on the device.

        Returns ``(energies (nsys,) FP64, [dE/dR (natoms, 3) FP64 per system])``
        on the calculator's device; raises if any system fails or does not
        converge (the autograd path needs every value).
        """
        if self._closed:
            raise RuntimeError("prepared batch is closed")
        if len(coordinates) != len(self._molecules):
            raise ValueError("coordinates must give one tensor per system")
        dev = self._calc.device
        energies = torch.empty(len(self._molecules), dtype=torch.float64, device=dev)
        grads: list = [None] * len(self._molecules)
        with torch.cuda.device(dev):
            for chunk in self._chunks:
                parts = []
                for i in chunk.indices:
                    c = coordinates[i].to(device=dev, dtype=torch.float64)
                    if tuple(c.shape) != (self._natoms[i], 3) or not bool(torch.isfinite(c).all()):
                        raise ValueError(f"system {i}: coordinates must be finite ({self._natoms[i]}, 3)")
                    parts.append(c)
                xyz = torch.cat(parts, dim=0).contiguous()
                out, g = self._run_chunk(chunk, xyz, True)
                if not bool(out["converged"].all()):
                    raise RuntimeError("SCF did not converge for a system of the batch")
                self._retain(chunk, out["density"], out["converged"].cpu().numpy(), coordinates)
                off = 0
                for j, i in enumerate(chunk.indices):
                    energies[i] = out["energy"][j]
                    grads[i] = g[off:off + self._natoms[i]]
                    off += self._natoms[i]
        return energies, grads

    def execute(self, coordinates=None, *, strict: bool = False,
                properties: Iterable[str] | None = None) -> BatchResult:
        if self._closed:
            raise RuntimeError("prepared batch is closed")
        props = {"energy", "forces"} if properties is None else set(properties)
        want_forces = "forces" in props
        coords = self._coords_for(coordinates)
        calc = self._calc
        items: list = [None] * len(self._molecules)
        dev = calc.device
        with torch.cuda.device(dev):
            for bucket, chunk in enumerate(self._chunks):
                # an item with non-finite coordinates fails alone: its slot in
                # the chunk computes the prepared geometry, its peers continue
                bad = {i for i in chunk.indices if not np.isfinite(coords[i]).all()}
                if len(bad) == len(chunk.indices):
                    for i in chunk.indices:
                        items[i] = _failed(i, bucket, STATUS_INVALID_ARGUMENT, "non-finite coordinates")
                    continue
                xyz_h = np.concatenate([self._molecules[i].coordinates if i in bad else coords[i]
                                        for i in chunk.indices], axis=0)
                xyz = torch.as_tensor(xyz_h, dtype=torch.float64).to(dev, non_blocking=True)
                try:
                    out, grad = self._run_chunk(chunk, xyz, want_forces)
                except (_lib.VqcError, FloatingPointError, torch.linalg.LinAlgError) as e:
                    status = getattr(e, "status", STATUS_NUMERICAL_FAILURE)
                    for i in chunk.indices:
                        items[i] = _failed(i, bucket, status, str(e))
                    continue
                energy = out["energy"].cpu().numpy()
                conv = out["converged"].cpu().numpy()
                iters = out["iterations"].cpu().numpy()
                de = out["energy_change"].cpu().numpy()
                drms = out["density_rms"].cpu().numpy()
                g = grad.cpu().numpy() if grad is not None else None
                used = out["warm_used"].cpu().numpy()
                fallback = out["warm_fallback"].cpu().numpy()
                self._retain(chunk, out["density"], conv, coords, skip=bad)
                off = 0
                for j, i in enumerate(chunk.indices):
                    na = self._natoms[i]
                    forces = None if g is None else -g[off:off + na].copy()
                    off += na
                    if i in bad:
                        items[i] = _failed(i, bucket, STATUS_INVALID_ARGUMENT, "non-finite coordinates")
                        continue
                    ok = bool(conv[j])
                    items[i] = BatchItemResult(
                        index=i,
                        status=STATUS_SUCCESS if ok else STATUS_NOT_CONVERGED,
                        status_message="success" if ok else "SCF did not converge",
                        energy=float(energy[j]),
                        forces=forces,
                        converged=ok,
                        iterations=int(iters[j]),
                        energy_change=float(de[j]),
                        density_rms=float(drms[j]),
                        executed_backend="cuda",
                        bucket_id=bucket,
                        warm_start_used=bool(used[j]),
                        warm_start_fallback=bool(fallback[j]),
                        basis_metadata={"nao": chunk.nao, "naux": chunk.naux,
                                        "metric_rank": int(out["metric_rank"][j]),
                                        "metric_condition": float(out["metric_condition"][j]),
                                        "metric_factor": out["metric_kind"]},
                        precision={"mode": chunk.precision, "requested": calc.precision},
                    )
        result = BatchResult(tuple(items))
        if strict:
            result.raise_for_failures()
        return result


# limits of the mixed-precision kernels: MMA N = round_up(n_occ, 16) <= 128 and
# FP32 B rows round_up(N, 4) <= 512 (Coulomb / fitted-density accumulators)
MIXED_MAX_NOCC = 128
MIXED_MAX_NAO = 512


def chunk_precision(requested: str, nao: int, nocc: int) -> str:
    """Precision a chunk runs in: "mixed" only inside the mixed kernels' limits.

    Molecules beyond them (more than 128 occupied orbitals or 512 basis
    functions) run the FP64 GPU path; each item's ``precision`` record says so.
    """
    if requested != "mixed":
        return requested
    if (nocc + 15) // 16 * 16 > MIXED_MAX_NOCC or (nao + 3) // 4 * 4 > MIXED_MAX_NAO:
        return "fp64"
    return "mixed"


def _device_bytes_per_molecule(nao: int, naux: int, precision: str,
                               unrestricted: bool = False) -> int:
    """Peak device bytes one molecule holds during a chunk (integrals to gradient)."""
    p = nao * (nao + 1) // 2
    # fp64: full FP64 B (16) + packed A during whitening / packed Abar (8) + K temporaries;
    # mixed: full FP64 B (16) + full FP32 B (8) + anchor/increment buffers of
    # N*o*X elements (~2o/N * 24 per packed element) + anchor temporaries;
    # the FP32 buffers are released before the packed Abar (8) is formed
    per_px = 30 if precision == "fp64" else 40
    if unrestricted:
        per_px += 8  # a second spin channel's anchor and U buffers
    return int(per_px * p * naux + 64 * nao * nao)


def _failed(i, bucket, status, msg) -> BatchItemResult:
    return BatchItemResult(i, status, msg, float("nan"), None, False, 0, float("nan"),
                           float("nan"), "cuda", bucket)
