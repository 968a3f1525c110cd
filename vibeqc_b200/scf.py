"""DF-RHF driver on the GPU: integrals -> metric factor -> whitened B -> SCF.

One :class:`Chunk` is a group of molecules with identical (N, X, n_occ) that
share one native plan and run their SCF iterations as batched device work
(the reference solves a homogeneous bucket with one batched plan,
``src/scf/rhf.cpp:2162``; ``src/scf/fleet.cpp:27-35`` buckets the batch).

SCF semantics follow ``src/scf/solver/mean_field_driver.cpp:233``: core-
Hamiltonian guess, F = H + J - K/2, E = 1/2 tr D(H + F) + E_nn, Pulay DIIS on
the orthogonalised commutator X^T (FDS - SDF) X with ``diis_history`` vectors,
and convergence when |dE| < energy_tolerance + 16 eps max(1, |E|, |E_old|),
rms(dD) < density_tolerance and max|FDS - SDF| <= min(1e-8, density_tolerance)
(``src/scf/cuda/scf_convergence_policy.cuh:18-37``, constants
``src/scf/cuda/scf_constants.hpp:16-17``).
"""

from __future__ import annotations

import os

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from . import jk as jkmod
from .plan import MoleculeSpec, NativePlan
from .timing import TIMER


def _stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


def _dptr(t: torch.Tensor) -> int:
    assert t.is_cuda and t.is_contiguous()
    return t.data_ptr()


@dataclass
class MoleculeResult:
    energy: float
    forces: np.ndarray | None
    converged: bool
    iterations: int
    energy_change: float
    density_rms: float
    status: int = 0
    status_message: str = "success"
    extra: dict = field(default_factory=dict)


@dataclass
class ChunkIntegrals:
    s: torch.Tensor       # (nb, N, N)
    h: torch.Tensor       # (nb, N, N)
    metric: torch.Tensor  # (nb, X, X)
    a_packed: torch.Tensor  # (nb, P, X)


def compute_integrals(plan: NativePlan, xyz: torch.Tensor) -> ChunkIntegrals:
    """Run the native integral kernels for every molecule of ``plan``."""
    lay = plan.layout
    nb = len(lay)
    n, x = lay[0].nao, lay[0].naux
    dev = xyz.device
    s = torch.empty(plan.mat_total, dtype=torch.float64, device=dev)
    t = torch.empty_like(s)
    v = torch.empty_like(s)
    m = torch.empty(plan.met_total, dtype=torch.float64, device=dev)
    a = torch.empty(plan.a_total, dtype=torch.float64, device=dev)
    st = _stream_ptr()
    with TIMER.stage("int1e"):
        _lib.call("vqc_int1e", plan.handle, _dptr(xyz), _dptr(s), _dptr(t), _dptr(v), st)
    with TIMER.stage("int2c"):
        _lib.call("vqc_int2c", plan.handle, _dptr(xyz), _dptr(m), st)
    with TIMER.stage("int3c"):
        _lib.call("vqc_int3c", plan.handle, _dptr(xyz), _dptr(a), st)
    p = n * (n + 1) // 2
    return ChunkIntegrals(
        s.view(nb, n, n), (t + v).view(nb, n, n), m.view(nb, x, x), a.view(nb, p, x)
    )


def nuclear_repulsion(z: torch.Tensor, xyz: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """E_nn and its gradient for one molecule (device tensors)."""
    d = xyz[:, None, :] - xyz[None, :, :]
    r = torch.linalg.norm(d, dim=-1)
    n = len(z)
    eye = torch.eye(n, dtype=torch.bool, device=xyz.device)
    zz = z[:, None] * z[None, :]
    inv = torch.where(eye, torch.zeros_like(r), 1.0 / torch.where(eye, torch.ones_like(r), r))
    e = 0.5 * (zz * inv).sum()
    g = -((zz * inv**3)[:, :, None] * d).sum(dim=1)
    return e, g


@dataclass
class MetricFactor:
    eigenvalues: torch.Tensor | None   # (nb, X); None for the Cholesky factor
    eigenvectors: torch.Tensor | None  # (nb, X, X)
    keep: torch.Tensor                 # (nb, X) bool
    inv_sqrt: torch.Tensor             # (nb, X, X) whitening W with W W^T = M^+
    rank: list
    condition: list                    # exact (eigen) or certified upper bound (Cholesky)
    kind: str = "eigen"
    chol: torch.Tensor | None = None   # (nb, X, X) lower Cholesky factor (kind "cholesky")


def factor_metric(metric: torch.Tensor, relative_threshold: float = 1e-10) -> MetricFactor:
    """FP64 whitening factor W (W W^T = M^+) with the reference's relative cutoff.

    The reference keeps eigenvectors with lambda > rel * lambda_max
    (``src/integrals/density_fitting_metric.cpp:101-154``; CUDA
    ``src/scf/cuda/df_plan_setup.cpp:595-726``).  When a rigorous certificate
    shows that no eigenvalue is cut -- lambda_min >= 1/tr(M^-1) exceeds
    rel * max_i sum_j |M_ij| >= rel * lambda_max -- the eigen factor and the
    Cholesky factor W = L^-T span the same fitting space and give identical
    J, K, energies and forces, so the cheaper Cholesky factor is used.
    Otherwise the eigen factor with the cutoff is formed.
    """
    if not torch.isfinite(metric).all():
        raise FloatingPointError("non-finite metric")
    m = 0.5 * (metric + metric.transpose(1, 2))
    nb, x, _ = m.shape
    l, info = torch.linalg.cholesky_ex(m)
    if bool((info == 0).all()):
        eye = torch.eye(x, dtype=m.dtype, device=m.device).expand(nb, x, x)
        linv = torch.linalg.solve_triangular(l, eye, upper=False)
        lam_min_lower = 1.0 / (linv * linv).sum(dim=(1, 2))
        lam_max_upper = m.abs().sum(dim=2).max(dim=1).values
        if bool((lam_min_lower > relative_threshold * lam_max_upper).all()):
            w = linv.transpose(1, 2).contiguous()
            keep = torch.ones(nb, x, dtype=torch.bool, device=m.device)
            cond = (lam_max_upper / lam_min_lower).tolist()
            return MetricFactor(None, None, keep, w, [x] * nb, cond, "cholesky", l)
    lam, vec = torch.linalg.eigh(m)
    lmax = lam[:, -1:]
    keep = lam > relative_threshold * lmax
    scale = torch.where(keep, 1.0 / torch.sqrt(torch.where(keep, lam, torch.ones_like(lam))),
                        torch.zeros_like(lam))
    inv_sqrt = (vec * scale[:, None, :]) @ vec.transpose(1, 2)
    rank = keep.sum(dim=1).tolist()
    lmin = torch.where(keep, lam, torch.full_like(lam, float("inf"))).min(dim=1).values
    cond = (lmax[:, 0] / lmin).tolist()
    return MetricFactor(lam, vec, keep, inv_sqrt, rank, cond, "eigen")


# energy-change roundoff allowance of the reference's stopping rule:
# 16 * DBL_EPSILON * max(1, |E|, |E_old|)
ENERGY_ROUNDOFF_FACTOR = 16.0
DOUBLE_EPS = 2.220446049250313e-16

MIXED_ITERATION_CAP = 40  # plain tensor-core iterations before the anchor is forced
ANCHOR_COMMUTATOR = 1e-5  # max|FDS - SDF| at which the FP64 anchor is formed
ANCHOR_DIIS_RESET = False  # restart DIIS at the anchor
# anchored builds after which a chunk that has not converged is re-anchored
# (a fresh FP64 build at the current density): the increments' split-precision
# error scales with |D - D0|, so a stalled chunk converges to FP64 noise
REANCHOR_EVERY = 8


def exact_energy(jk, d: torch.Tensor, c: torch.Tensor, h: torch.Tensor,
                 enuc: torch.Tensor) -> torch.Tensor:
    """E = tr(D H) + |rho|^2 / 2 - sum_{Q,i,j} (C^T B_Q C)_{ij}^2 + E_nn in FP64 arithmetic."""
    rho, u = jk.half_transform(c)
    e1 = torch.einsum("bmn,bmn->b", d, h)
    ej = 0.5 * (rho * rho).sum(dim=1)
    ek = torch.zeros_like(ej)
    for m in range(d.shape[0]):
        bij = torch.einsum("mi,mjq->qij", c[m], u[m])
        ek[m] = -(bij * bij).sum()
    return e1 + ej + ek + enuc, (rho, u)


class Chunk:
    """A homogeneous group of molecules sharing one native plan."""

    def __init__(self, molecules: list[MoleculeSpec], indices: list[int], spherical: bool = True):
        self.molecules = molecules
        self.indices = indices
        self.plan = NativePlan(molecules, spherical)
        lay = self.plan.layout
        self.nb = len(molecules)
        self.nao, self.naux, self.nocc = lay[0].nao, lay[0].naux, lay[0].nocc
        for l_ in lay:
            if (l_.nao, l_.naux, l_.nocc) != (self.nao, self.naux, self.nocc):
                raise ValueError("a chunk must be homogeneous in (N, X, n_occ)")
        self.natoms = [len(m.atomic_numbers) for m in molecules]
        spins = {(m.nalpha, m.nbeta) for m in molecules}
        if len(spins) != 1:
            raise ValueError("a chunk must be homogeneous in (n_alpha, n_beta)")
        self.nalpha, self.nbeta = spins.pop()
        self.precision = "fp64"  # set by the prepared batch from the requested precision

    def close(self):
        self.plan.close()


def _orthogonalizer(s: torch.Tensor) -> torch.Tensor:
    """X with X^T S X = I: inverse transposed Cholesky factor (eigen fallback)."""
    l, info = torch.linalg.cholesky_ex(s)
    if bool((info == 0).all()):
        eye = torch.eye(s.shape[-1], dtype=s.dtype, device=s.device).expand_as(s)
        return torch.linalg.solve_triangular(l, eye, upper=False).transpose(1, 2)
    lam, vec = torch.linalg.eigh(s)
    return (vec * lam.rsqrt()[:, None, :]) @ vec.transpose(1, 2)


SP2_GRAPH_STEPS = 8  # SP2 steps per captured CUDA graph (even: ends in the same buffer)
SP2_SLICES = 7  # 7-bit slices per operand of the int8 tensor-core X^2 (FP64-accurate products)
# native kernels launched by graph replays (the library's own launch counter
# sees only direct launches)
GRAPH_LAUNCHES = [0]


class _SP2Graph:
    """SP2_GRAPH_STEPS SP2 steps (X^2 + vqc_sp2_update) as one CUDA graph.

    The iterate lives in static buffers; converged molecules are copied
    unchanged by the update kernel, so extra steps are harmless and the host
    reads the device flags once per replay.  ``gemm`` selects how X^2 is
    formed: "fp64" (batched DGEMM) or "int8" (FP64-accurate products of
    SP2_SLICES 7-bit slices on the int8 tensor cores, vqc_ozaki_slice_rows +
    vqc_ozaki_gemm; X is symmetric, so X X^T = X^2, and the sliced product is
    exactly symmetric because both operands carry the same slices).
    """

    def __init__(self, nb: int, n: int, nocc: int, tol: float, device, steps: int = SP2_GRAPH_STEPS,
                 gemm: str = "fp64"):
        self.steps = int(steps)
        self.gemm = gemm
        self.x = torch.zeros(nb, n, n, dtype=torch.float64, device=device)
        self.x2 = torch.empty_like(self.x)
        self.xn = torch.empty_like(self.x)
        self.done = torch.zeros(nb, dtype=torch.int32, device=device)
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        if gemm == "int8":
            self.ldk = (n + 15) // 16 * 16
            self.sl = torch.zeros(nb * SP2_SLICES * n * self.ldk, dtype=torch.int8, device=device)
            self.ex = torch.zeros(nb * n, dtype=torch.int32, device=device)
        self.args = (nb, n, float(nocc), float(tol))
        self.graph = None
        if os.environ.get("VQC_SP2_GRAPHS", "1") == "0":
            return  # eager launches (e.g. under a kernel profiler)
        side = torch.cuda.Stream(device=device)
        side.wait_stream(torch.cuda.current_stream(device))
        with torch.cuda.stream(side):  # warm-up outside capture (cuBLAS handles, workspaces)
            self._steps()
        torch.cuda.current_stream(device).wait_stream(side)
        try:
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                self._steps()
            self.graph = graph
        except Exception:  # a capture the runtime refuses: run the same launches eagerly
            torch.cuda.synchronize(device)
            self.graph = None

    def run(self):
        """``steps`` steps: one graph replay, or eager launches."""
        if self.graph is not None:
            self.graph.replay()
            GRAPH_LAUNCHES[0] += self.steps * (3 if self.gemm == "int8" else 1)
        else:
            self._steps()

    def _square(self, x):
        nb, n = self.args[0], self.args[1]
        if self.gemm != "int8":
            torch.bmm(x, x, out=self.x2)
            return
        st = torch.cuda.current_stream().cuda_stream
        _lib.call("vqc_ozaki_slice_rows", x.data_ptr(), nb, n, n, n, n * n, None, SP2_SLICES,
                  self.sl.data_ptr(), self.ldk, self.ex.data_ptr(), st)
        # symmetric output: only the tiles on or above the diagonal, mirrored
        _lib.call("vqc_ozaki_gemm", self.sl.data_ptr(), self.ex.data_ptr(), n, self.sl.data_ptr(),
                  self.ex.data_ptr(), n, n, self.ldk, nb, SP2_SLICES, 2, self.x2.data_ptr(), n, n * n,
                  self.err.data_ptr(), st)

    def _steps(self):
        nb, n, nocc, tol = self.args
        st = torch.cuda.current_stream().cuda_stream
        x, xn = self.x, self.xn
        for _ in range(self.steps):
            self._square(x)
            _lib.call("vqc_sp2_update", x.data_ptr(), self.x2.data_ptr(), xn.data_ptr(), nb, n,
                      nocc, tol, self.done.data_ptr(), st)
            x, xn = xn, x


# captured SP2 graphs by (chunk shape, n_occ, tolerance, device); kept for the
# process so repeated executions of a prepared batch replay them
_SP2_GRAPHS: dict = {}
SP2_GRAPH_CACHE_BYTES = 4 << 30  # drop the cache when its buffers would exceed this


def purify_sp2(fo: torch.Tensor, nocc: int, max_steps: int = 96, tol: float = 1e-11,
               graphs: dict | None = None, steps: int = SP2_GRAPH_STEPS,
               gemm: str = "fp64") -> torch.Tensor:
    """Projector onto the lowest ``nocc`` eigenvectors of symmetric ``fo``.

    Second-order spectral projection (Niklasson, Phys. Rev. B 66, 155115
    (2002)): map the spectrum into [0, 1] with Gershgorin bounds, then apply
    X <- X^2 or X <- 2X - X^2, whichever moves tr X toward ``nocc``, until
    tr(X) - tr(X^2) < tol.  Per step: one batched GEMM and one native update
    kernel (vqc_sp2_update); convergence flags stay on the device.  Steps run
    in CUDA graphs of SP2_GRAPH_STEPS (cached in ``graphs``, one per shape and
    tolerance), and the flags are read once per graph replay.  ``steps`` (even)
    is the number of steps per graph and ``gemm`` the X^2 product ("fp64"
    DGEMM or "int8" sliced tensor-core products), both autotuned schedule
    choices.
    """
    nb, n, _ = fo.shape
    diag = torch.diagonal(fo, dim1=1, dim2=2)
    radius = fo.abs().sum(dim=2) - diag.abs()
    emin = (diag - radius).min(dim=1).values
    emax = (diag + radius).max(dim=1).values
    eye = torch.eye(n, dtype=fo.dtype, device=fo.device)
    key = (nb, n, int(nocc), float(tol), str(fo.device), int(steps), gemm)
    if graphs is None:
        graphs = {}
    g = graphs.get(key)
    if g is None:
        held = sum(3 * v.x.numel() * 8 for v in graphs.values())
        if held + 3 * nb * n * n * 8 > SP2_GRAPH_CACHE_BYTES:
            graphs.clear()
        g = graphs[key] = _SP2Graph(nb, n, nocc, tol, fo.device, steps, gemm)
    torch.div(emax[:, None, None] * eye - fo, (emax - emin)[:, None, None], out=g.x)
    g.done.zero_()
    for _ in range(0, max_steps, int(steps)):
        g.run()
        if bool(g.done.all()):
            break
    if gemm == "int8" and int(g.err.item()) != 0:
        raise _lib.VqcError(6, f"tensor-core purification wait expired (code {int(g.err.item())})")
    return 0.5 * (g.x + g.x.transpose(1, 2))


def _cholqr2(y: torch.Tensor):
    """Two Cholesky-QR passes (orthonormal columns); ok[b] False where a Gram factor failed."""
    ok = torch.ones(y.shape[0], dtype=torch.bool, device=y.device)
    eye = torch.eye(y.shape[-1], dtype=y.dtype, device=y.device)
    for _ in range(2):
        g = torch.bmm(y.transpose(1, 2), y)
        u, info = torch.linalg.cholesky_ex(g, upper=True)
        ok &= info == 0
        u = torch.where((info == 0)[:, None, None], u, eye)
        y = torch.linalg.solve_triangular(u, y, upper=True, left=False)
    return y, ok


class _OccGraph:
    """proj @ (guess + scale * noise) made orthonormal, as one CUDA graph per shape."""

    def __init__(self, nb: int, n: int, o: int, scale: float, device):
        f64 = dict(dtype=torch.float64, device=device)
        self.proj = torch.zeros(nb, n, n, **f64)
        self.guess = torch.zeros(nb, n, o, **f64)
        self.noise = torch.zeros(nb, n, o, **f64)
        self.scale = scale
        self.out = None
        self.graph = None
        self.guess[:, :o, :] = torch.eye(o, **f64)[None]  # well-posed warm-up input
        self.proj[:, :, :] = torch.eye(n, **f64)[None]
        if _graphs_enabled() and torch.device(device).type == "cuda":
            try:
                side = torch.cuda.Stream(device=device)
                side.wait_stream(torch.cuda.current_stream(device))
                with torch.cuda.stream(side):
                    self._step()
                torch.cuda.current_stream(device).wait_stream(side)
                graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(graph):
                    self.out = self._step()
                self.graph = graph
            except Exception:  # a capture the runtime refuses: run the same ops eagerly
                torch.cuda.synchronize(device)
                self.graph = None

    def _step(self):
        return _cholqr2(torch.bmm(self.proj, self.guess + self.scale * self.noise))

    def run(self, proj, guess, gen):
        self.proj.copy_(proj)
        self.guess.copy_(guess)
        torch.randn(self.noise.shape, dtype=self.noise.dtype, device=self.noise.device,
                    generator=gen, out=self.noise)
        if self.graph is not None:
            self.graph.replay()
            y, ok = self.out
            return y.clone(), ok
        return self._step()


_OCC: dict = {}


def occupied_factor(proj: torch.Tensor, guess: torch.Tensor, gen: torch.Generator,
                    noise_scale: float = 0.3) -> torch.Tensor:
    """Orthonormal basis of range(proj) by Cholesky-QR2 of proj @ (guess + noise).

    The previous occupied factor plus a random component keeps proj @ guess
    full rank even when the occupied space rotates far between iterations;
    a molecule whose factorisation still fails is retried with a purely random
    start.  With ``noise_scale=0`` the result is the projected guess made
    orthonormal, so it stays within O(|proj - guess guess^T|) of ``guess``.
    The first attempt runs as a cached CUDA graph per (shape, noise scale).
    """
    nb, n, o = guess.shape
    key = (nb, n, o, float(noise_scale), str(guess.device))
    og = _OCC.get(key)
    if og is None:
        if len(_OCC) > 64:
            _OCC.clear()
        og = _OCC[key] = _OccGraph(nb, n, o, float(noise_scale), guess.device)
    y, ok = og.run(proj, guess, gen)
    if bool(ok.all()):
        return y
    # retry the failed molecules from a purely random start
    noise = og.noise.clone()
    start = torch.where(ok[:, None, None], guess + noise_scale * noise, noise)
    y, ok = _cholqr2(torch.bmm(proj, start))
    if bool(ok.all()):
        return y
    raise FloatingPointError("occupied-space factorisation failed")


WHITEN_COLUMN_BLOCK = 256
# the mixed path whitens on the int8 tensor cores (whiten_tensor_cores); the
# FP64 comparator path keeps plain FP64 GEMMs (whiten_in_place)
WHITEN_TENSOR_CORES = os.environ.get("VQC_WHITEN_TC", "1") != "0"


def whiten_in_place(a: torch.Tensor, mf: MetricFactor) -> None:
    """B = A W over the packed rows of every molecule, in place (FP64 GEMMs).

    Row blocks of all molecules of the chunk go through batched GEMMs with
    bounded temporaries.  The Cholesky factor W = L^-T is upper triangular, so
    column block [c0, c1) of B needs only columns < c1 of A: blocks are formed
    right to left (each reads columns that are still unwhitened), which skips
    the structural zeros of W and halves the flops of the dense product.
    """
    nb, p_rows, x = a.shape
    w = mf.inv_sqrt
    cb = WHITEN_COLUMN_BLOCK
    # rows are views; only the (nb, blk, cb) product block is a temporary
    # (~512 MB), so the GEMMs are tall enough to run near the FP64 peak
    blk = max(256, (1 << 29) // (8 * max(cb, 1) * nb))
    if mf.kind != "cholesky":
        blk = max(256, (1 << 29) // (8 * x * nb))
    for r0 in range(0, p_rows, blk):
        rows = a[:, r0:r0 + blk]
        if mf.kind != "cholesky":
            rows.copy_(torch.matmul(rows, w))
            continue
        for c0 in range(((x - 1) // cb) * cb, -1, -cb):
            c1 = min(x, c0 + cb)
            rows[:, :, c0:c1].copy_(torch.matmul(rows[:, :, :c1], w[:, :c1, c0:c1]))


OZAKI_SLICES = 7  # 7-bit int8 slices per FP64 operand of the tensor-core whitening
OZAKI_GROUP_BYTES = 4 << 30  # bound on the A-slice workspace (rows are sliced in groups)
OZAKI_STATS = {"launches": 0, "int8_macs": 0}  # tensor-core whitening work since process start


def whiten_tensor_cores(a: torch.Tensor, mf: MetricFactor, metric: torch.Tensor) -> None:
    """B = A W over the packed rows of every molecule, in place, on the int8 tensor cores.

    FP64 accuracy from exact integer pieces (vqc_ozaki_slice_rows /
    vqc_ozaki_gemm): rows of A and columns of W are scaled by powers of two
    and cut into OZAKI_SLICES 7-bit slices; the slice products accumulate
    exactly in int32 and only their FP64 recombination rounds.  Before
    slicing, A W = (A S)(S^-1 W) with S_i = 2^round(log2 sqrt(max_c |W_ic| /
    sqrt(M_ii))) balances the column scale of A (|(mu nu|P)| <= sqrt((mu nu|mu nu)
    M_PP) by the Schwarz inequality) against the row scale of W; powers of two
    keep the rescaling exact.  With the Cholesky factor W = L^-T is upper
    triangular and each output column tile reads only the rows of W above it.
    The rows of A are sliced and multiplied in groups (slice workspace <=
    OZAKI_GROUP_BYTES); a group's FP64 rows are overwritten only after they
    were sliced.  Relative error ~1e-11 of each row's largest element at 7
    slices; the resulting Coulomb/exchange energies differ from the FP64
    product by ~1e-11 of their size.
    """
    nb, p_rows, x = a.shape
    dev = a.device
    ns = OZAKI_SLICES
    w = mf.inv_sqrt
    diag = torch.diagonal(metric, dim1=1, dim2=2).clamp_min(1e-300)
    wmax = w.abs().amax(dim=2).clamp_min(1e-300)
    scale = torch.exp2(torch.round(0.5 * (torch.log2(wmax) - 0.5 * torch.log2(diag)))).contiguous()
    wt = (w / scale[:, :, None]).transpose(1, 2).contiguous()  # [c][i] = W[i][c] / S_i
    ldk = (x + 15) // 16 * 16
    st = _stream_ptr()
    b_sl = torch.empty(nb, ns, x, ldk, dtype=torch.int8, device=dev)
    b_exp = torch.empty(nb, x, dtype=torch.int32, device=dev)
    _lib.call("vqc_ozaki_slice_rows", wt.data_ptr(), nb, x, x, x, x * x, None, ns, b_sl.data_ptr(),
              ldk, b_exp.data_ptr(), st)
    del wt
    grp = max(128, (OZAKI_GROUP_BYTES // (nb * ns * ldk)) // 128 * 128)
    grp = min(grp, p_rows)
    a_sl = torch.empty(nb * ns * grp * ldk, dtype=torch.int8, device=dev)
    a_exp = torch.empty(nb * grp, dtype=torch.int32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    upper = 1 if mf.kind == "cholesky" else 0
    assert a.is_contiguous()
    for r0 in range(0, p_rows, grp):
        m = min(p_rows, r0 + grp) - r0
        base = a.data_ptr() + r0 * x * 8
        _lib.call("vqc_ozaki_slice_rows", base, nb, m, x, x, p_rows * x, scale.data_ptr(), ns,
                  a_sl.data_ptr(), ldk, a_exp.data_ptr(), st)
        _lib.call("vqc_ozaki_gemm", a_sl.data_ptr(), a_exp.data_ptr(), m, b_sl.data_ptr(),
                  b_exp.data_ptr(), x, x, ldk, nb, ns, upper, base, x, p_rows * x, err.data_ptr(), st)
        OZAKI_STATS["launches"] += 2
        OZAKI_STATS["int8_macs"] += nb * m * x * x * ns * (ns + 1) // 2 // (2 if upper else 1)
    if int(err.item()) != 0:
        raise _lib.VqcError(6, f"tensor-core whitening wait expired (code {int(err.item())})")


def _graphs_enabled() -> bool:
    return (os.environ.get("VQC_CUDA_GRAPHS", "1") != "0"
            and os.environ.get("VQC_SP2_GRAPHS", "1") != "0")


class _SCFPost:
    """Fock, energy, commutator and DIIS extrapolation of one SCF iteration.

    Everything between a J/K build and the density update runs on static
    buffers and, when CUDA graphs are enabled, as one captured graph: the
    per-iteration work is ~25 small kernels whose host dispatch cost more
    than their GPU time.  DIIS keeps its error and Fock vectors in a ring of
    ``hist`` slots with an incrementally updated Gram matrix; slots not yet
    filled get identity rows in the Pulay system, so their weights are
    exactly zero and the extrapolation equals the usual one over the last
    ``min(count, hist)`` iterations (the order of the vectors does not
    matter).  ``with_rho`` selects the energy formula of the anchored phase,
    E = tr(DH) + |rho|^2/2 - tr(DK)/4 + E_nn, instead of tr(D(H+F))/2 + E_nn.
    """

    def __init__(self, nb: int, n: int, x: int, hist: int, with_rho: bool, device):
        f64 = dict(dtype=torch.float64, device=device)
        self.h, self.s, self.xo = (torch.zeros(nb, n, n, **f64) for _ in range(3))
        self.enuc = torch.zeros(nb, **f64)
        self.j, self.k, self.d = (torch.zeros(nb, n, n, **f64) for _ in range(3))
        self.rho = torch.zeros(nb, x, **f64)
        self.e_ring = torch.zeros(nb, hist, n, n, **f64)
        self.f_ring = torch.zeros(nb, hist, n, n, **f64)
        self.gram = torch.zeros(nb, hist, hist, **f64)
        self.count = torch.zeros(1, dtype=torch.int64, device=device)
        self.hist, self.with_rho = hist, with_rho
        self.eye = torch.eye(hist, **f64)
        self.out = None
        self.graph = None
        if _graphs_enabled() and torch.device(device).type == "cuda":
            try:
                side = torch.cuda.Stream(device=device)
                side.wait_stream(torch.cuda.current_stream(device))
                with torch.cuda.stream(side):  # warm-up outside capture
                    self._step()
                torch.cuda.current_stream(device).wait_stream(side)
                self.reset()
                graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(graph):
                    self.out = self._step()
                self.graph = graph
            except Exception:  # a capture the runtime refuses: run the same ops eagerly
                torch.cuda.synchronize(device)
                self.graph = None
        self.reset()

    def reset(self) -> None:
        self.count.zero_()
        self.gram.zero_()

    def load(self, h, s, xo, enuc) -> None:
        self.h.copy_(h)
        self.s.copy_(s)
        self.xo.copy_(xo)
        self.enuc.copy_(enuc)
        # empty slots carry weight 0; zeros keep a previous chunk's values out
        self.e_ring.zero_()
        self.f_ring.zero_()
        self.reset()

    def _step(self):
        hist = self.hist
        f = self.h + self.j - 0.5 * self.k
        if self.with_rho:
            energy = (torch.einsum("bmn,bmn->b", self.d, self.h)
                      + 0.5 * (self.rho * self.rho).sum(dim=1)
                      - 0.25 * torch.einsum("bmn,bmn->b", self.d, self.k) + self.enuc)
        else:
            energy = 0.5 * torch.einsum("bmn,bmn->b", self.d, self.h + f) + self.enuc
        fds = f @ self.d @ self.s
        comm = fds - fds.transpose(1, 2)
        cmax = comm.abs().amax(dim=(1, 2))
        err = self.xo.transpose(1, 2) @ comm @ self.xo
        slot = torch.remainder(self.count, hist)
        self.e_ring.index_copy_(1, slot, err[:, None])
        self.f_ring.index_copy_(1, slot, f[:, None])
        g_new = torch.einsum("bmn,bhmn->bh", err, self.e_ring)
        self.gram.index_copy_(1, slot, g_new[:, None, :])
        self.gram.index_copy_(2, slot, g_new[:, :, None])
        self.count.add_(1)
        valid = torch.arange(hist, device=self.count.device) < torch.clamp(self.count, max=hist)
        vf = valid.to(torch.float64)
        pair = vf[:, None] * vf[None, :]
        nb = f.shape[0]
        bmat = torch.zeros(nb, hist + 1, hist + 1, dtype=torch.float64, device=f.device)
        bmat[:, :hist, :hist] = self.gram * pair + self.eye * (1.0 - vf)[None, :, None]
        bmat[:, hist, :hist] = -vf
        bmat[:, :hist, hist] = -vf
        rhs = torch.zeros(nb, hist + 1, 1, dtype=torch.float64, device=f.device)
        rhs[:, hist, 0] = -1.0
        w, info = torch.linalg.solve_ex(bmat, rhs)
        w = w[:, :hist, 0] * vf
        ok = (info == 0) & torch.isfinite(w).all(dim=1)
        ext = torch.einsum("bh,bhmn->bmn", w, self.f_ring)
        f_ext = torch.where(ok[:, None, None], ext, f)
        return f, energy, cmax, f_ext

    def run(self, j, k, d, rho=None):
        """(F, energy, max|FDS - SDF|, extrapolated F); outputs are overwritten next call."""
        self.j.copy_(j)
        self.k.copy_(k)
        self.d.copy_(d)
        if rho is not None:
            self.rho.copy_(rho)
        if self.graph is not None:
            self.graph.replay()
            return self.out
        return self._step()


_POST: dict = {}
POST_CACHE_BYTES = 4 << 30
POST_STATS = {"graphs": 0, "eager": 0}  # how the cached post-build blocks run


def _scf_post(nb, n, x, hist, with_rho, device) -> _SCFPost:
    key = (nb, n, x, hist, with_rho, str(device))
    p = _POST.get(key)
    if p is None:
        held = sum(2 * v.e_ring.numel() * 8 for v in _POST.values())
        if held + 2 * nb * hist * n * n * 8 > POST_CACHE_BYTES:
            _POST.clear()
        p = _POST[key] = _SCFPost(nb, n, x, hist, with_rho, device)
        POST_STATS["graphs" if p.graph is not None else "eager"] += 1
    return p


def run_scf(chunk: Chunk, ints: ChunkIntegrals, xyz: torch.Tensor, *, precision: str = "fp64",
            max_iterations: int = 100, energy_tolerance: float = 1e-10,
            density_tolerance: float = 1e-8, diis_history: int = 8,
            relative_threshold: float = 1e-10, trace: list | None = None,
            warm_density: torch.Tensor | None = None,
            warm_mask: torch.Tensor | None = None, schedule=None) -> dict:
    """Batched SCF over one chunk; returns device tensors per molecule.

    ``warm_density`` (nb, N, N) with ``warm_mask`` (nb,) bool: molecules whose
    mask is set start from the occupied space of that density (a converged
    density of an earlier execution, possibly at another geometry) instead of
    the core-Hamiltonian guess -- the same purification as the cold guess,
    applied to F0 = -S D S / 2, whose lowest n_occ eigenvectors span the
    S-orthogonalised occupied space of D.  A non-finite warm density falls
    back to the cold guess (``warm_fallback``).  ``schedule`` (a
    ``tuning.Schedule``, default the untuned one) picks the whitening
    kernels of the mixed path, the SP2 steps per graph and the Gram split.
    """
    from .tuning import DEFAULT, apply_library_knobs

    sched = DEFAULT if schedule is None else schedule
    apply_library_knobs(sched)
    nb, n, x, nocc = chunk.nb, chunk.nao, chunk.naux, chunk.nocc
    dev = xyz.device
    with TIMER.stage("metric_factor"):
        mf = factor_metric(ints.metric, relative_threshold)
    with TIMER.stage("whiten"):
        b_packed = ints.a_packed  # whitened in place: B = A W
        ints.a_packed = None  # the raw tensor is not needed after whitening
        if precision == "mixed" and WHITEN_TENSOR_CORES and sched.whiten == "int8":
            whiten_tensor_cores(b_packed, mf, ints.metric)
        else:
            whiten_in_place(b_packed, mf)
        jk = jkmod.make_builder(precision, b_packed, n, x, nocc)
        del b_packed
    s, h = ints.s, ints.h
    xo = _orthogonalizer(s)
    enuc = []
    off = 0
    zs = []
    for i, mol in enumerate(chunk.molecules):
        na = chunk.natoms[i]
        z = torch.as_tensor(mol.atomic_numbers, dtype=torch.float64, device=dev)
        e, _ = nuclear_repulsion(z, xyz[off:off + na])
        enuc.append(e)
        zs.append(z)
        off += na
    enuc = torch.stack(enuc)

    gen = torch.Generator(device=dev)
    gen.manual_seed(1234)
    guess = torch.randn(nb, n, nocc, dtype=torch.float64, device=dev, generator=gen)

    sp2_graphs = _SP2_GRAPHS
    # the FP64 comparator path keeps plain DGEMMs; the mixed path may take
    # the sliced tensor-core products (FP64-accurate as well)
    sp2_gemm = sched.sp2_gemm if precision == "mixed" else "fp64"

    def density_from(f, guess, tol=1e-11, noise_scale=0.3):
        with TIMER.stage("purify"):
            proj = purify_sp2(xo.transpose(1, 2) @ f @ xo, nocc, tol=tol, graphs=sp2_graphs,
                              steps=sched.sp2_steps, gemm=sp2_gemm)
        with TIMER.stage("occupied_factor"):
            co = occupied_factor(proj, guess, gen, noise_scale)  # orthonormal, orthogonal basis
        return 2.0 * (xo @ proj @ xo.transpose(1, 2)), co

    warm_used = torch.zeros(nb, dtype=torch.bool, device=dev)
    warm_fallback = torch.zeros(nb, dtype=torch.bool, device=dev)
    f0 = h
    if warm_density is not None and warm_mask is not None and bool(warm_mask.any()):
        finite = torch.isfinite(warm_density).flatten(1).all(dim=1)
        warm_used = warm_mask & finite
        warm_fallback = warm_mask & ~finite
        wd = torch.where(warm_used[:, None, None], warm_density, torch.zeros_like(h))
        f0 = torch.where(warm_used[:, None, None], -0.5 * (s @ wd @ s), h)
    d, co = density_from(f0, guess)
    c = xo @ co  # AO occupied factor, D = 2 C C^T
    active = torch.ones(nb, dtype=torch.bool, device=dev)
    e_old = torch.full((nb,), float("nan"), dtype=torch.float64, device=dev)
    final_e = torch.zeros(nb, dtype=torch.float64, device=dev)
    final_de = torch.full((nb,), float("inf"), dtype=torch.float64, device=dev)
    final_drms = torch.full((nb,), float("inf"), dtype=torch.float64, device=dev)
    iters = torch.zeros(nb, dtype=torch.int64, device=dev)
    converged = torch.zeros(nb, dtype=torch.bool, device=dev)
    d_final = d.clone()
    c_final = c.clone()
    f_final = torch.zeros_like(d)
    post = None
    comm_tol = min(1e-8, density_tolerance)
    # mixed precision runs two phases per chunk:
    #   "tc":     plain tensor-core J/K until max|FDS-SDF| <= ANCHOR_COMMUTATOR
    #             for every active molecule (or MIXED_ITERATION_CAP).  Their
    #             split-precision error (~1e-7 relative, varying with D) makes
    #             the energy jitter, so no convergence test runs here.
    #   "anchor": one FP64 J/K build at the current density, then tensor-core
    #             increments about it (MixedBuilder.build_incremental) with the
    #             occupied factor aligned to the anchor's; the operators are
    #             FP64-accurate and the reference's criteria apply.
    # the FP64 path runs "exact" FP64 builds throughout.
    phase = "tc" if jk.precision == "mixed" else "exact"
    mixed_iterations = 0
    phase_iterations = 0
    co_anchor = None
    anchored = False
    anchor_builds = 0
    anchors = 0
    for it in range(1, max_iterations + 1):
        rho = None
        if phase == "exact":
            j, k = jk.build_exact(d, c)
        elif phase == "anchor":
            if anchored and anchor_builds >= REANCHOR_EVERY:
                anchored, co_anchor, anchor_builds = False, None, 0
            if not anchored:
                j, k, rho = jk.anchor(d, c)
                anchored = True
                anchors += 1
            else:
                j, k, rho = jk.build_incremental(d, c)
                mixed_iterations += 1
                anchor_builds += 1
        else:
            j, k = jk.build(d, c)
            mixed_iterations += 1
        phase_iterations += 1
        TIMER_ctx = TIMER.stage("scf_other")
        TIMER_ctx.__enter__()
        # Fock, energy, commutator, DIIS: one captured graph per (shape, formula);
        # the anchored phase (E from the FP64-accurate rho and K) has its own,
        # which continues the DIIS history of the tensor-core phase
        with_rho = rho is not None
        if post is None or post.with_rho != with_rho:
            prev = post
            post = _scf_post(nb, n, x, diis_history, with_rho, dev)
            post.load(h, s, xo, enuc)
            if prev is not None and not ANCHOR_DIIS_RESET:
                post.e_ring.copy_(prev.e_ring)
                post.f_ring.copy_(prev.f_ring)
                post.gram.copy_(prev.gram)
                post.count.copy_(prev.count)
        f, energy, cmax, f_ext = post.run(j, k, d, rho)
        energy = energy.clone()
        TIMER_ctx.__exit__(None, None, None)
        # the tensor-core phase only needs the projector to its own accuracy
        if phase == "anchor":
            if co_anchor is None:
                co_anchor = co
            d_new, co = density_from(f_ext, co_anchor, 1e-11, 0.0)
        else:
            d_new, co = density_from(f_ext, co, 1e-11 if phase == "exact" else 1e-8)
        TIMER_ctx = TIMER.stage("scf_other")
        TIMER_ctx.__enter__()
        c_new = xo @ co
        de = (energy - e_old).abs()
        de = torch.where(torch.isnan(de), torch.full_like(de, float("inf")), de)
        drms = ((d_new - d) ** 2).mean(dim=(1, 2)).sqrt()
        guard = ENERGY_ROUNDOFF_FACTOR * DOUBLE_EPS * torch.clamp(
            torch.maximum(energy.abs(), e_old.abs().nan_to_num(0.0)), min=1.0)
        done = (de < energy_tolerance + guard) & (drms < density_tolerance) & (cmax <= comm_tol)
        if phase == "tc":
            loose = cmax <= ANCHOR_COMMUTATOR
            if bool((loose | ~active).all()) or phase_iterations >= MIXED_ITERATION_CAP:
                phase, phase_iterations = "anchor", 0
            done = torch.zeros_like(done)
        if trace is not None:
            trace.append((it, phase, float(de[active].max()) if bool(active.any()) else 0.0,
                          float(cmax[active].max()) if bool(active.any()) else 0.0,
                          int(active.sum())))
        newly = done & active
        # record the state of molecules that are still active
        final_e = torch.where(active, energy, final_e)
        final_de = torch.where(active, de, final_de)
        final_drms = torch.where(active, drms, final_drms)
        iters = torch.where(active, torch.full_like(iters, it), iters)
        d_final = torch.where(active[:, None, None], d, d_final)
        c_final = torch.where(active[:, None, None], c, c_final)
        f_final = torch.where(active[:, None, None], f, f_final)
        converged |= newly
        active &= ~newly
        e_old = energy
        if not bool(active.any()):
            TIMER_ctx.__exit__(None, None, None)
            break
        d = torch.where(active[:, None, None], d_new, d)
        c = torch.where(active[:, None, None], c_new, c)
        TIMER_ctx.__exit__(None, None, None)
    if jk.precision == "mixed" and anchored:
        # rho and U = B C at the converged orbitals for the gradient: the
        # anchor's FP64 U0 plus the tensor-core increment
        exact_half = jk.anchored_half(c_final)
        jk.release_tensor_core_buffers()
    elif jk.precision == "mixed":
        # never anchored (iteration limit in the plain tensor-core phase):
        # re-evaluate E[D] in FP64 at the last density
        final_e, exact_half = exact_energy(jk, d_final, c_final, h, enuc)
    else:
        exact_half = None
    return {
        "energy": final_e, "converged": converged, "iterations": iters,
        "energy_change": final_de, "density_rms": final_drms, "density": d_final,
        "orbitals": c_final, "fock": f_final, "exact_half": exact_half,
        "mixed_iterations": mixed_iterations, "anchors": anchors,
        "warm_used": warm_used, "warm_fallback": warm_fallback,
        "metric": mf, "orthogonalizer": xo, "enuc": enuc, "charges": zs, "jk": jk,
        "relative_threshold": relative_threshold,
    }
