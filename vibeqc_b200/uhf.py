"""Unrestricted DF-HF (UHF) on the GPU: the same integrals, whitening and J/K kernels.

Semantics follow the reference's unrestricted DF path: F_s = H + J[D_a + D_b]
- K[D_s] for s in (alpha, beta) (``src/scf/density_fitting.cpp:844``; CUDA
``src/scf/cuda/df_uhf_scf.cpp`` with ``assemble_uhf_fock_kernel``,
``src/scf/cuda/df_scf_kernels.cu:154``), E = 1/2 tr(D_t H) + 1/2 sum_s
tr(D_s F_s) + E_nn (``compute_device_uhf_energy_kernel``, ``:211``), one set of
Pulay weights over both spins' residuals (``src/scf/cuda/df_scf_diis.cpp:110-185``)
and convergence on |dE|, the rms change of both spin densities and the
larger spin residual (``update_device_uhf_convergence_kernel``, ``:296-340``).

Each spin is a channel of the restricted J/K builders: with the spin's
occupied factor C_s (D_s = C_s C_s^T) scaled to c_s = C_s / sqrt(2), the
builders' restricted convention D = 2 c c^T gives exactly D_s, their exchange
2 (B c)(B c)^T is K[D_s] and their fitted density is that of D_s.  The beta
factor is padded with zero columns to the alpha count (zero columns add
nothing to K, rho or the gradient weights), so both channels share the
builder's buffers; the mixed path keeps one FP64 anchor per channel.
"""

from __future__ import annotations

import math

import torch

from . import jk as jkmod
from .timing import TIMER

INV_SQRT2 = 1.0 / math.sqrt(2.0)


def _pad_columns(c: torch.Tensor, width: int) -> torch.Tensor:
    if c.shape[2] == width:
        return c
    out = torch.zeros(c.shape[0], c.shape[1], width, dtype=c.dtype, device=c.device)
    out[:, :, :c.shape[2]] = c
    return out


class _UHFPost:
    """Fock, energy, residuals and two-spin DIIS of one UHF iteration (one CUDA graph).

    Like the restricted block: static buffers, a ring of ``hist`` DIIS slots
    with an incrementally updated Gram matrix over the concatenated spin
    residuals X^T (F_s D_s S - S D_s F_s) X, one set of weights applied to
    both spins' Fock matrices.  ``with_rho`` selects the anchored-phase energy
    tr(D_t H) + |rho|^2 / 2 - 1/2 sum_s tr(D_s K_s) + E_nn.
    """

    def __init__(self, nb: int, n: int, x: int, hist: int, with_rho: bool, device):
        from .scf import _graphs_enabled

        f64 = dict(dtype=torch.float64, device=device)
        self.h, self.s, self.xo = (torch.zeros(nb, n, n, **f64) for _ in range(3))
        self.enuc = torch.zeros(nb, **f64)
        self.j = torch.zeros(nb, n, n, **f64)
        self.k = torch.zeros(2, nb, n, n, **f64)
        self.d = torch.zeros(2, nb, n, n, **f64)
        self.rho = torch.zeros(nb, x, **f64)
        self.e_ring = torch.zeros(nb, hist, 2, n, n, **f64)
        self.f_ring = torch.zeros(nb, hist, 2, n, n, **f64)
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
                with torch.cuda.stream(side):
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
        self.e_ring.zero_()
        self.f_ring.zero_()
        self.reset()

    def _step(self):
        hist = self.hist
        f = self.h[None] + self.j[None] - self.k  # (2, nb, N, N)
        dt = self.d[0] + self.d[1]
        e1 = torch.einsum("bmn,bmn->b", dt, self.h)
        if self.with_rho:
            energy = (e1 + 0.5 * (self.rho * self.rho).sum(dim=1)
                      - 0.5 * torch.einsum("sbmn,sbmn->b", self.d, self.k) + self.enuc)
        else:
            energy = 0.5 * e1 + 0.5 * torch.einsum("sbmn,sbmn->b", self.d, f) + self.enuc
        fds = f @ self.d @ self.s[None]
        comm = fds - fds.transpose(2, 3)
        cmax = comm.abs().amax(dim=(2, 3)).amax(dim=0)
        err = (self.xo.transpose(1, 2)[None] @ comm @ self.xo[None]).transpose(0, 1)  # (nb, 2, N, N)
        slot = torch.remainder(self.count, hist)
        self.e_ring.index_copy_(1, slot, err[:, None])
        self.f_ring.index_copy_(1, slot, f.transpose(0, 1)[:, None])
        g_new = torch.einsum("bsmn,bhsmn->bh", err, self.e_ring)
        self.gram.index_copy_(1, slot, g_new[:, None, :])
        self.gram.index_copy_(2, slot, g_new[:, :, None])
        self.count.add_(1)
        valid = torch.arange(hist, device=self.count.device) < torch.clamp(self.count, max=hist)
        vf = valid.to(torch.float64)
        pair = vf[:, None] * vf[None, :]
        nb = f.shape[1]
        bmat = torch.zeros(nb, hist + 1, hist + 1, dtype=torch.float64, device=f.device)
        bmat[:, :hist, :hist] = self.gram * pair + self.eye * (1.0 - vf)[None, :, None]
        bmat[:, hist, :hist] = -vf
        bmat[:, :hist, hist] = -vf
        rhs = torch.zeros(nb, hist + 1, 1, dtype=torch.float64, device=f.device)
        rhs[:, hist, 0] = -1.0
        w, info = torch.linalg.solve_ex(bmat, rhs)
        w = w[:, :hist, 0] * vf
        ok = (info == 0) & torch.isfinite(w).all(dim=1)
        ext = torch.einsum("bh,bhsmn->sbmn", w, self.f_ring)
        f_ext = torch.where(ok[None, :, None, None], ext, f)
        return f, energy, cmax, f_ext

    def run(self, j, k_alpha, k_beta, d_alpha, d_beta, rho=None):
        """(F (2, nb, N, N), energy, max residual, extrapolated F); overwritten next call."""
        self.j.copy_(j)
        self.k[0].copy_(k_alpha)
        self.k[1].copy_(k_beta)
        self.d[0].copy_(d_alpha)
        self.d[1].copy_(d_beta)
        if rho is not None:
            self.rho.copy_(rho)
        if self.graph is not None:
            self.graph.replay()
            return self.out
        return self._step()


_POST: dict = {}


def _uhf_post(nb, n, x, hist, with_rho, device) -> _UHFPost:
    from .scf import POST_CACHE_BYTES, POST_STATS

    key = (nb, n, x, hist, with_rho, str(device))
    p = _POST.get(key)
    if p is None:
        held = sum(2 * v.e_ring.numel() * 8 for v in _POST.values())
        if held + 4 * nb * hist * n * n * 8 > POST_CACHE_BYTES:
            _POST.clear()
        p = _POST[key] = _UHFPost(nb, n, x, hist, with_rho, device)
        POST_STATS["graphs" if p.graph is not None else "eager"] += 1
    return p


def _coulomb_fp32(jk, drho: torch.Tensor) -> torch.Tensor:
    """B rho from the mixed builder's FP32 tensor (FP64 accumulation)."""
    nb, n = jk.nb, jk.n
    out = torch.empty(nb, n, n, dtype=torch.float64, device=drho.device)
    with TIMER.stage("J_fp32"):
        jk._lib.call("vqc_coulomb_tma", jk.b.data_ptr(), drho.contiguous().data_ptr(), nb, n,
                     jk.ld, jk.x, out.data_ptr(), jk.err.data_ptr(), jk.st)
    return out


def run_scf_uhf(chunk, ints, xyz: torch.Tensor, *, precision: str = "fp64",
                max_iterations: int = 100, energy_tolerance: float = 1e-10,
                density_tolerance: float = 1e-8, diis_history: int = 8,
                relative_threshold: float = 1e-10, warm_density: torch.Tensor | None = None,
                warm_mask: torch.Tensor | None = None, schedule=None) -> dict:
    """Batched UHF over one chunk (equal N, X, n_alpha, n_beta); device tensors out.

    ``warm_density`` (nb, 2, N, N) holds per-item alpha and beta densities of
    an earlier execution (used where ``warm_mask`` is set): the same
    purification as the cold guess applied to F0_s = -S D_s S.
    """
    from . import scf as scfm
    from .tuning import DEFAULT, apply_library_knobs

    sched = DEFAULT if schedule is None else schedule
    apply_library_knobs(sched)
    nb, n, x = chunk.nb, chunk.nao, chunk.naux
    occ = (chunk.nalpha, chunk.nbeta)
    width = max(1, occ[0])
    dev = xyz.device
    with TIMER.stage("metric_factor"):
        mf = scfm.factor_metric(ints.metric, relative_threshold)
    with TIMER.stage("whiten"):
        b_packed = ints.a_packed
        ints.a_packed = None
        if precision == "mixed" and scfm.WHITEN_TENSOR_CORES and sched.whiten == "int8":
            scfm.whiten_tensor_cores(b_packed, mf, ints.metric)
        else:
            scfm.whiten_in_place(b_packed, mf)
        jk = jkmod.make_builder(precision, b_packed, n, x, width)
        del b_packed
    s, h = ints.s, ints.h
    xo = scfm._orthogonalizer(s)
    enuc, zs = [], []
    off = 0
    for i, mol in enumerate(chunk.molecules):
        na = chunk.natoms[i]
        z = torch.as_tensor(mol.atomic_numbers, dtype=torch.float64, device=dev)
        e, _ = scfm.nuclear_repulsion(z, xyz[off:off + na])
        enuc.append(e)
        zs.append(z)
        off += na
    enuc = torch.stack(enuc)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234)
    guesses = [torch.randn(nb, n, o, dtype=torch.float64, device=dev, generator=gen) for o in occ]

    def density_from(f, guess, nocc, tol=1e-11, noise_scale=0.3):
        """(spin density X P X^T, orthonormal occupied factor) for ``nocc`` electrons."""
        if nocc == 0:
            return torch.zeros_like(f), torch.zeros(nb, n, 0, dtype=f.dtype, device=dev)
        with TIMER.stage("purify"):
            proj = scfm.purify_sp2(xo.transpose(1, 2) @ f @ xo, nocc, tol=tol,
                                   graphs=scfm._SP2_GRAPHS, steps=sched.sp2_steps,
                                   gemm=sched.sp2_gemm if precision == "mixed" else "fp64")
        with TIMER.stage("occupied_factor"):
            co = scfm.occupied_factor(proj, guess, gen, noise_scale)
        return xo @ proj @ xo.transpose(1, 2), co

    warm_used = torch.zeros(nb, dtype=torch.bool, device=dev)
    warm_fallback = torch.zeros(nb, dtype=torch.bool, device=dev)
    f0 = [h, h]
    if warm_density is not None and warm_mask is not None and bool(warm_mask.any()):
        finite = torch.isfinite(warm_density).flatten(1).all(dim=1)
        warm_used = warm_mask & finite
        warm_fallback = warm_mask & ~finite
        for sp in range(2):
            wd = torch.where(warm_used[:, None, None], warm_density[:, sp], torch.zeros_like(h))
            f0[sp] = torch.where(warm_used[:, None, None], -(s @ wd @ s), h)
    ds, cos = [], []
    for sp in range(2):
        d_, co_ = density_from(f0[sp], guesses[sp], occ[sp])
        ds.append(d_)
        cos.append(co_)

    def channel_factors(cos_):
        # builder channel factors c_s = X C'_s / sqrt(2), beta padded to the alpha width
        return [_pad_columns(xo @ c_, width) * INV_SQRT2 for c_ in cos_]

    cs = channel_factors(cos)
    active = torch.ones(nb, dtype=torch.bool, device=dev)
    e_old = torch.full((nb,), float("nan"), dtype=torch.float64, device=dev)
    final_e = torch.zeros(nb, dtype=torch.float64, device=dev)
    final_de = torch.full((nb,), float("inf"), dtype=torch.float64, device=dev)
    final_drms = torch.full((nb,), float("inf"), dtype=torch.float64, device=dev)
    iters = torch.zeros(nb, dtype=torch.int64, device=dev)
    converged = torch.zeros(nb, dtype=torch.bool, device=dev)
    d_final = [d_.clone() for d_ in ds]
    c_final = [c_.clone() for c_ in cs]
    f_final = [torch.zeros_like(h), torch.zeros_like(h)]
    post = None
    comm_tol = min(1e-8, density_tolerance)
    phase = "tc" if jk.precision == "mixed" else "exact"
    phase_iterations = 0
    mixed_iterations = 0
    co_anchor = None
    anchored = False
    anchor_builds = 0
    anchors = 0
    j_anchor = rho_anchor = None
    for it in range(1, max_iterations + 1):
        rho = None
        dt = ds[0] + ds[1]
        if phase == "exact":
            j, ka = jk.build_exact(dt, cs[0])
            _, kb = jk.build_exact(ds[1], cs[1], with_j=False)
        elif phase == "anchor":
            if anchored and anchor_builds >= scfm.REANCHOR_EVERY:
                anchored, co_anchor, anchor_builds = False, None, 0
            if not anchored:
                ja, ka, ra = jk.anchor(ds[0], cs[0], 0)
                jb, kb, rb = jk.anchor(ds[1], cs[1], 1)
                j_anchor, rho_anchor = ja + jb, ra + rb
                j, rho = j_anchor, rho_anchor
                anchored = True
                anchors += 1
            else:
                _, ka, ra = jk.build_incremental(ds[0], cs[0], 0, with_j=False)
                _, kb, rb = jk.build_incremental(ds[1], cs[1], 1, with_j=False)
                rho = ra + rb
                j = j_anchor + _coulomb_fp32(jk, rho - rho_anchor)
                mixed_iterations += 1
                anchor_builds += 1
        else:
            j, ka = jk.build(dt, cs[0])
            _, kb = jk.build(ds[1], cs[1], with_j=False)
            mixed_iterations += 1
        phase_iterations += 1
        ctx = TIMER.stage("scf_other")
        ctx.__enter__()
        with_rho = rho is not None
        if post is None or post.with_rho != with_rho:
            prev = post
            post = _uhf_post(nb, n, x, diis_history, with_rho, dev)
            post.load(h, s, xo, enuc)
            if prev is not None:
                post.e_ring.copy_(prev.e_ring)
                post.f_ring.copy_(prev.f_ring)
                post.gram.copy_(prev.gram)
                post.count.copy_(prev.count)
        f, energy, cmax, f_ext = post.run(j, ka, kb, ds[0], ds[1], rho)
        energy = energy.clone()
        f = f.clone()
        ctx.__exit__(None, None, None)
        new_d, new_co = [], []
        for sp in range(2):
            if phase == "anchor":
                if co_anchor is None:
                    co_anchor = list(cos)
                d_, co_ = density_from(f_ext[sp], co_anchor[sp], occ[sp], 1e-11, 0.0)
            else:
                d_, co_ = density_from(f_ext[sp], cos[sp], occ[sp],
                                       1e-11 if phase == "exact" else 1e-8)
            new_d.append(d_)
            new_co.append(co_)
        ctx = TIMER.stage("scf_other")
        ctx.__enter__()
        new_c = channel_factors(new_co)
        de = (energy - e_old).abs()
        de = torch.where(torch.isnan(de), torch.full_like(de, float("inf")), de)
        drms = ((((new_d[0] - ds[0]) ** 2).sum(dim=(1, 2)) + ((new_d[1] - ds[1]) ** 2).sum(dim=(1, 2)))
                / (2 * n * n)).sqrt()
        guard = scfm.ENERGY_ROUNDOFF_FACTOR * scfm.DOUBLE_EPS * torch.clamp(
            torch.maximum(energy.abs(), e_old.abs().nan_to_num(0.0)), min=1.0)
        done = (de < energy_tolerance + guard) & (drms < density_tolerance) & (cmax <= comm_tol)
        if phase == "tc":
            loose = cmax <= scfm.ANCHOR_COMMUTATOR
            if bool((loose | ~active).all()) or phase_iterations >= scfm.MIXED_ITERATION_CAP:
                phase, phase_iterations = "anchor", 0
            done = torch.zeros_like(done)
        newly = done & active
        final_e = torch.where(active, energy, final_e)
        final_de = torch.where(active, de, final_de)
        final_drms = torch.where(active, drms, final_drms)
        iters = torch.where(active, torch.full_like(iters, it), iters)
        keep = active[:, None, None]
        for sp in range(2):
            d_final[sp] = torch.where(keep, ds[sp], d_final[sp])
            c_final[sp] = torch.where(keep, cs[sp], c_final[sp])
            f_final[sp] = torch.where(keep, f[sp], f_final[sp])
        converged |= newly
        active &= ~newly
        e_old = energy
        if not bool(active.any()):
            ctx.__exit__(None, None, None)
            break
        for sp in range(2):
            ds[sp] = torch.where(keep & active[:, None, None], new_d[sp], ds[sp])
            cs[sp] = torch.where(keep & active[:, None, None], new_c[sp], cs[sp])
            cos[sp] = new_co[sp]
        ctx.__exit__(None, None, None)
    if jk.precision == "mixed" and anchored:
        exact_half = [jk.anchored_half(c_final[sp], sp) for sp in range(2)]
        jk.release_tensor_core_buffers()
    elif jk.precision == "mixed":
        final_e, exact_half = exact_energy_uhf(jk, d_final, c_final, h, enuc)
    else:
        exact_half = None
    return {
        "energy": final_e, "converged": converged, "iterations": iters,
        "energy_change": final_de, "density_rms": final_drms,
        "density": d_final[0] + d_final[1], "spin_densities": d_final,
        "orbitals": c_final, "fock": f_final, "exact_half": exact_half,
        "mixed_iterations": mixed_iterations, "anchors": anchors,
        "warm_used": warm_used, "warm_fallback": warm_fallback,
        "metric": mf, "orthogonalizer": xo, "enuc": enuc, "charges": zs, "jk": jk,
        "relative_threshold": relative_threshold,
    }


def exact_energy_uhf(jk, ds, cs, h, enuc):
    """FP64 E[D_a, D_b] from the FP64 whitened tensor, and each channel's (rho, U)."""
    halves = [jk.half_transform(c) for c in cs]
    dt = ds[0] + ds[1]
    rho = halves[0][0] + halves[1][0]
    e = torch.einsum("bmn,bmn->b", dt, h) + 0.5 * (rho * rho).sum(dim=1) + enuc
    for c, (_, u) in zip(cs, halves):
        for m in range(dt.shape[0]):
            bij = torch.einsum("mi,mjq->qij", c[m], u[m])
            e[m] = e[m] - 2.0 * (bij * bij).sum()  # -1/2 tr(D_s K_s), D_s = 2 c c^T
    return e, halves
