"""PyTorch autograd entry points with the native analytic adjoint as backward.

Same surface as the reference's ``python/generativeqc/torch.py:47-245``:
``energy(coordinates, atomic_numbers, calculator, charge=, multiplicity=)`` and
``batched_energy(coordinates, atomic_numbers, calculator, charges=,
multiplicities=, prepared_batch=)``.  The forward runs the DF-RHF energy and
analytic gradient (the hand-written derivative-contraction kernels); backward
returns dE/dR * grad_output.  Only first-order derivatives are supported.

Unlike the reference, CUDA coordinate tensors stay on the device: with a
prepared batch the forward feeds them straight to the device-resident
execution and the gradients never leave HBM.
"""

from __future__ import annotations

import typing
from typing import Sequence

import numpy as np
import torch

from .calculator import Calculator, PreparedBatch


def _require_first_order_backward() -> None:
    if torch.is_grad_enabled():
        raise RuntimeError(
            "only first-order coordinate derivatives are supported; higher-order "
            "derivatives through the analytic forces are unsupported"
        )


def _check_coordinates(coords: torch.Tensor, numbers: Sequence[int]) -> tuple[int, ...]:
    if not torch.is_floating_point(coords) or coords.dim() != 2 or coords.shape[1] != 3:
        raise ValueError("coordinates must be a real (natoms, 3) tensor")
    if coords.shape[0] != len(numbers):
        raise ValueError("atomic_numbers must match the coordinate rows")
    out = []
    for z in numbers:
        if isinstance(z, bool) or int(z) != z:
            raise ValueError("atomic numbers must be exact integers")
        out.append(int(z))
    return tuple(out)


class _BatchedEnergyFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, batch, *coordinates):  # type: ignore[override]
        ref = coordinates[0]
        for c in coordinates:
            if c.device != ref.device or c.dtype != ref.dtype:
                raise ValueError("all ragged coordinate tensors must share device and dtype")
        energies, grads = batch.execute_tensors([c.detach() for c in coordinates])
        ctx.save_for_backward(*[g.to(ref.dtype) for g in grads])
        return energies.to(device=ref.device, dtype=ref.dtype)

    @staticmethod
    def backward(ctx, grad_output):  # type: ignore[override]
        _require_first_order_backward()
        grads = tuple(g * grad_output[i] for i, g in enumerate(ctx.saved_tensors))
        return (None, *grads)


def batched_energy(
    coordinates: Sequence[torch.Tensor],
    atomic_numbers: Sequence[Sequence[int]],
    calculator: Calculator | None = None,
    *,
    charges: Sequence[int] | None = None,
    multiplicities: Sequence[int] | None = None,
    prepared_batch: PreparedBatch | None = None,
) -> torch.Tensor:
    """Energies of a ragged batch with the analytic coordinate gradient as backward."""
    if len(coordinates) != len(atomic_numbers) or not coordinates:
        raise ValueError("coordinates and atomic_numbers must have equal nonzero length")
    numbers = tuple(_check_coordinates(c, z) for c, z in zip(coordinates, atomic_numbers))
    n = len(coordinates)
    charges = tuple(0 for _ in range(n)) if charges is None else tuple(int(q) for q in charges)
    mults = tuple(1 for _ in range(n)) if multiplicities is None else tuple(int(m) for m in multiplicities)
    if len(charges) != n or len(mults) != n:
        raise ValueError("charges and multiplicities must match the ragged batch size")
    if prepared_batch is not None:
        if prepared_batch.atomic_numbers != numbers:
            raise ValueError("prepared batch topology does not match atomic numbers")
        if prepared_batch.charges != charges:
            raise ValueError("prepared batch charges do not match")
        if prepared_batch.multiplicities != mults:
            raise ValueError("prepared batch multiplicities do not match")
        batch = prepared_batch
    else:
        if calculator is None:
            raise ValueError("a calculator or a prepared batch is required")
        systems = [[(z, c[i].detach().cpu().tolist()) for i, z in enumerate(zs)]
                   for zs, c in zip(numbers, coordinates)]
        batch = calculator.prepare_batch(systems, charges=charges, multiplicities=mults)
    return _BatchedEnergyFunction.apply(batch, *coordinates)


def energy(
    coordinates: torch.Tensor,
    atomic_numbers: Sequence[int],
    calculator: Calculator | None = None,
    *,
    charge: int = 0,
    multiplicity: int = 1,
) -> torch.Tensor:
    """Single-system energy with the analytic coordinate gradient as backward."""
    return batched_energy([coordinates], [atomic_numbers], calculator, charges=[charge],
                          multiplicities=[multiplicity])[0]
