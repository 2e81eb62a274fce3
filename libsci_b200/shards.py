"""Folding per-GPU reduction results across ranks (one process per GPU, torch.distributed).

An elementwise chunk shards by contiguous element ranges with no exchange; a reduction over the
whole array is each rank's fold of its own range, then one exchange of those folds. This module is
that exchange. It keeps the single-device rules of libsci's reductions (core::Accumulator,
include/core/bytecode/accumulator.hpp:28-34; entries.slang:55-78): a NaN on any rank makes the
result NaN, sums add, minima and maxima take the extreme. A plain MIN/MAX all-reduce does not
promise that a NaN wins, so NaN is carried as a separate count.

Every rank issues the same four all-reduces in the same order, whatever folds it holds.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

SUM, MINIMUM, MAXIMUM = 0, 1, 2  # fold.hpp:11


def combine(values: torch.Tensor, folds, group=None) -> torch.Tensor:
    """values[i] is this rank's fold number i (double), of kind folds[i] (SUM, MINIMUM or MAXIMUM).
    Returns the folds over every rank's elements, on values' device."""
    kinds = torch.as_tensor(list(folds), device=values.device)
    nan = torch.isnan(values)
    nans = nan.to(values.dtype)
    dist.all_reduce(nans, op=dist.ReduceOp.SUM, group=group)
    clean = torch.where(nan, torch.zeros_like(values), values)
    total = torch.where(kinds == SUM, clean, torch.zeros_like(values))
    low = torch.where((kinds == MINIMUM) & ~nan, values, torch.full_like(values, float("inf")))
    high = torch.where((kinds == MAXIMUM) & ~nan, values, torch.full_like(values, float("-inf")))
    dist.all_reduce(total, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(low, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(high, op=dist.ReduceOp.MAX, group=group)
    out = torch.where(kinds == SUM, total, torch.where(kinds == MINIMUM, low, high))
    return torch.where(nans > 0, torch.full_like(values, float("nan")), out)
