"""Sharding of batched limb work across GPUs (one process per GPU).

Limbs, polynomials and ciphertexts are independent, so a batch is split into
contiguous, modulus-aligned ranges — no data-path collective.  Only the
timing (max over ranks) and, optionally, per-shard digests cross ranks.
"""
from __future__ import annotations


def shard_range(count: int, n_moduli: int, rank: int, world: int):
    """[begin, end) limb range of `rank`.  Boundaries fall on multiples of
    n_moduli so that limb i keeps modulus i % n_moduli on every rank (each
    shard starts at modulus 0).  Earlier ranks take the remainder."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank / world size")
    if count % n_moduli:
        raise ValueError("count must be a multiple of the number of moduli")
    units = count // n_moduli
    per, extra = divmod(units, world)
    begin = rank * per + min(rank, extra)
    end = begin + per + (1 if rank < extra else 0)
    return begin * n_moduli, end * n_moduli


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Largest `value` over all ranks (the job's wall time is the slowest rank's)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
