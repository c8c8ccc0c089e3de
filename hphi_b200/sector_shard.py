"""One sector's H*v split over the ranks of one node (one GPU each): partition and exchange
schedule.

Partition.  With world = 2^k ranks, rank r holds the configurations whose top k bits equal r,
and the rest of the configuration (the low nbits - k bits) indexes its slice.  This is the
split of the reference's MPI build, which gives the top sites to the process number (four
states per site for Hubbard and Kondo, two for spins, so it needs a power of 4 or of 2
processes: src/CheckMPI.c:49-105, 106-200); splitting by bits instead of whole sites also
allows 2 or 8 ranks for Hubbard sectors.  In a canonical sector a rank's slice is the
sub-sector whose particle numbers are reduced by the particles in its rank bits (the same
file: Nup, Ndown, Ne per process), so slices differ in size.

Terms.  A compiled term (cm, cv, flip, sm, coefficient) acts in gather form on the output
configuration c: if (c & cm) == cv, it adds coefficient * (-1)^popcount(c & sm) times the
source element at c ^ flip.  Its masks split at bit nlo = nbits - k:
  - rank condition (c >> nlo & cm_hi) == cv_hi is the same for every row of a rank;
  - the source lies on rank r ^ (flip >> nlo): the partner offset d;
  - the sign's rank part popcount(r & sm_hi) is fixed per rank and folds into the coefficient.
Terms with d == 0 read the rank's own slice.  The distinct d != 0 are the exchange rounds: in
round d every rank sends its whole slice to r ^ d and receives r ^ d's (pairs of ranks, so a
round has no conflicts), then applies the round's terms from the received slice.  The
reference moves whole vectors the same way (MPI_Sendrecv of v1 with the partner process,
src/mltplyMPISpinCore.c:124,152-159; the dimension first, :152, since canonical slices differ).

On GPUs a round is a send / receive pair of torch.distributed (NCCL) into a buffer in the
rank's own HBM, never a load from a peer's memory, and the local terms of the sector run while
the first round is in flight.  Only the partition and the schedule are built here; the
per-rank term application is the caller's (a callback), so the exchange logic is tested on
CPU ranks over gloo against the full-sector product.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Dict, List, Sequence, Tuple


@dataclass(frozen=True)
class LocalTerm:
    """The low-bit part of a term on one rank: it acts on the slice's configuration x
    (low bits) if (x & cm) == cv, reads the source slice at x ^ flip and adds
    coef * (-1)^popcount(x & sm) (coef already carries the rank part of the sign)."""
    cm: int
    cv: int
    flip: int
    sm: int
    re: float
    im: float


@dataclass
class ShardPlan:
    nbits: int
    world: int
    k: int                                  # rank bits
    nlo: int                                # local bits
    own: List[List[LocalTerm]] = field(default_factory=list)               # per rank: d == 0
    rounds: List[int] = field(default_factory=list)                        # partner offsets d != 0
    remote: List[Dict[int, List[LocalTerm]]] = field(default_factory=list)  # per rank, per d


def rank_bits(world: int) -> int:
    """k with world = 2^k; the split needs a power of two."""
    if world < 1 or world & (world - 1):
        raise ValueError(f"world size {world} is not a power of two")
    return world.bit_length() - 1


def plan(terms: Sequence[Tuple[int, int, int, int, float, float]], nbits: int, world: int) -> ShardPlan:
    """Splits terms (cm, cv, flip, sm, re, im) over world ranks of an nbits configuration."""
    k = rank_bits(world)
    if k > nbits:
        raise ValueError("more ranks than configurations")
    nlo = nbits - k
    lo = (1 << nlo) - 1
    p = ShardPlan(nbits=nbits, world=world, k=k, nlo=nlo)
    ds = set()
    for r in range(world):
        own: List[LocalTerm] = []
        rem: Dict[int, List[LocalTerm]] = {}
        for cm, cv, flip, sm, re, im in terms:
            if ((r & (cm >> nlo)) != (cv >> nlo)):
                continue
            sg = -1.0 if bin(r & (sm >> nlo)).count("1") & 1 else 1.0
            t = LocalTerm(cm & lo, cv & lo, flip & lo, sm & lo, sg * re, sg * im)
            d = flip >> nlo
            if d == 0:
                own.append(t)
            else:
                rem.setdefault(d, []).append(t)
                ds.add(d)
        p.own.append(own)
        p.remote.append(rem)
    p.rounds = sorted(ds)
    return p


def partner(plan_: ShardPlan, rank: int, d: int) -> int:
    return rank ^ d


def sharded_hv(plan_: ShardPlan, rank: int, v1, slice_dims: Sequence[int],
               apply: Callable[[List[LocalTerm], object, int], object], dist=None):
    """(H v1) on this rank's slice.  apply(terms, source, source_rank) returns the
    contribution of terms (gather form) to this rank's rows, reading source = the slice of
    source_rank.  Rounds run in plan order; every rank takes part in every round (sending
    even when it has no term for it), so the collectives match on all ranks."""
    import torch
    if plan_.rounds and dist is None:
        raise ValueError("terms cross ranks: a process group is needed")
    out = apply(plan_.own[rank], v1, rank)
    send = v1.contiguous()
    for d in plan_.rounds:
        q = partner(plan_, rank, d)
        buf = torch.empty(slice_dims[q], dtype=v1.dtype, device=v1.device)
        # complex slices travel as (re, im) pairs of their real dtype
        s_view = torch.view_as_real(send) if send.is_complex() else send
        r_view = torch.view_as_real(buf) if buf.is_complex() else buf
        ops = [dist.P2POp(dist.isend, s_view, q), dist.P2POp(dist.irecv, r_view, q)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        terms = plan_.remote[rank].get(d, [])
        if terms:
            out = out + apply(terms, buf, q)
    return out
