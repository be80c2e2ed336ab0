"""Row-block closure of one large query over several processes (one per GPU).

The rows of every nonterminal matrix are cut into `world` contiguous blocks of
whole 64-row tile-rows; rank p owns block p and keeps full copies of all
matrices in its GPU's memory.  Iteration t (semi-naive, like the single-GPU
engine):

  1. delta_X = X & ~prev_X, then prev_X = X, for every nonterminal X.  After
     the previous exchange every rank holds the same matrices, so the deltas
     are the same on every rank.
  2. For every rule C -> A B, on this rank's rows R_p:
        C[R_p] |= delta_A[R_p] * B   and   C[R_p] |= A[R_p] * delta_B
     (in the first iteration delta = everything and only the first term runs).
  3. Exchange: one OR all-reduce of the per-matrix changed flags (one word per
     matrix), then an all-gather of the row blocks of the matrices that some
     rank changed; every rank writes the other ranks' blocks into its copies.
  4. Stop after an iteration in which no rank changed anything.

Completeness is the semi-naive argument of the engine: a pair (bit of A, bit
of B) is combined in the iteration after the later of the two appeared,
because that bit is in the delta and every rank sees it after the exchange.
The exchange is host-driven collectives between iterations (NCCL over NVLink
for device buffers, gloo for host buffers); no kernel waits on another rank,
and no TMA or bulk copy ever reads another GPU's memory: the all-gather lands
every remote block in this GPU's own memory before any product reads it.

The reference has no multi-GPU path (one query on one GPU per process,
cuda/naive-gpu/main.cpp:9-10); this module is the row-block partition of the
products C |= A * B (cfpq-cpp/Grammar.h:58-69 semantics) across GPUs.

Engines implement:  n, nmats, block_bytes(r0, r1), begin_iteration(),
product(head, body1, body2, term, r0, r1) -> bool, export(m, r0, r1, buf),
import_(m, r0, r1, buf), sync(), and `device` ("cuda" or "cpu": where the
exchange buffers live).  DeviceRowEngine is the GPU engine over the C ABI.
"""
from __future__ import annotations

import dataclasses
from typing import Sequence

from . import capi


def row_blocks(n: int, world: int) -> list[tuple[int, int]]:
    """Row range [r0, r1) of every rank: whole 64-row tile-rows, the tile-rows
    dealt in contiguous blocks of ceil(T / world); ranks past the last
    tile-row get the empty range (n, n)."""
    T = (n + 63) // 64
    per = -(-T // world) if T else 0
    out = []
    for p in range(world):
        a, b = min(p * per, T), min((p + 1) * per, T)
        out.append((min(a * 64, n), min(b * 64, n)))
    return out


class DeviceRowEngine:
    """The matrices of one query on this process's GPU (C ABI): current
    matrices (the caller's), plus a previous-iteration copy and a delta per
    nonterminal."""

    device = "cuda"

    def __init__(self, ctx: capi.Context, mats: Sequence[capi.Matrix], variant: str = "lop3"):
        self.ctx, self.mats, self.variant = ctx, list(mats), variant
        self.n = mats[0].n if mats else 0
        self.nmats = len(mats)
        self.prev = [ctx.matrix(self.n) for _ in mats]
        self.delta = [ctx.matrix(self.n) for _ in mats]

    def close(self) -> None:
        for m in self.prev + self.delta:
            m.destroy()
        self.prev, self.delta = [], []

    def block_bytes(self, r0: int, r1: int) -> int:
        return self.mats[0].block_bytes(r0, r1) if self.mats else 0

    def begin_iteration(self) -> None:
        for x in range(self.nmats):
            self.ctx.delta(self.delta[x], self.mats[x], self.prev[x])

    def product(self, head: int, body1: int, body2: int, term: int, r0: int, r1: int) -> bool:
        a = self.delta[body1] if term == 0 else self.mats[body1]
        b = self.mats[body2] if term == 0 else self.delta[body2]
        return self.ctx.add_mul_rows(self.mats[head], a, b, r0, r1, self.variant)

    def export(self, m: int, r0: int, r1: int, buf) -> None:
        self.mats[m].export_block(r0, r1, buf.data_ptr())

    def import_(self, m: int, r0: int, r1: int, buf) -> None:
        self.mats[m].import_block(r0, r1, buf.data_ptr())

    def sync(self) -> None:
        self.ctx.synchronize()


@dataclasses.dataclass
class RowBlockStats:
    iterations: int = 0
    products: int = 0
    gathered_blocks: int = 0
    exchanged_bytes: int = 0  # bytes this rank received in all-gathers


def closure(engine, rules: Sequence[tuple[int, int, int]], dist=None, group=None,
            max_iterations: int = 0) -> RowBlockStats:
    """Close the query held by `engine` with the row-block partition over the
    ranks of `group` (dist = torch.distributed, None for a single process).
    Every rank must call this with the same rules and an engine over the same
    initial matrices; on return every rank holds the whole fixpoint."""
    import torch

    world = dist.get_world_size(group) if dist else 1
    rank = dist.get_rank(group) if dist else 0
    blocks = row_blocks(engine.n, world)
    r0, r1 = blocks[rank]
    chunk = max((engine.block_bytes(a, b) for a, b in blocks), default=0)
    nccl = dist is not None and dist.get_backend(group) == "nccl"
    # exchange buffers: device memory only for NCCL (a device engine's blocks
    # then never leave the GPUs); otherwise host memory, pinned when a device
    # engine copies into it.  The collective runs on torch's stream, the
    # engine's copies on its own: every hand-over below is synchronised.
    dev = "cuda" if nccl and engine.device == "cuda" else "cpu"
    pinned = dev == "cpu" and engine.device == "cuda"
    send = torch.zeros(max(chunk, 1), dtype=torch.uint8, device=dev, pin_memory=pinned)
    recv = (torch.zeros(max(chunk, 1) * world, dtype=torch.uint8, device=dev, pin_memory=pinned)
            if world > 1 else None)
    flags = torch.zeros(max(engine.nmats, 1), dtype=torch.int32, device="cuda" if nccl else "cpu")
    st = RowBlockStats()
    while True:
        engine.begin_iteration()
        changed = [0] * engine.nmats
        for head, b1, b2 in rules:
            for term in ((0,) if st.iterations == 0 else (0, 1)):
                if r1 > r0:  # a rank past the last tile-row owns no rows
                    st.products += 1
                    if engine.product(head, b1, b2, term, r0, r1):
                        changed[head] = 1
        st.iterations += 1
        flags.copy_(torch.tensor(changed or [0], dtype=torch.int32))
        if dist is not None and world > 1:
            dist.all_reduce(flags, op=dist.ReduceOp.MAX, group=group)
        any_changed = [m for m in range(engine.nmats) if int(flags[m]) != 0]
        if not any_changed:
            break
        if world > 1:
            for m in any_changed:
                # (bytes of send past this rank's block are never imported)
                if r1 > r0:
                    engine.export(m, r0, r1, send)
                engine.sync()
                if dev == "cuda":
                    dist.all_gather_into_tensor(recv, send, group=group)
                    torch.cuda.current_stream().synchronize()
                else:
                    dist.all_gather(list(recv.view(world, -1).unbind(0)), send, group=group)
                for p, (a, b) in enumerate(blocks):
                    if p != rank and b > a:
                        engine.import_(m, a, b, recv[p * chunk:(p + 1) * chunk])
                st.gathered_blocks += world - 1
                st.exchanged_bytes += (world - 1) * chunk
            engine.sync()
        if max_iterations and st.iterations >= max_iterations:
            break
    return st
