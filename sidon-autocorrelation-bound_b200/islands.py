"""Islands across ranks: one process per GPU, torch.distributed for the
exchange (NCCL between GPUs; gloo for the CPU tests).

Each rank holds ``n_islands_local`` islands of P/n_islands_local
consecutive candidates, and the islands of all ranks form one global ring
(global island g = rank * n_islands_local + i).  A migration step ranks and
migrates inside the rank on the device (``kernels.island_migrate``, whose
local ring also sends the last island's migrants to the first), then
replaces that local wrap by the cross-rank hop: every rank all-gathers the
top-k rows + fitness of its last island and writes the rows of rank
(r - 1) mod W over the k worst of its first island.  The result is the
single-process migration over all W * n_islands_local islands
(src/main.cu:676-692 for one ring of islands).  Rows cross the link once,
into local memory, then into their slots.

Only the migrants (k * n * 4 bytes + 8 k bytes per rank) and the global
best's (F, rank, index) cross ranks; the search itself never communicates.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def _ws(group):
    if not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def ring_exchange(send_rows: torch.Tensor, send_fit: torch.Tensor, group=None):
    """All-gather every rank's migrants; return those of rank (r - 1) mod W."""
    W, r = _ws(group)
    rows = [torch.empty_like(send_rows) for _ in range(W)]
    fits = [torch.empty_like(send_fit) for _ in range(W)]
    dist.all_gather(rows, send_rows.contiguous(), group=group)
    dist.all_gather(fits, send_fit.contiguous(), group=group)
    src = (r - 1) % W
    return rows[src], fits[src]


def migrate_across_ranks(pop: torch.Tensor, fit: torch.Tensor, n_islands_local: int, k: int,
                         group=None, local_migrate=None) -> torch.Tensor:
    """Global-ring island migration of a uniform [P, n] population, in place
    on pop and fit.  ``local_migrate(pop, fit, n_islands, k) -> order`` is the
    in-rank step (default: the device kernel).  Returns the local ranking."""
    if local_migrate is None:
        from .kernels import island_migrate as local_migrate
    order = local_migrate(pop, fit, n_islands_local, k)
    W, _ = _ws(group)
    if W == 1 or k == 0:
        return order
    P = pop.shape[0]
    PI = P // n_islands_local
    order_l = order.to(torch.long)
    last = order_l[(n_islands_local - 1) * PI:(n_islands_local - 1) * PI + k]
    recv_rows, recv_fit = ring_exchange(pop.index_select(0, last), fit.index_select(0, last),
                                        group)
    dst = torch.stack([order_l[PI - 1 - j] for j in range(k)])
    pop.index_copy_(0, dst, recv_rows)
    fit.index_copy_(0, dst, recv_fit)
    return order


def global_best(fit: torch.Tensor, group=None) -> tuple[float, int, int]:
    """(F, rank, local index) of the smallest fitness over all ranks; NaN
    never wins; ties go to the lower rank, then the lower index."""
    W, r = _ws(group)
    f = fit.detach().double()
    if W == 1:
        f1 = torch.where(torch.isnan(f), torch.full_like(f, float("inf")), f)
        i = int(torch.argmin(f1).item())
        return (f1[i].item(), 0, i)
    f = torch.where(torch.isnan(f), torch.full_like(f, float("inf")), f)
    idx = int(torch.argmin(f).item())
    mine = torch.tensor([f[idx].item(), float(r), float(idx)], dtype=torch.float64,
                        device=fit.device)
    allv = [torch.empty_like(mine) for _ in range(W)]
    dist.all_gather(allv, mine, group=group)
    best = min((v[0].item(), int(v[1].item()), int(v[2].item())) for v in allv)
    return best


def broadcast_row(row: torch.Tensor, src_rank: int, group=None) -> torch.Tensor:
    """The global best's heights on every rank."""
    dist.broadcast(row, src=src_rank, group=group)
    return row


def max_over_ranks(ms: float, device="cpu", group=None) -> float:
    """The slowest rank's time (the multi-GPU figure of merit)."""
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return t.item()


def shard(P_total: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of this rank's candidates when P_total are split as
    evenly as possible (weak scaling fixes P per rank instead)."""
    base, extra = divmod(P_total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)
