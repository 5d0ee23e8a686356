"""Multi-GPU plumbing around the C ABI: one process per GPU, torch.distributed
for the collectives (NCCL on GPUs, gloo on CPU).

* ``halo_exchange``: before a part of a sharded map (ff_set_shard) meshes,
  the bricks each part changed since its last export reach every other part.
  Each part exports its records into a device buffer (ff_halo_export), the
  buffers are all-gathered -- every record lands in each GPU's own memory,
  no peer loads -- and each part imports the others' records
  (ff_halo_import).  With hash ownership nearly every brick borders bricks
  of other parts, so the records are the part's changed bricks.
* ``lpt_placement``: independent maps of uneven size over ranks, longest
  processing time first (each map to the least-loaded rank, by an estimated
  cost such as frames x pixels).
"""
from __future__ import annotations


def lpt_placement(costs, ranks: int) -> list[list[int]]:
    """Indices of `costs` per rank: the largest cost first, each to the rank
    with the least total so far (ties: the lower rank; equal costs keep their
    order).  Deterministic, so every rank computes the same placement."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * ranks
    out = [[] for _ in range(ranks)]
    for i in order:
        r = min(range(ranks), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(costs[i])
    for lst in out:
        lst.sort()
    return out


def halo_exchange(part, device, group=None) -> dict:
    """All-gather the parts' halo records over the process group and import
    the other ranks' into `part` (a FusionMipMapCPU, or any object with
    halo_count / halo_export / halo_import over device pointers).  Collective:
    every rank of the group calls it at the same point.  Returns the record
    counts per rank and the bytes one rank sent."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n, rb = part.halo_count()
    counts = torch.tensor([n], dtype=torch.int64, device=device)
    gathered = [torch.zeros_like(counts) for _ in range(world)]
    dist.all_gather(gathered, counts, group=group)
    ns = [int(c.item()) for c in gathered]
    cap = max(max(ns), 1)
    send = torch.zeros(cap * rb, dtype=torch.uint8, device=device)
    wrote = part.halo_export(send.data_ptr(), cap)
    if wrote != n:
        raise RuntimeError(f"halo export wrote {wrote} records, counted {n}")
    recv = torch.empty(world * cap * rb, dtype=torch.uint8, device=device)
    dist.all_gather_into_tensor(recv, send, group=group)
    for r in range(world):
        if r != rank and ns[r]:
            part.halo_import(recv[r * cap * rb:].data_ptr(), ns[r])
    return {"records": ns, "record_bytes": rb, "bytes_sent": cap * rb}
