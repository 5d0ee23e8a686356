"""The multi-GPU host logic of fastfusion_b200/shard.py on CPU ranks (gloo,
world size 2 and 3, 127.0.0.1): the halo all-gather delivers every other
rank's records and none of its own, with uneven record counts, an empty rank
and repeated rounds; and the LPT placement of maps over ranks.

The parts here are stand-ins with the C ABI's halo contract (records of a
fixed size: a leaf index, padding, then the brick; export writes the bricks
changed since the last export; import writes records into the pool), kept in
host memory, so the collective and the bookkeeping run without a GPU."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

REC = 64  # record bytes of the stand-in (index + padding + 48 bytes of brick)


class FakePart:
    """A part of a sharded map: `owned` bricks it changes, a pool of all."""

    def __init__(self, rank, nleaves, owned):
        self.rank = rank
        self.pool = np.zeros((nleaves, REC - 16), np.uint8)
        self.owned = owned
        self.changed = set()

    def touch(self, leaves, value):
        for b in leaves:
            assert b in self.owned
            self.pool[b] = value
            self.changed.add(b)

    def halo_count(self):
        return len(self.changed), REC

    def halo_export(self, ptr, cap):
        recs = sorted(self.changed)
        assert len(recs) <= cap
        buf = np.zeros((len(recs), REC), np.uint8)
        for k, b in enumerate(recs):
            buf[k, :4] = np.frombuffer(np.uint32(b).tobytes(), np.uint8)
            buf[k, 16:] = self.pool[b]
        ctypes.memmove(ptr, buf.ctypes.data, buf.nbytes)
        self.changed.clear()
        return len(recs)

    def halo_import(self, ptr, n):
        buf = np.frombuffer((ctypes.c_uint8 * (n * REC)).from_address(ptr), np.uint8).reshape(n, REC).copy()
        for rec in buf:
            b = int(rec[:4].view(np.uint32)[0])
            assert b not in self.owned, "a part's own brick came back"
            self.pool[b] = rec[16:]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from fastfusion_b200.shard import halo_exchange
    nleaves = 60
    owner = np.arange(nleaves) % world
    part = FakePart(rank, nleaves, set(np.nonzero(owner == rank)[0].tolist()))
    whole = np.zeros((nleaves, REC - 16), np.uint8)
    rng = np.random.default_rng(5)
    ok = True
    for rnd in range(3):
        # every rank knows what every rank changes this round (the same rng);
        # rank world-1 changes nothing in round 1
        for r in range(world):
            mine = np.nonzero(owner == r)[0]
            k = 0 if (rnd == 1 and r == world - 1) else int(rng.integers(1, len(mine)))
            sel = rng.choice(mine, size=k, replace=False)
            val = rng.integers(1, 255, size=(k, REC - 16), dtype=np.uint8)
            for b, v in zip(sel, val):
                whole[b] = v
            if r == rank:
                for b, v in zip(sel, val):
                    part.touch([int(b)], v)
        info = halo_exchange(part, "cpu")
        ok = ok and np.array_equal(part.pool, whole) and info["record_bytes"] == REC
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ok))


@pytest.mark.timeout(240)
@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_over_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=200) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [ok for _, ok in out] == [True] * world


def test_lpt_placement():
    from fastfusion_b200.shard import lpt_placement
    costs = [7, 3, 9, 1, 4, 4, 8, 2]
    pl = lpt_placement(costs, 3)
    assert sorted(i for lst in pl for i in lst) == list(range(len(costs)))
    loads = [sum(costs[i] for i in lst) for lst in pl]
    assert max(loads) - min(loads) <= max(costs) and max(loads) == 13
    assert pl == lpt_placement(costs, 3)  # deterministic
    assert lpt_placement(costs, 1) == [list(range(len(costs)))]
    assert lpt_placement([5], 4) == [[0], [], [], []]
