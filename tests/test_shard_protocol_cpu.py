"""The peer-memory exchange of the sharded step (csrc/shard.cu) as a
protocol, checked on the CPU: ranks run their kernels' memory operations as
separate events, interleaved at random, and every exchange must read the
exact integer total of its own step.  The model holds what the GPU code
relies on and nothing more:

* a rank's kernels run in stream order: deposit adds, then the signal
  stores, then the exchange (its reads and clears in any order, after its
  wait), then the next step;
* different ranks' events interleave arbitrarily;
* the exchange of step s waits until every rank has signalled s.

With three slots no schedule breaks a total; with two slots some schedule
does (the model can tell the difference), which is why the library keeps
three.  Also checked: the IPC handle exchange over gloo."""
import os
import random
import socket

import pytest

torch = pytest.importorskip("torch")


def owner(cell, cells, world):
    # cells stand for grids here: grid i belongs to rank floor(i * world / k)
    return cell * world // cells


def first_cell(rank, cells, world):
    return -(-rank * cells // world)


class Rank:
    def __init__(self, r, world, cells, steps, rng, slots):
        self.r, self.world, self.cells, self.slots = r, world, cells, slots
        self.flags = [0] * world
        self.accum = [[0] * cells for _ in range(slots)]
        # this rank's particles' cell contributions per step
        self.contrib = [[rng.randrange(0, 4) for _ in range(cells)] for _ in range(steps)]
        self.step = 0
        self.phase = "deposit"
        self.pending = []
        self.local = [0] * cells

    def events(self, ranks, steps):
        """The rank's next enabled events (a list of thunks), or None when done."""
        if self.step >= steps:
            return None
        epoch = self.step + 1
        slot = epoch % self.slots
        if self.phase == "deposit":
            if not self.pending:
                self.pending = [("add", c) for c in range(self.cells) if self.contrib[self.step][c]]
                self.pending += [("signal", q) for q in range(self.world)]
            return self.pending
        if self.phase == "wait":
            if all(f >= epoch for f in self.flags):
                self.phase = "exchange"
                prev = (slot + self.slots - 1) % self.slots
                lo, hi = first_cell(self.r, self.cells, self.world), first_cell(self.r + 1, self.cells,
                                                                                 self.world)
                self.pending = [("read", c) for c in range(self.cells)]
                self.pending += [("clear", (prev, c)) for c in range(lo, hi)]
                return self.pending
            return []
        return self.pending

    def run(self, ev, ranks, expect):
        kind, arg = ev
        epoch = self.step + 1
        slot = epoch % self.slots
        if kind == "add":
            c = arg
            ranks[owner(c, self.cells, self.world)].accum[slot][c] += self.contrib[self.step][c]
        elif kind == "signal":
            ranks[arg].flags[self.r] = epoch
        elif kind == "read":
            c = arg
            self.local[c] = ranks[owner(c, self.cells, self.world)].accum[slot][c]
        elif kind == "clear":
            s, c = arg
            self.accum[s][c] = 0
        self.pending.remove(ev)
        if self.phase == "deposit" and not any(k == "add" for k, _ in self.pending) \
                and not self.pending:
            self.phase = "wait"
        elif self.phase == "exchange" and not self.pending:
            assert self.local == expect[self.step], (self.r, self.step)
            self.step += 1
            self.phase = "deposit"


def simulate(world, cells, steps, seed, slots=3):
    rng = random.Random(seed)
    ranks = [Rank(r, world, cells, steps, rng, slots) for r in range(world)]
    expect = [[sum(rk.contrib[s][c] for rk in ranks) for c in range(cells)] for s in range(steps)]
    while True:
        choices = []
        done = 0
        for rk in ranks:
            evs = rk.events(ranks, steps)
            if evs is None:
                done += 1
                continue
            if rk.phase == "deposit":
                # stream order inside the deposit: adds (any order), then signals
                adds = [e for e in evs if e[0] == "add"]
                evs = adds if adds else evs
            choices += [(rk, e) for e in evs]
        if done == world:
            return
        assert choices, "deadlock"
        rk, ev = rng.choice(choices)
        rk.run(ev, ranks, expect)


@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_three_slots_give_every_step_its_exact_total(world):
    for seed in range(300):
        simulate(world, cells=5, steps=6, seed=seed)


def test_two_slots_are_not_enough():
    """The model is sharp enough to see the hazard three slots avoid: with
    two, a fast rank's next deposit lands in a slot a slow rank is still
    reading or clearing."""
    failures = 0
    for seed in range(300):
        try:
            simulate(3, cells=5, steps=6, seed=seed, slots=2)
        except AssertionError:
            failures += 1
    assert failures > 0


def test_ownership_partitions_the_grids():
    """floor(i * world / k) and ceil(r * k / world) describe the same split:
    each grid has one owner and the owners' ranges tile [0, k)."""
    for k in (1, 2, 5, 16, 240):
        for world in range(1, 9):
            owned = []
            for r in range(world):
                lo, hi = first_cell(r, k, world), first_cell(r + 1, k, world)
                owned += list(range(lo, hi))
                assert all(owner(i, k, world) == r for i in range(lo, hi))
            assert owned == list(range(k))


def _handles_worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta

    from mog_solver_b200.sharded import exchange_handles

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        a, f = exchange_handles(bytes([rank]) * 64, bytes([100 + rank]) * 64)
        q.put((rank, a, f))
    finally:
        dist.destroy_process_group()


def test_ipc_handles_are_exchanged_in_rank_order():
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    world = 3
    procs = [ctx.Process(target=_handles_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get() for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    want_a = b"".join(bytes([r]) * 64 for r in range(world))
    want_f = b"".join(bytes([100 + r]) * 64 for r in range(world))
    for _, a, f in got:
        assert a == want_a and f == want_f


def test_exchange_handles_checks_sizes():
    from mog_solver_b200.sharded import exchange_handles

    with pytest.raises(ValueError):
        exchange_handles(b"\0" * 63, b"\0" * 64)


def test_shard_entry_points_reject_bad_arguments_without_a_gpu():
    """Argument checks come before any CUDA call."""
    from mog_solver_b200 import _lib

    lib = _lib.lib()
    assert lib.mog_shard_init(None, 0, 2) == _lib.MOG_ERR_ARG
    assert lib.mog_shard_deposit(None, None, 0, None) == _lib.MOG_ERR_ARG
    assert lib.mog_shard_exchange(None, None) == _lib.MOG_ERR_ARG
    assert lib.mog_shard_finish(None, None, None, 0, 0.0, None) == _lib.MOG_ERR_ARG
    assert lib.mog_shard_connect(None, None, None) == _lib.MOG_ERR_ARG
    assert lib.mog_shard_connect_local(None, None) == _lib.MOG_ERR_ARG
    assert lib.mog_shard_export(None, None, None) == _lib.MOG_ERR_ARG
