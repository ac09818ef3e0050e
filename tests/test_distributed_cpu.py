"""Multi-rank host logic on CPU (gloo, world size 2): sharding, per-rank
Philox streams, the grid all-reduce (bit-identical to the one-process grid
of the whole population) and failure detection on the host (a rank that
leaves makes the other's next collective end with an error, no GPU
involved)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from flexpart_gpu import distributed as fd
from flexpart_gpu import synthetic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port, timeout_s=30):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def test_shard_range_covers_every_slot_once():
    for n in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            ranges = [fd.shard_range(n, world, r) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [hi - lo for lo, hi in ranges]
            assert max(sizes) - min(sizes) <= 1


def test_shard_scenarios_balances_and_partitions():
    ens = synthetic.config2(n_scenarios=256)
    counts = [s.particle_count for s in ens.sources]
    for world in (2, 4, 8):
        parts = fd.shard_scenarios(counts, world)
        flat = sorted(s for p in parts for s in p)
        assert flat == list(range(256))
        loads = [sum(counts[s] for s in p) for p in parts]
        assert max(loads) - min(loads) <= max(counts)
        assert fd.shard_scenarios(counts, world) == parts


def test_rank_counters_are_distinct_streams():
    from oracle import orc

    c0 = fd.rank_counter([5, 0, 0, 0], 0)
    c1 = fd.rank_counter([5, 0, 0, 0], 1)
    assert c0 != c1 and c0[:3] == c1[:3]
    assert orc.philox(c0, (42, 0)) != orc.philox(c1, (42, 0))
    # a year of 900 s steps over 1e9 slots (2 blocks each) never carries into the top word
    far = orc.counter_add(c0, 2 * 10**9 * 35_040)
    assert far[3] == c0[3] and far[:3] != c0[:3]


def _grid_worker(rank, world, port, q):
    dist = _init(rank, world, port)
    try:
        _grid_body(rank, world, q, dist)
    except Exception as e:  # noqa: BLE001 - reported to the parent
        q.put(("error", repr(e)))
        raise
    finally:
        dist.destroy_process_group()


def _grid_body(rank, world, q, dist):
    from oracle import orc

    scn = synthetic.config1(particles=40_000)
    rec = synthetic.particles_at_sources(scn, 40_000, seed=9)
    st = orc.State.from_records(rec)
    lo, hi = fd.shard_range(len(rec), world, rank)
    part = orc.State.from_records(rec[lo:hi])
    c, m, _ = orc.grid(part, hi - lo, 0, 1e6, scn.outheights, scn.out_shape)
    c, m = fd.allreduce_grids(c, m)
    if rank == 0:
        c1, m1, _ = orc.grid(st, len(rec), 0, 1e6, scn.outheights, scn.out_shape)
        q.put((bool(np.array_equal(c, c1)), bool(np.array_equal(m, m1)), int(c.sum())))


def test_sharded_grid_allreduce_is_bit_identical_to_one_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_grid_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert res[0] is True and res[1] is True, res
    assert res[2] == 40_000


def _leaving_worker(rank, world, port, q):
    dist = _init(rank, world, port, timeout_s=5)
    import torch

    t = torch.ones(4)
    dist.all_reduce(t)                    # both ranks take part in the first step
    if rank == 1:
        os._exit(0)                       # rank 1 leaves between steps, no collective in flight
    try:
        dist.all_reduce(t)                # rank 0's next collective cannot complete
        q.put("completed")
    except Exception as e:                # noqa: BLE001 - any error is the detection
        q.put("error: " + type(e).__name__)


def test_a_rank_that_leaves_is_detected_by_the_next_collective():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_leaving_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert res.startswith("error"), res


def _gradient_worker(rank, world, port, q):
    dist = _init(rank, world, port)
    try:
        rng = np.random.default_rng(100 + rank)
        g = rng.standard_normal(5000) * 10.0 ** rng.uniform(-6, 2, 5000)
        s = fd.allreduce_gradient_fixed_point(g)
        if rank == 0:
            parts = [np.random.default_rng(100 + r) for r in range(world)]
            arrays = [p.standard_normal(5000) * 10.0 ** p.uniform(-6, 2, 5000) for p in parts]
            ref = fd.fixed_point_sum(arrays)
            flipped = fd.fixed_point_sum(arrays[::-1])
            exact = np.sum(np.array(arrays, np.float64), axis=0)
            q.put((bool(np.array_equal(s, ref)), bool(np.array_equal(ref, flipped)),
                   float(np.max(np.abs(s - exact)) / np.max(np.abs(exact)))))
    except Exception as e:  # noqa: BLE001 - reported to the parent
        q.put(("error", repr(e)))
        raise
    finally:
        dist.destroy_process_group()


def test_wind_bias_gradient_sum_over_ranks_is_order_independent():
    """The one exchange of an inversion sharded by instance: the wind-bias
    gradient summed in fixed point equals the one-process fixed-point sum
    bit for bit (in either rank order) and the float sum to ~1e-16."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gradient_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert res[0] is True and res[1] is True, res
    assert res[2] < 1e-15, res
