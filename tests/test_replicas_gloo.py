"""The multi-GPU mode runs independent replicas (one process per GPU): the
process group carries only the barrier around the timed region and the
maximum of the per-rank times.  This drives that coordination with two
gloo ranks on the CPU: every rank gets the slowest time, the whole-job rate
counts the units of all ranks over that time, and each replica gets its own
seed."""
import multiprocessing as mp
import os
import socket


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from paratt_b200.replicas import Replicas

    r = Replicas("gloo", timeout_s=60)
    r.barrier()
    slowest = r.max(1.5 + rank)
    rate = r.job_rate(8, 2.0 + rank)
    q.put((rank, slowest, rate, r.seed(3), r.world))
    r.barrier()
    r.close()


def test_two_replicas_over_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert [x[1] for x in res] == [2.5, 2.5]
    assert [x[2] for x in res] == [world * 8 / 3.0] * world
    assert [x[3] for x in res] == [3, 4]
    assert [x[4] for x in res] == [world] * world


def test_single_process_needs_no_group():
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    from paratt_b200.replicas import Replicas

    r = Replicas("gloo")
    assert r.world == 1 and r.rank == 0
    r.barrier()
    assert r.max(4.0) == 4.0
    assert r.job_rate(10, 2.0) == 5.0
    r.close()


def _batch_worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from paratt_b200 import workloads as W
    from paratt_b200.replicas import Replicas

    r = Replicas("gloo", timeout_s=60)
    shapes = W.batch_shapes(64, 4)
    shards = W.shard_by_cost([W.rounding_cost(s) for s in shapes], r.world)
    mine = shards[r.rank]
    # stand-in for the rounding of this rank's trains: the result of train i
    # is its index and its rank caps (what the benchmark gathers per train)
    results = [(i, list(shapes[i][3])) for i in mine]
    allres = r.gather(results)
    q.put((rank, shards, allres))
    r.close()


def test_batch_instances_sharded_over_two_ranks():
    """The batched-rounding workload split over 2 gloo ranks by instance,
    balanced by rounding cost: the shards are disjoint and cover all 64
    trains, every rank computes the same split, the heavier shard carries at
    most 10 % more than half the work, and rank 0 gathers every train's
    result."""
    from paratt_b200 import workloads as W

    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_batch_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    shards = res[0][1]
    assert res[1][1] == shards
    assert sorted(shards[0] + shards[1]) == list(range(64))
    shapes = W.batch_shapes(64, 4)
    cost = [W.rounding_cost(s) for s in shapes]
    loads = [sum(cost[i] for i in sh) for sh in shards]
    assert max(loads) <= 1.1 * sum(cost) / world
    gathered = [t for part in res[0][2] for t in part]
    assert sorted(i for i, _ in gathered) == list(range(64))
    assert all(caps == list(shapes[i][3]) for i, caps in gathered)
