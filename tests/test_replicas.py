"""bench.py's N > 1 path on CPU: world_size-2 gloo process groups run the
replica helpers the GPU run uses -- disjoint sample frames per rank, every
timing reduced to its maximum over ranks, clean teardown.  No GPU needed."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local = bench.init_replicas("gloo")
    times = [10.0 + r, 5.0 - r]  # rank 1 is slower in the first timing, faster in the second
    out[r] = (w, r, local, bench.frame_base(r), bench.max_over_ranks(times, device="cpu"))
    bench.finish_replicas()


@pytest.mark.parametrize("world", [2])
def test_replica_helpers_with_gloo(world):
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert sorted(res) == list(range(world))
    bases = {res[r][3] for r in range(world)}
    assert len(bases) == world                      # disjoint sample frames
    for r in range(world):
        w, rr, local, base, mx = res[r]
        assert (w, rr, local) == (world, r, r)
        assert mx == [10.0 + world - 1, 5.0]        # max over ranks, same on every rank


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.5], device="cpu") == [1.5, 2.5]
    assert bench.frame_base(0) == 0

