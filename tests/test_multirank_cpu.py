"""The multi-rank path on CPU: two gloo ranks (spawned processes, 127.0.0.1) exercise the
same helpers bench.py uses under torchrun -- rank discovery, the max-over-ranks device
time, the barrier -- and the z-slab ownership splits a volume exactly."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch

    from fastcone_b200 import dist as fd

    assert fd.env_ranks() == (rank, world, rank)
    assert fd.init("gloo", timeout_s=60)
    fd.barrier()
    t = fd.max_over_ranks(1.5 + rank, torch.device("cpu"))
    z0, z1 = fd.z_slab(1024, world, rank)
    fd.barrier()
    out.put((rank, t, z0, z1))
    import torch.distributed as dist

    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_max_and_split_slabs():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.5, 2.5]
    assert [(r[2], r[3]) for r in res] == [(0, 512), (512, 1024)]


@pytest.mark.parametrize("nz,world", [(1024, 8), (1000, 3), (64, 4), (7, 2), (384, 5)])
def test_z_slabs_partition_the_volume(nz, world):
    from fastcone_b200 import dist as fd

    covered = []
    for r in range(world):
        z0, z1 = fd.z_slab(nz, world, r)
        assert 0 <= z0 <= z1 <= nz
        if z1 > z0 and z1 < nz:
            assert (z1 - z0) % 32 == 0
        covered.extend(range(z0, z1))
    assert covered == list(range(nz))


def test_single_process_needs_no_group():
    import torch

    from fastcone_b200 import dist as fd

    assert not fd.init("gloo")
    assert fd.max_over_ranks(3.0, torch.device("cpu")) == 3.0
    with pytest.raises(ValueError):
        fd.z_slab(10, 2, 2)
