"""The multi-GPU path shards samples per pixel across ranks (disjoint iteration ranges, the
RNG is keyed on the iteration) and sums the FP32 images with one all-reduce. Checked here with
world_size-2 gloo ranks on the CPU, each rank rendering its share with the CPU oracle as the
stand-in for its GPU: the reduced image equals the single-process image of all samples."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

SPP = 4


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def rank_iters(rank: int, spp: int):
    """Iterations a rank renders, the partition bench.py uses for weak scaling."""
    return 1 + rank * 1000 * spp, spp


def worker(rank, world, port, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, here)
    import torch
    import luxion_b200 as lx
    import oracle_lib as ol
    from luxion_b200._ffi import default_options
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    s = lx.cornell36(16, 16)
    first, n = rank_iters(rank, SPP)
    img, _ = ol.OracleScene(s).render(default_options(direct_light_sampling=1), first, n, threads=1)
    t = torch.from_numpy(img.copy())
    dist.all_reduce(t)
    if rank == 0:
        np.save(out, t.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_spp_sharded_reduce_equals_single_process(tmp_path):
    import luxion_b200 as lx
    import oracle_lib as ol
    from luxion_b200._ffi import default_options
    out = str(tmp_path / "img.npy")
    mp.start_processes(worker, args=(2, free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    s = lx.cornell36(16, 16)
    o = ol.OracleScene(s)
    opt = default_options(direct_light_sampling=1)
    want = np.zeros_like(got)
    for rank in range(2):
        first, n = rank_iters(rank, SPP)
        want += o.render(opt, first, n, threads=1)[0]
    assert np.allclose(got, want, rtol=1e-6, atol=1e-6)
    assert not np.array_equal(got, 2 * o.render(opt, 1, SPP, threads=1)[0])  # disjoint streams


def test_rank_partition_is_disjoint():
    spans = [range(a, a + n) for a, n in (rank_iters(r, 16) for r in range(8))]
    seen = set()
    for sp in spans:
        assert not (seen & set(sp))
        seen |= set(sp)
