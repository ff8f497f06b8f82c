"""The spp-sharded multi-GPU path with its GPU side: two ranks as two processes, each rendering
its own iteration range on the device, copying its FP32 sum device to device
(lux_copy_image_device, as bench.py does before the all-reduce) and summing over gloo. The
reduced image equals the sum of the two ranges rendered apart, bit for bit.

Both ranks use the one GPU of the test box; their renders are independent (no kernel waits on
the other rank) and the exchange is the host all-reduce, so nothing here depends on two
GPUs running together."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

SPP = 6


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def rank_iters(rank: int):
    """First iteration and count of a rank's samples (the partition bench.py uses)."""
    return 1 + rank * 1000 * SPP, SPP


def scene():
    import luxion_b200 as lx
    return lx.random_scene(seed=17, num_instances=10, total_tris=20000, min_tris=1000, max_tris=4000,
                           num_emissive=2, num_textures=2, texture_size=32, env_width=64, env_height=32,
                           width=48, height=32, trace_depth=6)


def options(**kw):
    from luxion_b200._ffi import default_options
    return default_options(direct_light_sampling=1, env_importance_sampling=1, spp_per_wave=2, **kw)


def worker(rank, world, port, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    import torch
    import luxion_b200 as lx
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    s = scene()
    r = lx.Renderer(s, options())
    first, n = rank_iters(rank)
    r.render(first, n)
    img = torch.zeros(s.width * s.height * 3, dtype=torch.float32, device="cuda")
    r.copy_image_device(img.data_ptr())
    torch.cuda.synchronize()
    r.close()
    t = img.cpu()
    dist.all_reduce(t)
    if rank == 0:
        np.save(out, t.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_on_the_device_reduce_to_the_sum_of_their_ranges(tmp_path):
    import luxion_b200 as lx
    out = str(tmp_path / "img.npy")
    mp.start_processes(worker, args=(2, free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    s = scene()
    parts = []
    for rank in range(2):
        r = lx.Renderer(s, options())
        first, n = rank_iters(rank)
        r.render(first, n)
        parts.append(r.image_sum().reshape(-1))
        r.close()
    want = parts[0] + parts[1]
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert float(want.sum()) > 0
