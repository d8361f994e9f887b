"""The multi-GPU sample split on CPU: two gloo ranks render disjoint sample ranges of the
Cornell box with the CPU oracle (the same per-pixel PCG32 streams as the GPU kernels) and
reduce their FP64 films; the sum equals one render of all the samples. Also the max-over-
ranks timing helper."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

SPP = 4


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (os.path.join(root, "oracle"), os.path.join(root, "filianore-core_b200")):
        sys.path.insert(0, p)
    import oracle
    import filianore_b200 as fb
    from filianore_b200 import dist as fdist, scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        tab = oracle.Tables(fb.reference_tables())
        sc = scenes.cornell(24, 24)
        p = scenes.render_params(SPP, 8, fb.FL_SPECTRAL_HERO4, sample_offset=fdist.rank_sample_offset(rank, SPP))
        xyz, _ = oracle.render(sc, tab, p, nthreads=2)
        t = torch.from_numpy(np.ascontiguousarray(xyz))
        fdist.reduce_film(t, dst=0)
        slowest = fdist.max_over_ranks(1.0 + rank)
        if rank == 0:
            np.save(out_path, t.numpy())
            np.save(out_path + ".max.npy", np.array([slowest]))
    finally:
        dist.destroy_process_group()


def test_two_rank_sample_split_equals_single_render(tmp_path):
    import oracle
    import filianore_b200 as fb
    from filianore_b200 import scenes
    out = str(tmp_path / "film.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    summed = np.load(out)
    tab = oracle.Tables(fb.reference_tables())
    whole, _ = oracle.render(scenes.cornell(24, 24), tab, scenes.render_params(2 * SPP, 8, fb.FL_SPECTRAL_HERO4),
                             nthreads=2)
    assert np.allclose(summed, whole, rtol=1e-12, atol=1e-15)
    assert float(np.load(out + ".max.npy")[0]) == 2.0
