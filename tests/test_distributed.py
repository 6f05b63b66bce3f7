"""Distributed image formation over output-row blocks (the reference's
`cuda_distributed` schedule: output_img.distribute(y).send_to(0)), on the
CPU: gloo ranks as separate processes, each forming its block with the
reference-precision oracle, gathered on rank 0 and compared bit for bit
with the oracle's whole image (every pixel is formed independently, so the
split must not change a single value).  World sizes 2 and 3, including an
image whose rows do not divide evenly and a rank with an empty block."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case(nv):
    from sarbp_b200 import synth
    d = synth.make("plain_small", seed=8, with_r=False,
                   overrides=dict(P=60, S=96, n=64, extent=12.0, taylor=17))
    u = d["u"][:48]
    v = d["v"][:nv]
    r = synth.pixel_locs(u, v, d["u_hat"], d["v_hat"])
    return d, u, v, r


def _worker(rank, world, port, nv):
    import torch.distributed as dist
    import oracle
    from sarbp_b200.distributed import distributed_backprojection
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d, u, v, r = _case(nv)
        k32, p32 = d["k_r"].astype(np.float32), d["pos"].astype(np.float32)

        def compute(v_rows, r_rows):
            return oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], p32, r_rows,
                                         len(u), len(v_rows), nthreads=1)

        img = distributed_backprojection(compute, u, v, r)
        if rank == 0:
            full = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], p32, r,
                                         len(u), len(v), nthreads=1)
            assert img.shape == (len(v), len(u))
            assert np.array_equal(img, full), "gathered image differs from the whole-image oracle"
        else:
            assert img is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nv", [(2, 40), (2, 37), (3, 4), (3, 50)])
def test_row_blocks_gathered_on_rank0(world, nv):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), nv), nprocs=world, join=True)


def test_block_split_matches_distribute():
    from sarbp_b200.distributed import output_row_blocks, pixel_rows
    assert output_row_blocks(10, 3) == [(0, 4), (4, 8), (8, 10)]
    assert output_row_blocks(4, 3) == [(0, 2), (2, 4), (4, 4)]
    assert pixel_rows(10, 0, 4) == (6, 10)
