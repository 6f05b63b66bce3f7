"""Distributed image formation over output-row blocks (the reference's
`cuda_distributed` schedule: output_img.distribute(y).send_to(0)), on the
CPU: gloo ranks as separate processes.

* Each rank forms its block with the reference-precision oracle straight
  into its send buffer; the blocks gathered on rank 0 equal the oracle's
  whole image bit for bit (every pixel is formed independently, so the
  split must not change a single value).
* The split and gather logic with a stand-in compute that records the pixel
  rows it was asked for and writes each pixel's own coordinates: every rank
  is asked for exactly its pixel rows, and rank 0 finds every output row
  where the reference's row flip puts it.
World sizes 2 and 3, including an image whose rows do not divide evenly and
a rank with an empty block."""
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


def _init(rank, world, port):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)


def _oracle_worker(rank, world, port, nv):
    import torch.distributed as dist
    import oracle
    from sarbp_b200.distributed import distributed_backprojection, oracle_compute
    _init(rank, world, port)
    try:
        d, u, v, r = _case(nv)
        k32, p32 = d["k_r"].astype(np.float32), d["pos"].astype(np.float32)
        compute = oracle_compute(oracle.backprojection, d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"],
                                 u, v, p32, r, nthreads=1)
        img = distributed_backprojection(compute, len(u), len(v))
        if rank == 0:
            full = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], p32, r,
                                         len(u), len(v), nthreads=1)
            assert img.shape == (len(v), len(u))
            assert np.array_equal(img, full), "gathered image differs from the whole-image oracle"
        else:
            assert img is None
    finally:
        dist.destroy_process_group()


def _fake_worker(rank, world, port, nu, nv):
    import torch
    import torch.distributed as dist
    from sarbp_b200.distributed import distributed_backprojection, output_row_blocks, pixel_rows
    _init(rank, world, port)
    try:
        calls = []

        def compute(a, b, out):
            calls.append((a, b))
            assert tuple(out.shape) == (b - a, nu, 2)
            # block row j holds pixel row b - 1 - j (the reference's row flip)
            rows = np.arange(b - a)
            out[..., 0] = torch.from_numpy(
                np.repeat((b - 1 - rows)[:, None], nu, axis=1).astype(np.float64))
            out[..., 1] = torch.from_numpy(np.tile(np.arange(nu, dtype=np.float64), (b - a, 1)))

        img = distributed_backprojection(compute, nu, nv)
        y0, y1 = output_row_blocks(nv, world)[rank]
        assert calls == ([pixel_rows(nv, y0, y1)] if y1 > y0 else [])
        want = (nv - 1 - np.arange(nv))[:, None] + 1j * np.arange(nu)[None, :]
        if rank == 0:
            assert np.array_equal(img, want)
        else:
            assert img is None
        # again into a caller's buffer on the destination rank, in place
        out = np.full((nv, nu), np.nan, np.complex128) if rank == 0 else None
        img = distributed_backprojection(compute, nu, nv, out=out)
        if rank == 0:
            assert img is out and np.array_equal(out, want)
        else:
            assert img is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nv", [(2, 40), (2, 37), (3, 4), (3, 50)])
def test_row_blocks_gathered_on_rank0(world, nv):
    import torch.multiprocessing as mp
    mp.spawn(_oracle_worker, args=(world, _free_port(), nv), nprocs=world, join=True)


@pytest.mark.parametrize("world,nu,nv", [(2, 5, 9), (3, 7, 3), (3, 4, 100)])
def test_split_and_gather_logic(world, nu, nv):
    import torch.multiprocessing as mp
    mp.spawn(_fake_worker, args=(world, _free_port(), nu, nv), nprocs=world, join=True)


def test_block_split_matches_distribute():
    from sarbp_b200.distributed import output_row_blocks, pixel_rows
    assert output_row_blocks(10, 3) == [(0, 4), (4, 8), (8, 10)]
    assert output_row_blocks(4, 3) == [(0, 2), (2, 4), (4, 4)]
    assert pixel_rows(10, 0, 4) == (6, 10)
