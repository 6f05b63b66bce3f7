"""Distributed image formation: one image split into output-row slabs over
the ranks of a torch.distributed group and gathered on one rank -- the
`-s cuda_distributed` schedule of the reference (backprojection.cpp:239-243:
`output_img.distribute(y).send_to(0)` splits the image's y extent into one
contiguous block per rank and sends every block to rank 0).

Every rank forms the whole range compression (the phase history is small
next to the image) and the pixels of its own block of output rows; no data
crosses between ranks before the gather.  Output row y holds pixel row
nv - 1 - y (the reference's row flip, backprojection.cpp:130), so the block
[y0, y1) is the job over pixel rows [nv - y1, nv - y0), whose own flipped
rows are exactly that block in order.
"""
import numpy as np


def output_row_blocks(nv, world):
    """[(y0, y1)] per rank: blocks of ceil(nv / world) output rows, the last
    one shorter (Halide's distribute() split)."""
    step = -(-nv // world)
    return [(min(nv, k * step), min(nv, (k + 1) * step)) for k in range(world)]


def pixel_rows(nv, y0, y1):
    """Pixel rows [a, b) that produce output rows [y0, y1)."""
    return nv - y1, nv - y0


def cuda_compute(ctx, phs, k_r, taylor_s_l, n_fft, delta_r, u, pos, **kw):
    """compute(v_rows, r_rows) on this rank's GPU through the host entry
    point (Context.backprojection_cuda)."""
    def compute(v_rows, r_rows):
        return ctx.backprojection_cuda(phs, k_r, taylor_s_l, n_fft, delta_r, u, v_rows, pos, r_rows, **kw)
    return compute


def cuda_compute_plane(ctx, phs, k_r, taylor_s_l, n_fft, delta_r, u, u_hat, v_hat, pos, **kw):
    """compute(v_rows, None) on this rank's GPU from the image-plane axes
    (Context.backprojection_plane): no pixel-position array at all."""
    def compute(v_rows, r_rows):
        return ctx.backprojection_plane(phs, k_r, taylor_s_l, n_fft, delta_r, u, v_rows, u_hat, v_hat, pos, **kw)
    return compute


def distributed_backprojection(compute, u, v, r, group=None, dst=0):
    """Forms this rank's block of output rows with compute(v_rows, r_rows)
    (-> complex128 [rows, nu]) and gathers the blocks on rank `dst`, which
    returns the whole image complex128 [nv, nu]; the other ranks return None.
    r is SoA [3, nu * nv] (pixel_locs) or None when compute forms the
    positions itself (then r_rows is None)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    nu, nv = len(u), len(v)
    blocks = output_row_blocks(nv, world)
    y0, y1 = blocks[rank]
    a, b = pixel_rows(nv, y0, y1)
    rows = y1 - y0
    if rows > 0:
        r_rows = None if r is None else np.ascontiguousarray(
            np.asarray(r).reshape(3, nv, nu)[:, a:b, :].reshape(3, rows * nu))
        img = np.ascontiguousarray(compute(np.asarray(v)[a:b], r_rows), np.complex128)
    else:
        img = np.zeros((0, nu), np.complex128)
    # equal-size blocks for the collective: pad to the first block's rows
    step = blocks[0][1] - blocks[0][0]
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    send = torch.zeros((step, nu, 2), dtype=torch.float64, device=dev)
    if rows:
        send[:rows] = torch.from_numpy(img.view(np.float64).reshape(rows, nu, 2)).to(dev)
    gather = [torch.empty_like(send) for _ in range(world)] if rank == dst else None
    dist.gather(send, gather_list=gather, dst=dst, group=group)
    if rank != dst:
        return None
    out = np.empty((nv, nu), np.complex128)
    for k, (g0, g1) in enumerate(blocks):
        if g1 > g0:
            out[g0:g1] = gather[k][: g1 - g0].cpu().numpy().view(np.complex128)[..., 0]
    return out
