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

The data path stays on the device: each rank's kernels write its block
straight into its slice of an equal-size send buffer in device memory, the
blocks are gathered device to device (NCCL gather; with gloo, on the CPU,
the same buffers live in host memory), and the destination rank copies the
assembled image to the host once.
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


class DeviceCompute:
    """compute(a, b, out) on this rank's GPU: forms pixel rows [a, b) of the
    job into `out`, a float64 CUDA tensor [b - a, nu, 2] (complex128 rows in
    output order), through the device entry point.  The phase history, k_r,
    antenna positions and image-plane axes (or pixel positions r, SoA
    [3, nu * nv]) are uploaded once; the context launches on torch's current
    stream, so the gather that follows is ordered after the kernels."""

    def __init__(self, ctx, phs, k_r, taylor_s_l, n_fft, delta_r, u, v, pos, u_hat=None, v_hat=None, r=None,
                 precision=None, taylor_mode=0):
        import torch
        import sarbp_b200 as sb
        self.sb, self.torch, self.ctx = sb, torch, ctx
        dev = torch.device("cuda", torch.cuda.current_device())
        to = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt)).to(dev)
        phs = np.ascontiguousarray(phs, np.complex64)
        self.P, self.S = phs.shape
        self.phs = to(phs.view(np.float32), np.float32)
        wide = np.asarray(pos).dtype == np.float64
        self.precision = (sb.PREC_PRECISE if wide else sb.PREC_COMPAT) if precision is None else precision
        self.k32, self.p32 = to(k_r, np.float32), to(pos, np.float32)
        self.k64, self.p64 = to(k_r, np.float64), to(pos, np.float64)
        self.u, self.v = to(u, np.float64), to(v, np.float64)
        self.nu, self.nv = len(u), len(v)
        self.r = to(r, np.float64).reshape(3, self.nv, self.nu) if r is not None else None
        self.u_hat = (0.0, 0.0, 0.0) if u_hat is None else tuple(u_hat)
        self.v_hat = (0.0, 0.0, 0.0) if v_hat is None else tuple(v_hat)
        self.taylor, self.n_fft, self.delta_r, self.taylor_mode = taylor_s_l, n_fft, delta_r, taylor_mode
        ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)

    def __call__(self, a, b, out):
        sb = self.sb
        rows = b - a
        kw = {}
        keep = None
        if self.r is not None:
            keep = self.r[:, a:b, :].contiguous()  # rows a..b of each coordinate
            kw["r"] = keep.data_ptr()
        else:
            kw.update(u=self.u.data_ptr(), v=self.v.data_ptr() + 8 * a, u_hat=self.u_hat, v_hat=self.v_hat)
        job = sb.make_job(self.S, self.P, self.n_fft, self.taylor, self.nu, rows, self.delta_r,
                          self.phs.data_ptr(), self.k32.data_ptr(), self.p32.data_ptr(), out.data_ptr(),
                          k_r64=self.k64.data_ptr(), pos64=self.p64.data_ptr(), precision=self.precision,
                          taylor_mode=self.taylor_mode, **kw)
        self.ctx.run_jobs([job])
        self.ctx.synchronize()  # raises on a kernel status error; `keep` is read by then


def form_block(compute, nu, nv, world, rank, device="cpu"):
    """This rank's equal-size send buffer (float64 [ceil(nv/world), nu, 2]
    on `device`) with its block of output rows formed by compute(a, b, out)
    into the leading rows."""
    import torch
    blocks = output_row_blocks(nv, world)
    y0, y1 = blocks[rank]
    step = blocks[0][1] - blocks[0][0]
    send = torch.zeros((step, nu, 2), dtype=torch.float64, device=device)
    if y1 > y0:
        a, b = pixel_rows(nv, y0, y1)
        compute(a, b, send[: y1 - y0])
    return send


def assemble(gathered, nu, nv, out=None):
    """The image complex128 [nv, nu] (host) from the ranks' send buffers in
    rank order, each block copied once into its rows of `out` (a C-order
    complex128 [nv, nu] host array, written in place; page-locked memory
    makes the device-to-host copies fastest) or of a new array."""
    import torch
    world = len(gathered)
    if out is None:
        out = np.empty((nv, nu), np.complex128)
    if out.shape != (nv, nu) or out.dtype != np.complex128 or not out.flags.c_contiguous:
        raise ValueError("out must be a C-order complex128 [nv, nu] array")
    o = torch.from_numpy(out.view(np.float64).reshape(nv, nu, 2))
    for g, (y0, y1) in zip(gathered, output_row_blocks(nv, world)):
        if y1 > y0:
            o[y0:y1].copy_(g[: y1 - y0])
    return out


def distributed_backprojection(compute, nu, nv, group=None, dst=0, out=None):
    """Forms this rank's block of output rows with compute(a, b, out) (pixel
    rows [a, b) into the float64 tensor out [b - a, nu, 2], on the CUDA
    device for an NCCL group, in host memory for gloo) and gathers the
    blocks on rank `dst`, which returns the whole image complex128 [nv, nu]
    (in `out` when given, see assemble); the other ranks return None."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    device = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    send = form_block(compute, nu, nv, world, rank, device)
    gather = [torch.empty_like(send) for _ in range(world)] if rank == dst else None
    dist.gather(send, gather_list=gather, dst=dst, group=group)
    if rank != dst:
        return None
    return assemble(gather, nu, nv, out)


def oracle_compute(backprojection, phs, k_r, taylor_s_l, n_fft, delta_r, u, v, pos, r, **kw):
    """compute(a, b, out) from a CPU backprojection function with the
    oracle's signature (phs, k_r, taylor, n_fft, delta_r, pos, r, nu, nv):
    pixel rows [a, b) of r (SoA [3, nu * nv]) written into a host tensor."""
    nu, nv = len(u), len(v)
    r3 = np.asarray(r).reshape(3, nv, nu)

    def compute(a, b, out):
        import torch
        rr = np.ascontiguousarray(r3[:, a:b, :].reshape(3, (b - a) * nu))
        img = backprojection(phs, k_r, taylor_s_l, n_fft, delta_r, pos, rr, nu, b - a, **kw)
        out.copy_(torch.from_numpy(np.ascontiguousarray(img).view(np.float64).reshape(b - a, nu, 2)))
    return compute
