"""Device-resident jobs for the batched and served forms.

A DeviceJob synthesises one image-formation job (synth.make_from), uploads
its phase history, k_r and antenna positions, describes its image plane by
its axes (u, v, u_hat, v_hat: the device forms the pixel positions) and
owns its complex128 output (and optional u8 image) on the device.
"""
import numpy as np

from . import PREC_COMPAT, make_job, synth


class DeviceJob:
    def __init__(self, cfg, torch, device="cuda", u8=False, data=None):
        d = data if data is not None else synth.make_from(cfg)
        self.cfg, self.data = cfg, d
        f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device)
        f64 = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64)).to(device)
        self.phs = f32(d["phs"].view(np.float32))
        self.k_r = f32(d["k_r"])
        self.pos = f32(d["pos"])
        self.u, self.v = f64(d["u"]), f64(d["v"])
        self.nu, self.nv, self.P, self.S = d["nu"], d["nv"], d["P"], d["S"]
        self.out = torch.zeros((self.nv, self.nu, 2), dtype=torch.float64, device=device)
        self.out_u8 = torch.zeros((self.nv, self.nu), dtype=torch.uint8, device=device) if u8 else None
        db = d.get("db", (-40.0, 0.0))
        self.job = make_job(self.S, self.P, d["N_fft"], d["taylor"], self.nu, self.nv, d["delta_r"],
                            self.phs.data_ptr(), self.k_r.data_ptr(), self.pos.data_ptr(),
                            self.out.data_ptr(), u=self.u.data_ptr(), v=self.v.data_ptr(),
                            u_hat=d["u_hat"], v_hat=d["v_hat"],
                            out_u8=self.out_u8.data_ptr() if u8 else 0, dB_min=db[0], dB_max=db[1],
                            precision=-1, taylor_mode=d.get("taylor_mode", 0))
        self.units = self.nu * self.nv * self.P

    def image(self):
        return self.out.cpu().numpy().view(np.complex128)[..., 0]

    def device_bytes(self):
        """Inputs and outputs held on the device for this job."""
        n = self.phs.numel() * 4 + self.k_r.numel() * 4 + self.pos.numel() * 4
        n += (self.nu + self.nv) * 8 + self.out.numel() * 8
        return n + (self.out_u8.numel() if self.out_u8 is not None else 0)


class HostJob:
    """A job in host memory for the serving loop: phase history, k_r and
    positions (f32, and f64 for PREC_PRECISE), image-plane axes, and the
    host output images.  `alloc(shape, dtype)` makes the host arrays (pass
    a pinned allocator for asynchronous copies); several requests may share
    one HostJob's inputs, each with its own outputs (new_outputs)."""

    def __init__(self, cfg, alloc=None, u8=False, data=None):
        d = data if data is not None else synth.make_from(cfg)
        self.cfg, self.data = cfg, d
        self.alloc = alloc or (lambda shape, dtype: np.empty(shape, dtype))

        def put(a, dtype):
            a = np.asarray(a, dtype)
            h = self.alloc(a.shape, dtype)
            h[...] = a
            return h

        self.phs = put(d["phs"], np.complex64)
        self.k32, self.k64 = put(d["k_r"], np.float32), put(d["k_r"], np.float64)
        self.p32, self.p64 = put(d["pos"], np.float32), put(d["pos"], np.float64)
        self.u, self.v = put(d["u"], np.float64), put(d["v"], np.float64)
        self.nu, self.nv, self.P, self.S = d["nu"], d["nv"], d["P"], d["S"]
        self.units = self.nu * self.nv * self.P
        self.u8 = u8

    def new_outputs(self):
        out = self.alloc((self.nv, self.nu), np.complex128)
        u8 = self.alloc((self.nv, self.nu), np.uint8) if self.u8 else None
        return out, u8

    def job(self, out, out_u8=None, precision=-1):
        d = self.data
        db = d.get("db", (-40.0, 0.0))
        p = lambda a: a.ctypes.data
        return make_job(self.S, self.P, d["N_fft"], d["taylor"], self.nu, self.nv, d["delta_r"],
                        p(self.phs), p(self.k32), p(self.p32), p(out), u=p(self.u), v=p(self.v),
                        u_hat=d["u_hat"], v_hat=d["v_hat"], k_r64=p(self.k64), pos64=p(self.p64),
                        out_u8=p(out_u8) if out_u8 is not None else 0, dB_min=db[0], dB_max=db[1],
                        precision=precision, taylor_mode=d.get("taylor_mode", 0))
