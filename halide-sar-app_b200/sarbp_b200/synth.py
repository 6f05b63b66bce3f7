"""Seeded synthetic inputs at the benchmark configurations' shapes.

The reference is exercised on recorded AFRL / Sandia phase histories (the
Sandia phase history is not even shipped); these generators stand in for
them with stepped-frequency data of the same shapes, value distributions
and geometry scale:

  plain_small  469 x 424, f0 9.29 GHz, 1.5 MHz step, 10 km, 30 deg
               depression, 4 deg span, 20 scatterers in +-25 m, 20 dB SNR,
               512^2 image over 50 m, Taylor 17, upsample 2, dB -30..0
  plain_large  1999 x 1024, f0 16.7 GHz, 0.59 MHz step, 8 km, 45 deg,
               3 deg span, 200 scatterers + uniform-amplitude clutter grid,
               2048^2 image over 100 m, Taylor 30, upsample 2, dB -45..0
  plain_mid    plain_large's aperture on a 1024^2 image over 50 m
  precision    4000 x 2048 at 20 km, 300 scatterers, 4096^2 image
  sandia_8192  8192 x 8192 (the reference's Sandia 8192^2 runs), 8192^2 over 400 m
  sandia_2048  1999 x 1800 (the reference's one-node Sandia run, whose CLI
               forms a 2048^2 image over the 254 m range swath), 200
               scatterers in +-100 m
  batch        96 uneven jobs (image 256^2..2048^2, 128-2000 pulses,
               256/512/1024 samples, Taylor 17-35 dB, 5-15 km, 20-50 deg)

Each scene is a list of point scatterers (x, y, z, Re a, Im a); the phase
history is S(f, p) = sum_i a_i exp(+j 4 pi f / c (|p| - |p - x_i|)) plus
complex Gaussian noise, generated by libsarbp_b200's host generator.
"""
import ctypes

import numpy as np

from . import img_plane_create, n_fft_for, pixel_locs
from ._lib import TAYLOR_FLOAT, TAYLOR_REF, check, lib

C = 299792458.0

CONFIGS = {
    "plain_small": dict(P=469, S=424, f0=9.29e9, df=1.5e6, R0=10e3, dep=30.0, span=4.0,
                        nscat=20, half=25.0, clutter=0, snr=20.0, n=512, extent=50.0,
                        taylor=17, upsample=2, db=(-30.0, 0.0)),
    "plain_large": dict(P=1999, S=1024, f0=16.7e9, df=0.59e6, R0=8e3, dep=45.0, span=3.0,
                        nscat=200, half=45.0, clutter=32, snr=20.0, n=2048, extent=100.0,
                        taylor=30, upsample=2, db=(-45.0, 0.0)),
    # plain_large's aperture on a 1024^2 image over 50 m (profiling captures)
    "plain_mid": dict(P=1999, S=1024, f0=16.7e9, df=0.59e6, R0=8e3, dep=45.0, span=3.0,
                      nscat=200, half=22.0, clutter=32, snr=20.0, n=1024, extent=50.0,
                      taylor=30, upsample=2, db=(-45.0, 0.0)),
    "precision": dict(P=4000, S=2048, f0=16.7e9, df=0.59e6, R0=20e3, dep=45.0, span=3.0,
                      nscat=300, half=45.0, clutter=32, snr=20.0, n=4096, extent=100.0,
                      taylor=30, upsample=2, db=(-45.0, 0.0)),
    # the shape of the reference's Sandia 8192^2 runs (8192 pulses x 8192
    # samples; N_fft 32768 by the reference's sizing rule): plain_large's band over 8x the samples, so the
    # range swath (2 km) covers a 8192^2 image over 400 m
    "sandia_8192": dict(P=8192, S=8192, f0=16.7e9, df=0.59e6 / 8, R0=8e3, dep=45.0, span=3.0,
                        nscat=60, half=180.0, clutter=0, snr=20.0, n=8192, extent=400.0,
                        taylor=30, upsample=2, db=(-45.0, 0.0)),
    "sandia_2048": dict(P=1999, S=1800, f0=16.7e9, df=0.59e6, R0=8e3, dep=45.0, span=3.0,
                        nscat=200, half=100.0, clutter=0, snr=20.0, n=2048, extent=254.0,
                        taylor=30, upsample=2, db=(-45.0, 0.0)),
}


def scene(nscat, half, clutter, seed):
    """Point scatterers uniform in +-half (x, y), complex-normal amplitudes,
    plus a clutter x clutter grid of unit-amplitude, random-phase points of
    amplitude 0.1 spread over the same square."""
    rng = np.random.default_rng(seed)
    pts = np.zeros((nscat, 5))
    pts[:, 0:2] = rng.uniform(-half, half, size=(nscat, 2))
    pts[:, 3] = rng.normal(size=nscat) / np.sqrt(2)
    pts[:, 4] = rng.normal(size=nscat) / np.sqrt(2)
    if clutter:
        g = np.linspace(-half, half, clutter)
        gx, gy = np.meshgrid(g, g)
        ph = rng.uniform(0, 2 * np.pi, size=gx.size)
        cl = np.zeros((gx.size, 5))
        cl[:, 0], cl[:, 1] = gx.ravel(), gy.ravel()
        cl[:, 3], cl[:, 4] = 0.1 * np.cos(ph), 0.1 * np.sin(ph)
        pts = np.concatenate([pts, cl])
    return pts


def phase_history(S, P, f0, df, R0, dep, span, scat, snr_db, seed, nthreads=0):
    """Returns (phs complex64 [P, S], pos f64 [P, 3], k_r f64 [S])."""
    scat = np.ascontiguousarray(scat, np.float64)
    phs = np.empty((P, S), np.complex64)
    pos = np.empty((P, 3), np.float64)
    k_r = np.empty(S, np.float64)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    check(lib().sarbp_synth_phase_history(int(S), int(P), float(f0), float(df), float(R0),
                                          float(dep), float(span), p(scat), int(scat.shape[0]),
                                          float(snr_db), ctypes.c_uint64(int(seed)), p(phs), p(pos),
                                          p(k_r), int(nthreads)))
    return phs, pos, k_r


def grid_plane(n, extent, pos, delta_r, S, P):
    """Explicit square image plane: n x n pixels over extent metres, axes
    from the reference's image-plane construction (ImgPlane.cpp) with
    R_c = mid-aperture position and n_hat = (0, 0, 1)."""
    R_c = pos[P // 2].astype(np.float32)
    ip = img_plane_create(S, P, delta_r, R_c, with_pixel_locs=False)
    d = extent / n
    u = (np.arange(n) - n // 2) * d
    v = (np.arange(n) - n // 2) * d
    return dict(u=u, v=v, u_hat=ip["u_hat"], v_hat=ip["v_hat"], R_c=R_c, nu=n, nv=n)


def make(name="plain_small", seed=1, with_r=True, overrides=None, nthreads=0):
    """Synthesises one configuration; returns a dict with phs, pos (f64),
    k_r (f64), delta_r, N_fft, taylor, u, v, u_hat, v_hat, r (SoA, optional),
    nu, nv, db, scat."""
    cfg = dict(CONFIGS[name])
    if overrides:
        cfg.update(overrides)
    scat = scene(cfg["nscat"], cfg["half"], cfg["clutter"], seed)
    phs, pos, k_r = phase_history(cfg["S"], cfg["P"], cfg["f0"], cfg["df"], cfg["R0"], cfg["dep"],
                                  cfg["span"], scat, cfg["snr"], seed, nthreads)
    if cfg.get("az"):
        # the whole geometry turned by az degrees about z (the phase history
        # only sees relative positions): the image plane's axes turn with it
        a = np.deg2rad(cfg["az"])
        rot = np.array([[np.cos(a), -np.sin(a), 0.0], [np.sin(a), np.cos(a), 0.0], [0.0, 0.0, 1.0]])
        pos = pos @ rot.T
        scat = scat.copy()
        scat[:, :3] = scat[:, :3] @ rot.T
    delta_r = C / (2.0 * cfg["S"] * cfg["df"])
    g = grid_plane(cfg["n"], cfg["extent"], pos, delta_r, cfg["S"], cfg["P"])
    out = dict(cfg=cfg, name=name, phs=phs, pos=pos, k_r=k_r, delta_r=delta_r,
               N_fft=n_fft_for(cfg["S"], cfg["upsample"]), taylor=cfg["taylor"], db=cfg["db"],
               scat=scat, S=cfg["S"], P=cfg["P"], **g)
    if with_r:
        out["r"] = pixel_locs(g["u"], g["v"], g["u_hat"], g["v_hat"])
    return out


def taylor_mode_for(level):
    """The reference's Taylor window (TAYLOR_REF) where it is defined, up to
    30 dB; above that its F_m denominator divides by zero (the Int32
    division of signal.h:40) and the float-quotient window (TAYLOR_FLOAT)
    is used."""
    return TAYLOR_REF if level <= 30 else TAYLOR_FLOAT


def batch_jobs(njobs=96, seed=7, sizes=(256, 512, 1024, 2048), pulses=(128, 2000),
               samples=(256, 512, 1024), taylors=(17, 35), ranges=(5e3, 15e3), deps=(20.0, 50.0)):
    """Parameters of uneven jobs (no data): list of dicts.  Taylor levels
    17-35 dB; each job's taylor_mode is taylor_mode_for(level)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(njobs):
        n = int(rng.choice(sizes))
        S = int(rng.choice(samples))
        df = float(rng.uniform(0.5e6, 1.5e6))
        delta_r = C / (2 * S * df)
        # image extent: a pixel of about half the range resolution
        extent = n * delta_r * 0.5
        jobs.append(dict(P=int(rng.integers(pulses[0], pulses[1] + 1)), S=S,
                         f0=float(rng.uniform(9e9, 17e9)), df=df,
                         R0=float(rng.uniform(*ranges)), dep=float(rng.uniform(*deps)),
                         span=float(rng.uniform(2.0, 4.0)), nscat=16, half=extent * 0.4,
                         clutter=0, snr=20.0, n=n, extent=extent,
                         taylor=int(rng.integers(taylors[0], taylors[1] + 1)), upsample=2,
                         db=(-40.0, 0.0), seed=int(seed * 1000 + i)))
        jobs[-1]["taylor_mode"] = taylor_mode_for(jobs[-1]["taylor"])
    return jobs


def make_from(cfg, with_r=False, nthreads=0):
    """Synthesises a job described by a batch_jobs() dict."""
    scat = scene(cfg["nscat"], cfg["half"], cfg["clutter"], cfg["seed"])
    phs, pos, k_r = phase_history(cfg["S"], cfg["P"], cfg["f0"], cfg["df"], cfg["R0"], cfg["dep"],
                                  cfg["span"], scat, cfg["snr"], cfg["seed"], nthreads)
    delta_r = C / (2.0 * cfg["S"] * cfg["df"])
    g = grid_plane(cfg["n"], cfg["extent"], pos, delta_r, cfg["S"], cfg["P"])
    out = dict(cfg=cfg, phs=phs, pos=pos, k_r=k_r, delta_r=delta_r,
               N_fft=n_fft_for(cfg["S"], cfg["upsample"]), taylor=cfg["taylor"], db=cfg["db"],
               taylor_mode=cfg.get("taylor_mode", TAYLOR_REF), scat=scat, S=cfg["S"], P=cfg["P"], **g)
    if with_r:
        out["r"] = pixel_locs(g["u"], g["v"], g["u_hat"], g["v_hat"])
    return out
