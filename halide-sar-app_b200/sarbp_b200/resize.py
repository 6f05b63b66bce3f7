#!/usr/bin/env python3
"""Resize RITSAR-formatted platform data to other pulse and sample counts:
the reference's data/resize.py (data/resize.py:14-99), same arguments and
outputs, with the resampling on the device (sarbp_resize).

    python -m sarbp_b200.resize INDIR OUTDIR [-P PULSES | -p SCALE] [-S SAMPLES | -s SCALE]

Reads delta_r, k_r, n_hat (optional), npulses, nsamples, phs, pos and R_c
(.npy), and writes them resized: delta_r / scale_s; k_r * scale_s resampled
to the new sample count; phs (real and imaginary parts separately) to
(pulses, samples); pos to (pulses, 3); the rest unchanged.  The numpy
arithmetic around the resampling (scale factors, dtypes) is the reference's.
"""
import argparse
import os

import numpy as np


def resize(idir, odir, p, s, scale_p=1.0, scale_s=1.0, ctx=None):
    """Resize data from idir and save to odir (data/resize.py:14-70)."""
    from . import Context
    own = ctx is None
    ctx = ctx or Context(0)
    try:
        delta_r = np.load(os.path.join(idir, 'delta_r.npy'))
        k_r = np.load(os.path.join(idir, 'k_r.npy'))
        try:
            n_hat = np.load(os.path.join(idir, 'n_hat.npy'))
        except FileNotFoundError:
            n_hat = None
        npulses = np.load(os.path.join(idir, 'npulses.npy'))
        nsamples = np.load(os.path.join(idir, 'nsamples.npy'))
        phs = np.load(os.path.join(idir, 'phs.npy'))
        pos = np.load(os.path.join(idir, 'pos.npy'))
        R_c = np.load(os.path.join(idir, 'R_c.npy'))

        # p takes precedence over scale_p
        if p is not None and p > 0:
            scale_p = p / npulses
        else:
            p = int(npulses * scale_p)
            if p <= 0:
                raise ValueError('Scaling pulses resulted in count <= 0')
        print('pulses = ' + str(p))
        # s takes precedence over scale_s
        if s is not None and s > 0:
            scale_s = s / nsamples
        else:
            s = int(nsamples * scale_s)
            if s <= 0:
                raise ValueError('Scaling samples resulted in count <= 0')
        print('samples = ' + str(s))

        # delta_r and k_r are functions of frequency: adjust values and shape
        delta_r = delta_r / scale_s
        k_r = ctx.resize(k_r * scale_s, (s,))
        npulses = p
        nsamples = s
        phs = ctx.resize(np.real(phs), (p, s)) + 1j * ctx.resize(np.imag(phs), (p, s))
        pos = ctx.resize(pos, (p, pos.shape[1]))

        os.mkdir(odir)
        np.save(os.path.join(odir, 'delta_r.npy'), delta_r)
        np.save(os.path.join(odir, 'k_r.npy'), k_r)
        if n_hat is not None:
            np.save(os.path.join(odir, 'n_hat.npy'), n_hat)
        np.save(os.path.join(odir, 'npulses.npy'), npulses)
        np.save(os.path.join(odir, 'nsamples.npy'), nsamples)
        np.save(os.path.join(odir, 'phs.npy'), phs)
        np.save(os.path.join(odir, 'pos.npy'), pos)
        np.save(os.path.join(odir, 'R_c.npy'), R_c)
    finally:
        if own:
            ctx.close()


def main(argv=None):
    def positive(v):
        if v <= 0:
            raise argparse.ArgumentTypeError("Expected value > 0, got %s" % v)
        return v

    def positive_int(v):
        return positive(int(v))

    def positive_float(v):
        return positive(float(v))

    parser = argparse.ArgumentParser()
    parser.add_argument('indir', help='Data input directory')
    parser.add_argument('outdir', help='Data output directory')
    group = parser.add_mutually_exclusive_group()
    group.add_argument('-P', '--pulses', type=positive_int, help='The number of pulses')
    group.add_argument('-p', '--scale-pulses', default=1, type=positive_float,
                       help='The scale factor for number of pulses')
    group = parser.add_mutually_exclusive_group()
    group.add_argument('-S', '--samples', type=positive_int, help='The number of samples')
    group.add_argument('-s', '--scale-samples', default=1, type=positive_float,
                       help='The scale factor for number of samples')
    args = parser.parse_args(argv)
    resize(args.indir, args.outdir, args.pulses, args.samples, scale_p=args.scale_pulses,
           scale_s=args.scale_samples)


if __name__ == '__main__':
    main()
