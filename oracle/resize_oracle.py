"""CPU oracle of the reference's data/resize.py resampling.

TEST INFRASTRUCTURE ONLY: the parity checker of sarbp_resize (tests/);
the product library never imports it.

The reference resizes platform arrays with scikit-image
(`skimage.transform.resize(a, shape, preserve_range=True)`,
data/resize.py:50-58), a third-party dependency it does not vendor or pin
(data/resize.py:7 imports it; no version is named anywhere in the
reference) and which is absent here.  This module restates the published
algorithm of skimage's `resize` (skimage >= 0.19, skimage/transform/
_warps.py) for the arguments the reference passes -- order 1 (linear),
mode 'reflect', anti-aliasing on by default when the output is smaller on
any axis, clip to the input range, preserve_range -- on scipy.ndimage, the
library skimage itself calls for these steps:
  * f32 / f64 input is kept as is (preserve_range), other types become f64;
  * anti-aliasing: ndimage.gaussian_filter(image, sigma = max(0, (f - 1) / 2)
    per axis, f = in / out, mode 'mirror' -- numpy's 'reflect');
  * ndimage.zoom(filtered, out / in, order=1, mode='mirror', grid_mode=True);
  * clip to [min, max] of the input.
Parity of this restatement with the reference's own environment is
unpinned (the reference ships no resized data); it is pinned to
scipy.ndimage's implementation of the same steps.
"""
import numpy as np
from scipy import ndimage as ndi


def sk_resize(image, output_shape):
    """skimage.transform.resize(image, output_shape, preserve_range=True)
    with its default order 1, mode 'reflect', anti_aliasing and clip."""
    image = np.asarray(image)
    output_shape = tuple(int(x) for x in output_shape)
    input_shape = image.shape
    if image.dtype.char not in "df":
        image = image.astype(np.float64)
    lo, hi = image.min(), image.max()
    factors = np.divide(input_shape, output_shape)
    if any(o < i for o, i in zip(output_shape, input_shape)):
        sigma = np.maximum(0, (factors - 1) / 2)
        filtered = ndi.gaussian_filter(image, sigma, cval=0, mode="mirror")
    else:
        filtered = image
    out = ndi.zoom(filtered, [1 / f for f in factors], order=1, mode="mirror", cval=0, grid_mode=True)
    np.clip(out, lo, hi, out=out)
    return out


def resize_platform(delta_r, k_r, npulses, nsamples, phs, pos, p=None, s=None, scale_p=1.0, scale_s=1.0):
    """The array arithmetic of data/resize.py:14-58 on loaded arrays; returns
    (delta_r, k_r, npulses, nsamples, phs, pos)."""
    if p is not None and p > 0:
        scale_p = p / npulses
    else:
        p = int(npulses * scale_p)
    if s is not None and s > 0:
        scale_s = s / nsamples
    else:
        s = int(nsamples * scale_s)
    delta_r = delta_r / scale_s
    k_r = sk_resize(k_r * scale_s, (s,))
    phs = sk_resize(np.real(phs), (p, s)) + 1j * sk_resize(np.imag(phs), (p, s))
    pos = sk_resize(pos, (p, pos.shape[1]))
    return delta_r, k_r, p, s, phs, pos
