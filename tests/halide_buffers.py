"""ctypes view of halide_buffer_t (the public layout declared in
include/sarbp_halide.h) over numpy arrays, for calling the shim library the
way Halide-generated callers do.  A C-order numpy array of shape
(..., b, a) becomes a Halide buffer with dim 0 = a (stride 1), dim 1 = b, ..."""
import ctypes

import numpy as np


class HalideType(ctypes.Structure):
    _fields_ = [("code", ctypes.c_uint8), ("bits", ctypes.c_uint8), ("lanes", ctypes.c_uint16)]


class HalideDim(ctypes.Structure):
    _fields_ = [("min", ctypes.c_int32), ("extent", ctypes.c_int32), ("stride", ctypes.c_int32),
                ("flags", ctypes.c_uint32)]


class HalideBufferT(ctypes.Structure):
    _fields_ = [("device", ctypes.c_uint64), ("device_interface", ctypes.c_void_p),
                ("host", ctypes.c_void_p), ("flags", ctypes.c_uint64), ("type", HalideType),
                ("dimensions", ctypes.c_int32), ("dim", ctypes.POINTER(HalideDim)),
                ("padding", ctypes.c_void_p)]


_CODES = {"i": 0, "u": 1, "f": 2}


class HalideBuffer:
    """Keeps the array and the dim array alive as long as the buffer."""

    def __init__(self, arr):
        self.arr = np.ascontiguousarray(arr)
        shape = self.arr.shape[::-1]
        self.dims = (HalideDim * len(shape))()
        stride = 1
        for i, n in enumerate(shape):
            self.dims[i] = HalideDim(0, n, stride, 0)
            stride *= n
        self.buf = HalideBufferT()
        self.buf.host = self.arr.ctypes.data
        self.buf.type = HalideType(_CODES[self.arr.dtype.kind], self.arr.dtype.itemsize * 8, 1)
        self.buf.dimensions = len(shape)
        self.buf.dim = self.dims

    def ptr(self):
        return ctypes.byref(self.buf)
