"""Frame development on the GPU: the path tracer's accumulation image to
8-bit sRGB (src/post.rs:25-160) with the kernels of libpyro_b200.so.

    dev = Developer(w, h)
    cam = Camera(auto_exposure, ev, glare)           # pyro_b200.post
    rgb8 = dev.develop(cam, renderer.accum.data_ptr(), frame_dt, stream)

Per frame: the mean radiance and the exact 99.5th luminance percentile on
the device (pyro_post_select), the exposure state's update on the host
(Camera.exposure_from, the same arithmetic as the CPU path), then exposure,
glare, ACES, sRGB, dither and quantisation on the device
(pyro_post_develop), and one read-back of the 8-bit image.  The CPU
restatement in pyro_b200.post is the check: every value up to the sRGB
curve agrees bit for bit, and the 8-bit image within one level where the
device's and the host's powf differ in the last place.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _abi
from .post import Camera, percentile_rank

F32 = np.float32


class Developer:
    """Device buffers for frames of w x h pixels (torch memory)."""

    def __init__(self, w: int, h: int):
        import torch
        self.w, self.h = int(w), int(h)
        n = self.w * self.h
        dev = torch.device("cuda")
        self.img = torch.empty(3 * n, dtype=torch.float32, device=dev)
        self.keys = torch.empty(n, dtype=torch.int32, device=dev)
        self.sel = torch.empty(_abi.POST_SEL_WORDS, dtype=torch.int32, device=dev)
        self.scratch = torch.empty(12 * n, dtype=torch.float32, device=dev)
        self.out = torch.empty(3 * n, dtype=torch.uint8, device=dev)
        self._lib = _abi.load()

    def select(self, accum_ptr: int, stream: Optional[int] = None) -> np.float32:
        """Mean radiance into self.img and the 99.5th luminance percentile."""
        n = self.w * self.h
        v = ctypes.c_float()
        _abi.check("pyro_post_select", self._lib.pyro_post_select(
            ctypes.c_void_p(accum_ptr), self.w, self.h, percentile_rank(n),
            ctypes.c_void_p(self.img.data_ptr()), ctypes.c_void_p(self.keys.data_ptr()),
            ctypes.c_void_p(self.sel.data_ptr()), ctypes.byref(v),
            ctypes.c_void_p(stream) if stream else None))
        return F32(v.value)

    def develop(self, cam: Camera, accum_ptr: int, frame_dt: float,
                stream: Optional[int] = None, lin_out: Optional[int] = None) -> np.ndarray:
        """(h, w, 3) uint8 sRGB of one frame; updates cam's exposure state."""
        import torch
        v = self.select(accum_ptr, stream)
        ev = cam.exposure_from(v, frame_dt)
        gain = np.power(F32(2.0), ev)
        _abi.check("pyro_post_develop", self._lib.pyro_post_develop(
            ctypes.c_void_p(self.img.data_ptr()), self.w, self.h, float(gain), float(cam.glare),
            ctypes.c_void_p(self.scratch.data_ptr()), ctypes.c_void_p(self.out.data_ptr()),
            ctypes.c_void_p(lin_out) if lin_out else None,
            ctypes.c_void_p(stream) if stream else None))
        if stream:
            torch.cuda.ExternalStream(stream).synchronize()
        else:
            torch.cuda.synchronize()
        return self.out.cpu().numpy().reshape(self.h, self.w, 3)
