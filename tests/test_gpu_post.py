"""Frame development on the GPU (pyro_post_select / pyro_post_develop)
against the CPU restatement of src/post.rs (pyro_b200.post): the mean
radiance and the 99.5th luminance percentile exactly, the linear image after
exposure and glare bit for bit (the box filters' running sums in the
reference's order), and the 8-bit sRGB image within one level (powf of the
sRGB curve may round differently on the device), over a sequence of frames
so the exposure state's smoothing is exercised."""
import ctypes

import numpy as np
import pytest
import torch

from gpu_util import require_cuda
from pyro_b200 import _abi
from pyro_b200.develop import Developer
from pyro_b200.post import Camera, glare, percentile_rank

pytestmark = pytest.mark.gpu
F32 = np.float32


def _accum(h, w, seed):
    rng = np.random.default_rng(seed)
    acc = np.zeros((h * w, 4), F32)
    n = rng.integers(0, 9, size=h * w).astype(F32)          # some pixels with no sample
    rad = rng.gamma(0.6, 0.4, size=(h * w, 3)).astype(F32)
    hot = rng.random(h * w) < 0.01                          # a few bright sources
    rad[hot] *= F32(40.0)
    acc[:, :3] = rad * n[:, None]
    acc[:, 3] = n
    return acc


@pytest.mark.parametrize("auto,glare_w", [(True, 0.04), (True, 0.0), (False, 0.04)])
def test_device_development_matches_the_cpu_restatement(auto, glare_w):
    require_cuda()
    h, w = 90, 160
    dev = Developer(w, h)
    cam_d, cam_h = Camera(auto, 0.5, glare_w), Camera(auto, 0.5, glare_w)
    lin_d = torch.empty(h * w * 3, dtype=torch.float32, device="cuda")
    for frame in range(3):
        acc = _accum(h, w, 10 + frame)
        acc_d = torch.from_numpy(acc).cuda()
        rgb8 = dev.develop(cam_d, acc_d.data_ptr(), 1.0 / 30.0, lin_out=lin_d.data_ptr())
        # the CPU restatement from the same accumulation image
        img = (acc[:, :3] / np.maximum(acc[:, 3:4], F32(1.0))).reshape(h, w, 3)
        assert np.array_equal(dev.img.cpu().numpy().reshape(h, w, 3), img)
        if auto:
            p = img.reshape(-1, 3)
            l = F32(0.2126) * p[:, 0] + F32(0.7152) * p[:, 1] + F32(0.0722) * p[:, 2]
            k = percentile_rank(l.size)
            assert dev.select(acc_d.data_ptr()) == np.partition(l, k)[k]
        want = cam_h.develop(img, 1.0 / 30.0)
        assert cam_d.ev == cam_h.ev
        k_gain = np.power(F32(2.0), F32(cam_h.ev + cam_h.ev_offset) if auto else cam_h.ev_offset)
        lin = img * k_gain
        if glare_w > 0.0:
            lin = lin * (F32(1.0) - F32(glare_w)) + glare(lin) * F32(glare_w)
        assert np.array_equal(lin_d.cpu().numpy().reshape(h, w, 3), lin)
        diff = np.abs(rgb8.astype(np.int16) - want.astype(np.int16))
        assert diff.max() <= 1 and (diff > 0).mean() < 0.01, (diff.max(), (diff > 0).mean())


def test_select_rejects_bad_arguments():
    lib = require_cuda()
    v = ctypes.c_float()
    buf = torch.zeros(64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    assert lib.pyro_post_select(p, 4, 4, 16, p, p, p, ctypes.byref(v), None) == \
        _abi.PYRO_E_INVALID
    assert lib.pyro_post_develop(p, 4, 4, 1.0, 2.0, p, p, None, None) == _abi.PYRO_E_INVALID
