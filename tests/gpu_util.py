"""Device helpers for the GPU tests: torch tensors are only device memory;
every computation goes through the C ABI of libpyro_b200.so."""
import ctypes

import numpy as np
import torch

from pyro_b200 import _abi


def require_cuda():
    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    lib = _abi.load()
    return lib


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def zeros_like_dev(a):
    return torch.zeros(a.shape, dtype=torch.from_numpy(a[:0] if a.ndim else a).dtype, device="cuda")


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def params_dev(P):
    return torch.frombuffer(bytearray(P.to_bytes()), dtype=torch.uint8).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def stats_dev():
    return torch.zeros(_abi.STATS_N, dtype=torch.float32, device="cuda")
