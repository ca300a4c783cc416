"""tcgen05 implicit-GEMM convolutions against a plain PyTorch FP32 reference
(torch.nn.functional.conv3d on the same BF16-rounded inputs).  Input
channel counts that are multiples of 16 take the TMA-staged kernel, 2 -> 16
and 16 -> 1 the direct CUDA-core kernel, the others the gathering one; all
are covered.  Products of
BF16 values are exact in FP32, so the only differences are FP32 summation
order: 1e-3 relative of each output's magnitude."""
import numpy as np
import pytest
import torch
import torch.nn.functional as Fn

from gpu_util import ptr, require_cuda

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    return require_cuda()


def _close(got, exp, tol=1e-3):
    got = got.double()
    exp = exp.double()
    scale = exp.abs().max().item() + 1e-30
    err = (got - exp).abs().max().item() / scale
    assert err <= tol, err


def _tensors(nb, C, nz, ny, nx, Cout, seed):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn(nb, C, nz, ny, nx, generator=g).bfloat16().float()
    w = (torch.randn(Cout, C, 3, 3, 3, generator=g) / np.sqrt(27 * C)).bfloat16().float()
    b = torch.randn(Cout, generator=g) * 0.1
    return x.cuda(), w.cuda(), b.cuda()


def _cl(x):
    """(nb, C, z, y, x) -> the library's BF16 activation layout: C / 8 planes
    of [voxel][8 channels] when C is a multiple of 8, else [voxel][C]."""
    nb, C = x.shape[:2]
    if C % 8:
        return x.permute(0, 2, 3, 4, 1).contiguous().bfloat16()
    return x.reshape(nb, C // 8, 8, *x.shape[2:]).permute(1, 0, 3, 4, 5, 2).contiguous().bfloat16()


def _wk(w):   # (Cout, C, 3, 3, 3) -> [Cout][27][C] bf16
    return w.permute(0, 2, 3, 4, 1).reshape(w.shape[0], 27, w.shape[1]).contiguous().bfloat16()


@pytest.mark.parametrize("C,Cout,dims,nb", [(16, 32, (8, 10, 12), 2), (2, 16, (9, 7, 11), 1),
                                            (96, 32, (6, 8, 8), 1), (16, 1, (8, 8, 8), 2),
                                            (32, 64, (8, 16, 8), 1), (48, 16, (4, 8, 8), 1),
                                            (32, 16, (5, 9, 13), 2), (16, 96, (6, 6, 40), 1),
                                            (64, 128, (4, 8, 8), 1),
                                            # many tiles per CTA: every stage and both
                                            # accumulators of the persistent kernel cycle
                                            (48, 16, (40, 64, 64), 1), (16, 16, (24, 40, 48), 2),
                                            (32, 64, (16, 32, 32), 1), (2, 16, (33, 35, 37), 1),
                                            (16, 1, (33, 35, 37), 1)])
def test_forward(lib, C, Cout, dims, nb):
    nz, ny, nx = dims
    x, w, b = _tensors(nb, C, nz, ny, nx, Cout, 1)
    ref = torch.relu(Fn.conv3d(x, w, b, padding=1))
    y = torch.empty(nb, nz, ny, nx, Cout, dtype=torch.float32, device="cuda")
    xc, wk = _cl(x), _wk(w)      # held until the call returns
    rc = lib.pyro_conv3_forward(ptr(xc), C, nx, ny, nz, nb, ptr(wk), Cout, ptr(b), 1,
                                ptr(y), 1, None)
    assert rc == 0, lib.pyro_last_error()
    _close(y.permute(0, 4, 1, 2, 3), ref)


@pytest.mark.parametrize("Cin,Cout,dims", [(16, 32, (8, 10, 12)), (48, 16, (6, 8, 8)),
                                           (96, 32, (4, 8, 8)), (32, 64, (8, 8, 8)),
                                           (16, 8, (5, 7, 9)), (64, 16, (3, 17, 20)),
                                           (48, 16, (20, 32, 32))])
def test_backward_data_and_weight(lib, Cin, Cout, dims):
    nz, ny, nx = dims
    nb = 1
    x, w, _ = _tensors(nb, Cin, nz, ny, nx, Cout, 2)
    g = torch.Generator().manual_seed(3)
    dy = torch.randn(nb, Cout, nz, ny, nx, generator=g).bfloat16().float().cuda()
    xr = x.clone().requires_grad_(True)
    wr = w.clone().requires_grad_(True)
    out = Fn.conv3d(xr, wr, None, padding=1)
    out.backward(dy)
    dx = torch.empty(nb, nz, ny, nx, Cin, dtype=torch.float32, device="cuda")
    dyc, wk, xc = _cl(dy), _wk(w), _cl(x)
    rc = lib.pyro_conv3_backward_data(ptr(dyc), Cout, nx, ny, nz, nb, ptr(wk), Cin, None,
                                      ptr(dx), 1, None)
    assert rc == 0, lib.pyro_last_error()
    _close(dx.permute(0, 4, 1, 2, 3), xr.grad)
    # masked by the input activation (ReLU derivative)
    rc = lib.pyro_conv3_backward_data(ptr(dyc), Cout, nx, ny, nz, nb, ptr(wk), Cin,
                                      ptr(xc), ptr(dx), 1, None)
    assert rc == 0
    _close(dx.permute(0, 4, 1, 2, 3), xr.grad * (x > 0))
    dw = torch.zeros(Cout, 27, Cin, dtype=torch.float32, device="cuda")
    rc = lib.pyro_conv3_backward_weight(ptr(xc), Cin, ptr(dyc), Cout, nx, ny, nz, nb,
                                        ptr(dw), None)
    assert rc == 0, lib.pyro_last_error()
    _close(dw, wr.grad.permute(0, 2, 3, 4, 1).reshape(Cout, 27, Cin))
