"""The tensor-core GEMM tile of the learned correction (tcgen05, BF16 inputs,
FP32 accumulation in tensor memory) against a float64 product of the same
BF16-rounded inputs: the only difference is FP32 accumulation order."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k", [(128, 16, 16), (256, 32, 112), (128, 112, 128), (384, 32, 32),
                                   (128, 256, 256), (256, 16, 32)])
def test_tensor_core_gemm_matches_float64(m, n, k):
    from dev_field_efvm_b200 import abi
    from dev_field_efvm_b200.device import load

    L = load()
    g = torch.Generator().manual_seed(m * 1000 + n * 10 + k)
    a = torch.randn(m, k, generator=g).to(torch.bfloat16).cuda()
    b = torch.randn(n, k, generator=g).to(torch.bfloat16).cuda()
    d = torch.full((m, n), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = L.efvm_nn_gemm_bf16(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), C.c_void_p(d.data_ptr()), m, n, k,
                             None)
    assert rc == abi.OK, L.efvm_last_error(None).decode()
    ref = a.double().cpu().numpy() @ b.double().cpu().numpy().T
    got = d.cpu().numpy().astype(np.float64)
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < 1e-5, err
