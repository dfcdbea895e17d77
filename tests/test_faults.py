"""Failure paths on the GPU, each forced without a device fault:

* allocation failure: a per-context device memory cap refuses an allocation
  (SOLAR_GPU_ERR_OOM) before cudaMalloc is called, and the context stays
  usable once the cap is raised;
* an expired device wait: a GEMM tile whose operand loads are withheld lets
  its bounded mbarrier wait run out (about a second); the kernel records the
  error and exits normally, the call returns SOLAR_GPU_ERR_DEVICE_CHECK, and
  the next GEMM on the same device is correct.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import device_arrays, load_scene

pytestmark = pytest.mark.gpu


def test_memory_limit_refuses_then_recovers(cuda_lib):
    import torch
    from solargpu_b200 import api
    s = load_scene("dsm64")
    dev = device_arrays(s)
    want = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
    with api.Context(0) as ref:
        ref.run_device(s, dev, want)
        held = ref.memory_held()
    assert held > 0
    out = torch.zeros_like(want)
    with api.Context(0) as c:
        c.set_memory_limit(1 << 20)
        with pytest.raises(api.SolarGPUError) as e:
            c.run_device(s, dev, out)
        assert e.value.code == -4
        assert "memory limit" in str(e.value)
        assert c.memory_held() <= 1 << 20
        c.set_memory_limit(2 * held)          # room for this scene
        c.run_device(s, dev, out)
        assert c.memory_held() <= 2 * held
        assert torch.equal(out, want)
        with pytest.raises(api.SolarGPUError) as e:
            c.set_memory_limit(-1)
        assert e.value.code == -1


def test_expired_device_wait_is_reported_and_device_stays_usable(cuda_lib):
    import torch
    from solargpu_b200 import api
    L = api.lib()
    L.solar_gpu_selftest_bounded_wait.argtypes = [C.c_void_p]
    rc = L.solar_gpu_selftest_bounded_wait(None)
    assert rc == -5
    assert "bounded wait expired" in L.solar_gpu_last_error().decode()
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(256, 128, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(128, 128, device="cuda", generator=g).to(torch.bfloat16)
    got = api.gemm_bf16(A, B)
    torch.testing.assert_close(got, A.float() @ B.float().T, rtol=1e-4, atol=1e-3)
    assert np.isfinite(got.cpu().numpy()).all()
