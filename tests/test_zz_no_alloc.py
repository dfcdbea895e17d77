"""solar_gpu_barle_encode_noalloc: ba-RLE encoding that allocates no device memory.

It exists for callers that may not allocate on the GPU themselves or through
us -- a host framework that owns the device memory through its own pool, or a
real-time loop that cannot take the device-wide stalls of cudaMalloc/cudaFree.
Its scratch is one static device array, so it is limited to 1024 lists of at
most 2592 ids per call.

The checks call it through the C ABI, twice in a row on different voxel
ranges (the second call reuses the scratch the first one left behind), and
compare its bytes with the ba-RLE lists the library's own trace entry point
builds for the same voxels.  Integer/byte work: the tolerance is bit-exact.
This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from conftest import device_arrays, load_scene

pytestmark = pytest.mark.gpu


def _encode(lib, off_d, ids_d, n, out_off_d, out_bytes_d, cap, stream):
    total = C.c_longlong(-1)
    rc = lib.solar_gpu_barle_encode_noalloc(C.c_void_p(off_d.data_ptr()), C.c_void_p(ids_d.data_ptr()), n,
                                            C.c_void_p(out_off_d.data_ptr()), C.c_void_p(out_bytes_d.data_ptr()),
                                            C.c_longlong(cap), C.byref(total), C.c_void_p(stream))
    return rc, total.value


@pytest.fixture(scope="module")
def traced():
    from solargpu_b200 import api
    s = load_scene("dsm64")
    with api.Context(0) as ctx:
        r = ctx.trace(s, device_arrays(s), neighbor_format=api.BOTH)
    return s, r


def test_no_alloc_encoder_matches_library_lists(cuda_lib, traced):
    import torch
    s, r = traced
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row: tops of the first rows, then the last 1024 voxels (walls)
    for a, b in ((0, 1024), (s.num_total - 1024, s.num_total)):
        off = r["csr_off"][a:b + 1] - r["csr_off"][a]
        ids = r["csr_ids"][r["csr_off"][a]:r["csr_off"][b]]
        want = r["barle"][r["barle_off"][a]:r["barle_off"][b]]
        want_off = r["barle_off"][a:b + 1] - r["barle_off"][a]
        off_d = torch.from_numpy(off.astype(np.int64)).cuda()
        ids_d = torch.from_numpy(ids.astype(np.int32)).cuda()
        out_off = torch.zeros(b - a + 1, dtype=torch.int64, device="cuda")
        cap = int(want.size) + 64
        out_b = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        rc, total = _encode(cuda_lib, off_d, ids_d, b - a, out_off, out_b, cap, stream)
        assert rc == 0, cuda_lib.solar_gpu_last_error()
        assert total == want.size
        np.testing.assert_array_equal(out_off.cpu().numpy(), want_off)
        np.testing.assert_array_equal(out_b.cpu().numpy()[:total], want)


def test_no_alloc_encoder_rejects_oversize(cuda_lib, traced):
    import torch
    s, r = traced
    stream = torch.cuda.current_stream().cuda_stream
    off_d = torch.zeros(1026, dtype=torch.int64, device="cuda")
    ids_d = torch.zeros(1, dtype=torch.int32, device="cuda")
    out_off = torch.zeros(1026, dtype=torch.int64, device="cuda")
    out_b = torch.zeros(16, dtype=torch.uint8, device="cuda")
    rc, _ = _encode(cuda_lib, off_d, ids_d, 1025, out_off, out_b, 16, stream)
    assert rc == -1
    assert b"1024" in cuda_lib.solar_gpu_last_error()
    # a capacity too small reports the needed size and writes nothing
    a, b = 0, 64
    off_d = torch.from_numpy((r["csr_off"][a:b + 1] - r["csr_off"][a]).astype(np.int64)).cuda()
    ids_d = torch.from_numpy(r["csr_ids"][r["csr_off"][a]:r["csr_off"][b]].astype(np.int32)).cuda()
    out_off = torch.zeros(b - a + 1, dtype=torch.int64, device="cuda")
    rc, total = _encode(cuda_lib, off_d, ids_d, b - a, out_off, out_b, 16, stream)
    assert rc == -1
    assert total == r["barle_off"][b] - r["barle_off"][a]
    assert int(out_b.sum().item()) == 0
