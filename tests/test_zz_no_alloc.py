"""solar_gpu_barle_encode_noalloc: ba-RLE encoding that allocates no device memory.

It exists for callers that may not allocate on the GPU themselves or through
us -- a host framework that owns the device memory through its own pool, or a
real-time loop that cannot take the device-wide stalls of cudaMalloc/cudaFree.
Its scratch is one static device array, so it is limited to 1024 lists of at
most 2592 ids per call.

The checks call it through the C ABI, twice in a row on different voxel
ranges (the second call reuses the scratch the first one left behind), and
compare its bytes with the ba-RLE lists the library's own trace entry point
builds for the same voxels, and with the reference encoder's own bytes
(tests/golden/barle_golden.npz: every width class, 2592-id lists, ids near
2^31).  Integer/byte work: the tolerance is bit-exact.  Rejected calls
(too many lists, a list over 2592 ids, repeated or zero ids, a capacity too
small) are each followed by a valid call on the same scratch.
This file is collected last on purpose."""
import os
import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN, device_arrays, load_scene

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


def _encode_host(lib, off, ids, cap, stream):
    """Encodes host CSR lists through device copies; returns (rc, total, offsets, bytes)."""
    import torch
    n = off.size - 1
    off_d = torch.from_numpy(off.astype(np.int64)).cuda()
    ids_d = torch.from_numpy(ids.astype(np.int32) if ids.size else np.zeros(1, np.int32)).cuda()
    out_off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    out_b = torch.zeros(max(1, cap), dtype=torch.uint8, device="cuda")
    rc, total = _encode(lib, off_d, ids_d, n, out_off, out_b, cap, stream)
    return rc, total, out_off.cpu().numpy(), out_b.cpu().numpy()


def test_no_alloc_encoder_matches_reference_encoder_bytes(cuda_lib):
    import torch
    g = np.load(os.path.join(GOLDEN, "barle_golden.npz"))
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):   # two calls in a row on the same scratch
        rc, total, boff, b = _encode_host(cuda_lib, g["off"], g["ids"], int(g["bytes"].size) + 64, stream)
        assert rc == 0, cuda_lib.solar_gpu_last_error()
        assert total == g["bytes"].size
        np.testing.assert_array_equal(boff, g["boff"])
        np.testing.assert_array_equal(b[:total], g["bytes"])


def test_no_alloc_encoder_rejects_bad_lists_and_recovers(cuda_lib):
    import torch
    g = np.load(os.path.join(GOLDEN, "barle_golden.npz"))
    stream = torch.cuda.current_stream().cuda_stream
    cap = int(g["bytes"].size) + 64

    def valid_again():
        rc, total, boff, b = _encode_host(cuda_lib, g["off"], g["ids"], cap, stream)
        assert rc == 0 and total == g["bytes"].size
        np.testing.assert_array_equal(b[:total], g["bytes"])

    # a list of 2593 ids (one more than there are traced directions)
    long_ids = np.arange(2593, 0, -1, dtype=np.int32)
    rc, _, _, _ = _encode_host(cuda_lib, np.array([0, 2593], np.int64), long_ids, 1 << 16, stream)
    assert rc == -1
    assert b"2592" in cuda_lib.solar_gpu_last_error()
    valid_again()
    # a repeated id, and a zero id
    for bad in (np.array([9, 5, 9], np.int32), np.array([3, 0, 7], np.int32)):
        rc, _, _, _ = _encode_host(cuda_lib, np.array([0, 1, 1 + bad.size], np.int64),
                                   np.concatenate([[4], bad]).astype(np.int32), 256, stream)
        assert rc == -1
        assert b"id" in cuda_lib.solar_gpu_last_error()
        valid_again()
    # no lists at all: nothing to encode
    rc, total, boff, _ = _encode_host(cuda_lib, np.zeros(1, np.int64), np.zeros(0, np.int32), 16, stream)
    assert rc == 0 and total == 0 and boff[0] == 0
    valid_again()
