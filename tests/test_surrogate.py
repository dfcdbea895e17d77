"""The tensor-core (tcgen05) BF16 GEMM of the sky-bin visibility surrogate
against torch's FP32 product of the same bf16 inputs."""
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("bn", ["64", "128", "256"])
@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 320), (384, 256, 1024), (256, 512, 1600),
                                   (5120, 1024, 320)])
def test_gemm_bf16_matches_fp32_product(M, N, K, bn, monkeypatch):
    """Every tile width (SGB_GEMM_BN forces one where N allows it); the last
    shape has more tiles than SMs, so it runs the persistent kernel."""
    monkeypatch.setenv("SGB_GEMM_BN", bn)
    import torch
    from solargpu_b200 import api
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    want = A.float() @ B.float().T
    got = api.gemm_bf16(A, B)
    torch.cuda.synchronize()
    torch.testing.assert_close(got, want, rtol=1e-4, atol=1e-3)
    got2 = api.gemm_bf16(A, B, bias=bias, relu=True)
    torch.testing.assert_close(got2, torch.relu(want + bias), rtol=1e-4, atol=1e-3)
    hb = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    api.gemm_bf16(A, B, out_bf16=hb, bias=bias)
    torch.testing.assert_close(hb.float(), (want + bias).to(torch.bfloat16).float(), rtol=1e-2, atol=1e-2)


@pytest.mark.gpu
@pytest.mark.parametrize("bn", ["64", "256"])
def test_persistent_gemm_equals_one_tile_per_cta(bn, monkeypatch):
    """The persistent kernel (two TMEM accumulators, CTAs walking tiles)
    issues the same MMAs in the same order as one CTA per tile: equal bits."""
    import torch
    from solargpu_b200 import api
    monkeypatch.setenv("SGB_GEMM_BN", bn)
    g = torch.Generator(device="cuda").manual_seed(9)
    A = torch.randn(128 * 80, 448, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(512, 448, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(512, device="cuda", generator=g)
    got = api.gemm_bf16(A, B, bias=bias, relu=True)
    monkeypatch.setenv("SGB_GEMM_ONE_TILE_PER_CTA", "1")
    want = api.gemm_bf16(A, B, bias=bias, relu=True)
    assert torch.equal(got, want)


def test_gemm_rejects_bad_shapes():
    from solargpu_b200 import api
    import ctypes as C
    rc = api.lib().solar_gpu_gemm_bf16(C.c_void_p(16), C.c_void_p(32), C.c_void_p(64), None, None, 100, 128, 64, 0,
                                       None)
    assert rc in (-1, -2, -3)


def _bf16(x):
    """Round float values to bfloat16 (nearest even), returned as float64."""
    import numpy as np
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


@pytest.mark.gpu
def test_surrogate_gradients_match_fp64():
    """Backward pass (all products on the tensor cores) against an FP64 numpy
    restatement that rounds to bf16 where the GPU path stores bf16."""
    import numpy as np
    import torch
    from solargpu_b200 import surrogate as S
    M, active = 128, 100
    m = S.Surrogate(active=active, hidden=128, layers=1, feat=128, outw=128, seed=3, conv=None, share_units=0)
    g = torch.Generator(device="cpu").manual_seed(7)
    X = torch.randn(M, 128, generator=g).to(torch.bfloat16).cuda()
    Y = (torch.rand(M, 128, generator=g) > 0.5).float().cuda()
    m.b[0].copy_(torch.randn(128, generator=g) * 0.1)
    m.b[1].copy_(torch.randn(128, generator=g) * 0.1)
    loss, dW, db = m.gradients(X, Y)
    x = X.float().cpu().numpy().astype(np.float64)
    y = Y.cpu().numpy().astype(np.float64)
    w1, w2 = (w.float().cpu().numpy().astype(np.float64) for w in m.Wb)
    b1, b2 = (b.cpu().numpy().astype(np.float64) for b in m.b)
    h1 = _bf16(np.maximum(x @ w1.T + b1, 0.0))
    z = h1 @ w2.T + b2
    mask = np.arange(128) < active
    p = 1.0 / (1.0 + np.exp(-z))
    dz = _bf16(np.where(mask, (p - y) / (M * active), 0.0))
    ref_loss = np.sum(np.where(mask, np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))), 0.0)) / (M * active)
    g1 = _bf16(np.where(h1 > 0, dz @ w2, 0.0))
    refs = [(g1.T @ x, g1.sum(0)), (dz.T @ h1, dz.sum(0))]
    assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss)
    for l, (rw, rb) in enumerate(refs):
        gw = dW[l].cpu().numpy()
        gb = db[l].cpu().numpy()
        assert np.abs(gw - rw).max() <= 2e-2 * np.abs(rw).max(), l
        assert np.abs(gb - rb).max() <= 2e-2 * np.abs(rb).max(), l
        assert np.abs(gw - rw).mean() <= 2e-3 * np.abs(rw).mean(), l


def _im2col(x, kp):
    """NHWC x [B][H][W][C] -> [B (H/2) (W/2)][kp], 4 x 4 taps, stride 2, padding 1."""
    import numpy as np
    B, H, W, Cc = x.shape
    Ho, Wo = H // 2, W // 2
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    cols = np.zeros((B, Ho, Wo, kp))
    for ky in range(4):
        for kx in range(4):
            t = ky * 4 + kx
            cols[..., t * Cc:(t + 1) * Cc] = xp[:, ky:ky + 2 * Ho:2, kx:kx + 2 * Wo:2, :]
    return cols.reshape(B * Ho * Wo, kp)


def _col2im(d, B, H, W, Cc):
    """Adjoint of _im2col."""
    import numpy as np
    Ho, Wo = H // 2, W // 2
    d = d.reshape(B, Ho, Wo, -1)
    xp = np.zeros((B, H + 2, W + 2, Cc))
    for ky in range(4):
        for kx in range(4):
            t = ky * 4 + kx
            xp[:, ky:ky + 2 * Ho:2, kx:kx + 2 * Wo:2, :] += d[..., t * Cc:(t + 1) * Cc]
    return xp[:, 1:H + 1, 1:W + 1, :]


@pytest.mark.gpu
def test_conv_surrogate_gradients_match_fp64():
    """Two stride-2 convolutions (im2col + GEMM forward, GEMM + col2im
    backward) and a one-hidden-layer MLP against an FP64 numpy restatement
    that rounds to bf16 where the GPU path stores bf16."""
    import numpy as np
    import torch
    from solargpu_b200 import surrogate as S
    B, active = 128, 100
    m = S.Surrogate(active=active, hidden=128, layers=1, outw=128, seed=5, conv=(64, 64), share_units=0)
    assert m.feat == 16 * 16 * 64 + S.NRM and m.kp == [128, 1024]
    g = torch.Generator(device="cpu").manual_seed(11)
    img = torch.randn(B, 64, 64, 2, generator=g).to(torch.bfloat16).cuda()
    nrm = torch.zeros(B, S.NRM)
    nrm[:, :3] = torch.randn(B, 3, generator=g)
    nrm = nrm.to(torch.bfloat16).cuda()
    Y = (torch.rand(B, 128, generator=g) > 0.5).float().cuda()
    for b in m.b:
        b.copy_(torch.randn(b.numel(), generator=g) * 0.1)
    loss, dW, db = m.gradients(img, Y, nrm)
    w = [x.float().cpu().numpy().astype(np.float64) for x in m.Wb]
    bs = [x.cpu().numpy().astype(np.float64) for x in m.b]
    x0 = img.float().cpu().numpy().astype(np.float64)
    nr = nrm.float().cpu().numpy().astype(np.float64)
    y = Y.cpu().numpy().astype(np.float64)
    c1 = _im2col(x0, 128)
    y1 = _bf16(np.maximum(c1 @ w[0].T + bs[0], 0.0))                       # [B 1024][64]
    c2 = _im2col(y1.reshape(B, 32, 32, 64), 1024)
    y2 = _bf16(np.maximum(c2 @ w[1].T + bs[1], 0.0))                       # [B 256][64]
    flat = np.concatenate([y2.reshape(B, -1), nr], axis=1)
    h1 = _bf16(np.maximum(flat @ w[2].T + bs[2], 0.0))
    z = h1 @ w[3].T + bs[3]
    mask = np.arange(128) < active
    p = 1.0 / (1.0 + np.exp(-z))
    dz = _bf16(np.where(mask, (p - y) / (B * active), 0.0))
    ref_loss = np.sum(np.where(mask, np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))), 0.0)) / (B * active)
    g3 = _bf16(np.where(h1 > 0, dz @ w[3], 0.0))
    g2 = _bf16(np.where(y2.reshape(B, -1) > 0, (g3 @ w[2])[:, :16 * 16 * 64], 0.0)).reshape(B * 256, 64)
    g1 = _bf16(np.where(y1 > 0, _col2im(g2 @ w[1], B, 32, 32, 64).reshape(B * 1024, 64), 0.0))
    refs = [(g1.T @ c1, g1.sum(0)), (g2.T @ c2, g2.sum(0)), (g3.T @ flat, g3.sum(0)), (dz.T @ h1, dz.sum(0))]
    assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss)
    for l, (rw, rb) in enumerate(refs):
        gw = dW[l].cpu().numpy()
        gb = db[l].cpu().numpy()
        assert gw.shape == rw.shape, l
        assert np.abs(gw - rw).max() <= 2e-2 * np.abs(rw).max(), l
        assert np.abs(gb - rb).max() <= 2e-2 * np.abs(rb).max(), l
        assert np.abs(gw - rw).mean() <= 2e-3 * np.abs(rw).mean(), l
    assert np.all(dW[0].cpu().numpy()[:, 32:] == 0)        # the zero-padded columns of the first layer


@pytest.mark.gpu
def test_surrogate_image_matches_numpy():
    """The conv model's input image (1 m heights and 8 x 8 context maxima
    around the voxel) and normal, against numpy."""
    import numpy as np
    import torch
    from conftest import device_arrays, load_scene
    from solargpu_b200 import surrogate as S
    s = load_scene("dsm64")
    dev = device_arrays(s)
    m = S.Surrogate(active=8, hidden=128, layers=1, outw=128, conv=(64, 64))
    rng = np.random.default_rng(2)
    vox = rng.choice(s.num_total, 128, replace=False).astype(np.int32)
    img, nrm = m.inputs(s, dev, torch.from_numpy(vox).cuda())
    img = img.float().cpu().numpy()
    nrm = nrm.float().cpu().numpy()
    W, H = s.width, s.height
    grid = s.grid.reshape(H, W).astype(np.float64)
    hc, wc = (H + 7) // 8, (W + 7) // 8
    coarse = np.full((hc * 8, wc * 8), -np.inf)
    coarse[:H, :W] = grid
    coarse = coarse.reshape(hc, 8, wc, 8).max(axis=(1, 3))
    for i, v in enumerate(vox):
        top = int(s.pixel_parent[v])
        gx, gy = top % W, top // W
        z = float(s.grid[top]) if v < s.num_top else float(s.wall_z[v - s.num_top])
        d = np.arange(64) - 32
        ys, xs = gy + d[:, None], gx + d[None, :]
        inside = (ys >= 0) & (ys < H) & (xs >= 0) & (xs < W)
        h = np.where(inside, grid[np.clip(ys, 0, H - 1), np.clip(xs, 0, W - 1)], 0.0)
        cy, cx = gy // 8 + d[:, None], gx // 8 + d[None, :]
        cin = (cy >= 0) & (cy < hc) & (cx >= 0) & (cx < wc)
        hcv = np.where(cin, coarse[np.clip(cy, 0, hc - 1), np.clip(cx, 0, wc - 1)], 0.0)
        want0 = _bf16(np.clip((h - z) / 50.0, -2, 2))
        want1 = _bf16(np.clip((hcv - z) / 50.0, -2, 2))
        np.testing.assert_allclose(img[i, :, :, 0], want0, atol=1e-2, rtol=0)
        np.testing.assert_allclose(img[i, :, :, 1], want1, atol=1e-2, rtol=0)
        sl, asp = np.radians(s.slopes[v]), np.radians(s.aspects[v])
        np.testing.assert_allclose(nrm[i, :3], [np.sin(sl) * np.sin(asp), -np.sin(sl) * np.cos(asp), np.cos(sl)],
                                   atol=1e-2)
        assert np.all(nrm[i, 3:] == 0)


@pytest.mark.gpu
def test_surrogate_learns_and_fallback_is_exact():
    """A short training run lowers the loss; with a zero error threshold the
    guarded prediction falls back everywhere and equals the exact DDA bits."""
    import numpy as np
    import torch
    from conftest import device_arrays, load_scene
    from solargpu_b200 import api
    from solargpu_b200 import surrogate as S
    s = load_scene("dsm64")
    dev = device_arrays(s)
    with api.Context(0) as ctx:
        r = ctx.trace(s, dev, neighbor_format=0)
        sh = torch.from_numpy(r["shadow"].view(np.int32)).cuda()
        m = S.Surrogate(active=r["active_bins"], seed=1)
        losses = m.train([(s, dev, sh, r["shadow_words"])], steps=60, batch=256, lr=1e-3)
        assert np.mean(losses[-10:]) < np.mean(losses[:10])
        res = S.predict_with_fallback(m, ctx, s, dev, tile=32, spot=16, max_err=0.0)
        allv = torch.arange(s.num_total, dtype=torch.int32, device="cuda")
        exact, w = S.exact_bits(ctx, s, dev, allv)
        assert w == r["shadow_words"]
        assert torch.equal(exact.cpu(), sh.cpu())
        # every tile whose sample showed any error was replaced by exact bits
        for t in res["tiles"]:
            if t["sampled_error"] > 0:
                assert t["fallback"]


@pytest.mark.gpu
def test_surrogate_learns_the_reflected_share():
    """The share units: targets 1 - own / total from the pipeline's runs with
    and without reflection, soft cross-entropy; a short training run brings
    the predicted share of the scene's voxels closer to the exact one."""
    import numpy as np
    import torch
    from conftest import device_arrays, load_scene
    from solargpu_b200 import api
    from solargpu_b200 import surrogate as S
    s = load_scene("dsm64")
    dev = device_arrays(s)
    with api.Context(0) as ctx:
        tot = torch.zeros(s.num_total, dtype=torch.float32, device="cuda")
        own = torch.zeros_like(tot)
        ctx.run_device(s, dev, tot, neighbor_format=0)
        ctx.run_device(s, dev, own, neighbor_format=0, reflection=api.REFL_NONE)
        share = (1.0 - own / tot).clamp_min(0.0)
        assert float(share.max()) > 0.0 and float(share.min()) >= 0.0
        r = ctx.trace(s, dev, neighbor_format=0)
        sh = torch.from_numpy(r["shadow"].view(np.int32)).cuda()
        m = S.Surrogate(active=r["active_bins"], seed=2, conv=None)
        allv = torch.arange(s.num_total, dtype=torch.int32, device="cuda")
        before = float((m.predict_share(s, dev, allv) - share).abs().mean())
        m.train([(s, dev, sh, r["shadow_words"], share)], steps=150, batch=256, lr=1e-3)
        p = m.predict_share(s, dev, allv)
        after = float((p - share).abs().mean())
        assert p.shape == (s.num_total,) and float(p.min()) >= 0.0 and float(p.max()) <= 1.0
        assert after < 0.5 * before, (before, after)
