"""Sky-bin visibility surrogate: a BF16 conv net on the tcgen05 GEMM.

For a voxel, the model predicts its 265 sun-bin shadow bits (the DDA's
shadow words: 1 = a ray toward that bin hits terrain) and its reflected
irradiance share (the part of its annual irradiance that inter-reflection
adds: 1 - own / total, own = the run with reflection=none).  Two inputs:

* conv model (the default): a 64 x 64 x 2 image around the voxel, channel 0
  the 1 m cell heights, channel 1 the maxima of 8 x 8-cell context cells
  (a 512 m window, so that long low-sun shadows are in view), both relative
  to the voxel's base height / 50 m; and its normal.  Four 4 x 4, stride-2
  convolutions (64, 64, 128, 128 channels, ReLU; 64 -> 32 -> 16 -> 8 -> 4
  pixels), the 4 x 4 x 128 map and the normal (2048 + 64 columns) into
  512 -> 512 -> 512 -> 384 logits;
* MLP model (`conv=None`): the 64 x 64 heights and the normal, zero-padded
  to 4224 columns, into the same MLP.

The first `active` logits are the sun bins, the next `share_units` (16) all
learn the reflected share (soft binary cross-entropy targets; the prediction
is the mean of their sigmoids, which gives the one scalar the weight of 16
bins in the loss); ReLU between layers.  Every
product, forward and backward, runs on the tensor cores through
`solar_gpu_gemm_bf16` (bf16 operands, f32 accumulation in TMEM); a
convolution is im2col + GEMM, its input gradient GEMM + col2im (fused with
the ReLU mask below it).  Images, labels, the loss, transposes, bias sums
and Adam are small CUDA kernels of the library.  Master weights and Adam
moments are FP32, the GEMMs read bf16 copies.

`predict_with_fallback` is the guarded use: bits for every voxel from the
model, then per 256 x 256-cell tile a random sample of voxels traced exactly
(`solar_gpu_trace_shadow_subset`); a tile whose sampled bit error exceeds the
threshold (2%) is traced exactly in full.  The result is exact on fallback
tiles and within the sampled error elsewhere.  The share is a preview only:
the exact irradiance needs the exact neighbor lists.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import api

FEAT = 4224      # 64 * 64 + 3, padded to a multiple of 128 (MLP model)
OUTW = 384       # >= 265 active sun bins, a multiple of 128
CONV = (64, 64, 128, 128)   # channels of the four stride-2 convolutions
IMG = 64         # image side (pixels); 2 channels
NRM = 64         # normal columns (3 used)


def _lib():
    L = api.lib()
    if not getattr(L, "_sg_bound", False):
        vp, i, f, ll = C.c_void_p, C.c_int, C.c_float, C.c_longlong
        L.solar_gpu_sg_features.argtypes = [vp, i, i, i, vp, vp, vp, vp, vp, i, i, vp, vp]
        L.solar_gpu_sg_labels.argtypes = [vp, i, vp, i, i, i, vp, vp]
        L.solar_gpu_sg_bce.argtypes = [vp, vp, i, i, i, vp, vp, vp]
        L.solar_gpu_sg_relu_grad.argtypes = [vp, vp, ll, vp, vp]
        L.solar_gpu_sg_transpose.argtypes = [vp, i, i, vp, vp]
        L.solar_gpu_sg_colsum.argtypes = [vp, i, i, vp, vp]
        L.solar_gpu_sg_adam.argtypes = [vp, vp, vp, vp, ll, f, f, f, f, i, vp, vp]
        L.solar_gpu_sg_coarse.argtypes = [vp, i, i, vp, vp]
        L.solar_gpu_sg_image.argtypes = [vp, vp, i, i, i, vp, vp, vp, vp, vp, i, vp, vp, vp]
        L.solar_gpu_sg_im2col.argtypes = [vp, i, i, i, i, i, vp, vp]
        L.solar_gpu_sg_col2im_relu.argtypes = [vp, vp, i, i, i, i, i, vp, vp]
        L.solar_gpu_sg_hcat.argtypes = [vp, i, vp, i, i, vp, vp]
        L.solar_gpu_sg_relu_grad_cols.argtypes = [vp, i, vp, i, i, i, vp, vp]
        L.solar_gpu_sg_transpose_f32.argtypes = [vp, i, i, vp, vp]
        L.solar_gpu_trace_shadow_subset.argtypes = [vp, C.POINTER(api.SceneDesc), vp, i, vp, C.POINTER(i), vp]
        L._sg_bound = True
    return L


def _p(t):
    return None if t is None else C.c_void_p(int(t.data_ptr()))


def _t(torch, x):
    """Transpose of a 2-D bf16 CUDA tensor through the library kernel."""
    R, Cc = x.shape
    out = torch.empty(Cc, R, dtype=torch.bfloat16, device=x.device)
    api._check(_lib().solar_gpu_sg_transpose(_p(x), R, Cc, _p(out), None))
    return out


def _t32(torch, x):
    """Transpose of a 2-D f32 CUDA tensor through the library kernel."""
    R, Cc = x.shape
    out = torch.empty(Cc, R, dtype=torch.float32, device=x.device)
    api._check(_lib().solar_gpu_sg_transpose_f32(_p(x), R, Cc, _p(out), None))
    return out


def _round_up(x: int, m: int) -> int:
    return (x + m - 1) // m * m


class Surrogate:
    """conv: channels of the stride-2 convolutions (None: MLP on `feat`
    flat features).  Parameters W[l] / b[l] run over the convolutions
    (W [Cout][Kp], Kp = 16 Cin rounded up to 128) then the MLP layers."""

    def __init__(self, active: int, hidden: int = 512, layers: int = 3, feat: int = FEAT, outw: int = OUTW,
                 seed: int = 0, device: int = 0, conv: tuple | None = CONV, share_units: int = 16):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.active, self.outw = active, outw
        if active + share_units > outw:
            raise ValueError(f"{active} sun bins + {share_units} share units exceed {outw} outputs")
        self.share_units = share_units
        self.loss_cols = active + share_units
        self.conv = tuple(conv) if conv else ()
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.W, self.b = [], []
        self.kp, self.sides, self.cins = [], [], []
        side, cin = IMG, 2
        for cout in self.conv:
            if side % 2 or cout % 64:
                raise ValueError("conv: even image sides and channels multiple of 64")
            kp = _round_up(16 * cin, 128)
            w = torch.zeros(cout, kp)
            w[:, :16 * cin] = torch.randn(cout, 16 * cin, generator=g) * math.sqrt(2.0 / (16 * cin))
            self.W.append(w.to(self.dev))
            self.b.append(torch.zeros(cout, device=self.dev))
            self.kp.append(kp)
            self.sides.append(side)
            self.cins.append(cin)
            side, cin = side // 2, cout
        self.feat = side * side * cin + NRM if self.conv else feat
        self.flat = side * side * cin
        self.dims = [self.feat] + [hidden] * layers + [outw]
        for a, o in zip(self.dims[:-1], self.dims[1:]):
            self.W.append((torch.randn(o, a, generator=g) * math.sqrt(2.0 / a)).to(self.dev))
            self.b.append(torch.zeros(o, device=self.dev))
        self.Wb = [w.to(torch.bfloat16) for w in self.W]
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.step_count = 0

    # -- data -----------------------------------------------------------------

    def inputs(self, scene, dev: dict, voxels) -> tuple:
        """Model inputs of the listed voxels (device int32 ids): (image,
        normal) for the conv model, (features,) for the MLP model."""
        torch = self.torch
        M = voxels.numel()
        if not self.conv:
            out = torch.empty(M, self.feat, dtype=torch.bfloat16, device=self.dev)
            api._check(_lib().solar_gpu_sg_features(_p(dev["grid"]), scene.width, scene.height, scene.num_top,
                                                    _p(dev["pixel_parent"]), _p(dev["wall_z"]), _p(dev["slopes"]),
                                                    _p(dev["aspects"]), _p(voxels), M, self.feat, _p(out), None))
            return (out,)
        if "coarse" not in dev:
            wc, hc = (scene.width + 7) // 8, (scene.height + 7) // 8
            dev["coarse"] = torch.empty(hc * wc, dtype=torch.float32, device=self.dev)
            api._check(_lib().solar_gpu_sg_coarse(_p(dev["grid"]), scene.width, scene.height, _p(dev["coarse"]), None))
        img = torch.empty(M, IMG, IMG, 2, dtype=torch.bfloat16, device=self.dev)
        nrm = torch.empty(M, NRM, dtype=torch.bfloat16, device=self.dev)
        api._check(_lib().solar_gpu_sg_image(_p(dev["grid"]), _p(dev["coarse"]), scene.width, scene.height,
                                             scene.num_top, _p(dev["pixel_parent"]), _p(dev["wall_z"]),
                                             _p(dev["slopes"]), _p(dev["aspects"]), _p(voxels), M, _p(img), _p(nrm),
                                             None))
        return img, nrm

    def features(self, scene, dev: dict, voxels):
        """Flat features of the MLP model."""
        return self.inputs(scene, dev, voxels)[0]

    def labels(self, shadow_dev, words32: int, voxels, share=None):
        """Bit targets of the sun bins and, when `share` (per voxel, on the
        device) is given, the reflected share in the share units."""
        torch = self.torch
        M = voxels.numel()
        y = torch.empty(M, self.outw, dtype=torch.float32, device=self.dev)
        api._check(_lib().solar_gpu_sg_labels(_p(shadow_dev), words32, _p(voxels), M, self.active, self.outw,
                                              _p(y), None))
        if share is not None and self.share_units:
            y[:, self.active:self.loss_cols] = share[voxels.long()].unsqueeze(1)
        return y

    # -- model ----------------------------------------------------------------

    def forward(self, X, nrm=None):
        """GEMM inputs of every layer (im2col columns for the convolutions,
        activations for the MLP), the bf16 post-ReLU outputs of every hidden
        layer, and the f32 logits."""
        torch = self.torch
        L = _lib()
        ins, outs = [], []
        h = X
        B = X.shape[0]
        for l, cout in enumerate(self.conv):
            side, cin, kp = self.sides[l], self.cins[l], self.kp[l]
            rows = B * (side // 2) ** 2
            cols = torch.empty(rows, kp, dtype=torch.bfloat16, device=self.dev)
            api._check(L.solar_gpu_sg_im2col(_p(h), B, side, side, cin, kp, _p(cols), None))
            y = torch.empty(rows, cout, dtype=torch.bfloat16, device=self.dev)
            api.gemm_bf16(cols, self.Wb[l], out_bf16=y, bias=self.b[l], relu=True)
            ins.append(cols)
            outs.append(y)
            h = y
        if self.conv:
            flat = torch.empty(B, self.feat, dtype=torch.bfloat16, device=self.dev)
            api._check(L.solar_gpu_sg_hcat(_p(h), self.flat, _p(nrm), NRM, B, _p(flat), None))
            h = flat
        nc = len(self.conv)
        for l in range(nc, len(self.Wb) - 1):
            hn = torch.empty(B, self.dims[l - nc + 1], dtype=torch.bfloat16, device=self.dev)
            api.gemm_bf16(h, self.Wb[l], out_bf16=hn, bias=self.b[l], relu=True)
            ins.append(h)
            outs.append(hn)
            h = hn
        ins.append(h)
        Z = api.gemm_bf16(h, self.Wb[-1], bias=self.b[-1])
        return ins, outs, Z

    def gradients(self, X, Y, nrm=None):
        """Loss and the gradients of every weight and bias (f32)."""
        torch = self.torch
        L = _lib()
        B = X.shape[0]
        ins, outs, Z = self.forward(X, nrm)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        g = torch.empty(B, self.outw, dtype=torch.bfloat16, device=self.dev)
        api._check(L.solar_gpu_sg_bce(_p(Z), _p(Y), B, self.outw, self.loss_cols, _p(g), _p(loss), None))
        nc = len(self.conv)
        dW = [None] * len(self.W)
        db = [None] * len(self.W)
        for l in range(len(self.W) - 1, -1, -1):
            a = ins[l]
            rows, n_out = g.shape
            if l < nc:
                dW[l] = _t32(torch, api.gemm_bf16(_t(torch, a), _t(torch, g)))   # ([K, rows] [rows, N])^T
            else:
                dW[l] = api.gemm_bf16(_t(torch, g), _t(torch, a))                # [N, K] = g^T a
            db[l] = torch.empty(n_out, dtype=torch.float32, device=self.dev)
            api._check(L.solar_gpu_sg_colsum(_p(g), rows, n_out, _p(db[l]), None))
            if l == 0:
                break
            dA = api.gemm_bf16(g, _t(torch, self.Wb[l]))                         # [rows, K] = g W
            below = outs[l - 1]
            if l > nc:                  # MLP layer over an MLP layer
                gn = torch.empty(rows, dA.shape[1], dtype=torch.bfloat16, device=self.dev)
                api._check(L.solar_gpu_sg_relu_grad(_p(dA), _p(below), dA.numel(), _p(gn), None))
            elif l == nc:               # first MLP layer over the last convolution
                gn = torch.empty_like(below)    # [B * 16][128] = [B][flat]
                api._check(L.solar_gpu_sg_relu_grad_cols(_p(dA), self.feat, _p(below), self.flat, B, self.flat,
                                                         _p(gn), None))
            else:                       # convolution over a convolution
                side, cin, kp = self.sides[l], self.cins[l], self.kp[l]
                gn = torch.empty(B * side * side, cin, dtype=torch.bfloat16, device=self.dev)
                api._check(L.solar_gpu_sg_col2im_relu(_p(dA), _p(below), B, side, side, cin, kp, _p(gn), None))
            g = gn
        return float(loss.item()), dW, db

    def apply(self, dW, db, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        self.step_count += 1
        L = _lib()
        for l in range(len(self.W)):
            api._check(L.solar_gpu_sg_adam(_p(self.W[l]), _p(dW[l]), _p(self.mW[l]), _p(self.vW[l]),
                                           self.W[l].numel(), lr, b1, b2, eps, self.step_count, _p(self.Wb[l]),
                                           None))
            api._check(L.solar_gpu_sg_adam(_p(self.b[l]), _p(db[l]), _p(self.mb[l]), _p(self.vb[l]),
                                           self.b[l].numel(), lr, b1, b2, eps, self.step_count, None, None))

    def train(self, data: list, steps: int, batch: int = 1024, lr: float = 1e-3, seed: int = 0, log_every: int = 0):
        """data: (scene, dev arrays, shadow words on the device, words32[,
        reflected share per voxel on the device]) per training scene; batches
        of `batch` voxels (a multiple of 128) drawn uniformly."""
        torch = self.torch
        rng = np.random.default_rng(seed)
        losses = []
        for it in range(steps):
            scene, dev, shadow, words32, *rest = data[it % len(data)]
            vox = torch.from_numpy(rng.integers(0, scene.num_total, batch, dtype=np.int32)).to(self.dev)
            Y = self.labels(shadow, words32, vox, rest[0] if rest else None)
            inp = self.inputs(scene, dev, vox)
            loss, dW, db = self.gradients(inp[0], Y, *inp[1:])
            self.apply(dW, db, lr)
            losses.append(loss)
            if log_every and (it + 1) % log_every == 0:
                print(f"step {it + 1}: loss {np.mean(losses[-log_every:]):.4f}", flush=True)
        return losses

    def predict_share(self, scene, dev: dict, voxels, batch: int | None = None):
        """Predicted reflected share per voxel (float32, on the device)."""
        torch = self.torch
        batch = batch or (4096 if self.conv else 16384)
        n = voxels.numel()
        out = torch.zeros(n, dtype=torch.float32, device=self.dev)
        for i0 in range(0, n, batch):
            v = voxels[i0:i0 + batch]
            m = v.numel()
            pad = (-m) % 128
            if pad:
                v = torch.cat([v, v[:1].expand(pad)])
            _, _, Z = self.forward(*self.inputs(scene, dev, v))
            out[i0:i0 + m] = torch.sigmoid(Z[:m, self.active:self.loss_cols]).mean(1)
        return out

    def predict_bits(self, scene, dev: dict, voxels, batch: int | None = None):
        """Predicted shadow words [n][ceil(active/32)] (uint32, on the device)."""
        torch = self.torch
        batch = batch or (4096 if self.conv else 16384)
        n = voxels.numel()
        words = (self.active + 31) // 32
        out = torch.zeros(n, words, dtype=torch.int64, device=self.dev)
        shifts = (torch.arange(32, device=self.dev, dtype=torch.int64))
        for i0 in range(0, n, batch):
            v = voxels[i0:i0 + batch]
            m = v.numel()
            pad = (-m) % 128
            if pad:
                v = torch.cat([v, v[:1].expand(pad)])
            _, _, Z = self.forward(*self.inputs(scene, dev, v))
            bits = (Z[:m, :self.active] > 0).to(torch.int64)
            bits = torch.nn.functional.pad(bits, (0, 32 * words - self.active))
            out[i0:i0 + m] = (bits.view(m, words, 32) << shifts).sum(-1)
        return out.to(torch.int32)   # low 32 bits carry the word


def exact_bits(ctx, scene, dev: dict, voxels) -> tuple:
    """Exact DDA shadow words of the listed voxels (device int32 ids)."""
    import torch
    n = voxels.numel()
    words = C.c_int(0)
    d, keep = api._scene_desc(scene, dev)
    # first call sizes the words: trace zero voxels
    api._check(_lib().solar_gpu_trace_shadow_subset(ctx.h, C.byref(d), _p(voxels), 0, _p(voxels), C.byref(words),
                                                    None))
    out = torch.zeros(max(1, n), words.value, dtype=torch.int32, device=voxels.device)
    api._check(_lib().solar_gpu_trace_shadow_subset(ctx.h, C.byref(d), _p(voxels), n, _p(out), C.byref(words),
                                                    None))
    return out[:n], words.value


def bit_error(pred, exact, active: int) -> float:
    """Fraction of the active sun bins whose bit differs."""
    import torch
    x = (pred ^ exact).to(torch.int64) & 0xFFFFFFFF
    diff = sum(int(((x >> k) & 1).sum()) for k in range(32))
    return diff / (pred.shape[0] * active)


def predict_with_fallback(model: Surrogate, ctx, scene, dev: dict, tile: int = 256, spot: int = 64,
                          max_err: float = 0.02, seed: int = 0) -> dict:
    """Shadow words of every voxel: the model's, checked per tile on `spot`
    random voxels against the exact tracer; tiles above `max_err` traced
    exactly.  Returns the words and per-tile statistics."""
    import torch
    t0 = time.perf_counter()
    allv = torch.arange(scene.num_total, dtype=torch.int32, device=model.dev)
    words = model.predict_bits(scene, dev, allv)
    torch.cuda.synchronize()
    t_model = time.perf_counter() - t0
    pp = scene.pixel_parent.astype(np.int64)
    tid = (pp % scene.width) // tile + ((pp // scene.width) // tile) * ((scene.width + tile - 1) // tile)
    rng = np.random.default_rng(seed)
    stats = []
    for t in np.unique(tid):
        members = np.nonzero(tid == t)[0].astype(np.int32)
        smp = torch.from_numpy(rng.choice(members, min(spot, members.size), replace=False).astype(np.int32)).to(model.dev)
        ex, _ = exact_bits(ctx, scene, dev, smp)
        err = bit_error(words[smp.long()], ex, model.active)
        fell_back = err > max_err
        if fell_back:
            mv = torch.from_numpy(members).to(model.dev)
            exm, _ = exact_bits(ctx, scene, dev, mv)
            words[mv.long()] = exm
        stats.append({"tile": int(t), "voxels": int(members.size), "sampled_error": err, "fallback": bool(fell_back)})
    torch.cuda.synchronize()
    return {"words": words, "tiles": stats, "model_s": t_model, "total_s": time.perf_counter() - t0}


def main(argv=None) -> int:
    """Train on some synthetic cities, then the guarded prediction on another
    against the exact tracer (the ablation):

        python -m solargpu_b200.surrogate [--model conv|mlp] [--train dsm256,dsm512] [--test dsm1024]
                                          [--steps 3000]
    """
    import argparse
    import json
    import torch
    from . import inputs
    ap = argparse.ArgumentParser(description="sky-bin visibility surrogate: train and ablation")
    ap.add_argument("--model", choices=("conv", "mlp"), default="conv")
    ap.add_argument("--train", default="dsm256,dsm512")
    ap.add_argument("--test", default="dsm1024")
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--max-err", type=float, default=0.02)
    ap.add_argument("--log-every", type=int, default=0)
    ap.add_argument("--gemm-only", type=int, default=0, metavar="SIZE",
                    help="only time the tensor-core GEMM on SIZE x SIZE x SIZE (profiling)")
    a = ap.parse_args(argv)
    if a.gemm_only:
        return _gemm_bench(a.gemm_only, a.gemm_only, a.gemm_only)

    def staged(name):
        s = inputs.make_scene(name)
        d = {"grid": torch.from_numpy(s.grid).cuda(), "pixel_parent": torch.from_numpy(s.pixel_parent).cuda(),
             "wall_z": torch.from_numpy(s.wall_z if s.wall_z.size else np.zeros(1, np.float32)).cuda(),
             "slopes": torch.from_numpy(s.slopes).cuda(), "aspects": torch.from_numpy(s.aspects).cuda()}
        return s, d

    def share_of(ctx, s, d):
        """1 - own / total per voxel: the reflected share of the annual irradiance."""
        tot = torch.zeros(s.num_total, dtype=torch.float32, device="cuda")
        own = torch.zeros_like(tot)
        ctx.run_device(s, d, tot, neighbor_format=0)
        ctx.run_device(s, d, own, neighbor_format=0, reflection=api.REFL_NONE)
        return (1.0 - own.double() / tot.double().clamp_min(1.0)).clamp_min(0.0).float()

    res = {}
    with api.Context(0) as ctx:
        data = []
        shares = []
        for name in a.train.split(","):
            s, d = staged(name)
            share = share_of(ctx, s, d)
            r = ctx.trace(s, d, neighbor_format=0)
            data.append((s, d, torch.from_numpy(r["shadow"].view(np.int32)).cuda(), r["shadow_words"], share))
            shares.append(share)
            active = r["active_bins"]
        model = Surrogate(active=active, seed=0, conv=CONV if a.model == "conv" else None)
        t0 = time.perf_counter()
        losses = model.train(data, a.steps, a.batch, a.lr, log_every=a.log_every)
        torch.cuda.synchronize()
        res["train"] = {"model": a.model, "parameters": int(sum(w.numel() + b.numel() for w, b in zip(model.W, model.b))),
                        "scenes": a.train, "steps": a.steps, "batch": a.batch, "s": round(time.perf_counter() - t0, 2),
                        "loss_first100": float(np.mean(losses[:100])), "loss_last100": float(np.mean(losses[-100:]))}
        s, d = staged(a.test)
        allv = torch.arange(s.num_total, dtype=torch.int32, device="cuda")
        # exact shadow words of every voxel (chunks of 2^20), timed
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        exact = torch.cat([exact_bits(ctx, s, d, allv[i:i + (1 << 20)])[0] for i in range(0, s.num_total, 1 << 20)])
        torch.cuda.synchronize()
        t_exact = time.perf_counter() - t0
        t0 = time.perf_counter()
        pred = model.predict_bits(s, d, allv)
        torch.cuda.synchronize()
        t_pred = time.perf_counter() - t0
        guarded = predict_with_fallback(model, ctx, s, d, max_err=a.max_err)
        share_true = share_of(ctx, s, d)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        share_pred = model.predict_share(s, d, allv)
        torch.cuda.synchronize()
        t_share = time.perf_counter() - t0
        err = (share_pred - share_true).abs()
        mean_train = float(torch.cat(shares).mean())
        base = (share_true - mean_train).abs()
        res["test"] = {"scene": a.test, "voxels": s.num_total, "active_bins": active,
                       "exact_trace_s": round(t_exact, 4), "model_only_s": round(t_pred, 4),
                       "model_bit_error": bit_error(pred, exact, active),
                       "guarded_s": round(guarded["total_s"], 4),
                       "guarded_bit_error": bit_error(guarded["words"], exact, active),
                       "tiles": len(guarded["tiles"]),
                       "fallback_tiles": sum(t["fallback"] for t in guarded["tiles"]),
                       "reflected_share": {"mean": float(share_true.mean()), "max": float(share_true.max()),
                                           "model_abs_error_mean": float(err.mean()),
                                           "model_abs_error_p99": float(err.quantile(0.99)) if err.numel() <= 1 << 24
                                           else None,
                                           "model_abs_error_max": float(err.max()),
                                           "training_mean_abs_error_mean": float(base.mean()),
                                           "model_only_s": round(t_share, 4)}}
        res["gemm"] = _gemm_stats(8192, 8192, 4096)
    print(json.dumps(res))
    return 0


def _gemm_stats(Mg: int, Ng: int, Kg: int, reps: int = 5) -> dict:
    """Time of C = A B^T on the tensor cores (CUDA events, after one warm run)."""
    import torch
    A = torch.randn(Mg, Kg, device="cuda").to(torch.bfloat16)
    B = torch.randn(Ng, Kg, device="cuda").to(torch.bfloat16)
    Cg = torch.empty(Mg, Ng, device="cuda")
    api.gemm_bf16(A, B, out=Cg)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        api.gemm_bf16(A, B, out=Cg)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    return {"M": Mg, "N": Ng, "K": Kg, "ms": round(ms, 3), "tflops": round(2.0 * Mg * Ng * Kg / ms / 1e9, 1)}


def _gemm_bench(Mg: int, Ng: int, Kg: int) -> int:
    import json
    print(json.dumps({"gemm": _gemm_stats(Mg, Ng, Kg, reps=3)}))
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
