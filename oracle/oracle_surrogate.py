"""CPU oracle for the learned surrogate denoiser and the GPU scene generator.

TEST INFRASTRUCTURE ONLY: the checker for cpipe_b200/csrc/surrogate.cu and
cpipe_b200/csrc/scene.cu; the product never imports it.  There is no reference
counterpart for either (the reference's AI denoise node is not implemented), so
the network oracle restates the definition in cpipe_b200_params.h
(cpipe_SurrogateHeader): 8 zero-padded 3x3 convolutions, ReLU after all but the
last, residual output.  Arithmetic is float64; with bf16=True every tensor the
GPU stores as bfloat16 (weights, the input map, activations, the loss gradient
and the backward gradients) is rounded to bfloat16 at the same point, so the
GPU's FP32-accumulated results agree to accumulation-order rounding.
"""
import numpy as np

LAYERS = 8
SHAPES = [(32, 4)] + [(32, 32)] * 6 + [(3, 32)]  # (cout, cin)


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def prep(rgba, ab):
    """Network input [n,h,w,4]: R, G, B, sigma/0.03 in float32 as the GPU
    computes them (sigma = sqrt(max(0, b + a*max(L,0))), L = ((R+G)+B)/3)."""
    x = np.asarray(rgba, np.float32)
    r, g, b = x[..., 0], x[..., 1], x[..., 2]
    L = ((r + g) + b) * np.float32(1.0 / 3.0)
    a_ = np.asarray([p[0] for p in ab], np.float32)[:, None, None]
    b_ = np.asarray([p[1] for p in ab], np.float32)[:, None, None]
    var = np.maximum(np.float32(0.0), b_ + a_ * np.maximum(L, np.float32(0.0)))
    s = np.sqrt(var) * np.float32(1.0 / 0.03)
    return np.stack([r, g, b, s], -1).astype(np.float64)


def conv(x, W, b):
    n, h, w, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((n, h, w, W.shape[0]))
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("nhwc,oc->nhwo", xp[:, ky:ky + h, kx:kx + w, :], W[:, :, ky, kx], optimize=True)
    return out + b


def conv_input_grad(dy, W):
    n, h, w, _ = dy.shape
    dp = np.pad(dy, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dx = np.zeros((n, h, w, W.shape[1]))
    for ky in range(3):
        for kx in range(3):
            dx += np.einsum("nhwo,oc->nhwc", dp[:, 2 - ky:2 - ky + h, 2 - kx:2 - kx + w, :], W[:, :, ky, kx],
                            optimize=True)
    return dx


def conv_weight_grad(x, dy):
    n, h, w, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dW = np.zeros((dy.shape[-1], x.shape[-1], 3, 3))
    for ky in range(3):
        for kx in range(3):
            dW[:, :, ky, kx] = np.einsum("nhwo,nhwc->oc", dy, xp[:, ky:ky + h, kx:kx + w, :], optimize=True)
    return dW, dy.sum(axis=(0, 1, 2))


def forward(params, rgba, ab, bf=True):
    """Returns (output RGB [n,h,w,3], activations a0..a7)."""
    rnd = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    acts = [rnd(prep(rgba, ab))]
    for l in range(LAYERS - 1):
        W, b = params[l]
        acts.append(rnd(np.maximum(conv(acts[-1], rnd(W), np.asarray(b, np.float64)), 0.0)))
    W, b = params[-1]
    res = conv(acts[-1], rnd(W), np.asarray(b, np.float64))
    x = np.asarray(rgba, np.float64)[..., :3]
    return x + res, acts


def loss_and_grads(params, rgba, target, ab, bf=True):
    """Mean squared error over RGB and its gradients [(dW, db)] per layer."""
    rnd = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    out, acts = forward(params, rgba, ab, bf)
    t = np.asarray(target, np.float64)[..., :3]
    if bf:  # the GPU forms the output and the difference in float32
        res = (out - np.asarray(rgba, np.float64)[..., :3]).astype(np.float32)
        o32 = np.asarray(rgba, np.float32)[..., :3] + res
        d = (o32 - np.asarray(target, np.float32)[..., :3]).astype(np.float64)
    else:
        d = out - t
    count = d.shape[0] * d.shape[1] * d.shape[2] * 3
    loss = float(np.sum(d * d) / count)
    g = rnd(d * (2.0 / count))
    grads = [None] * LAYERS
    for l in range(LAYERS - 1, -1, -1):
        W, _ = params[l]
        grads[l] = conv_weight_grad(acts[l], g)
        if l == 0:
            break
        g = rnd(conv_input_grad(g, rnd(W)) * (acts[l] > 0))
    return loss, grads


# ------------------------------------------------------------ GPU scene
M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85


def philox(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 (Salmon et al., SC 2011) on numpy uint64 arrays holding
    32-bit words."""
    mask = np.uint64(0xFFFFFFFF)
    c = [np.asarray(v, np.uint64) & mask for v in (c0, c1, c2, c3)]
    k0, k1 = np.uint64(k0) & mask, np.uint64(k1) & mask
    for _ in range(10):
        p0 = c[0] * np.uint64(M0)
        p1 = c[2] * np.uint64(M1)
        hi0, lo0 = p0 >> np.uint64(32), p0 & mask
        hi1, lo1 = p1 >> np.uint64(32), p1 & mask
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
        k0 = (k0 + np.uint64(W0)) & mask
        k1 = (k1 + np.uint64(W1)) & mask
    return c


def unit(u):
    return ((np.asarray(u, np.float64) + 1.0) * (1.0 / 4294967296.0)).astype(np.float32)


def scene_clean(w, h, seed, cfa=(0, 1, 1, 2), rects=20):
    """The noise-free mosaic of cpipe_cuda_scene_raw, float32 in [0, 1]."""
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    f32 = np.float32
    y, x = np.mgrid[0:h, 0:w]
    fx = (x.astype(f32) / f32(w - 1)) if w > 1 else np.zeros((h, w), f32)
    fy = (y.astype(f32) / f32(h - 1)) if h > 1 else np.zeros((h, w), f32)
    rgb = np.stack([f32(0.15) + f32(0.55) * fx + f32(0.1) * fy, f32(0.2) + f32(0.4) * fy + f32(0.15) * fx,
                    f32(0.1) + f32(0.3) * (f32(1.0) - fx) + f32(0.25) * fy], -1)
    painted = np.zeros((h, w), bool)
    for i in range(rects - 1, -1, -1):
        g = philox(i, 1, 0, 0, k0, k1)
        xa, xb = int(g[0]) % w, int(g[1]) % w
        ya, yb = int(g[2]) % h, int(g[3]) % h
        c = philox(i, 2, 0, 0, k0, k1)
        refl = [f32(0.05) + f32(0.85) * unit(c[k]) for k in range(3)]
        m = (x >= min(xa, xb)) & (x <= max(xa, xb)) & (y >= min(ya, yb)) & (y <= max(ya, yb)) & ~painted
        rgb[m] = np.array(refl, f32)
        painted |= m
    cy, cx, rr = f32(h) * f32(0.5), f32(w) * f32(0.5), f32(min(h, w)) / f32(6.0)
    yf, xf = y.astype(f32), x.astype(f32)
    zm = (np.abs(yf - cy) < rr) & (np.abs(xf - cx) < rr)
    d2 = ((yf - cy) * (yf - cy) + (xf - cx) * (xf - cx)) / (rr * rr)
    zp = f32(0.5) + f32(0.4) * np.cos(f32(3.14159265358979) * f32(0.5) * rr * d2).astype(f32)
    for k, s in enumerate((0.9, 0.85, 0.8)):
        rgb[..., k][zm] = (zp * f32(s))[zm]
    idx = np.asarray(cfa)[(y & 1) * 2 + (x & 1)]
    clean = np.take_along_axis(rgb, idx[..., None], -1)[..., 0]
    return np.clip(clean, 0.0, 1.0).astype(f32)


def scene_raw(w, h, seed, bits=10, black=16, a=4e-3, b=4e-5, cfa=(0, 1, 1, 2), rects=20):
    f32 = np.float32
    clean = scene_clean(w, h, seed, cfa, rects)
    p = np.arange(w * h, dtype=np.uint64)
    r = philox(p & np.uint64(0xFFFFFFFF), p >> np.uint64(32), 3, 0, seed & 0xFFFFFFFF, seed >> 32)
    u1, u2 = unit(r[0]).reshape(h, w), unit(r[1]).reshape(h, w)
    nrm = (np.sqrt(f32(-2.0) * np.log(u1)) * np.cos(f32(6.28318530717959) * u2)).astype(f32)
    noisy = clean + np.sqrt(np.maximum(f32(a) * clean + f32(b), f32(0.0))) * nrm
    white = (1 << bits) - 1
    v = np.rint(noisy * f32(white - black)) + f32(black)
    return np.clip(v, 0, white).astype(np.uint16), clean
