"""FP64 restatement of the learned denoiser (test infrastructure only).

The oracle the BF16 tensor-core network is checked against: every layer and
the whole kernel-predicting U-Net, forward and backward, in float64 numpy,
with bf16 rounding applied at exactly the points where the device stores a
bf16 tensor (`rounded=True`), so that the only differences left are the
device's fp32 accumulation order. Nothing in the product imports this file.

phiray has no learned denoiser; what it pins here is the build's own network.
The inputs come from phiray's px image planes (src/trace/read.rs:37-56:
sums n..4n, albedo 7n..10n, normal 10n..13n, depth 13n..14n, sample count
31n..32n, missed samples 33n..34n) and the radiance the loss compares is
Tracer::radiance (read.rs:241-251). The compose step restates the last
a-trous round's write-back (src/kernel/denoise.wgsl, Standard view).
"""

from __future__ import annotations

import numpy as np

LAYERS = [(16, 32), (32, 32), (32, 64), (64, 64), (64, 96), (96, 96), (96, 128), (128, 128), (128, 160),
          (160, 160), (288, 128), (128, 128), (224, 96), (96, 96), (160, 64), (64, 64), (96, 32), (32, 32), (32, 32)]
LEVEL_CH = [32, 64, 96, 128, 160]
CAT_CH = [96, 160, 224, 288]
UP_CH = [64, 96, 128, 160]
LN2 = 0.693147182


def bf16(x) -> np.ndarray:
    """Round to the nearest bf16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)
    nan = np.isnan(f)
    if nan.any():
        out = np.where(nan, f, out)
    return out.astype(np.float64)


def bf16_bits(x) -> np.ndarray:
    """uint16 bit patterns of bf16(x)."""
    return (bf16(x).astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(b) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32).astype(np.float64)


# ---- layers ----

def im2col(x: np.ndarray) -> np.ndarray:
    """(B, H, W, C) -> (B, H, W, 9 C), k = (3 ty + tx) C + c, zero padding 1."""
    B, H, W, C = x.shape
    p = np.zeros((B, H + 2, W + 2, C), dtype=np.float64)
    p[:, 1:-1, 1:-1] = x
    return np.concatenate([p[:, ty:ty + H, tx:tx + W] for ty in range(3) for tx in range(3)], axis=-1)


def conv(x: np.ndarray, w: np.ndarray, b: np.ndarray | None, relu: bool, acc=np.float64) -> np.ndarray:
    """3x3 convolution, stride 1, same size: w is (cout, 9 cin). `acc` is the
    accumulation type (float32 gives a second, equally valid summation for
    measuring how far bf16 rounding amplifies accumulation-order noise)."""
    y = np.einsum("bhwk,ok->bhwo", im2col(x).astype(acc), w.astype(acc), optimize=True).astype(np.float64)
    if b is not None:
        y = y + b
    return np.maximum(y, 0.0) if relu else y


def conv_wgrad(x: np.ndarray, dy: np.ndarray, acc=np.float64) -> np.ndarray:
    """dW (cout, 9 cin) = sum over pixels of dy[p, o] im2col(x)[p, k]."""
    return np.einsum("bhwk,bhwo->ok", im2col(x).astype(acc), dy.astype(acc), optimize=True).astype(np.float64)


def flip(w: np.ndarray, cin: int) -> np.ndarray:
    """W2 (cin, 9 cout) with W2[ci, (8 - tap) cout + co] = W[co, tap cin + ci]."""
    cout = w.shape[0]
    w4 = w.reshape(cout, 9, cin)  # [co, tap, ci]
    return w4[:, ::-1, :].transpose(2, 1, 0).reshape(cin, 9 * cout)


def conv_dgrad(dy: np.ndarray, w: np.ndarray, cin: int, acc=np.float64) -> np.ndarray:
    """dX = the 3x3 convolution of dy by flip(w)."""
    return conv(dy, flip(w, cin), None, False, acc)


def pool(x: np.ndarray) -> np.ndarray:
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4)) * 0.25


def pool_bwd(dy: np.ndarray) -> np.ndarray:
    return np.repeat(np.repeat(dy, 2, axis=1), 2, axis=2) * 0.25


def up(x: np.ndarray) -> np.ndarray:
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up_bwd(dy: np.ndarray) -> np.ndarray:
    B, H, W, C = dy.shape
    return dy.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


def kpn(logits, irr, alb, h, w, ref=None, err_weight=0.0):
    """Softmax-weighted 5x5 filter of irr (clamped to the valid h x w) times
    alb; error estimate exp(logit 25) - 1e-3; with ref: (loss, dlogits)."""
    B, Hp, Wp, _ = logits.shape
    lg = logits[:, :h, :w, :25]
    mx = lg.max(axis=-1, keepdims=True)
    e = np.exp(lg - mx)
    wt = e / e.sum(axis=-1, keepdims=True)  # (B, h, w, 25)
    ys = np.arange(h)
    xs = np.arange(w)
    taps = []
    for t in range(25):
        yy = np.clip(ys + t // 5 - 2, 0, h - 1)
        xx = np.clip(xs + t % 5 - 2, 0, w - 1)
        taps.append(irr[:, yy][:, :, xx][:, :, :, :3])
    nb = np.stack(taps, axis=3)  # (B, h, w, 25, 3)
    a = alb[:, :h, :w]
    s = np.einsum("bhwt,bhwtc->bhwc", wt, nb)
    o = a * s
    out = np.zeros((B, Hp, Wp, 3))
    out[:, :h, :w] = o
    err = np.zeros((B, Hp, Wp))
    err[:, :h, :w] = np.maximum(np.exp(logits[:, :h, :w, 25]) - 1e-3, 0.0)
    if ref is None:
        return out, err
    r = ref[:, :h, :w]
    den = r * r + 0.01
    d = o - r
    scale = 1.0 / (3.0 * B * h * w)
    rel = (d * d / den).sum(axis=-1)
    loss = rel.sum() * scale
    go = 2.0 * d / den * scale * a
    gw = np.einsum("bhwc,bhwtc->bhwt", go, nb)
    dot = (wt * gw).sum(axis=-1, keepdims=True)
    dl = np.zeros((B, Hp, Wp, 32))
    dl[:, :h, :w, :25] = wt * (gw - dot)
    target = np.log(rel / 3.0 + 1e-3)
    dl[:, :h, :w, 25] = 2.0 * err_weight * (logits[:, :h, :w, 25] - target) * (3.0 * scale)
    return out, err, loss, dl


def _fin(a):
    return np.where(np.isfinite(a), a, 0.0)


def features(px: np.ndarray, w: int, h: int, Hp: int, Wp: int, half: np.ndarray | None = None):
    """(feat (Hp, Wp, 16), irr (Hp, Wp, 3), alb (Hp, Wp, 3)) from px planes;
    `half` (n, 4): sums and met-sample counts part way through the samples."""
    n = w * h
    f = px.view(np.float32).astype(np.float64)
    cnt_raw = px[31 * n:32 * n].astype(np.float64)
    cnt = np.maximum(cnt_raw, 1.0)
    gone = f[33 * n:34 * n]
    met = np.maximum(cnt - gone, 1.0)
    sums = f[n:4 * n].reshape(n, 3)
    with np.errstate(invalid="ignore", over="ignore", divide="ignore"):
        rad = _fin(np.maximum(sums / met[:, None], 0.0))
        al = _fin(f[7 * n:10 * n].reshape(n, 3) / cnt[:, None])
    ad = np.maximum(al, 0.05)
    ir = rad / ad
    nr = _fin(f[10 * n:13 * n].reshape(n, 3))
    nn = (nr * nr).sum(axis=1)
    nr = nr * np.where(nn > 0, 1.0 / np.sqrt(np.where(nn > 0, nn, 1.0)), 0.0)[:, None]
    d = _fin(f[13 * n:14 * n] / cnt)
    feat = np.zeros((Hp, Wp, 16))
    v = feat[:h, :w]
    if half is not None:
        hs = half.astype(np.float64)
        met_total = cnt_raw - gone
        spread = (hs[:, 3] >= 1.0) & (met_total - hs[:, 3] >= 1.0)
        with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
            ra = np.maximum(hs[:, :3] / hs[:, 3:4], 0.0)
            rb = np.maximum((sums - hs[:, :3]) / (met_total - hs[:, 3])[:, None], 0.0)
            sp = _fin(np.abs(ra - rb) * 0.5 / np.maximum(al, 0.05))
        v[..., 0:3] = np.where(spread[:, None], np.log1p(np.where(spread[:, None], sp, 0.0)), 0.0).reshape(h, w, 3)
        v[..., 15] = spread.astype(np.float64).reshape(h, w)
    v[..., 3:6] = np.log1p(ir).reshape(h, w, 3)
    v[..., 6:9] = al.reshape(h, w, 3)
    v[..., 9:12] = nr.reshape(h, w, 3)
    v[..., 12] = (d / (1.0 + np.abs(d))).reshape(h, w)
    v[..., 13] = np.maximum(1.0 - gone / cnt, 0.0).reshape(h, w)
    v[..., 14] = (np.log2(cnt) * 0.125).reshape(h, w)
    irr = np.zeros((Hp, Wp, 3))
    alb = np.zeros((Hp, Wp, 3))
    irr[:h, :w] = ir.reshape(h, w, 3)
    alb[:h, :w] = ad.reshape(h, w, 3)
    return feat, irr, alb


# ---- the network ----

def firefly(irr: np.ndarray, h: int, w: int) -> np.ndarray:
    """The a-trous Denoise's first-round firefly clamp (denoise.wgsl:47-134,
    its FIRST pass) on padded (B, Hp, Wp, 3) irradiance, in float32 with the
    device's order of operations: inside the h x w image, a pixel whose luma
    0.2126 r + 0.7152 g + 0.0722 b exceeds 1.5 x the brightest in-image
    8-neighbour's + 0.05 takes the neighbours' mean (summed row by row);
    other pixels are copied."""
    x = np.asarray(irr, dtype=np.float32)
    out = x.copy()
    B = x.shape[0]
    k = [np.float32(0.2126), np.float32(0.7152), np.float32(0.0722)]

    def luma(v):
        return (v[..., 0] * k[0] + v[..., 1] * k[1]) + v[..., 2] * k[2]

    top = np.zeros((B, h, w), np.float32)
    acc = np.zeros((B, h, w, 3), np.float32)
    cnt = np.zeros((B, h, w), np.float32)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            if dy == 0 and dx == 0:
                continue
            ys, xs = np.arange(h) + dy, np.arange(w) + dx
            ok = ((ys >= 0) & (ys < h))[:, None] & ((xs >= 0) & (xs < w))[None, :]
            nb = x[:, np.clip(ys, 0, h - 1)][:, :, np.clip(xs, 0, w - 1)]
            top = np.where(ok, np.maximum(top, luma(nb)), top)
            acc = np.where(ok[..., None], acc + nb, acc)
            cnt = np.where(ok, cnt + np.float32(1.0), cnt)
    centre = x[:, :h, :w]
    hit = (cnt > 0) & (luma(centre) > np.float32(1.5) * top + np.float32(0.05))
    mean = acc / np.maximum(cnt, np.float32(1.0))[..., None]
    out[:, :h, :w] = np.where(hit[..., None], mean, centre)
    return out


def split_params(blob: np.ndarray):
    """Blob (per layer W (cout, 9 cin) then b (cout,)) -> [(W, b)]."""
    out, o = [], 0
    for cin, cout in LAYERS:
        W = blob[o:o + cout * 9 * cin].reshape(cout, 9 * cin).astype(np.float64)
        o += cout * 9 * cin
        b = blob[o:o + cout].astype(np.float64)
        o += cout
        out.append((W, b))
    assert o == blob.size
    return out


def join_params(pairs) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in pairs])


def forward(params, feat, rounded=True, acc=np.float64):
    """Logits (B, H, W, 32) and the activations backward needs."""
    R = bf16 if rounded else (lambda a: np.asarray(a, dtype=np.float64))
    P = [(R(W), b) for W, b in params]
    act = {"feat": feat}
    x = feat
    for l in range(4):
        A = R(conv(x, *P[2 * l], True, acc))
        S = R(conv(A, *P[2 * l + 1], True, acc))
        act[f"A{l}"], act[f"S{l}"] = A, S
        x = R(pool(S))
        act[f"pool{l + 1}"] = x
    A4 = R(conv(x, *P[8], True, acc))
    B4 = R(conv(A4, *P[9], True, acc))
    act["A4"], act["B4"] = A4, B4
    below = B4
    for l in range(3, -1, -1):
        cat = np.concatenate([up(below), act[f"S{l}"]], axis=-1)
        d = 10 + 2 * (3 - l)
        Da = R(conv(cat, *P[d], True, acc))
        Db = R(conv(Da, *P[d + 1], True, acc))
        act[f"cat{l}"], act[f"Da{l}"], act[f"Db{l}"] = cat, Da, Db
        below = Db
    logits = conv(below, *P[18], False, acc)
    if rounded:
        logits = logits.astype(np.float32).astype(np.float64)
    return logits, act, P


def backward(P, act, dlogits, rounded=True, acc=np.float64):
    """Gradients [(dW, db)] of every layer, dlogits the head's output gradient."""
    R = bf16 if rounded else (lambda a: np.asarray(a, dtype=np.float64))
    grads = [None] * len(LAYERS)

    def layer(i, x, dy, want_dx):
        cin = LAYERS[i][0]
        grads[i] = (conv_wgrad(x, dy, acc), dy.sum(axis=(0, 1, 2)))
        return R(conv_dgrad(dy, P[i][0], cin, acc)) if want_dx else None

    dy = R(dlogits)
    d = layer(18, act["Db0"], dy, True)
    for l in range(4):
        dn = 10 + 2 * (3 - l)
        d = d * (act[f"Db{l}"] > 0)
        dda = layer(dn + 1, act[f"Da{l}"], d, True)
        dda = dda * (act[f"Da{l}"] > 0)
        dcat = layer(dn, act[f"cat{l}"], dda, True)
        act[f"dskip{l}"] = dcat[..., UP_CH[l]:]
        d = R(up_bwd(dcat[..., :UP_CH[l]]))
    d = d * (act["B4"] > 0)
    dA4 = layer(9, act["A4"], d, True) * (act["A4"] > 0)
    dp = layer(8, act["pool4"], dA4, True)
    for l in range(3, -1, -1):
        ds = R(act[f"dskip{l}"] + pool_bwd(dp))
        ds = ds * (act[f"S{l}"] > 0)
        dA = layer(2 * l + 1, act[f"A{l}"], ds, True) * (act[f"A{l}"] > 0)
        if l > 0:
            dp = layer(2 * l, act[f"pool{l}"], dA, True)
        else:
            layer(0, act["feat"], dA, False)
    return grads


def adam(w, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    return w - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v


def compose(px, w, h, out, err, tile, threshold, keep=False, exposure=0.0, gamma=1.0):
    """Tiles whose mean error estimate is within threshold: the learned
    radiance replaces the px sums (unless keep); returns the px copy with the
    sums written and the tile mask (True = learned). The shown and packed
    planes are checked through the sums on the device side."""
    px = px.copy()
    n = w * h
    ty, tx = (h + tile - 1) // tile, (w + tile - 1) // tile
    mask = np.zeros((ty, tx), dtype=bool)
    for j in range(ty):
        for i in range(tx):
            e = err[j * tile:(j + 1) * tile, i * tile:(i + 1) * tile]
            mask[j, i] = e.mean() <= threshold
    cnt = np.maximum(px[31 * n:32 * n].astype(np.float64), 1.0)
    f = px.view(np.float32)
    gone = f[33 * n:34 * n].astype(np.float64)
    metf = 1.0 - gone / cnt
    m = np.maximum(cnt - gone, 1.0)
    if not keep:
        lin = out[:h, :w].reshape(n, 3).copy()
        lin[~(metf > 0.5 / cnt)] = 0.0
        sums = f[n:4 * n].reshape(n, 3)
        pm = np.repeat(np.repeat(mask, tile, 0), tile, 1)[:h, :w].reshape(n)
        sums[pm] = (lin * m[:, None])[pm].astype(np.float32)
    return px, mask
