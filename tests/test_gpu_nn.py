"""The tcgen05 BF16 engine and the learned denoiser's kernels against the
FP64 oracle (oracle/nn.py) on the same bf16 inputs: each layer forward and
backward, the per-pixel kernel step and its loss gradient, Adam, the
feature planes, the whole network's logits and gradients, and the per-tile
fallback to the a-trous Denoise."""

import ctypes as C

import numpy as np
import pytest

from phiray_b200 import _native as N
from tests import oracle_lib

pytestmark = pytest.mark.gpu
nn = oracle_lib.nn()


def _t(a, dtype=None):
    """A CUDA tensor of a numpy array (bf16 from float64 via the oracle's rounding)."""
    import torch

    if dtype == "bf16":
        bits = nn.bf16_bits(a).view(np.int16)
        return torch.from_numpy(bits.copy()).cuda().view(torch.bfloat16)
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _np(t):
    import torch

    torch.cuda.synchronize()
    if t.dtype == torch.bfloat16:
        return nn.from_bf16_bits(t.view(torch.int16).cpu().numpy().view(np.uint16))
    return t.cpu().numpy().astype(np.float64)


def _sync(gpu):
    import torch

    torch.cuda.synchronize()
    gpu.wait()


def _round64(k):
    return (k + 63) // 64 * 64


@pytest.mark.parametrize("n", [32, 64, 96, 128, 160])
@pytest.mark.parametrize("m,k", [(128, 64), (256, 576), (1024, 1472)])
def test_gemm_bf16_matches_fp32_product(gpu, m, n, k):
    import torch

    g = torch.Generator(device="cpu").manual_seed(m * 1000 + n + k)
    a = torch.randn(m, k, generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, generator=g).to(torch.bfloat16)
    want = a.double() @ b.double().T
    da, db = a.cuda(), b.cuda()
    d = torch.empty(m, n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_gemm_bf16(gpu.handle, da.data_ptr(), db.data_ptr(), d.data_ptr(), m, n, k))
    gpu.wait()
    got = d.cpu().double()
    err = (got - want).abs().max().item()
    scale = want.abs().max().item()
    assert err <= 1e-5 * scale + 1e-4, (err, scale)  # fp32 accumulation of exact bf16 products


def _weights(rng, cout, cin):
    K = 9 * cin
    Kp = _round64(K)
    w = nn.bf16(rng.normal(size=(cout, K)) * np.sqrt(2.0 / K))
    wp = np.zeros((cout, Kp))
    wp[:, :K] = w
    return w, wp, Kp


CONV_CASES = [
    (16, 32, True, False),
    (32, 64, True, False),
    (64, 96, False, False),
    (96, 128, True, False),
    (128, 160, True, False),
    (288, 128, True, False),
    (224, 96, True, False),
    (32, 32, False, True),
    (96, 32, True, False),
    (160, 64, True, False),
]


@pytest.mark.parametrize("cin,cout,relu,f32", CONV_CASES)
def test_conv_fwd(gpu, cin, cout, relu, f32):
    """Implicit-GEMM 3x3 convolution on the tensor cores, reading a channel
    window of a wider buffer and writing into another: rounding of the
    exact product only (bf16 out) or fp32 accumulation error (fp32 out);
    the channels outside the window are untouched."""
    import torch

    rng = np.random.default_rng(cin * 1000 + cout)
    B, H, W = 2, 12, 20  # 480 pixels: 3 full 128-row tiles and a partial one
    xs, xo = cin + 16, 8
    xbuf = nn.bf16(rng.normal(size=(B, H, W, xs)))
    x = xbuf[..., xo:xo + cin]
    w, wp, Kp = _weights(rng, cout, cin)
    bias = rng.normal(size=cout).astype(np.float32) * 0.1
    ys, yo = cout + 16, 8
    X, Wt, bb = _t(xbuf, "bf16"), _t(wp, "bf16"), _t(bias)
    sentinel = 1024.0  # exact in bf16 and fp32
    if f32:
        Y = torch.full((B, H, W, ys), sentinel, dtype=torch.float32, device="cuda")
    else:
        Y = torch.full((B, H, W, ys), sentinel, dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_conv_fwd(gpu.handle, X.data_ptr(), xs, xo, cin, Wt.data_ptr(), Kp, bb.data_ptr(),
                                    Y.data_ptr(), ys, yo, cout, B, H, W, int(relu), int(f32)))
    _sync(gpu)
    got = _np(Y)
    want = nn.conv(x, w, bias.astype(np.float64), relu)
    mag = nn.conv(np.abs(x), np.abs(w), np.abs(bias), False)
    g = got[..., yo:yo + cout]
    if f32:
        assert np.all(np.abs(g - want) <= 1e-5 * mag + 1e-30)
    else:
        assert np.all(np.abs(g - want) <= 2.0 ** -8 * np.abs(want) + 1e-5 * mag + 1e-30)
    assert np.all(got[..., :yo] == sentinel) and np.all(got[..., yo + cout:] == np.float32(sentinel))


@pytest.mark.parametrize("cin,cout,shape", [(16, 32, (2, 256, 384)), (32, 64, (1, 256, 256)),
                                            (96, 32, (1, 256, 256))])
def test_conv_fwd_many_tiles_per_block(gpu, cin, cout, shape):
    """Images with more 16 x 8 tiles than resident blocks: the persistent,
    weight-stationary form walks several tiles per block through its two
    patch buffers and two tensor-memory accumulators."""
    import torch

    rng = np.random.default_rng(cin * 31 + cout)
    B, H, W = shape
    x = nn.bf16(rng.normal(size=(B, H, W, cin)))
    w, wp, Kp = _weights(rng, cout, cin)
    bias = rng.normal(size=cout).astype(np.float32) * 0.1
    X, Wt, bb = _t(x, "bf16"), _t(wp, "bf16"), _t(bias)
    Y = torch.empty((B, H, W, cout), dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_conv_fwd(gpu.handle, X.data_ptr(), cin, 0, cin, Wt.data_ptr(), Kp, bb.data_ptr(),
                                    Y.data_ptr(), cout, 0, cout, B, H, W, 1, 0))
    _sync(gpu)
    got = _np(Y)
    want = nn.conv(x, w, bias.astype(np.float64), True)
    mag = nn.conv(np.abs(x), np.abs(w), np.abs(bias), False)
    assert np.all(np.abs(got - want) <= 2.0 ** -8 * np.abs(want) + 1e-5 * mag + 1e-30)


@pytest.mark.parametrize("cin,cout,shape", [(16, 32, (2, 12, 20)), (96, 96, (1, 16, 24)), (288, 128, (2, 8, 8)),
                                            (32, 160, (1, 64, 96)), (64, 64, (1, 64, 96))])
def test_conv_wgrad(gpu, cin, cout, shape):
    """Weight gradient: im2col(X)^T dY on the tensor cores, split over the
    pixels with fp32 atomics; rows past K stay zero."""
    import torch

    rng = np.random.default_rng(cin * 7 + cout)
    B, H, W = shape
    xs, xo = cin + 8, 8
    xbuf = nn.bf16(rng.normal(size=(B, H, W, xs)))
    x = xbuf[..., xo:xo + cin]
    dys, dyo = cout + 32, 16
    dybuf = nn.bf16(rng.normal(size=(B, H, W, dys)))
    dy = dybuf[..., dyo:dyo + cout]
    K, Kp = 9 * cin, _round64(9 * cin)
    X, DY = _t(xbuf, "bf16"), _t(dybuf, "bf16")
    dWt = torch.zeros((Kp, cout), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_conv_wgrad(gpu.handle, X.data_ptr(), xs, xo, cin, DY.data_ptr(), dys, dyo, cout,
                                      dWt.data_ptr(), Kp, B, H, W))
    _sync(gpu)
    got = _np(dWt)
    want = nn.conv_wgrad(x, dy)  # (cout, K)
    mag = nn.conv_wgrad(np.abs(x), np.abs(dy))
    assert np.all(np.abs(got[:K].T - want) <= 1e-5 * mag + 1e-30)
    assert np.all(got[K:] == 0.0)


@pytest.mark.parametrize("cin,cout", [(32, 32), (96, 64), (160, 160), (64, 128)])
def test_conv_dgrad_by_flipped_weights(gpu, cin, cout):
    """Data gradient = the 3x3 convolution of dY by the flipped weights."""
    import torch

    rng = np.random.default_rng(cin + 31 * cout)
    B, H, W = 2, 10, 14
    w, wp, Kp = _weights(rng, cout, cin)
    dy = nn.bf16(rng.normal(size=(B, H, W, cout)))
    Kp2 = _round64(9 * cout)
    Wt, DY = _t(wp, "bf16"), _t(dy, "bf16")
    W2 = torch.empty((cin, Kp2), dtype=torch.bfloat16, device="cuda")
    zero = torch.zeros(cin, dtype=torch.float32, device="cuda")
    DX = torch.empty((B, H, W, cin), dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_flip(gpu.handle, Wt.data_ptr(), cout, cin, Kp, W2.data_ptr(), Kp2))
    N.check(N.lib().phx_nn_conv_fwd(gpu.handle, DY.data_ptr(), cout, 0, cout, W2.data_ptr(), Kp2, zero.data_ptr(),
                                    DX.data_ptr(), cin, 0, cin, B, H, W, 0, 0))
    _sync(gpu)
    w2 = _np(W2)
    assert np.array_equal(w2[:, :9 * cout], nn.flip(w, cin)) and np.all(w2[:, 9 * cout:] == 0)
    got = _np(DX)
    want = nn.conv_dgrad(dy, w, cin)
    mag = nn.conv_dgrad(np.abs(dy), np.abs(w), cin)
    assert np.all(np.abs(got - want) <= 2.0 ** -8 * np.abs(want) + 1e-5 * mag + 1e-30)


def test_pool_up_relu_bias(gpu):
    """The elementwise layers: pooling and upsampling (and their gradients,
    pooling's added into a channel window), ReLU's gradient, bias gradient."""
    import torch

    rng = np.random.default_rng(5)
    B, H, W, C = 2, 8, 12, 32
    pitch, off = 96, 64
    buf = nn.bf16(rng.normal(size=(B, H, W, pitch)))
    X = _t(buf, "bf16")
    Y = torch.empty((B, H // 2, W // 2, C), dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_pool_fwd(gpu.handle, X.data_ptr(), pitch, off, C, B, H, W, Y.data_ptr()))
    _sync(gpu)
    assert np.array_equal(_np(Y), nn.bf16(nn.pool(buf[..., off:off + C])))

    dy = nn.bf16(rng.normal(size=(B, H // 2, W // 2, C)))
    DY = _t(dy, "bf16")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_pool_bwd(gpu.handle, DY.data_ptr(), C, B, H, W, X.data_ptr(), pitch, off))
    _sync(gpu)
    got = _np(X)
    want = buf.copy()
    want[..., off:off + C] = nn.bf16(buf[..., off:off + C] + nn.pool_bwd(dy))
    assert np.array_equal(got, want)

    small = nn.bf16(rng.normal(size=(B, H // 2, W // 2, C)))
    S = _t(small, "bf16")
    U = torch.zeros((B, H, W, pitch), dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_up_fwd(gpu.handle, S.data_ptr(), C, B, H, W, U.data_ptr(), pitch, 0))
    _sync(gpu)
    u = _np(U)
    assert np.array_equal(u[..., :C], nn.up(small)) and np.all(u[..., C:] == 0)

    D = torch.empty((B, H // 2, W // 2, C), dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_up_bwd(gpu.handle, X.data_ptr(), pitch, off, C, B, H, W, D.data_ptr()))
    _sync(gpu)
    assert np.array_equal(_np(D), nn.bf16(nn.up_bwd(got[..., off:off + C])))

    yv = nn.bf16(rng.normal(size=(B * H * W, pitch)))
    dv = nn.bf16(rng.normal(size=(B * H * W, pitch)))
    Yt, Dt = _t(yv, "bf16"), _t(dv, "bf16")
    db = torch.zeros(C, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_relu_bwd(gpu.handle, Yt.data_ptr(), pitch, 8, Dt.data_ptr(), pitch, off, C, B * H * W))
    N.check(N.lib().phx_nn_bias_grad(gpu.handle, Dt.data_ptr(), pitch, off, C, B * H * W, db.data_ptr()))
    _sync(gpu)
    want = dv.copy()
    want[:, off:off + C] *= yv[:, 8:8 + C] > 0
    assert np.array_equal(_np(Dt), want)
    sums = want[:, off:off + C].sum(axis=0)
    assert np.allclose(_np(db), sums, rtol=1e-5, atol=1e-4)


def test_kpn_and_loss_gradient(gpu):
    """Per-pixel 5x5 kernels on demodulated radiance, the error estimate, the
    relMSE loss and its logit gradient, with padding pixels zero."""
    import torch

    rng = np.random.default_rng(11)
    B, Hp, Wp, h, w = 2, 16, 32, 13, 27
    logits = rng.normal(size=(B, Hp, Wp, 32)).astype(np.float32)
    irr = rng.gamma(1.0, size=(B, Hp, Wp, 3)).astype(np.float32)
    alb = rng.uniform(0.05, 1.0, size=(B, Hp, Wp, 3)).astype(np.float32)
    ref = rng.gamma(1.0, size=(B, Hp, Wp, 3)).astype(np.float32)
    L, I, A, R = _t(logits), _t(irr), _t(alb), _t(ref)
    out = torch.empty((B, Hp, Wp, 3), dtype=torch.float32, device="cuda")
    err = torch.empty((B, Hp, Wp), dtype=torch.float32, device="cuda")
    dl = torch.empty((B, Hp, Wp, 32), dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_kpn(gpu.handle, L.data_ptr(), I.data_ptr(), A.data_ptr(), R.data_ptr(), B, Hp, Wp, h, w,
                               out.data_ptr(), err.data_ptr(), dl.data_ptr(), loss.data_ptr(), 0.25))
    _sync(gpu)
    o, e, lo, d = nn.kpn(logits.astype(np.float64), irr.astype(np.float64), alb.astype(np.float64), h, w,
                         ref.astype(np.float64), 0.25)
    assert np.allclose(_np(out), o, rtol=2e-5, atol=1e-6)
    assert np.allclose(_np(err), e, rtol=2e-5, atol=1e-7)
    assert abs(_np(loss)[0] - lo) <= 1e-4 * lo
    got = _np(dl)
    assert np.all(np.abs(got - d) <= 2.0 ** -8 * np.abs(d) + 1e-4 * np.abs(d).max())
    assert np.all(got[:, h:] == 0) and np.all(got[:, :, w:] == 0) and np.all(got[..., 26:] == 0)


def test_head_with_kpn_epilogue_equals_head_then_kpn(gpu):
    """The fused head + kernel-prediction step gives the outputs of the head
    convolution (fp32 logits) followed by the kernel-prediction kernel."""
    import torch

    rng = np.random.default_rng(21)
    B, Hp, Wp, h, w = 2, 32, 48, 29, 41
    x = nn.bf16(rng.normal(size=(B, Hp, Wp, 32)) * 0.5)
    wgt, wp, Kp = _weights(rng, 32, 32)
    bias = (rng.normal(size=32) * 0.1).astype(np.float32)
    irr = rng.gamma(1.0, size=(B, Hp, Wp, 3)).astype(np.float32)
    alb = rng.uniform(0.05, 1.0, size=(B, Hp, Wp, 3)).astype(np.float32)
    X, Wt, bb, I, A = _t(x, "bf16"), _t(wp, "bf16"), _t(bias), _t(irr), _t(alb)
    logits = torch.empty((B, Hp, Wp, 32), dtype=torch.float32, device="cuda")
    o1 = torch.empty((B, Hp, Wp, 3), dtype=torch.float32, device="cuda")
    e1 = torch.empty((B, Hp, Wp), dtype=torch.float32, device="cuda")
    o2 = torch.empty_like(o1)
    e2 = torch.empty_like(e1)
    torch.cuda.synchronize()
    L = N.lib()
    N.check(L.phx_nn_conv_fwd(gpu.handle, X.data_ptr(), 32, 0, 32, Wt.data_ptr(), Kp, bb.data_ptr(), logits.data_ptr(),
                              32, 0, 32, B, Hp, Wp, 0, 1))
    N.check(L.phx_nn_kpn(gpu.handle, logits.data_ptr(), I.data_ptr(), A.data_ptr(), None, B, Hp, Wp, h, w,
                         o1.data_ptr(), e1.data_ptr(), None, None, 0.0))
    N.check(L.phx_nn_conv_kpn(gpu.handle, X.data_ptr(), 32, 0, 32, Wt.data_ptr(), Kp, bb.data_ptr(), I.data_ptr(),
                              A.data_ptr(), B, Hp, Wp, h, w, o2.data_ptr(), e2.data_ptr()))
    _sync(gpu)
    assert np.allclose(_np(o1), _np(o2), rtol=1e-6, atol=1e-7)
    assert np.allclose(_np(e1), _np(e2), rtol=1e-6, atol=1e-9)
    o, e = nn.kpn(nn.conv(x, wgt, bias.astype(np.float64), False), irr.astype(np.float64), alb.astype(np.float64), h, w)
    assert np.allclose(_np(o2), o, rtol=1e-4, atol=1e-6)


def test_adam(gpu):
    import torch

    rng = np.random.default_rng(3)
    rows, K, Kp = 32, 144, 192
    w = rng.normal(size=(rows, Kp)).astype(np.float32)
    w[:, K:] = 0
    g = rng.normal(size=(Kp, rows)).astype(np.float32)
    m = rng.normal(size=(rows, Kp)).astype(np.float32) * 0.1
    v = rng.uniform(0, 0.1, size=(rows, Kp)).astype(np.float32)
    Wd, G, M, V = _t(w), _t(g), _t(m), _t(v)
    WB = torch.empty((rows, Kp), dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_adam(gpu.handle, Wd.data_ptr(), G.data_ptr(), M.data_ptr(), V.data_ptr(), WB.data_ptr(),
                                rows, Kp, K, 1, 1e-3, 0.9, 0.999, 1e-8, 7))
    _sync(gpu)
    b1, b2 = float(np.float32(0.9)), float(np.float32(0.999))  # the constants as the device holds them
    nw, nm, nv = nn.adam(w[:, :K].astype(np.float64), g.T[:, :K].astype(np.float64), m[:, :K].astype(np.float64),
                         v[:, :K].astype(np.float64), 1e-3, 7, b1, b2)
    gw = _np(Wd)
    assert np.allclose(gw[:, :K], nw, rtol=1e-6, atol=1e-6)
    assert np.allclose(_np(M)[:, :K], nm, rtol=1e-5, atol=1e-7)
    assert np.allclose(_np(V)[:, :K], nv, rtol=1e-5, atol=1e-9)
    assert np.array_equal(_np(WB)[:, :K], nn.bf16(gw[:, :K])) and np.all(_np(WB)[:, K:] == 0)


def _fake_px(rng, w, h):
    """A px image with the planes the features read: sample counts 1..16,
    missed samples, sums, albedo, normal and depth guides."""
    n = w * h
    px = np.zeros(34 * n + 1, dtype=np.uint32)
    f = px.view(np.float32)
    cnt = rng.integers(1, 17, size=n).astype(np.uint32)
    px[31 * n:32 * n] = cnt
    gone = np.minimum(rng.integers(0, 3, size=n), cnt).astype(np.float32)
    f[33 * n:34 * n] = gone
    f[n:4 * n] = (rng.gamma(0.5, size=(n, 3)) * cnt[:, None]).ravel()
    f[7 * n:10 * n] = (rng.uniform(0, 1, size=(n, 3)) * cnt[:, None]).ravel()
    f[10 * n:13 * n] = rng.normal(size=3 * n)
    f[13 * n:14 * n] = rng.uniform(0.5, 5, size=n) * cnt
    return px


@pytest.mark.parametrize("with_half", [False, True])
def test_features(gpu, with_half):
    """Feature planes from px planes, with and without the part-way snapshot
    (the snapshot taken on the device equals the host restatement's)."""
    import torch

    from phiray_b200.denoiser import snapshot_host

    rng = np.random.default_rng(9)
    w, h, Hp, Wp = 37, 21, 32, 48
    px = _fake_px(rng, w, h)
    n = w * h
    half = None
    if with_half:
        early = px.copy()  # a part-way image: fewer samples, part of the sums
        early[31 * n:32 * n] = px[31 * n:32 * n] // 2
        fe = early.view(np.float32)
        fe[n:4 * n] *= 0.4
        fe[33 * n:34 * n] = np.minimum(fe[33 * n:34 * n], early[31 * n:32 * n].astype(np.float32))
        E = _t(early.view(np.int32))
        S = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        N.check(N.lib().phx_nn_snapshot(gpu.handle, E.data_ptr(), w, h, S.data_ptr()))
        _sync(gpu)
        half = snapshot_host(early, w, h)
        assert np.array_equal(_np(S).astype(np.float32), half)
    P = _t(px.view(np.int32))
    H_ = _t(half) if half is not None else None
    feat = torch.empty((Hp, Wp, 16), dtype=torch.bfloat16, device="cuda")
    irr = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
    alb = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().phx_nn_features(gpu.handle, P.data_ptr(), H_.data_ptr() if H_ is not None else None, w, h, Hp, Wp,
                                    feat.data_ptr(), irr.data_ptr(), alb.data_ptr()))
    _sync(gpu)
    f, i, a = nn.features(px, w, h, Hp, Wp, half)
    assert np.all(np.abs(_np(feat) - f) <= 2.0 ** -8 * np.abs(f) + 1e-6)
    assert np.allclose(_np(irr), i, rtol=1e-6, atol=0)
    assert np.allclose(_np(alb), a, rtol=1e-6, atol=0)
    assert (f[..., 15] > 0).any() == with_half


def _net_inputs(rng, B, H, W):
    feat = nn.bf16(np.concatenate([rng.normal(size=(B, H, W, 15)) * 0.5, np.zeros((B, H, W, 1))], axis=-1))
    irr = rng.gamma(1.0, size=(B, H, W, 3))
    alb = rng.uniform(0.05, 1.0, size=(B, H, W, 3))
    ref = irr * alb * rng.uniform(0.5, 1.5, size=(B, H, W, 3))
    return feat, irr, alb, ref


def _random_params(rng):
    pairs = []
    for cin, cout in nn.LAYERS:
        pairs.append((rng.normal(size=(cout, 9 * cin)) * np.sqrt(2.0 / (9 * cin)), rng.normal(size=cout) * 0.05))
    return nn.join_params(pairs).astype(np.float32)


def test_unet_logits_and_gradients_match_fp64_oracle(gpu):
    """The whole network on the device (19 tensor-core convolutions forward,
    their weight and data gradients backward) against the FP64 oracle with
    bf16 rounding at the same tensors: logits and every layer's gradients."""
    import torch

    from phiray_b200.denoiser import Unet

    rng = np.random.default_rng(2024)
    B, H, W = 2, 32, 48
    feat, irr, alb, ref = _net_inputs(rng, B, H, W)
    blob = _random_params(rng)
    net = Unet(gpu, params=blob)
    F, I, A, R = _t(feat, "bf16"), _t(irr.astype(np.float32)), _t(alb.astype(np.float32)), _t(ref.astype(np.float32))
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    net.compute_grads(F, I, A, R, B, H, W, H, W, loss, err_weight=0.1)
    _sync(gpu)
    from phiray_b200 import GpuArray

    logits = GpuArray(gpu, B * H * W * 32 * 4, _wrap=net.logits()).read(np.float32).reshape(B, H, W, 32)
    grads = net.grads()
    params = nn.split_params(blob)
    want_logits, act, P = nn.forward(params, feat, rounded=True)
    scale = np.abs(want_logits).max()
    assert np.abs(logits - want_logits).max() <= 1e-2 * scale
    _, _, want_loss, dl = nn.kpn(logits.astype(np.float64), irr, alb, H, W, ref, 0.1)
    assert abs(_np(loss)[0] - want_loss) <= 1e-4 * want_loss
    want = nn.backward(P, act, dl, rounded=True)
    got = nn.split_params(grads)
    # The same network summed in fp32 instead of fp64 (same bf16 roundings):
    # how far one valid summation order drifts from another once bf16 storage
    # amplifies it (a rounding flip in one activation changes every sum
    # downstream). The device's drift from fp64 must be of that size.
    lg32, act32, P32 = nn.forward(params, feat, rounded=True, acc=np.float32)
    alt = nn.backward(P32, act32, dl, rounded=True, acc=np.float32)

    def rel(a, b):
        return np.linalg.norm(a - b) / np.linalg.norm(b)

    dev = np.array([rel(g[0], w[0]) for g, w in zip(got, want)])
    ref32 = np.array([rel(a[0], w[0]) for a, w in zip(alt, want)])
    print("weight-gradient drift from fp64 per layer: device", np.round(dev, 4), "fp32 oracle", np.round(ref32, 4))
    assert dev[-1] < 2e-3  # the head: its inputs agree, only accumulation order differs
    assert np.all(dev <= 2.0 * ref32 + 0.01), (dev, ref32)
    assert np.all([rel(g[1], w[1]) <= 2.0 * rel(a[1], w[1]) + 0.01 for g, w, a in zip(got, want, alt)])
    net.close()


def test_unet_training_lowers_the_loss(gpu):
    """A few Adam steps on one batch lower its loss (the optimiser and the
    gradients agree in sign and scale)."""
    import torch

    from phiray_b200.denoiser import Unet

    rng = np.random.default_rng(77)
    B, H, W = 2, 32, 32
    feat, irr, alb, ref = _net_inputs(rng, B, H, W)
    net = Unet(gpu, seed=1)
    F, I, A, R = _t(feat, "bf16"), _t(irr.astype(np.float32)), _t(alb.astype(np.float32)), _t(ref.astype(np.float32))
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    hist = []
    for _ in range(30):
        loss.zero_()
        net.train_step(F, I, A, R, B, H, W, H, W, loss, lr=2e-3)
        _sync(gpu)
        hist.append(float(_np(loss)[0]))
    assert hist[-1] < 0.7 * hist[0], hist
    net.close()


def test_learned_denoise_fallback_tiles(gpu):
    """Per-tile fallback: threshold below every estimate keeps the a-trous
    Denoise bit for bit; above every estimate gives the network's own output;
    in between, exactly the tiles over the threshold keep the a-trous result."""
    import torch

    import phiray_b200 as px
    from phiray_b200 import GpuArray, scenes
    from phiray_b200.denoiser import Unet, padded

    s = scenes.c1_plain(ntris=4096, width=72, height=40, spp=4)
    cam = px.camera(s)
    w, h = s.width, s.height
    tr = px.Tracer.of(gpu, s)
    net = Unet(gpu, seed=3)

    def traced():
        tr.trace(cam, w, h, 0, 4)

    traced()
    tr.denoise()
    plain = tr.image()
    traced()
    fb = net.denoise(tr, tile=16, threshold=-1.0, count=True)
    assert fb == 3 * 5
    assert np.array_equal(tr.image(), plain)

    traced()
    noisy = tr.image()
    Hp, Wp = padded(h), padded(w)
    feat = torch.empty((Hp, Wp, 16), dtype=torch.bfloat16, device="cuda")
    irr = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
    alb = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
    out = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
    err = torch.empty((Hp, Wp), dtype=torch.float32, device="cuda")
    pptr, _ = tr.device_image()
    torch.cuda.synchronize()
    px.denoiser.features(gpu, pptr, w, h, Hp, Wp, feat, irr, alb)
    net.forward(feat, irr, alb, 1, Hp, Wp, h, w, out, err)
    _sync(gpu)
    o, e = _np(out), _np(err)
    fb = net.denoise(tr, tile=16, threshold=1e30, count=True)
    assert fb == 0
    rad = tr.lit()
    n = w * h
    cnt = np.maximum(noisy[31 * n:32 * n].astype(np.float64), 1)
    gone = noisy.view(np.float32)[33 * n:34 * n]
    live = (1.0 - gone / cnt > 0.5 / cnt).reshape(h, w)
    assert np.allclose(rad[live], o[:h, :w][live], rtol=1e-6, atol=1e-7)

    tiles = sorted(e[j:min(j + 16, h), i:min(i + 16, w)].mean() for j in range(0, h, 16) for i in range(0, w, 16))
    thr = float(0.5 * (tiles[7] + tiles[8]))
    traced()
    fb = net.denoise(tr, tile=16, threshold=thr, count=True)
    mixed = tr.image()
    _, mask = nn.compose(noisy, w, h, o, e[:h, :w], 16, thr)
    assert fb == int((~mask).sum())
    pm = np.repeat(np.repeat(mask, 16, 0), 16, 1)[:h, :w].reshape(n)
    assert np.array_equal(mixed[:n][~pm], plain[:n][~pm])
    net.close()
    tr.close()


def test_unet_data_parallel_step_equals_one_batch(gpu):
    """Data-parallel training emulated on one GPU: two networks with the same
    weights take the gradients of two half batches, their gradient arenas are
    averaged (what the NCCL all-reduce average does between ranks) and each
    takes its Adam step. Both then hold identical weights, and the averaged
    gradient equals the whole batch's gradient on one network up to fp32
    summation order (the loss is a mean over the batch). The arena holds
    exactly the gradients phx_unet_get reports, in its own layout."""
    import torch

    from phiray_b200.denoiser import Unet

    rng = np.random.default_rng(31)
    B, H, W = 4, 32, 32
    feat, irr, alb, ref = _net_inputs(rng, B, H, W)
    blob = _random_params(rng)
    nets = [Unet(gpu, params=blob) for _ in range(3)]
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")

    def inputs(sl):
        return (_t(feat[sl], "bf16"), _t(irr[sl].astype(np.float32)), _t(alb[sl].astype(np.float32)),
                _t(ref[sl].astype(np.float32)))

    parts = [inputs(slice(0, 2)), inputs(slice(2, 4)), inputs(slice(0, 4))]
    torch.cuda.synchronize()
    for net, (F, I, A, R), b in zip(nets, parts, (2, 2, 4)):
        net.compute_grads(F, I, A, R, b, H, W, H, W, loss, err_weight=0.1)
    _sync(gpu)
    arenas = [n.grad_tensor() for n in nets]
    count = nets[0].grad_arena()[1]
    assert all(a.numel() == count for a in arenas)

    # the arena layout: per layer [Kp][cout] then [cout], each at a multiple of 64 floats
    host = arenas[0].cpu().numpy()
    want = nets[0].grads()
    at, q = 0, 0
    for cin, cout in nn.LAYERS:
        K, Kp = 9 * cin, _round64(9 * cin)
        gw = host[at:at + Kp * cout].reshape(Kp, cout)
        assert np.array_equal(gw[:K].T.reshape(-1), want[q:q + cout * K])
        assert not gw[K:].any()
        q += cout * K
        at += (Kp * cout + 63) // 64 * 64
        assert np.array_equal(host[at:at + cout], want[q:q + cout])
        q += cout
        at += (cout + 63) // 64 * 64
    assert at == count and q == want.size

    avg = (arenas[0] + arenas[1]) / 2
    whole = arenas[2]
    assert float(torch.linalg.norm(avg - whole) / torch.linalg.norm(whole)) < 1e-3
    arenas[0].copy_(avg)
    arenas[1].copy_(avg)
    torch.cuda.synchronize()
    for net in nets[:2]:
        net.adam(1e-3)
    _sync(gpu)
    p0, p1 = nets[0].params(), nets[1].params()
    assert np.array_equal(p0, p1)
    assert not np.array_equal(p0, blob)
    for net in nets:
        net.close()


def test_shipped_weights_beat_the_atrous_denoise_on_held_out_scenes(gpu):
    """The trained weights in the package on procedural scenes the training
    never saw (indices 100000 and 100003): at 4 spp with the part-way
    snapshot, the learned denoiser's relMSE against a 1024-spp reference is
    well below the a-trous Denoise's, which is below the noisy image's."""
    from phiray_b200 import scenes
    from phiray_b200 import train as T
    from phiray_b200.denoiser import Unet

    net = Unet.pretrained(gpu)
    scs = [scenes.procedural(i, width=256, height=256) for i in (100000, 100003)]
    noisy, halves, refs = T.render_group(gpu, scs, [4], 1024)
    ratios = []
    for k in range(len(scs)):
        r = T.evaluate(gpu, net, noisy[k][0], T.radiance(refs[k], 256, 256), 256, 256, halves[k][0])
        print(scs[k].name if hasattr(scs[k], "name") else k, {q: round(v, 5) for q, v in r.items()})
        assert r["learned"] < r["denoise"] < r["noisy"], r
        assert r["fallback_0.1"] < r["denoise"], r
        ratios.append(r["learned"] / r["denoise"])
    assert np.mean(ratios) < 0.75, ratios
    net.close()


def test_firefly_clamp_matches_the_oracle(gpu):
    """phx_nn_firefly against the oracle's float32 restatement, bit for bit:
    planted single-pixel fireflies (corners and edges included) take their
    neighbours' mean, a pixel no brighter than its neighbours is kept, and
    the padding outside the h x w image is copied."""
    import torch

    from phiray_b200.denoiser import firefly

    rng = np.random.default_rng(9)
    B, Hp, Wp, h, w = 2, 32, 48, 30, 45
    irr = rng.gamma(1.0, size=(B, Hp, Wp, 3)).astype(np.float32)
    for b, y, x in [(0, 0, 0), (0, 29, 44), (1, 15, 0), (1, 7, 22), (0, 12, 33)]:
        irr[b, y, x] = 1000.0  # a firefly
    irr[1, 20, 20] = irr[1, 19:22, 19:22].reshape(-1, 3).max(axis=0)  # no brighter than its neighbours
    src = torch.from_numpy(irr).cuda()
    dst = torch.full_like(src, -1.0)
    torch.cuda.synchronize()
    firefly(gpu, src, dst, B, Hp, Wp, h, w)
    _sync(gpu)
    got = dst.cpu().numpy()
    want = nn.firefly(irr, h, w)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    changed = (got != irr).any(axis=-1)
    assert changed[0, 0, 0] and changed[0, 29, 44] and changed[1, 15, 0] and changed[1, 7, 22]
    assert not changed[1, 20, 20]
    assert not changed[:, h:, :].any() and not changed[:, :, w:].any()


def test_learned_denoise_with_the_clamp_filters_clamped_irradiance(gpu):
    """With phx_unet_set_clamp on, the learned denoise equals the network run
    on the features with its kernels applied to the firefly-clamped
    irradiance (no tile falling back)."""
    import torch

    import phiray_b200 as px
    from phiray_b200 import scenes
    from phiray_b200.denoiser import Unet, padded

    s = scenes.c1_plain(ntris=4096, width=72, height=40, spp=4)
    cam = px.camera(s)
    w, h = s.width, s.height
    tr = px.Tracer.of(gpu, s)
    net = Unet(gpu, seed=3)
    net.set_clamp(True)
    tr.trace(cam, w, h, 0, 4)
    noisy = tr.image()
    Hp, Wp = padded(h), padded(w)
    feat = torch.empty((Hp, Wp, 16), dtype=torch.bfloat16, device="cuda")
    irr = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
    alb = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
    clamped = torch.empty_like(irr)
    out = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
    err = torch.empty((Hp, Wp), dtype=torch.float32, device="cuda")
    pptr, _ = tr.device_image()
    torch.cuda.synchronize()
    px.denoiser.features(gpu, pptr, w, h, Hp, Wp, feat, irr, alb)
    px.denoiser.firefly(gpu, irr, clamped, 1, Hp, Wp, h, w)
    net.forward(feat, clamped, alb, 1, Hp, Wp, h, w, out, err)
    _sync(gpu)
    o = _np(out)
    assert net.denoise(tr, tile=16, threshold=1e30, count=True) == 0
    rad = tr.lit()
    n = w * h
    cnt = np.maximum(noisy[31 * n:32 * n].astype(np.float64), 1)
    gone = noisy.view(np.float32)[33 * n:34 * n]
    live = (1.0 - gone / cnt > 0.5 / cnt).reshape(h, w)
    assert np.allclose(rad[live], o[:h, :w][live], rtol=1e-6, atol=1e-7)
    net.close()
    tr.close()


@pytest.mark.parametrize("flips", [2, 4])
def test_learned_denoise_flip_average(gpu, flips):
    """phx_unet_set_flips: the learned result is the mean of the network run
    on the frame and on its mirror images (in x; for 4 also in y and both),
    each mirrored result mirrored back (no tile falling back)."""
    import torch

    import phiray_b200 as px
    from phiray_b200 import scenes
    from phiray_b200.denoiser import Unet, padded

    s = scenes.c1_plain(ntris=4096, width=72, height=40, spp=4)
    cam = px.camera(s)
    w, h = s.width, s.height
    tr = px.Tracer.of(gpu, s)
    net = Unet(gpu, seed=3)
    net.set_flips(flips)
    tr.trace(cam, w, h, 0, 4)
    noisy = tr.image()
    Hp, Wp = padded(h), padded(w)
    feat = torch.empty((Hp, Wp, 16), dtype=torch.bfloat16, device="cuda")
    irr = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
    alb = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
    pptr, _ = tr.device_image()
    torch.cuda.synchronize()
    px.denoiser.features(gpu, pptr, w, h, Hp, Wp, feat, irr, alb)
    _sync(gpu)

    def mirror(t, f):
        m = t.clone()
        part = t[:h, :w]
        if f & 1:
            part = part.flip(1)
        if f & 2:
            part = part.flip(0)
        m[:h, :w] = part
        return m

    acc = None
    for f in range(flips):
        out = torch.empty((Hp, Wp, 3), dtype=torch.float32, device="cuda")
        err = torch.empty((Hp, Wp), dtype=torch.float32, device="cuda")
        net.forward(mirror(feat, f), mirror(irr, f), mirror(alb, f), 1, Hp, Wp, h, w, out, err)
        _sync(gpu)
        back = mirror(out, f)
        acc = back if acc is None else acc + back
    want = (acc * (1.0 / flips)).cpu().numpy()
    assert net.denoise(tr, tile=16, threshold=1e30, count=True) == 0
    rad = tr.lit()
    n = w * h
    cnt = np.maximum(noisy[31 * n:32 * n].astype(np.float64), 1)
    gone = noisy.view(np.float32)[33 * n:34 * n]
    live = (1.0 - gone / cnt > 0.5 / cnt).reshape(h, w)
    assert np.allclose(rad[live], want[:h, :w][live], rtol=1e-6, atol=1e-7)
    net.set_flips(1)
    with pytest.raises(px.PhxError):
        net.set_flips(3)
    net.close()
    tr.close()
