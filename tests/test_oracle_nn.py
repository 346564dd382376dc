"""The FP64 network oracle pinned on the CPU: its backward pass equals the
central finite difference of its own forward pass and loss (no rounding),
and its layers satisfy the identities the device kernels rely on."""

import numpy as np

from tests import oracle_lib

nn = oracle_lib.nn()


def _loss(params, feat, irr, alb, ref, H, W):
    logits, _, _ = nn.forward(params, feat, rounded=False)
    return nn.kpn(logits, irr, alb, H, W, ref, 0.0)[2]


def test_backward_equals_finite_differences():
    rng = np.random.default_rng(0)
    B, H, W = 1, 16, 16
    feat = rng.normal(size=(B, H, W, 16)) * 0.5
    irr = rng.gamma(1.0, size=(B, H, W, 3))
    alb = rng.uniform(0.05, 1.0, size=(B, H, W, 3))
    ref = irr * alb * rng.uniform(0.5, 1.5, size=(B, H, W, 3))
    params = []
    for cin, cout in nn.LAYERS:
        params.append((rng.normal(size=(cout, 9 * cin)) * np.sqrt(2.0 / (9 * cin)), rng.normal(size=cout) * 0.05))
    logits, act, P = nn.forward(params, feat, rounded=False)
    _, _, _, dl = nn.kpn(logits, irr, alb, H, W, ref, 0.0)
    grads = nn.backward(P, act, dl, rounded=False)
    eps = 1e-6
    for li in (0, 5, 9, 10, 16, 18):
        W0, b0 = params[li]
        for _ in range(3):
            idx = tuple(rng.integers(0, s) for s in W0.shape)
            Wp, Wm = W0.copy(), W0.copy()
            Wp[idx] += eps
            Wm[idx] -= eps
            pp = list(params)
            pp[li] = (Wp, b0)
            lp = _loss(pp, feat, irr, alb, ref, H, W)
            pp[li] = (Wm, b0)
            lm = _loss(pp, feat, irr, alb, ref, H, W)
            fd = (lp - lm) / (2 * eps)
            g = grads[li][0][idx]
            assert abs(fd - g) <= 1e-4 * max(abs(fd), abs(g)) + 1e-9, (li, idx, fd, g)
        j = int(rng.integers(0, b0.size))
        bp, bm = b0.copy(), b0.copy()
        bp[j] += eps
        bm[j] -= eps
        pp = list(params)
        pp[li] = (W0, bp)
        lp = _loss(pp, feat, irr, alb, ref, H, W)
        pp[li] = (W0, bm)
        lm = _loss(pp, feat, irr, alb, ref, H, W)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - grads[li][1][j]) <= 1e-4 * max(abs(fd), 1e-12) + 1e-9, (li, j)


def test_kpn_gradient_equals_finite_differences():
    rng = np.random.default_rng(1)
    B, Hp, Wp, h, w = 1, 8, 8, 7, 6
    logits = rng.normal(size=(B, Hp, Wp, 32))
    irr = rng.gamma(1.0, size=(B, Hp, Wp, 3))
    alb = rng.uniform(0.05, 1, size=(B, Hp, Wp, 3))
    ref = rng.gamma(1.0, size=(B, Hp, Wp, 3))
    ew = 0.3
    _, _, _, dl = nn.kpn(logits, irr, alb, h, w, ref, ew)

    def total(lg):
        _, _, loss, _ = nn.kpn(lg, irr, alb, h, w, ref, ew)
        # the error head's term, with its target held fixed at the base logits
        o, _ = nn.kpn(logits, irr, alb, h, w)
        r = ref[:, :h, :w]
        rel = (((o[:, :h, :w] - r) ** 2) / (r * r + 0.01)).sum(-1) / 3.0
        e = lg[:, :h, :w, 25]
        return loss + ew * ((e - np.log(rel + 1e-3)) ** 2).sum() / (B * h * w)

    eps = 1e-6
    for t in (0, 7, 12, 24, 25):
        y, x = 3, 2
        lp, lm = logits.copy(), logits.copy()
        lp[0, y, x, t] += eps
        lm[0, y, x, t] -= eps
        fd = (total(lp) - total(lm)) / (2 * eps)
        assert abs(fd - dl[0, y, x, t]) <= 1e-5 * abs(fd) + 1e-10, (t, fd, dl[0, y, x, t])


def test_flip_is_the_adjoint():
    """<conv(x, W), dy> == <x, conv(dy, flip(W))>: the data gradient."""
    rng = np.random.default_rng(2)
    cin, cout = 8, 16
    x = rng.normal(size=(1, 6, 7, cin))
    dy = rng.normal(size=(1, 6, 7, cout))
    Wt = rng.normal(size=(cout, 9 * cin))
    lhs = (nn.conv(x, Wt, None, False) * dy).sum()
    rhs = (x * nn.conv_dgrad(dy, Wt, cin)).sum()
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 1e-40, 3.0e38])
    r = nn.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6  # ties to even
    assert r[3] == -2.5 and r[4] == 0.0
    assert np.array_equal(nn.from_bf16_bits(nn.bf16_bits(v)), r)
