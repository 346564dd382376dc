"""The reference's own Rendered-path tests run on the CUDA tracer: the same
scenes and thresholds as tests/test_oracle_pins.py, and every image or hit
equal to the oracle's bit for bit (see tests/pins.py for the scenes)."""

import numpy as np
import pytest

import phiray_b200 as px
from tests import oracle_lib, pins

pytestmark = pytest.mark.gpu


def _walk(gpu, tri, rays):
    """Closest hits of `rays` (o, d pairs) against one triangle, on the device."""
    import torch

    n = len(rays)
    buf = np.zeros((n, 8), np.float32)
    for k, (o, d) in enumerate(rays):
        buf[k, 0:3], buf[k, 3], buf[k, 4:7] = o, 3.0e38, d
    tr = px.Tracer.of(gpu, pins.single_triangle_scene(tri))
    dr = torch.tensor(buf, device="cuda")
    hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    tr.trace_rays(dr, n, hits)
    gpu.wait()
    tr.close()
    return buf, hits.cpu().numpy()


def test_shared_edge_rays_on_the_device(gpu, orc):
    """tri.rs:201-227 on the device walk: 200,000 xorshift rays at the
    card's shared edge each hit one triangle or both; every hit equals the
    oracle's, and the Möller-Trumbore witness drops some of them."""
    a, b = pins.card()
    rays = pins.edge_rays(200_000)
    buf, ha = _walk(gpu, a, rays)
    _, hb = _walk(gpu, b, rays)
    one = ha.view(np.uint32)[:, 1] != 0xFFFFFFFF
    two = hb.view(np.uint32)[:, 1] != 0xFFFFFFFF
    assert np.all(one | two), np.nonzero(~(one | two))[0][:10]
    for tri, got in ((a, ha), (b, hb)):
        want = oracle_lib.TraceOracle(orc, pins.single_triangle_scene(tri)).trace_rays(buf)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    dropped = sum(pins.moller_trumbore(*a, o, d) is None and pins.moller_trumbore(*b, o, d) is None
                  for o, d in rays[:20000])
    assert dropped > 0


def test_shared_diagonal_on_the_device(gpu):
    """tri.rs:188-195: every preview ray on the diagonal hits the card, some
    both triangles."""
    a, b = pins.card()
    rays = [pins.preview_ray(x, y) for x, y in pins.diagonal()]
    _, ha = _walk(gpu, a, rays)
    _, hb = _walk(gpu, b, rays)
    one = ha.view(np.uint32)[:, 1] != 0xFFFFFFFF
    two = hb.view(np.uint32)[:, 1] != 0xFFFFFFFF
    assert np.all(one | two) and np.any(one & two)


def _trace(gpu, scene, cam, first, spp, tr=None):
    w, h = int(cam["w"][0]), int(cam["h"][0])
    tr = tr or px.Tracer.of(gpu, scene)
    tr.trace(cam, w, h, first, spp)
    return tr


@pytest.mark.parametrize("case", ["near", "far", "middle"])
def test_emitters_closed_form_on_the_device(gpu, orc, case):
    scene, cam, want, tol = pins.emitter_case(case)
    tr = _trace(gpu, scene, cam, 0, 1)
    first = pins.centre_red(tr.radiance())
    _trace(gpu, scene, cam, 1, pins.SAMPLE_COUNT - 1, tr)
    all_ = pins.centre_red(tr.radiance())
    T = oracle_lib.TraceOracle(orc, scene)
    img, _ = T.trace(cam, 0, 1)
    T.trace(cam, 1, pins.SAMPLE_COUNT - 1, px=img)
    assert np.array_equal(tr.image(), img)
    assert abs(all_ - want) < want * tol, (case, all_, want)
    if case == "near":
        assert abs(first - all_) < all_ * 0.15
    tr.close()


@pytest.mark.parametrize("persp", [False, True])
@pytest.mark.parametrize("kernel", [0, 1, 15, 16], ids=["megakernel", "state_machine", "mk16_sync", "wavefront"])
def test_box_floor_sky_and_grid_on_the_device(gpu, orc, persp, kernel):
    scene, cam = pins.box_scene(persp)
    want, _ = pins.render_oracle(orc, scene, cam, pins.SAMPLE_COUNT)
    tr = px.Tracer.of(gpu, scene)
    tr.set_kernel(kernel)
    tr.set_samples(pins.SAMPLE_COUNT)
    frames = 0
    done = False
    while not done:
        _, done = tr.sample(cam, 160, 120)
        frames += 1
    assert frames == pins.SAMPLE_COUNT
    rgba = tr.pixels().view(np.uint8).reshape(120, 160, 4)
    assert np.array_equal(rgba, want)
    centre, top = pins.box_checks(rgba, cam)
    assert centre[0] > centre[1] + 30 and abs(top[0] - top[2]) < 40 and top[2] > 40
    tr.close()


def test_denoise_behaviour_on_the_device(gpu, orc):
    scene, cam = pins.denoise_scene()
    side = pins.SIDE

    def render(samples, denoise):
        tr = _trace(gpu, scene, cam, 0, samples)
        if denoise:
            tr.denoise()
        out = tr.pixels().view(np.uint8).copy()
        tr.close()
        return out

    reference, noisy, cleaned = render(1024, False), render(12, False), render(12, True)
    assert np.array_equal(cleaned, pins.denoise_render_oracle(orc, 12, True))
    assert pins.byte_diff(cleaned, reference) < pins.byte_diff(noisy, reference) * 0.75
    left, right, step = pins.edge_numbers(cleaned)
    assert right - left > 40.0 and step > (right - left) * 0.5
    assert len(cleaned) == side * side * 4
