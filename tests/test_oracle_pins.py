"""The oracle pinned to the reference's own tests of the Rendered path.

Each test restates one of phiray's Rust tests — same scene, same inputs,
same thresholds — and runs it on the oracle (the C++ restatement the CUDA
kernels are checked against bit for bit), so the restatement is held to
what the reference itself asserts, not only to the CUDA code:

  src/trace/tri.rs:188-251   the watertight triangle test: no ray through a
                             quad's shared diagonal, 200,000 xorshift rays
                             at a shared edge, hits equal to Möller-Trumbore's
  tests/emitter.rs:30-57     glowing panels against closed-form irradiance
                             (near, far and middle), MIS counting each once
  tests/trace.rs:51-81       the lit box is red and the sky is sky, in both
                             projections, with the floor grid on
  tests/denoise.rs:79-106    the a-trous filter moves 12 spp towards 1024
                             spp by 25 % and keeps the albedo edge

The scenes are built in `tests/pins.py`, shared with the GPU twins of these
tests (`tests/test_gpu_pins.py`).
"""

import numpy as np
import pytest

from tests import pins

F32 = np.float32


# ---- src/trace/tri.rs:188-251 ----

def test_no_ray_falls_through_a_quads_shared_edge(orc):
    a, b = pins.card()
    holes, both = [], 0
    for x, y in pins.diagonal():
        o, d = pins.preview_ray(x, y)
        hits = sum(orc.tri_hit(*t, o, d) is not None for t in (a, b))
        if hits == 0:
            holes.append((x, y))
        both += hits == 2
    assert not holes, f"the shared diagonal leaks at {holes}"
    assert both > 0, "a ray on the edge is inside both triangles, not just inside one"


def test_a_ray_aimed_at_a_shared_edge_hits_one_side_or_both(orc):
    a, b = pins.card()
    dropped = 0
    for o, d in pins.edge_rays(200_000):
        one = orc.tri_hit(*a, o, d) is not None
        two = orc.tri_hit(*b, o, d) is not None
        assert one or two, f"a hole from {o} along {d}"
        old = pins.moller_trumbore(*a, o, d) is not None or pins.moller_trumbore(*b, o, d) is not None
        dropped += not old
    assert dropped > 0, "Möller-Trumbore let all of these through"


def test_the_hit_is_the_one_moller_trumbore_found(orc):
    a, _ = pins.card()
    agreed = 0
    for x in range(pins.W):
        for y in range(pins.W):
            o, d = pins.preview_ray(x, y)
            n = orc.tri_hit(*a, o, d)
            m = pins.moller_trumbore(*a, o, d)
            if n is None or m is None:
                continue
            agreed += 1
            assert abs(n[0] - m[0]) < 1e-3 * m[0], (x, y, n, m)
            assert abs(n[1] - m[1]) < 1e-3 and abs(n[2] - m[2]) < 1e-3, (x, y, n, m)
            w = F32(1.0) - F32(n[1]) - F32(n[2])
            px_ = w * a[0][0] + F32(n[1]) * a[1][0] + F32(n[2]) * a[2][0]
            assert abs(px_ - (o[0] + F32(n[0]) * d[0])) < 1e-3
    assert agreed > 400, agreed


# ---- tests/emitter.rs:30-57 ----

@pytest.mark.parametrize("case", ["near", "far", "middle"])
def test_emitters_are_counted_once_near_and_far(orc, case):
    scene, cam, want, tol = pins.emitter_case(case)
    first, all_ = pins.wall_view_oracle(orc, scene, cam)
    assert abs(all_ - want) < want * tol, f"{case}: converged {all_} vs expected {want}"
    if case == "near":
        assert abs(first - all_) < all_ * 0.15, f"near: one sample {first} vs converged {all_}"


# ---- tests/trace.rs:51-81 ----

@pytest.mark.parametrize("persp", [False, True])
def test_renders_box_floor_and_sky(orc, persp):
    scene, cam = pins.box_scene(persp)
    img, frames = pins.render_oracle(orc, scene, cam, pins.SAMPLE_COUNT)
    assert frames == pins.SAMPLE_COUNT
    centre, top = pins.box_checks(img, cam)
    assert centre[0] > centre[1] + 30, f"box is red: {centre}"
    assert abs(int(top[0]) - int(top[2])) < 40 and top[2] > 40, f"sky at the top: {top}"


def test_the_floor_grid_is_drawn(orc):
    # The grid overlay is part of that frame: with it off, floor pixels change.
    scene, cam = pins.box_scene(True)
    on, _ = pins.render_oracle(orc, scene, cam, 2)
    off_cam = cam.copy()
    off_cam["grid"] = 0.0
    off, _ = pins.render_oracle(orc, scene, off_cam, 2)
    assert np.mean(on != off) > 0.01


# ---- tests/denoise.rs:79-106 ----

def test_denoising_moves_a_noisy_render_towards_the_converged_one(orc):
    reference = pins.denoise_render_oracle(orc, 1024, False)
    noisy = pins.denoise_render_oracle(orc, 12, False)
    cleaned = pins.denoise_render_oracle(orc, 12, True)
    before = pins.byte_diff(noisy, reference)
    after = pins.byte_diff(cleaned, reference)
    assert after < before * 0.75, f"denoised is {after:.2f} from the reference, noisy was {before:.2f}"


def test_demodulation_keeps_the_albedo_edge(orc):
    cleaned = pins.denoise_render_oracle(orc, 12, True)
    left, right, step = pins.edge_numbers(cleaned)
    assert right - left > 40.0, f"the edge flattened: left {left:.1f}, right {right:.1f}"
    assert step > (right - left) * 0.5, f"the seam ramped over {step:.1f} of {right - left:.1f}"
