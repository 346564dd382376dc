"""The CUDA tracer == the oracle on the shader paths the benchmark scenes
leave unused: sun, point and elliptical spot lamps and a round area lamp
(light.wgsl:14-30, 118-167), the studio rig (count 0, black world,
light.wgsl:87-90), glass, partial transmission and alpha cut-outs
(shade.wgsl:345-369, bvh.wgsl:158-162), coat, sheen and subsurface layers
(brdf.wgsl:109-208) and smooth vertex normals. Every px plane bit for bit,
on every render kernel form, and the rays traced equal in number."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import scenes
from tests import oracle_lib
from tests.test_gpu_trace import cam_of, check_image

pytestmark = pytest.mark.gpu

KINDS = ["lamps", "rig", "glass", "layers"]
KERNELS = list(range(20))


@pytest.fixture(scope="module")
def want(orc):
    out = {}
    for k in KINDS:
        s = scenes.features(k)
        cam = cam_of(s, s.width, s.height)
        out[k] = (s, cam) + oracle_lib.TraceOracle(orc, s).trace(cam, 0, s.spp)
    return out


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("kind", KINDS)
def test_feature_scene_matches_oracle(gpu, want, kind, kernel):
    s, cam, img, rays = want[kind]
    tr = px.Tracer.of(gpu, s)
    tr.set_kernel(kernel)
    tr.trace(cam, s.width, s.height, 0, s.spp)
    check_image(tr.image(), img, s.width * s.height)
    assert tr.time()[1] == rays
    tr.close()


@pytest.mark.parametrize("kind", KINDS)
def test_feature_scene_sample_by_sample(gpu, want, kind):
    # Tracer::sample one frame at a time, in slices, == the oracle's frames.
    s, cam, img, _ = want[kind]
    tr = px.Tracer.of(gpu, s)
    tr.set_samples(s.spp)
    while not tr.sample(cam, s.width, s.height, slices=3)[1]:
        pass
    check_image(tr.image(), img, s.width * s.height)
    tr.close()


def test_feature_scenes_in_one_batch(gpu, want):
    # The batched persistent launch over all four scenes == each one alone.
    from phiray_b200.batch import Batch

    trs = [px.Tracer.of(gpu, want[k][0]) for k in KINDS]
    b = Batch(gpu)
    for k, tr in zip(KINDS, trs):
        s, cam = want[k][0], want[k][1]
        b.add(tr, cam, s.width, s.height, 0, s.spp)
    b.trace()
    gpu.wait()
    for k, tr in zip(KINDS, trs):
        s = want[k][0]
        check_image(tr.image(), want[k][2], s.width * s.height)
        tr.close()
    b.close()
