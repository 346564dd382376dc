"""Scenes of instances on the device (phx_tracer_create_instanced): the
two-level walk, placed shading, per-instance shadow flags and emitter
entries, the top tree rebuilt on the device by reinstance, and a repose of
the meshes — every image, hit and walk equal to the oracle's bit for bit."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import scenes
from tests import oracle_lib
from tests.test_gpu_trace import cam_of, check_image

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    return scenes.instanced()


@pytest.fixture(scope="module")
def want(orc, scene):
    cam = cam_of(scene, scene.width, scene.height)
    return (cam,) + oracle_lib.TraceOracle(orc, scene).trace(cam, 0, scene.spp)


@pytest.mark.parametrize("kernel", list(range(17)))
def test_instanced_image_matches_oracle(gpu, scene, want, kernel):
    cam, img, rays = want
    tr = px.Tracer.of(gpu, scene)
    tr.set_kernel(kernel)
    tr.trace(cam, scene.width, scene.height, 0, scene.spp)
    check_image(tr.image(), img, scene.width * scene.height)
    assert tr.time()[1] == rays
    tr.close()


def test_instanced_primary_hits(gpu, orc, scene):
    import torch

    w, h = 128, 96
    cam = cam_of(scene, w, h)
    want_ids, want_t = oracle_lib.TraceOracle(orc, scene).primary(cam, 2)
    tr = px.Tracer.of(gpu, scene)
    ids = torch.empty(w * h, dtype=torch.int32, device="cuda")
    ts = torch.empty(w * h, dtype=torch.float32, device="cuda")
    tr.primary(cam, w, h, 2, ids, ts)
    gpu.wait()
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), want_ids)
    assert np.array_equal(ts.cpu().numpy(), want_t)
    tr.close()


@pytest.mark.parametrize("walk", [0, 1, 2], ids=["thread_per_ray", "persistent_fetch", "sorted"])
def test_instanced_ray_walks(gpu, orc, scene, walk):
    import torch

    rng = np.random.default_rng(21)
    n = 20000
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-1.5, 1.5, (n, 3)) + np.array([0.0, 0.8, 0.0])
    d = rng.standard_normal((n, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3] = 3.0e38
    rays[::4, 3] = 0.5
    tr = px.Tracer.of(gpu, scene)
    tr.set_walk(walk)
    dr = torch.tensor(rays, device="cuda")
    hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    T = oracle_lib.TraceOracle(orc, scene)
    for any_hit in (False, True):
        tr.trace_rays(dr, n, hits, any_hit)
        gpu.wait()
        got = hits.cpu().numpy()
        want = T.trace_rays(rays, any_hit)
        assert np.array_equal(got.view(np.uint32)[:, 1], want.view(np.uint32)[:, 1])
        if not any_hit:
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    tr.close()


def test_reinstance_rebuilds_the_top_tree_on_the_device(gpu, orc, scene):
    cam = cam_of(scene, scene.width, scene.height)
    moved = scene.insts.copy()
    moved[1] = scenes.instance(scenes.placement((-0.4, 0.5, 0.0), (0.0, 0.0, 1.0), 40.0), 1)[0]
    moved[6] = scenes.instance(scenes.placement((0.0, 1.6, -0.3), (1.0, 0.0, 0.0), 150.0), 3)[0]
    moved[3]["casts_shadow"] = 0
    tr = px.Tracer.of(gpu, scene)
    tr.trace(cam, scene.width, scene.height, 0, scene.spp)
    tr.reinstance(moved)
    tr.trace(cam, scene.width, scene.height, 0, scene.spp)
    T = oracle_lib.TraceOracle(orc, scene)
    T.reinstance(moved)
    want, _ = T.trace(cam, 0, scene.spp)
    check_image(tr.image(), want, scene.width * scene.height)
    bad = moved.copy()
    bad[0]["mesh"] = 1
    with pytest.raises(px.PhxError):
        tr.reinstance(bad)
    with pytest.raises(px.PhxError):
        tr.reinstance(moved[:-1])
    tr.close()


def test_instanced_repose_rebuild(gpu, orc, scene):
    import torch

    cam = cam_of(scene, scene.width, scene.height)
    v = scene.verts.copy()
    lo, hi = scene.meshes[1]
    used = np.unique(scene.faces[lo:hi, :3])
    v[used, 1] *= np.float32(1.3)  # the sphere mesh stretched: every instance of it moves
    tr = px.Tracer.of(gpu, scene)
    tr.repose_device(torch.tensor(v, device="cuda"), rebuild=True)
    tr.trace(cam, scene.width, scene.height, 0, scene.spp)
    want, _ = oracle_lib.TraceOracle(orc, scenes.Scene(**{**scene.__dict__, "verts": v})).trace(cam, 0, scene.spp)
    check_image(tr.image(), want, scene.width * scene.height)
    tr.close()


def test_instanced_and_flat_in_one_batch(gpu, orc, scene, want):
    from phiray_b200.batch import Batch

    flat = scenes.features("lamps")
    fcam = cam_of(flat, flat.width, flat.height)
    fwant, _ = oracle_lib.TraceOracle(orc, flat).trace(fcam, 0, flat.spp)
    a, b = px.Tracer.of(gpu, scene), px.Tracer.of(gpu, flat)
    bt = Batch(gpu)
    bt.add(a, want[0], scene.width, scene.height, 0, scene.spp)
    bt.add(b, fcam, flat.width, flat.height, 0, flat.spp)
    bt.trace()
    gpu.wait()
    check_image(a.image(), want[1], scene.width * scene.height)
    check_image(b.image(), fwant, flat.width * flat.height)
    for t in (a, b, bt):
        t.close()
