"""The oracle's scenes of instances (forest.rs, instance.rs, bvh.wgsl's
two-level walk, lamp.rs table_of per instance) against the same world laid
out flat: every primary hit agrees, distances to 1e-5, and the image within
the noise of the sample streams; the per-instance shadow flag, reinstancing
and instances of empty meshes behave as the reference's do."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import scenes
from tests import oracle_lib


def cam_of(s):
    c = px.camera(s)
    c["w"], c["h"] = s.width, s.height
    return c


def casting(s):
    ins = s.insts.copy()
    ins["casts_shadow"] = 1
    return scenes.Scene(**{**s.__dict__, "insts": ins})


def relmse(a, b):
    return float(np.mean((a - b) ** 2 / (b * b + 1e-2)))


@pytest.fixture(scope="module")
def scene():
    return casting(scenes.instanced(width=48, height=36))


def test_primary_hits_equal_the_flat_world(orc, scene):
    cam = cam_of(scene)
    ids, ts, inst = oracle_lib.TraceOracle(orc, scene).primary(cam, 0, True)
    ids2, ts2 = oracle_lib.TraceOracle(orc, scenes.flatten(scene)).primary(cam, 0)
    hit, hit2 = ids != 0xFFFFFFFF, ids2 != 0xFFFFFFFF
    assert np.array_equal(hit, hit2) and hit.mean() > 0.5
    assert np.max(np.abs(ts[hit] - ts2[hit]) / ts2[hit]) < 1e-5
    # every placed mesh instance that faces the camera is seen
    assert {0, 1, 2, 3, 4, 5} <= set(inst[hit].tolist())


def test_image_equals_the_flat_world_within_noise(orc, scene):
    cam = cam_of(scene)
    a, _ = oracle_lib.TraceOracle(orc, scene).trace(cam, 0, 128)
    b, _ = oracle_lib.TraceOracle(orc, scenes.flatten(scene)).trace(cam, 0, 128)
    w, h = scene.width, scene.height
    assert relmse(px.tracer.lit_of(a, w, h), px.tracer.lit_of(b, w, h)) < 3e-3


def test_an_instance_that_casts_no_shadow(orc):
    s = scenes.instanced(width=48, height=36)
    assert (s.insts["casts_shadow"] == 0).sum() == 1
    cam = cam_of(s)
    a, _ = oracle_lib.TraceOracle(orc, s).trace(cam, 0, 16)
    b, _ = oracle_lib.TraceOracle(orc, casting(s)).trace(cam, 0, 16)
    la, lb = px.tracer.lit_of(a, 48, 36), px.tracer.lit_of(b, 48, 36)
    assert np.mean(np.abs(la - lb).sum(-1) > 1e-6) > 0.05
    assert la.mean() > lb.mean()  # less shadow, more light


def test_reinstance_equals_a_scene_built_there(orc, scene):
    cam = cam_of(scene)
    moved = scene.insts.copy()
    moved[1] = scenes.instance(scenes.placement((-0.4, 0.5, 0.0), (0.0, 0.0, 1.0), 40.0), 1)[0]
    T = oracle_lib.TraceOracle(orc, scene)
    before, _ = T.trace(cam, 0, 4)
    T.reinstance(moved)
    after, _ = T.trace(cam, 0, 4)
    fresh, _ = oracle_lib.TraceOracle(orc, scenes.Scene(**{**scene.__dict__, "insts": moved})).trace(cam, 0, 4)
    assert np.array_equal(after, fresh)
    assert not np.array_equal(after, before)


def test_emitters_are_counted_per_instance(orc, scene):
    # the glowing panel mesh is placed twice: dropping one placement's
    # emission share changes the light (both are sampled)
    cam = cam_of(scene)
    panels = np.nonzero(scene.insts["mesh"] == 3)[0]
    assert len(panels) == 2
    one = np.delete(scene.insts, panels[1])
    a, _ = oracle_lib.TraceOracle(orc, scene).trace(cam, 0, 32)
    b, _ = oracle_lib.TraceOracle(orc, scenes.Scene(**{**scene.__dict__, "insts": one})).trace(cam, 0, 32)
    assert px.tracer.lit_of(a, 48, 36).mean() > px.tracer.lit_of(b, 48, 36).mean()
