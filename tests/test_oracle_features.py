"""The feature scenes reach the shader paths they are meant to reach: on
the oracle, switching each feature off changes the image. (The GPU tests
then compare the CUDA tracer with the oracle on these scenes bit for bit;
this file makes sure that comparison exercises the lamp, rig, glass,
cut-out and layer code and not just the plain surfaces around it.)"""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import scenes
from tests import oracle_lib


def render(orc, s, cam=None):
    if cam is None:
        cam = px.camera(s)
        cam["w"], cam["h"] = s.width, s.height
    img, rays = oracle_lib.TraceOracle(orc, s).trace(cam, 0, s.spp)
    return px.tracer.lit_of(img, s.width, s.height), rays


def differs(a, b, frac=0.02):
    return float(np.mean(np.abs(a - b).sum(-1) > 1e-6)) >= frac


@pytest.mark.parametrize("kind", ["lamps", "rig", "glass", "layers"])
def test_feature_scene_renders(orc, kind):
    s = scenes.features(kind)
    lit, rays = render(orc, s)
    assert np.all(np.isfinite(lit))
    assert float(np.mean(lit.sum(-1) > 0)) > 0.9
    assert rays > s.width * s.height * s.spp


def test_every_lamp_reaches_the_scene(orc):
    s = scenes.features("lamps")
    base, _ = render(orc, s)
    kinds = s.lights.view(np.uint32)[:, 3].tolist()
    assert sorted(kinds) == [0, 1, 2, 3]
    assert s.lights.view(np.uint32)[3, 16] == 4  # the area lamp is round
    for k in range(len(s.lights)):
        dark = s.lights.copy()
        dark[k, 4:7] = 0.0
        t = scenes.Scene(**{**s.__dict__, "lights": dark})
        lit, _ = render(orc, t)
        assert differs(lit, base), f"lamp {k} (kind {kinds[k]}) changes nothing"


def test_the_spot_cone_and_its_ellipse_matter(orc):
    s = scenes.features("lamps")
    base, _ = render(orc, s)
    for change in ({"cone": 0.5}, {"scale": (0.0, 0.0)}):
        l = s.lights.copy()
        if "cone" in change:
            l[2, 11] = change["cone"]
        else:
            l[2, 18:20] = change["scale"]
        lit, _ = render(orc, scenes.Scene(**{**s.__dict__, "lights": l}))
        assert differs(lit, base, 0.01), change


def test_the_studio_rig_lights_a_lampless_scene(orc):
    s = scenes.features("rig")
    assert len(s.lights) == 0 and s.env == (0.0, 0.0, 0.0)
    lit, _ = render(orc, s)
    off = scenes.Scene(**{**s.__dict__, "lights": np.stack([scenes.light_off()])})
    dark, _ = render(orc, off)
    assert float(lit.mean()) > 10 * float(dark.mean())


def test_glass_and_cut_outs_matter(orc):
    s = scenes.features("glass")
    base, base_rays = render(orc, s)
    m = s.mats.copy()
    glassy = np.nonzero(m[:, 6] > 0)[0]
    assert len(glassy) == 3
    m[:, 6] = 0.0
    opaque, rays = render(orc, scenes.Scene(**{**s.__dict__, "mats": m}))
    assert differs(opaque, base) and rays != base_rays
    m = s.mats.copy()
    cut = np.nonzero(m[:, 3] < 0.5)[0]
    assert len(cut) == 1
    m[cut, 3] = 1.0
    solid, _ = render(orc, scenes.Scene(**{**s.__dict__, "mats": m}))
    assert differs(solid, base, 0.005)


@pytest.mark.parametrize("word", [26, 21, 17], ids=["coat", "sheen", "subsurface"])
def test_material_layers_matter(orc, word):
    s = scenes.features("layers")
    base, _ = render(orc, s)
    m = s.mats.copy()
    assert np.any(m[:, word] > 0)
    m[:, word] = 0.0
    lit, _ = render(orc, scenes.Scene(**{**s.__dict__, "mats": m}))
    assert differs(lit, base)


def test_smooth_normals_matter(orc):
    s = scenes.features("layers")
    base, _ = render(orc, s)
    flat, _ = render(orc, scenes.Scene(**{**s.__dict__, "normals": None}))
    assert differs(flat, base)
