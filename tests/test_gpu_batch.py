"""Batched serving: many tracers' frames in one persistent launch give each
tracer's own image bit for bit, under every launch form the autotuner picks
from; the captured serving frame (gated rebuild/refit, trace, learned
denoise) replays the same images as the same calls made one by one."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import scenes
from phiray_b200.batch import PER_SCENE, PERSISTENT, PERSISTENT_DENSE, STACK_LOCAL, STACK_SHARED, Batch

pytestmark = pytest.mark.gpu


def _jobs():
    out = []
    for s, first in ((scenes.c1_plain(ntris=4096, width=64, height=64, spp=4), 0),
                     (scenes.c2_mesh(levels=4, width=64, height=48, spp=2), 3),
                     (scenes.procedural(7, width=48, height=40, spp=3), 0),
                     (scenes.procedural(8, width=80, height=16, spp=1), 5)):
        cam = px.camera(s)
        cam["w"], cam["h"] = s.width, s.height
        out.append((s, cam, first))
    return out


def _single(gpu, jobs):
    imgs = []
    for s, cam, first in jobs:
        tr = px.Tracer.of(gpu, s)
        tr.set_kernel(px.Tracer.MEGAKERNEL)
        tr.trace(cam, s.width, s.height, first, s.spp)
        imgs.append(tr.image())
        tr.close()
    return imgs


@pytest.mark.parametrize("kind,threads,stack", [(PERSISTENT, 64, STACK_LOCAL), (PERSISTENT, 128, STACK_SHARED),
                                                (PERSISTENT, 256, STACK_LOCAL), (PERSISTENT, 256, STACK_SHARED),
                                                (PER_SCENE, 128, STACK_LOCAL), (PERSISTENT_DENSE, 128, STACK_LOCAL),
                                                (PERSISTENT_DENSE, 256, STACK_SHARED)])
def test_batch_equals_single_traces(gpu, kind, threads, stack):
    jobs = _jobs()
    want = _single(gpu, jobs)
    b = Batch(gpu)
    trs = []
    for s, cam, first in jobs:
        tr = px.Tracer.of(gpu, s)
        trs.append(tr)
        b.add(tr, cam, s.width, s.height, first, s.spp)
    b.set_config(kind, threads, stack)
    b.trace()
    for tr, w in zip(trs, want):
        assert np.array_equal(tr.image(), w)
    b.close()
    for tr in trs:
        tr.close()


def test_batch_autotune_and_captured_frame(gpu):
    from phiray_b200.denoiser import Unet

    # A serving frame starts every image over (frame 0): a job that continued
    # an accumulation would add to whatever the last replay left.
    jobs = [(s, cam, 0) for s, cam, _ in _jobs()]
    b = Batch(gpu)
    trs = []
    for s, cam, first in jobs:
        tr = px.Tracer.of(gpu, s)
        trs.append(tr)
        b.add(tr, cam, s.width, s.height, first, s.spp)
    cfg, ms = b.autotune()
    assert len(ms) == 11 and all(v > 0 for v in ms.values())
    net = Unet(gpu, seed=5)
    b.capture(net, threshold=0.1)
    modes = [1, 0, 0, 1]
    b.replay(modes)
    lat, rays = b.results()
    got = [tr.image() for tr in trs]
    assert np.all(lat > 0) and np.all(rays > 0)

    # The same frame, call by call on fresh tracers.
    for (s, cam, first), mode, g, r in zip(jobs, modes, got, rays):
        tr = px.Tracer.of(gpu, s)
        tr.repose_device(px.GpuArray.from_(gpu, s.verts), rebuild=bool(mode))
        counts = tr.trace_stats(cam, s.width, s.height, first, s.spp)
        net.denoise(tr, threshold=0.1)
        assert np.array_equal(tr.image(), g)
        assert counts[0] == r
        tr.close()
    b.replay([0, 0, 1, 1])
    b.results()
    b.close()
    net.close()
    for tr in trs:
        tr.close()
