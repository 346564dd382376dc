"""Skin on the GPU == Skin::cpu (tests/gpu.rs:44-73): the reference's rig of
70,001 vertices, a replayed pass after new bone matrices, B-Bone blends."""

import numpy as np
import pytest

import phiray_b200 as px
from tests import gen

pytestmark = pytest.mark.gpu


def close(a, b, tol=1e-4):
    assert a.shape == b.shape
    assert np.all(np.abs(a - b) <= tol)


def test_skin_matches_cpu_and_replays(gpu, orc):
    n = 70_001
    rest, offsets, pairs = gen.rig(n)
    bones = np.stack([gen.translate(1.0, 0.0, 0.0), gen.translate(0.0, 2.0, -4.0)])
    r = px.GpuArray.from_(gpu, rest)
    o = px.GpuArray.from_(gpu, offsets)
    q = px.GpuArray.from_(gpu, pairs)
    b = px.GpuArray.from_(gpu, bones)
    out = px.GpuArray.zeroed(gpu, rest.nbytes)
    ps = px.Pass(gpu)
    ps.add(px.Skin, n, px.Skin.params(min=1e-4), [r, o, q, b, out])
    ps.run()
    got = out.read(np.float32).reshape(n, 4)
    want = orc.skin(rest, offsets, pairs, bones, 1e-4)
    close(got, want)
    assert np.array_equal(got, want)  # same operation order, no contraction
    bones[1] = gen.translate(-3.0, 0.5, 0.0)
    assert not b.write(bones)
    ps.run()
    got = out.read(np.float32).reshape(n, 4)
    want = orc.skin(rest, offsets, pairs, bones, 1e-4)
    close(got, want)
    assert np.array_equal(got, want)
    assert ps.compiled() == 1


def test_skin_bbone_blend_and_rotations(gpu, orc):
    rng = np.random.default_rng(3)
    n, nb = 20_000, 64
    rest = np.ones((n, 4), np.float32)
    rest[:, :3] = rng.standard_normal((n, 3)).astype(np.float32)
    counts = rng.integers(1, 5, n)
    offsets = np.zeros(n + 1, np.uint32)
    offsets[1:] = np.cumsum(counts)
    k = int(offsets[-1])
    pairs = np.zeros(k, dtype=gen.PAIR)
    pairs["bone"] = rng.integers(0, nb, k)
    pairs["next"] = rng.integers(0, nb, k)
    pairs["weight"] = rng.dirichlet(np.ones(4), k)[:, 0].astype(np.float32)
    pairs["blend"] = rng.random(k).astype(np.float32)
    bones = rng.standard_normal((nb, 16)).astype(np.float32)
    import torch

    d = {name: torch.tensor(np.ascontiguousarray(a).view(np.uint8), device="cuda") for name, a in
         dict(rest=rest, offsets=offsets, pairs=pairs, bones=bones).items()}
    out = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    px.skin(gpu, d["rest"], d["offsets"], d["pairs"], d["bones"], nb, out, n, 1e-4)
    gpu.wait()
    want = orc.skin(rest, offsets, pairs, bones, 1e-4)
    assert np.array_equal(out.cpu().numpy(), want)


def test_skin_bad_bone_is_reported(gpu):
    rest = np.ones((4, 4), np.float32)
    offsets = np.array([0, 1, 1, 1, 1], np.uint32)
    pairs = np.zeros(1, dtype=gen.PAIR)
    pairs["bone"] = 9
    pairs["weight"] = 1.0
    bones = gen.translate(0, 0, 0)[None]
    arr = [px.GpuArray.from_(gpu, a) for a in (rest, offsets, pairs, bones)]
    out = px.GpuArray.zeroed(gpu, rest.nbytes)
    px.skin(gpu, arr[0], arr[1], arr[2], arr[3], 1, out, 4, 1e-4)
    with pytest.raises(px.PhxError) as e:
        gpu.wait()
    assert e.value.code == px._native.PHX_ERR_KERNEL
    gpu.wait()  # the status word was cleared


def test_face_boxes(gpu):
    rng = np.random.default_rng(5)
    v = np.ones((300, 4), np.float32)
    v[:, :3] = rng.standard_normal((300, 3))
    f = rng.integers(0, 300, (1000, 4)).astype(np.uint32)
    vv, ff = px.GpuArray.from_(gpu, v), px.GpuArray.from_(gpu, f)
    boxes = px.GpuArray.zeroed(gpu, 1000 * 32)
    px.face_boxes(gpu, vv, ff, 1000, boxes)
    got = boxes.read(np.float32).reshape(-1, 8)
    a, b, c = v[f[:, 0], :3], v[f[:, 1], :3], v[f[:, 2], :3]
    assert np.array_equal(got[:, 0:3], np.minimum(np.minimum(a, b), c))
    assert np.array_equal(got[:, 4:7], np.maximum(np.maximum(a, b), c))
