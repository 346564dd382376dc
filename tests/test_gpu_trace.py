"""The CUDA tracer == the oracle's restatement of shade.wgsl and what it
calls, on the same seeded scenes and per-pixel sample streams: primary hit
ids exact, images within relMSE 1e-4 (and, with the shared deterministic
transcendentals, expected bit-identical), ray-buffer walks exact."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import scenes
from tests import oracle_lib

pytestmark = pytest.mark.gpu

RELMSE_TOL = 1e-4  # north-star image gate, on linear radiance


def relmse(x, r):
    return float(np.mean((x - r) ** 2 / (r * r + 1e-2)))


def radiance(img, n):
    f = img.view(np.float32)
    k = img[31 * n: 32 * n].astype(np.float32)
    gone = f[33 * n: 34 * n]
    return f[n: 4 * n].reshape(n, 3) / np.maximum(k - gone, 1.0)[:, None]


def cam_of(s, w, h):
    c = px.camera(s)
    c["w"], c["h"] = w, h
    c["aspect"] = w / h
    return c


def check_image(got, want, n, exact=True):
    rm = relmse(radiance(got, n), radiance(want, n))
    assert rm <= RELMSE_TOL, f"relMSE {rm}"
    if exact:
        planes = {"packed": (0, n), "linear": (n, 4 * n), "shown": (4 * n, 7 * n), "guides": (7 * n, 14 * n),
                  "film": (20 * n, 26 * n), "counts": (31 * n, 32 * n), "missed": (33 * n, 34 * n)}
        bad = {k: int(np.sum(got[a:b] != want[a:b])) for k, (a, b) in planes.items()}
        assert all(v == 0 for v in bad.values()), bad
    return rm


SCENES = {
    "c1_small": lambda: scenes.c1_plain(ntris=4096, width=64, height=64, spp=4),
    "c2_small": lambda: scenes.c2_mesh(levels=4, width=64, height=48, spp=4),
}


@pytest.mark.parametrize("kernel", list(range(20)),
                         ids=["megakernel", "state_machine", "sm6", "sm8", "mk3", "mk2", "mk_sync", "mk2_sync", "mk5",
                              "mk6", "mk6_sync", "mk8", "mk8_sync", "mk10_sync", "mk12_sync", "mk16_sync", "wavefront",
                              "mk_reg8", "mk8_sync_reg1", "mk16_sync_reg1"])
@pytest.mark.parametrize("name", list(SCENES))
def test_image_matches_oracle(gpu, orc, name, kernel):
    s = SCENES[name]()
    cam = cam_of(s, s.width, s.height)
    want, orays = oracle_lib.TraceOracle(orc, s).trace(cam, 0, s.spp)
    tr = px.Tracer.of(gpu, s)
    tr.set_kernel(kernel)
    tr.trace(cam, s.width, s.height, 0, s.spp)
    got = tr.image()
    check_image(got, want, s.width * s.height)
    ms, grays = tr.time()
    assert grays == orays, (grays, orays)


def test_samples_one_at_a_time_equal_one_launch(gpu):
    # Tracer::sample's per-frame accumulation == the in-kernel sample loop.
    s = SCENES["c1_small"]()
    cam = cam_of(s, s.width, s.height)
    a = px.Tracer.of(gpu, s)
    a.set_samples(4)
    frames = []
    while True:
        f, done = a.sample(cam, s.width, s.height)
        frames.append(f)
        if done:  # (frame, frame + 1 >= samples), sample.rs:223
            break
    assert frames == [0, 1, 2, 3]
    assert a.sample(cam, s.width, s.height) == (3, True)  # no more work
    b = px.Tracer.of(gpu, s)
    b.trace(cam, s.width, s.height, 0, 4)
    assert np.array_equal(a.image(), b.image())


def test_sliced_sample_equals_one_sample(gpu):
    # tests/slice.rs: a sample in slices is the same sample.
    s = SCENES["c2_small"]()
    cam = cam_of(s, s.width, s.height)
    a = px.Tracer.of(gpu, s)
    a.sample(cam, s.width, s.height, slices=1)
    b = px.Tracer.of(gpu, s)
    b.sample(cam, s.width, s.height, slices=7)
    assert np.array_equal(a.image(), b.image())


def test_cancel_between_slices(gpu):
    import ctypes as C

    s = SCENES["c2_small"]()
    cam = cam_of(s, s.width, s.height)
    t = px.Tracer.of(gpu, s)
    flag = C.c_int32(1)
    with pytest.raises(px.PhxError) as e:
        t.sample(cam, s.width, s.height, slices=4, cancel=C.addressof(flag))
    assert e.value.code == px._native.PHX_ERR_CANCELLED
    f, done = t.sample(cam, s.width, s.height)
    assert f == 0  # the abandoned sample starts over


@pytest.mark.parametrize("name", list(SCENES))
def test_primary_hit_ids(gpu, orc, name):
    import torch

    s = SCENES[name]()
    w, h = 128, 96
    cam = cam_of(s, w, h)
    want_ids, want_t = oracle_lib.TraceOracle(orc, s).primary(cam, 3)
    tr = px.Tracer.of(gpu, s)
    ids = torch.empty(w * h, dtype=torch.int32, device="cuda")
    ts = torch.empty(w * h, dtype=torch.float32, device="cuda")
    tr.primary(cam, w, h, 3, ids, ts)
    gpu.wait()
    got = ids.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, want_ids)
    assert np.array_equal(ts.cpu().numpy(), want_t)


def _chain_scene():
    """40 parallel triangles at x = 2^-k, overlapping in y and z: a tree 13
    levels deep whose boxes a ray along x nearly all enters, so it pushes at
    nearly every level (more entries than the register stack holds: its
    spill and refill)."""
    from tests import pins

    k = np.arange(40)
    x = (2.0 ** -k.astype(np.float64)).astype(np.float32)
    v = np.ones((120, 4), np.float32)
    v[0::3, :3] = np.stack([x, -np.ones(40), -np.ones(40)], 1)
    v[1::3, :3] = np.stack([x, np.ones(40), -np.ones(40)], 1)
    v[2::3, :3] = np.stack([x, np.zeros(40), np.ones(40)], 1)
    f = np.zeros((40, 4), np.uint32)
    f[:, 0], f[:, 1], f[:, 2] = 3 * k, 3 * k + 1, 3 * k + 2
    return scenes.Scene("chain", v, f, np.stack([scenes.lambert((0.5, 0.5, 0.5))]),
                        np.stack([scenes.light_off()]), None, pins.W, pins.W, 1, 1)


@pytest.mark.parametrize("place", [0, 1, 2], ids=["local", "shared", "register"])
@pytest.mark.parametrize("name", ["c2_small", "chain"])
def test_ray_walk_stack_placements(gpu, orc, name, place):
    """Thread-per-ray walks with the stack in local memory, shared memory or
    registers over a spill array: the oracle's hits, word for word."""
    import torch

    s = _chain_scene() if name == "chain" else SCENES[name]()
    rng = np.random.default_rng(21)
    n = 8000
    rays = np.zeros((n, 8), np.float32)
    if name == "chain":
        rays[:, 0] = np.where(np.arange(n) % 2 == 0, -1.0, 2.0)
        rays[:, 1:3] = rng.uniform(-0.3, 0.3, (n, 2))
        d = np.zeros((n, 3), np.float32)
        d[:, 0] = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
        d[:, 1:3] = rng.uniform(-0.05, 0.05, (n, 2))
    else:
        rays[:, 0:3] = rng.uniform(-1.0, 1.0, (n, 3))
        d = rng.standard_normal((n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3], rays[:, 4:7] = 3.0e38, d
    tr = px.Tracer.of(gpu, s)
    tr.set_stack(place)
    dr = torch.tensor(rays, device="cuda")
    hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    T = oracle_lib.TraceOracle(orc, s)
    for any_hit in (False, True):
        tr.trace_rays(dr, n, hits, any_hit)
        gpu.wait()
        got, want = hits.cpu().numpy(), T.trace_rays(rays, any_hit)
        assert np.array_equal(got.view(np.uint32)[:, 1], want.view(np.uint32)[:, 1])
        if not any_hit:
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    tr.close()


@pytest.mark.parametrize("walk", [0, 1, 2], ids=["thread_per_ray", "persistent_fetch", "sorted"])
def test_ray_buffer_walks(gpu, orc, walk):
    import torch

    s = SCENES["c2_small"]()
    rng = np.random.default_rng(9)
    n = 20000
    o = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    d = rng.standard_normal((n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 3], rays[:, 4:7] = o, 3.0e38, d
    rays[::5, 3] = 0.3  # some bounded rays
    tr = px.Tracer.of(gpu, s)
    tr.set_walk(walk)
    dr = torch.tensor(rays, device="cuda")
    hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    T = oracle_lib.TraceOracle(orc, s)
    for any_hit in (False, True):
        tr.trace_rays(dr, n, hits, any_hit)
        gpu.wait()
        got = hits.cpu().numpy()
        want = T.trace_rays(rays, any_hit)
        assert np.array_equal(got.view(np.uint32)[:, 1], want.view(np.uint32)[:, 1])
        hit = want.view(np.uint32)[:, 1] != 0xFFFFFFFF
        if not any_hit:
            assert np.array_equal(got[hit], want[hit])


def _same_closest_hits(got, want):
    """The closest t of every ray equal bit for bit; the face equal wherever
    no other face sits at that t (a tie is the only freedom the wide walk
    has), so at most a few in 10,000 rays may name another face."""
    gt, wt = got[:, 0], want[:, 0]
    assert np.array_equal(gt.view(np.uint32), wt.view(np.uint32))
    diff = got.view(np.uint32)[:, 1] != want.view(np.uint32)[:, 1]
    assert diff.sum() <= max(2, len(got) // 10000), diff.sum()


@pytest.mark.parametrize("mode", [3, 4], ids=["persistent", "thread_per_ray"])
@pytest.mark.parametrize("tree", [0, 1], ids=["lbvh", "sah"])
def test_wide_walk(gpu, orc, tree, mode):
    """PHX_WALK_WIDE over the 4-wide tree collapsed from either binary tree:
    closest hits == the oracle's binary walk (ties aside), any-hit rays hit
    or miss as the oracle's do; after a repose the wide tree follows the
    refitted binary one."""
    import torch

    s = SCENES["c2_small"]()
    rng = np.random.default_rng(9)
    n = 20000
    o = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    d = rng.standard_normal((n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 3], rays[:, 4:7] = o, 3.0e38, d
    rays[::5, 3] = 0.3
    tr = px.Tracer.of(gpu, s)
    tr.set_tree(tree)
    tr.set_walk(mode)
    dr = torch.tensor(rays, device="cuda")
    hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    T = oracle_lib.TraceOracle(orc, s, sah=bool(tree))
    for any_hit in (False, True):
        tr.trace_rays(dr, n, hits, any_hit)
        gpu.wait()
        got, want = hits.cpu().numpy(), T.trace_rays(rays, any_hit)
        if any_hit:
            assert np.array_equal(got.view(np.uint32)[:, 1] != 0xFFFFFFFF, want.view(np.uint32)[:, 1] != 0xFFFFFFFF)
        else:
            _same_closest_hits(got, want)
    c = tr.trace_rays_stats(dr, n, hits)
    tr.set_walk(px.Tracer.WALK_FETCH)
    c2 = tr.trace_rays_stats(dr, n, hits)
    assert c[0] == c2[0] == n and c[1] < c2[1]  # fewer (wider) steps
    moved = s.verts.copy()
    moved[:, 1] *= np.float32(1.07)
    tr.repose_device(torch.tensor(moved, device="cuda"), rebuild=False)
    tr.trace_rays(dr, n, hits)
    gpu.wait()
    binary = hits.cpu().numpy().copy()
    tr.set_walk(mode)
    tr.trace_rays(dr, n, hits)
    gpu.wait()
    _same_closest_hits(hits.cpu().numpy(), binary)
    tr.close()


def test_autotune_keeps_the_image(gpu, orc):
    s = SCENES["c2_small"]()
    cam = cam_of(s, s.width, s.height)
    tr = px.Tracer.of(gpu, s)
    chosen, ms = tr.autotune(cam, s.width, s.height, 2)
    assert chosen in range(20) and len(ms) == 20 and all(t > 0 for t in ms)
    tr.trace(cam, s.width, s.height, 0, s.spp)
    want, _ = oracle_lib.TraceOracle(orc, s).trace(cam, 0, s.spp)
    check_image(tr.image(), want, s.width * s.height)


def test_config1_full_image(gpu, orc):
    # Config 1 as specified: 65,536 triangles, 256 x 256, 16 spp, 4 bounces.
    s = scenes.c1_plain()
    cam = cam_of(s, s.width, s.height)
    want, _ = oracle_lib.TraceOracle(orc, s).trace(cam, 0, s.spp)
    tr = px.Tracer.of(gpu, s)
    tr.trace(cam, s.width, s.height, 0, s.spp)
    check_image(tr.image(), want, s.width * s.height)


def test_refit_after_repose_matches_a_fresh_tracer(gpu):
    # Tracer::repose on the device: new vertices, refit, same image as a
    # tracer built on those vertices (the tree is the refit one, so compare
    # images through the oracle-equal path: a rebuild must equal a fresh build).
    import torch

    s = SCENES["c2_small"]()
    cam = cam_of(s, s.width, s.height)
    moved = s.verts.copy()
    moved[:, 1] += 0.01
    t = px.Tracer.of(gpu, s)
    t.repose_device(torch.tensor(moved, device="cuda"), rebuild=True)
    t.trace(cam, s.width, s.height, 0, 2)
    s2 = scenes.Scene(s.name, moved, s.faces, s.mats, s.lights, s.view, s.width, s.height, s.spp, s.bounces, s.env)
    f = px.Tracer.of(gpu, s2)
    f.trace(cam, s.width, s.height, 0, 2)
    assert np.array_equal(t.image(), f.image())


ADAPT = [0.03, 4.0, 4.0, 1.0]  # Adaptive Sampling: threshold, min samples, step, on


def _check_adaptive(got, want, n):
    # every plane bit for bit but the open list, whose order is the GPU's;
    # the list as a set, and its length
    assert np.array_equal(got[:32 * n], want[:32 * n])
    assert np.array_equal(got[33 * n:34 * n], want[33 * n:34 * n])
    m = int(want[34 * n])
    assert int(got[34 * n]) == m and 0 < m < n
    assert np.array_equal(np.sort(got[32 * n:32 * n + m]), want[32 * n:32 * n + m])
    return m


@pytest.mark.parametrize("kernel", [0, 1, 12, 15], ids=["megakernel", "state_machine", "mk8_sync", "mk16_sync"])
def test_adaptive_sampling_matches_oracle(gpu, orc, kernel):
    """Adaptive Sampling (set_adaptive): the samples of one frame over two
    calls, settled pixels skipped through the open list, the convergence
    check and dilation at each step boundary — the image equals the
    oracle's, which runs the reference's per-sample tail, bit for bit."""
    s = scenes.c1_plain(ntris=2048, width=48, height=32, spp=4)
    w, h = s.width, s.height
    n = w * h
    cam = cam_of(s, w, h)
    ocam = cam.copy()
    ocam["adapt"] = ADAPT
    want, _ = oracle_lib.TraceOracle(orc, s).trace(ocam, 0, 32)
    tr = px.Tracer.of(gpu, s)
    tr.set_kernel(kernel)
    assert tr.unconverged() is None  # off
    tr.set_adaptive(ADAPT)
    tr.trace(cam, w, h, 0, 13)
    tr.trace(cam, w, h, 13, 19)
    m = _check_adaptive(tr.image(), want, n)
    assert tr.unconverged() == m
    tr.close()


def test_adaptive_sampling_sample_by_sample(gpu, orc):
    """Tracer::sample under Adaptive Sampling (slices are ignored: an
    adaptive sample traces the open list whole) == the oracle."""
    s = scenes.c1_plain(ntris=2048, width=48, height=32, spp=4)
    w, h = s.width, s.height
    cam = cam_of(s, w, h)
    ocam = cam.copy()
    ocam["adapt"] = ADAPT
    want, _ = oracle_lib.TraceOracle(orc, s).trace(ocam, 0, 20)
    tr = px.Tracer.of(gpu, s)
    tr.set_adaptive(ADAPT)
    tr.set_samples(20)
    for k in range(20):
        frame, done = tr.sample(cam, w, h, slices=3)
        assert frame == k and done == (k == 19)
    _check_adaptive(tr.image(), want, w * h)
    tr.close()


def test_show_matches_oracle(gpu, orc):
    """Tracer::show (phx_tracer_show): a composited linear image written back
    as sums scaled by the samples taken, then show.wgsl's display step —
    the sums, shown planes and packed pixels equal the oracle's bit for bit."""
    s = SCENES["c1_small"]()
    w, h = s.width, s.height
    n = w * h
    cam = cam_of(s, w, h)
    tr = px.Tracer.of(gpu, s)
    tr.trace(cam, w, h, 0, 5)
    before = tr.image()
    linear = (px.tracer.radiance_of(before, w, h) * np.float32(0.5)).reshape(n, 3).astype(np.float32)
    linear[::7] = 0.0
    tr.show(linear[: n - 10])  # the last pixels missing read as 0
    got = tr.image()
    want = before.copy()
    full = np.zeros((n, 3), np.float32)
    full[: n - 10] = linear[: n - 10]
    want.view(np.float32)[n:4 * n] = (full * np.float32(5.0)).reshape(-1)
    orc.lib.orc_show(cam.ctypes.data, want.ctypes.data)
    assert np.array_equal(got, want)
    tr.close()


@pytest.mark.parametrize("kernel", [0, 1, 15, 16, 19],
                         ids=["megakernel", "state_machine", "mk16_sync", "wavefront", "mk16_sync_reg1"])
@pytest.mark.parametrize("name", list(SCENES))
def test_sah_tree_image_matches_oracle(gpu, orc, name, kernel):
    """The tracer walking the binned SAH tree (phx_tracer_set_tree) == the
    oracle walking its restatement of sah.rs's tree, bit for bit."""
    s = SCENES[name]()
    cam = cam_of(s, s.width, s.height)
    want, orays = oracle_lib.TraceOracle(orc, s, sah=True).trace(cam, 0, s.spp)
    tr = px.Tracer.of(gpu, s)
    tr.set_tree(px.Tracer.TREE_SAH)
    tr.set_kernel(kernel)
    tr.trace(cam, s.width, s.height, 0, s.spp)
    check_image(tr.image(), want, s.width * s.height)
    assert tr.time()[1] == orays
    tr.close()


def test_sah_tree_repose_and_back_to_lbvh(gpu, orc):
    import torch

    s = SCENES["c2_small"]()
    cam = cam_of(s, s.width, s.height)
    moved = s.verts.copy()
    moved[:, 0] *= np.float32(1.1)
    tr = px.Tracer.of(gpu, s)
    tr.set_tree(px.Tracer.TREE_SAH)
    tr.repose_device(torch.tensor(moved, device="cuda"), rebuild=True)
    tr.trace(cam, s.width, s.height, 0, s.spp)
    s2 = scenes.Scene(**{**s.__dict__, "verts": moved})
    want, _ = oracle_lib.TraceOracle(orc, s2, sah=True).trace(cam, 0, s.spp)
    check_image(tr.image(), want, s.width * s.height)
    # a refit of the SAH tree: closest hits do not depend on the tree, so
    # the image stays within the relMSE gate of the rebuilt one
    back = s.verts.copy()
    back[:, 0] *= np.float32(1.05)
    tr.repose_device(torch.tensor(back, device="cuda"), rebuild=False)
    tr.trace(cam, s.width, s.height, 0, s.spp)
    s3 = scenes.Scene(**{**s.__dict__, "verts": back})
    want3, _ = oracle_lib.TraceOracle(orc, s3, sah=True).trace(cam, 0, s.spp)
    check_image(tr.image(), want3, s.width * s.height, exact=False)
    tr.set_tree(px.Tracer.TREE_LBVH)
    tr.trace(cam, s.width, s.height, 0, s.spp)
    want4, _ = oracle_lib.TraceOracle(orc, s3).trace(cam, 0, s.spp)
    check_image(tr.image(), want4, s.width * s.height)
    tr.close()


def test_autotune_tree_weighs_build_against_frames(gpu, orc):
    s = SCENES["c2_small"]()
    cam = cam_of(s, s.width, s.height)
    tr = px.Tracer.of(gpu, s)
    chosen, ms = tr.autotune_tree(cam, s.width, s.height, s.spp, 0)
    assert len(ms) == 4 and all(t > 0 for t in ms)
    assert chosen == (px.Tracer.TREE_SAH if ms[2] < ms[0] else px.Tracer.TREE_LBVH)
    many, ms2 = tr.autotune_tree(cam, s.width, s.height, s.spp, 10 ** 6)
    assert many == (px.Tracer.TREE_SAH if ms2[3] < ms2[1] else px.Tracer.TREE_LBVH)
    tr.trace(cam, s.width, s.height, 0, s.spp)
    want, _ = oracle_lib.TraceOracle(orc, s, sah=many == px.Tracer.TREE_SAH).trace(cam, 0, s.spp)
    check_image(tr.image(), want, s.width * s.height)
    tr.close()


def test_create_refuses_scenes_the_tracer_does_not_take(gpu):
    """The device check at create: a face naming a vertex or material out of
    range, a material with a texture or map word set, or one with a second
    lobe, each refused with PHX_ERR_INVALID; the scene otherwise builds."""
    s = SCENES["c1_small"]()
    px.Tracer.of(gpu, s).close()
    cases = []
    f = s.faces.copy()
    f[17, 1] = len(s.verts)
    cases.append((s.verts, f, s.mats, "vertex"))
    f = s.faces.copy()
    f[5, 3] = len(s.mats)
    cases.append((s.verts, f, s.mats, "material index"))
    m = s.mats.copy()
    m.view(np.uint32).reshape(len(m), -1)[len(m) - 1, 13] = 0
    cases.append((s.verts, s.faces, m, "texture"))
    m = s.mats.copy()
    m.view(np.uint32).reshape(len(m), -1)[0, 30] = 0
    cases.append((s.verts, s.faces, m, "second lobe"))
    for v, f, m, what in cases:
        with pytest.raises(px.PhxError) as e:
            px.Tracer(gpu, v, f, m)
        assert e.value.code == px._native.PHX_ERR_INVALID, what
    px.Tracer.of(gpu, s).close()  # the context is still good


@pytest.mark.parametrize("mode", [3, 4], ids=["persistent", "thread_per_ray"])
def test_wide_walk_when_the_root_is_a_leaf(gpu, orc, mode):
    """A scene of one face: the tree is a single leaf, the wide tree has no
    node, and the wide walks test the leaf as the binary walk does."""
    import torch

    from tests import pins

    a, _ = pins.card()
    s = pins.single_triangle_scene(a)
    rays = np.zeros((len(pins.edge_rays(2000)), 8), np.float32)
    for k, (o, d) in enumerate(pins.edge_rays(2000)):
        rays[k, 0:3], rays[k, 3], rays[k, 4:7] = o, 3.0e38, d
    tr = px.Tracer.of(gpu, s)
    tr.set_walk(mode)
    n = len(rays)
    dr = torch.tensor(rays, device="cuda")
    hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    tr.trace_rays(dr, n, hits)
    gpu.wait()
    want = oracle_lib.TraceOracle(orc, s).trace_rays(rays)
    assert np.array_equal(hits.cpu().numpy().view(np.uint32), want.view(np.uint32))
    tr.close()
