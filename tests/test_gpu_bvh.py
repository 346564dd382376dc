"""GPU LBVH == the oracle's Bvh::build, bit for bit (tests/bvh.rs:31-54 and
beyond): codes, sorted order, Karras links, packing, depth, refit bounds."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import scenes
from tests import gen

pytestmark = pytest.mark.gpu


def same_tree(g: px.Bvh, nodes, order, depth, orc):
    """tests/bvh.rs:21-29 (`same`: order, depth, every reachable node's links
    and bounds), then stronger: every node slot, reachable or not."""
    assert np.array_equal(g.order, order)
    assert g.depth == depth
    gw, cw = g.nodes.view(np.uint32), nodes.view(np.uint32)
    r = orc.reachable(nodes)
    assert np.array_equal(gw[r][:, [3, 7]], cw[r][:, [3, 7]]), "reachable links"
    assert np.array_equal(g.nodes[r][:, [0, 1, 2, 4, 5, 6]], nodes[r][:, [0, 1, 2, 4, 5, 6]]), "reachable bounds"
    # unreachable slots keep the reference's initial links and zero bounds
    assert np.array_equal(g.nodes, nodes)


@pytest.mark.parametrize("n", [1, 2, 3, 257, 100_003])
def test_gpu_build_and_refit_match_cpu(gpu, orc, n):
    p = gen.bvh_prims(n, 0.0)
    nodes, order, depth = orc.build(p, 4)
    g = px.GpuBvh.build(gpu, p, 4)
    same_tree(g.download(), nodes, order, depth, orc)
    moved = gen.bvh_prims(n, 2.5)
    assert g.update(moved)
    want = orc.refit(nodes, order, moved)
    same_tree(g.download(), want, order, depth, orc)
    # refit twice more (the parity counters carry across refits)
    g.refit()
    g.refit()
    same_tree(g.download(), want, order, depth, orc)


def test_update_with_another_count_asks_for_a_rebuild(gpu):
    g = px.GpuBvh.build(gpu, gen.bvh_prims(100, 0.0), 4)
    assert not g.update(gen.bvh_prims(101, 0.0))


def test_empty_build(gpu):
    g = px.GpuBvh.build(gpu, np.zeros((0, 8), np.float32), 4)
    b = g.download()
    assert len(b.nodes) == 0 and len(b.order) == 0 and b.depth == 0


@pytest.mark.parametrize("n", [7, 5000])
@pytest.mark.parametrize("leaf", [1, 4])
def test_test_rs_generator(gpu, orc, n, leaf):
    p = gen.test_prims(n)
    nodes, order, depth = orc.build(p, leaf)
    same_tree(px.GpuBvh.build(gpu, p, leaf).download(), nodes, order, depth, orc)


def test_all_equal_codes_hit_the_depth_cap(gpu, orc):
    p = np.tile(np.array([0, 0, 0, 0, 1, 1, 1, 0], np.float32), (1000, 1))
    nodes, order, depth = orc.build(p, 1)
    b = px.GpuBvh.build(gpu, p, 1).download()
    same_tree(b, nodes, order, depth, orc)


def test_deep_karras_chain_is_packed_at_stack(gpu, orc):
    # Exponentially spread centres make a Karras chain deeper than 32: the
    # packing must cut it at STACK - 1 exactly as assemble's DFS does.
    k = np.arange(40)
    lo = np.zeros((40, 3), np.float32)
    lo[:, 0] = (2.0 ** -k.astype(np.float64)).astype(np.float32)
    p = px.aabbs(lo, lo)
    p = np.concatenate([p, np.zeros((1, 8), np.float32)])
    for leaf in (1, 4):
        nodes, order, depth = orc.build(p, leaf)
        same_tree(px.GpuBvh.build(gpu, p, leaf).download(), nodes, order, depth, orc)


def test_config1_scene(gpu, orc):
    s = scenes.c1_plain()
    p = s.face_boxes()
    nodes, order, depth = orc.build(p, 4)
    same_tree(px.GpuBvh.build(gpu, p, 4).download(), nodes, order, depth, orc)


def test_large_scene_bit_exact(gpu, orc):
    # 1.31M random triangles: the size class of the single-mesh config.
    rng = np.random.default_rng(7)
    n = 1_310_722
    c = rng.random((n, 3), dtype=np.float32)
    e = rng.uniform(0.0, 0.01, (n, 3)).astype(np.float32)
    p = px.aabbs(c - e, c + e)
    p[::97] = p[5]  # collisions
    nodes, order, depth = orc.build(p, 4)
    same_tree(px.GpuBvh.build(gpu, p, 4).download(), nodes, order, depth, orc)


@pytest.mark.parametrize(
    "codes",
    [
        [7],
        [5] * 8,
        [9, 1, 8, 1, 7, 1, 0, 0xFFFFFFFF, 0, 3],
        [(i * 2654435761) % (1 << 32) % 97 for i in range(1000)],
    ],
    ids=["single", "equal", "mixed", "knuth97"],
)
def test_stable_radix_sort_small_sets(gpu, orc, codes):
    import torch

    c = torch.tensor(np.array(codes, dtype=np.uint32).view(np.int32), device="cuda")
    o = torch.empty_like(c)
    s = torch.empty_like(c)
    px.bvh.sort_codes(gpu, c, len(codes), o, s)
    order, sorted_ = orc.sort_codes(np.array(codes, dtype=np.uint32))
    assert np.array_equal(o.cpu().numpy().view(np.uint32), order)
    assert np.array_equal(s.cpu().numpy().view(np.uint32), sorted_)


@pytest.mark.parametrize("n", [4095, 4096, 4097, 1 << 22])
def test_stable_radix_sort_large(gpu, n):
    import torch

    rng = np.random.default_rng(n)
    codes = rng.integers(0, 1 << 30, n, dtype=np.uint32)
    codes[::3] = codes[7]  # heavy collisions: stability is what matters
    c = torch.tensor(codes.view(np.int32), device="cuda")
    o = torch.empty_like(c)
    s = torch.empty_like(c)
    px.bvh.sort_codes(gpu, c, n, o, s)
    want = np.argsort(codes, kind="stable").astype(np.uint32)
    assert np.array_equal(o.cpu().numpy().view(np.uint32), want)
    assert np.array_equal(s.cpu().numpy().view(np.uint32), codes[want])


def test_stage_morton_and_karras(gpu, orc):
    import torch

    p = gen.bvh_prims(50_000, 0.0)
    dp = torch.tensor(p, device="cuda")
    codes = torch.empty(len(p), dtype=torch.int32, device="cuda")
    px.bvh.morton(gpu, dp, len(p), codes)
    want = orc.codes(p)
    assert np.array_equal(codes.cpu().numpy().view(np.uint32), want)
    order, sorted_ = orc.sort_codes(want)
    ds = torch.tensor(sorted_.view(np.int32), device="cuda")
    links = torch.empty((len(p) - 1, 4), dtype=torch.int32, device="cuda")
    px.bvh.karras(gpu, ds, len(p), links)
    assert np.array_equal(links.cpu().numpy().view(np.uint32), orc.links(sorted_))


def test_pass_replays_reference_kernels(gpu, orc):
    # bvh::Morton / Karras / Refit recorded into a Pass (the reference's
    # GpuBvh flow, gpu.rs:36-85) give the oracle's codes, links and bounds.
    p = gen.bvh_prims(3000, 0.0)
    n = len(p)
    s = orc.scene(p)
    inv = [1.0 / (s[4 + k] - s[k]) if s[4 + k] - s[k] > 0 else 0.0 for k in range(3)]
    prims = px.GpuArray.from_(gpu, p)
    codes = px.GpuArray.zeroed(gpu, 4 * n)
    ps = px.Pass(gpu)
    ps.add(px.Morton, n, px.Morton.params(lo=s[0:3], inv=np.float32(inv)), [prims, codes])
    ps.run()
    want = orc.codes(p)
    assert np.array_equal(codes.read(np.uint32), want)
    order, sorted_ = orc.sort_codes(want)
    sc = px.GpuArray.from_(gpu, sorted_)
    links = px.GpuArray.zeroed(gpu, 16 * (n - 1))
    ps.clear()
    ps.add(px.Karras, n - 1, px.Karras.params(leaves=n), [sc, links])
    ps.run()
    assert np.array_equal(links.read(np.uint32).reshape(-1, 4), orc.links(sorted_))
    nodes, order2, depth = orc.build(p, 4)
    blank = nodes.copy()
    blank[:, [0, 1, 2, 4, 5, 6]] = 0.0
    a = px.GpuArray.from_(gpu, blank)
    b = px.GpuArray.from_(gpu, blank)
    og = px.GpuArray.from_(gpu, order2)
    ps.clear()
    steps = depth + 1 + ((depth + 1) % 2)
    for k in range(steps):
        src, dst = (a, b) if k % 2 == 0 else (b, a)
        ps.add(px.Refit, len(nodes), px.Refit.params(), [prims, og, src, dst])
    ps.run()
    got = a.read(np.float32).reshape(-1, 8)
    for i in orc.reachable(nodes):
        assert np.array_equal(got[i], nodes[i])
    assert ps.compiled() == 1


@pytest.mark.parametrize("n", [1, 2, 7, 100, 600, 5000, 70000])
@pytest.mark.parametrize("leaf", [0, 1, 4])
def test_sah_build_equals_the_reference_tree(gpu, orc, n, leaf):
    """phx_bvh_build_sah == Bvh::build_sah's restatement, word for word:
    nodes with their bounds, slot order, depth."""
    from phiray_b200.bvh import build_sah

    p = gen.test_prims(n)
    want_nodes, want_order, want_depth = orc.build_sah(p, leaf)
    got = build_sah(gpu, p, leaf)
    assert got.depth == want_depth
    assert np.array_equal(got.order, want_order)
    assert np.array_equal(got.nodes.view(np.uint32), want_nodes.view(np.uint32))


def test_sah_build_of_many_big_nodes(gpu, orc):
    """300,000 boxes (a spread, a dense clump, and 9,000 copies of one box):
    many levels of nodes cut over blocks, with several such nodes a level,
    flat ones among them, == the restatement word for word."""
    from phiray_b200.bvh import build_sah

    rng = np.random.default_rng(11)
    n = 300_000
    lo = rng.uniform(0.0, 100.0, (n, 3)).astype(np.float32)
    lo[: n // 4] = rng.normal(40.0, 0.5, (n // 4, 3)).astype(np.float32)
    size = rng.uniform(0.01, 2.0, (n, 3)).astype(np.float32)
    p = np.zeros((n, 8), np.float32)
    p[:, 0:3], p[:, 4:7] = lo, lo + size
    p[n - 9000:, 0:3], p[n - 9000:, 4:7] = 7.0, 7.5
    p = p[rng.permutation(n)]
    want_nodes, want_order, want_depth = orc.build_sah(p, 4)
    got = build_sah(gpu, p, 4)
    assert got.depth == want_depth
    assert np.array_equal(got.order, want_order)
    assert np.array_equal(got.nodes.view(np.uint32), want_nodes.view(np.uint32))


def test_sah_build_on_a_mesh(gpu, orc):
    from phiray_b200.bvh import build_sah

    p = gen.bvh_prims(20000, 0.0)
    want_nodes, want_order, want_depth = orc.build_sah(p, 4)
    got = build_sah(gpu, p, 4)
    assert got.depth == want_depth and np.array_equal(got.order, want_order)
    assert np.array_equal(got.nodes.view(np.uint32), want_nodes.view(np.uint32))
