"""The oracle's LBVH, pinned against the reference's own known answers:
src/bvh/node.rs:111-124 (layout, Morton KATs), src/bvh/sort.rs:156-182 (the
five radix code sets, CPU sort == radix model), src/bvh/test.rs:45-77
(valid trees, all-equal codes, compaction), plus hand-derived Karras cases.
"""

import numpy as np
import pytest

from tests import gen


def test_morton_known_answers(orc):
    # node.rs:119-124
    assert orc.morton([1.0, 1.0, 1.0]) == (1 << 30) - 1
    assert orc.morton([0.1] * 3) < orc.morton([0.9] * 3)
    assert orc.morton([1.0] * 3, 0) < orc.morton([0.0] * 3, 1)
    assert orc.morton([0.0] * 3) == 0
    # one axis at a time: x is the highest of each bit triple
    assert orc.morton([1.0, 0.0, 0.0]) == 0x24924924
    assert orc.morton([0.0, 1.0, 0.0]) == 0x12492492
    assert orc.morton([0.0, 0.0, 1.0]) == 0x09249249
    # clamping and NaN (Rust: clamp keeps NaN, `as u64` makes it 0)
    assert orc.morton([2.0, -1.0, float("nan")]) == 0x24924924


def test_node_layout_is_wgsl_sized():
    # node.rs:111-117: Half 16 bytes, Node 32, Aabb 32
    import ctypes as C

    from tests import oracle_lib

    assert oracle_lib.C.sizeof(C.c_float * 4) == 16
    import phiray_b200._native as N

    assert N.LEAF == 0x80000000 and N.STACK == 32


RADIX_SETS = [
    [],
    [7],
    [5, 5, 5, 5, 5, 5, 5, 5],
    [9, 1, 8, 1, 7, 1, 0, 0xFFFFFFFF, 0, 3],
    [(i * 2654435761) % (1 << 32) % 97 for i in range(1000)],
]


@pytest.mark.parametrize("codes", RADIX_SETS, ids=["empty", "single", "equal", "mixed", "knuth97"])
def test_sort_equals_radix_model(orc, codes):
    # sort.rs:156-173: the CPU sort (by code, then index) equals the
    # sequential model of the LSD radix, order and codes.
    codes = np.array(codes, dtype=np.uint32)
    order, sorted_ = orc.sort_codes(codes)
    morder, msorted = orc.radix_model(codes)
    assert np.array_equal(order, morder)
    assert np.array_equal(sorted_, msorted)
    # and it is the stable argsort
    want = np.argsort(codes, kind="stable").astype(np.uint32)
    assert np.array_equal(order, want)
    assert np.array_equal(sorted_, codes[want])


def test_delta_definition(orc):
    # mod.rs:33-43: -1 outside, clz of the xor, index tie-break past 32.
    codes = np.array([0b0001, 0b0001, 0b0011, 0xFFFFFFFF], dtype=np.uint32)
    assert orc.lib.orc_delta(codes.ctypes.data, 4, 0, -1) == -1
    assert orc.lib.orc_delta(codes.ctypes.data, 4, 0, 4) == -1
    assert orc.lib.orc_delta(codes.ctypes.data, 4, 1, 2) == 30
    assert orc.lib.orc_delta(codes.ctypes.data, 4, 0, 1) == 32 + 31  # equal codes, 0 ^ 1
    assert orc.lib.orc_delta(codes.ctypes.data, 4, 2, 3) == 0


def test_karras_small_cases(orc):
    # Two leaves: the root splits them (left = leaf n-1+0, right = leaf n+0).
    assert orc.links(np.array([3, 9], dtype=np.uint32)).tolist() == [[1, 2, 0, 1]]
    # Three distinct codes 0b00, 0b01, 0b11: root covers [0, 2], splits
    # after slot 1 (node 1 = {0,1}), node 1 splits 0 | 1.
    links = orc.links(np.array([0, 1, 3], dtype=np.uint32))
    assert links.tolist() == [[1, 4, 0, 2], [2, 3, 0, 1]]
    # Equal codes fall back to the index: still a valid binary tree.
    links = orc.links(np.zeros(8, dtype=np.uint32))
    assert sorted(np.concatenate([links[:, 0], links[:, 1]]).tolist()) == list(range(1, 15))


@pytest.mark.parametrize("n", [1, 2, 3, 7, 100, 5000])
@pytest.mark.parametrize("leaf", [1, 4])
def test_builds_valid_trees(orc, n, leaf):
    # test.rs:45-54
    p = gen.test_prims(n)
    nodes, order, depth = orc.build(p, leaf)
    gen.check_tree(nodes, order, depth, p, orc.reachable(nodes))


def test_empty_build(orc):
    nodes, order, depth = orc.build(np.zeros((0, 8), np.float32), 4)
    assert len(nodes) == 0 and len(order) == 0 and depth == 0


def test_all_equal_codes_stay_shallow(orc):
    # test.rs:56-61
    p = np.tile(np.array([0, 0, 0, 0, 1, 1, 1, 0], np.float32), (1000, 1))
    nodes, order, depth = orc.build(p, 1)
    gen.check_tree(nodes, order, depth, p, orc.reachable(nodes))


def test_compaction_keeps_the_tree(orc):
    # test.rs:63-77
    p = gen.test_prims(5000)
    nodes, order, depth = orc.build(p, 4)
    before = len(nodes)
    c = orc.compact(nodes)
    assert len(c) < before // 2 + 2
    assert len(orc.reachable(c)) == len(c)
    gen.check_tree(c, order, depth, p, orc.reachable(c))
    bc_nodes, bc_order, bc_depth = orc.build_compact(p, 4)
    assert np.array_equal(bc_nodes.view(np.uint32), c.view(np.uint32))
    assert np.array_equal(bc_order, order) and bc_depth == depth
    flat = np.tile(np.array([0, 0, 0, 0, 1, 1, 1, 0], np.float32), (1000, 1))
    nodes, order, depth = orc.build(flat, 1)
    deep = orc.compact(nodes)
    bc_nodes, _, _ = orc.build_compact(flat, 1)
    assert np.array_equal(bc_nodes.view(np.uint32), deep.view(np.uint32))


def test_refit_after_motion_is_exact(orc):
    # tests/bvh.rs:46-52 on the CPU side: the old topology refit over moved
    # prims contains them exactly.
    p = gen.bvh_prims(2000, 0.0)
    moved = gen.bvh_prims(2000, 2.5)
    nodes, order, depth = orc.build(p, 4)
    r = orc.refit(nodes, order, moved)
    gen.check_tree(r, order, depth, moved, orc.reachable(r))
    root_lo = moved[:, 0:3].min(axis=0)
    root_hi = moved[:, 4:7].max(axis=0)
    assert np.array_equal(r[0, 0:3], root_lo) and np.array_equal(r[0, 4:7], root_hi)


def test_golden_fixture(orc):
    # The oracle's own output for the reference generator at n = 257, kept
    # as a fixture (tests/golden/make_golden.py) so a change to the
    # restatement shows up as a diff.
    import os

    path = os.path.join(os.path.dirname(__file__), "golden", "bvh_257.npz")
    g = np.load(path)
    p = gen.bvh_prims(257, 0.0)
    assert np.array_equal(p, g["prims"])
    nodes, order, depth = orc.build(p, 4)
    assert np.array_equal(order, g["order"]) and depth == int(g["depth"])
    assert np.array_equal(nodes.view(np.uint32), g["nodes"].view(np.uint32))


@pytest.mark.parametrize("n", [1, 2, 3, 7, 100, 5000, 70000])
@pytest.mark.parametrize("leaf", [1, 4])
def test_sah_builds_valid_trees(orc, n, leaf):
    # test.rs:79-91: the binned SAH tree (sah.rs) the reference's tracer walks
    p = gen.test_prims(n)
    nodes, order, depth = orc.build_sah(p, leaf)
    gen.check_tree(nodes, order, depth, p, orc.reachable(nodes))
    assert len(orc.reachable(nodes)) == len(nodes)  # built compact: no unreachable nodes


def test_sah_empty_and_flat(orc):
    nodes, order, depth = orc.build_sah(np.zeros((0, 8), np.float32), 4)
    assert len(nodes) == 0 and len(order) == 0 and depth == 0
    # every centre in one point: no plane to split on, still a valid tree
    flat = np.tile(np.array([0, 0, 0, 0, 1, 1, 1, 0], np.float32), (1000, 1))
    nodes, order, depth = orc.build_sah(flat, 4)
    gen.check_tree(nodes, order, depth, flat, orc.reachable(nodes))


def _sah_cost(nodes):
    # test.rs:97-112 cost: each node's area against the root's, times what it holds
    w = nodes.view(np.uint32)

    def area(i):
        d = np.maximum(nodes[i, 4:7] - nodes[i, 0:3], 0.0).astype(np.float32)
        return np.float32(2.0) * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0])

    root = area(0)
    total = 0.0
    for i in range(len(nodes)):
        lo, hi = int(w[i, 3]), int(w[i, 7])
        held = (hi - (lo & 0x7FFFFFFF)) if lo & 0x80000000 else 1
        total += float(area(i) / root) * held
    return total


def test_sah_trees_are_cheaper_to_walk_than_morton_ones(orc):
    # test.rs:94-116
    p = gen.test_prims(20000)
    sah = _sah_cost(orc.build_sah(p, 4)[0])
    morton = _sah_cost(orc.build_compact(p, 4)[0])
    assert sah < morton * 0.9, (sah, morton)


@pytest.mark.parametrize("which", ["c1", "c2"])
def test_sah_tree_traces_the_same_image(orc, which):
    """The tree decides only which nodes a walk visits: with the SAH tree
    the oracle's image is the Morton tree's word for word, with fewer
    triangle tests."""
    import phiray_b200 as px
    from phiray_b200 import scenes
    from tests import oracle_lib

    s = (scenes.c1_plain(ntris=4096, width=64, height=64, spp=4) if which == "c1"
         else scenes.c2_mesh(levels=4, width=64, height=48, spp=4))
    cam = px.camera(s)
    cam["w"], cam["h"] = s.width, s.height
    a, ra, _, ta = oracle_lib.TraceOracle(orc, s).trace_walk(cam, 0, 4)
    b, rb, _, tb = oracle_lib.TraceOracle(orc, s, sah=True).trace_walk(cam, 0, 4)
    assert ra == rb and np.array_equal(a, b)
    assert tb < ta
