"""The device SAH builder's per-node code (phiray_b200/csrc/sah_core.cuh),
built for the host and run level by level as phx_bvh_build_sah launches it,
against the oracle's restatement of Bvh::build_sah: the same nodes, bounds,
slot order and depth, word for word."""

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests import gen

HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    out = tmp_path_factory.mktemp("sah") / "libsahemul.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                    "-o", str(out), str(HERE / "sah_emul.cpp")], check=True)
    lib = C.CDLL(str(out))
    lib.emul_build_sah.restype = C.c_uint32
    lib.emul_build_sah.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_uint32)]

    def build(prims, leaf):
        prims = np.ascontiguousarray(prims, np.float32).reshape(-1, 8)
        n = len(prims)
        nodes = np.zeros((max(1, 2 * n - 1), 8), np.float32)
        order = np.zeros(n, np.uint32)
        depth = C.c_uint32()
        m = lib.emul_build_sah(prims.ctypes.data, n, leaf, nodes.ctypes.data, order.ctypes.data, C.byref(depth))
        return nodes[:m].copy(), order, depth.value

    return build


@pytest.mark.parametrize("n", [1, 2, 3, 7, 100, 5000, 70000])
@pytest.mark.parametrize("leaf", [0, 1, 4])
def test_device_steps_build_the_reference_tree(orc, emul, n, leaf):
    p = gen.test_prims(n)
    want_nodes, want_order, want_depth = orc.build_sah(p, leaf)
    nodes, order, depth = emul(p, leaf)
    assert depth == want_depth
    assert np.array_equal(order, want_order)
    assert np.array_equal(nodes.view(np.uint32), want_nodes.view(np.uint32))


def test_device_steps_on_flat_and_mesh_input(orc, emul):
    flat = np.tile(np.array([0, 0, 0, 0, 1, 1, 1, 0], np.float32), (1000, 1))
    for p in (flat, gen.bvh_prims(3000, 0.0)):
        a = orc.build_sah(p, 4)
        b = emul(p, 4)
        assert a[2] == b[2] and np.array_equal(a[1], b[1])
        assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_device_steps_on_random_boxes(orc, emul, seed):
    """Spread boxes, a dense clump and repeated boxes: nodes whose slots
    fill few of the 16 bins, the case the occupied-bin sweep shortens."""
    rng = np.random.default_rng(seed)
    n = 20000
    lo = rng.uniform(0.0, 10.0, (n, 3)).astype(np.float32)
    lo[: n // 3] = rng.normal(4.0, 0.05, (n // 3, 3)).astype(np.float32)
    size = rng.uniform(0.0, 0.5, (n, 3)).astype(np.float32)
    p = np.zeros((n, 8), np.float32)
    p[:, 0:3], p[:, 4:7] = lo, lo + size
    p[n - 500:, 0:3], p[n - 500:, 4:7] = 2.0, 2.25
    p = p[rng.permutation(n)]
    for leaf in (1, 4):
        a = orc.build_sah(p, leaf)
        b = emul(p, leaf)
        assert a[2] == b[2] and np.array_equal(a[1], b[1])
        assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32))
