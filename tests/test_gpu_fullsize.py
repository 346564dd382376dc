"""Parity at the benchmark configurations' own sizes.

C2 as the bench times it — the 1,310,722-face displaced icosphere, 1920 x
1080, 8 bounces, on the LBVH and on the binned SAH tree — traced whole on
the GPU and compared with the oracle on a band of rows spread over the
frame (every px plane word of those rows),
plus every primary hit id of the 1080p frame. C3 as configured — 500,000
vertices (+ 4 of the ground), 999,002 faces, 64 bones, 1-4 influences a vertex — Skin, face
boxes and the LBVH refit, each bit for bit against the oracle, and the
rebuilt pose traced on a band of rows."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import scenes
from tests import oracle_lib
from tests.test_gpu_trace import cam_of

pytestmark = pytest.mark.gpu

# Per-pixel words of each plane range the tracer writes (read.rs:37-56).
PLANES = {"packed": (0, 1), "linear": (1, 3), "shown": (4, 3), "albedo": (7, 3), "normal": (10, 3),
          "depth": (13, 1), "overlay": (20, 3), "coverage": (23, 1), "film": (24, 1), "outline": (25, 1),
          "count": (31, 1), "missed": (33, 1)}


def rows_equal(got, want, w, n, rows):
    bad = {}
    for name, (plane, k) in PLANES.items():
        for r in rows:
            a = plane * n + k * r * w
            b = a + k * w
            d = int(np.sum(got[a:b] != want[a:b]))
            if d:
                bad[f"{name}@{r}"] = d
    assert not bad, bad


@pytest.fixture(scope="module")
def c2():
    return scenes.c2_mesh()


@pytest.mark.parametrize("tree", [0, 1], ids=["lbvh", "sah"])
def test_c2_1080p_rows_match_oracle(gpu, orc, c2, tree):
    """On either tree; the SAH tree is the one the bench's autotuner picks
    for this frame, so this is the headline step's image."""
    s = c2
    w, h, spp = 1920, 1080, 2
    cam = cam_of(s, w, h)
    rows = np.linspace(0, h - 1, 40).round().astype(int).tolist()
    T = oracle_lib.TraceOracle(orc, s, sah=bool(tree))
    want = np.zeros(34 * w * h + 1, np.uint32)
    for r in rows:
        T.trace(cam, 0, spp, px=want, rows=(r, 1))
    tr = px.Tracer.of(gpu, s)
    tr.set_tree(tree)
    tr.autotune(cam, w, h, 1)  # the form the bench picks
    tr.trace(cam, w, h, 0, spp)
    rows_equal(tr.image(), want, w, w * h, rows)
    tr.close()


def test_c2_1080p_primary_ids_exact(gpu, orc, c2):
    import torch

    s = c2
    w, h = 1920, 1080
    cam = cam_of(s, w, h)
    want_ids, want_t = oracle_lib.TraceOracle(orc, s).primary(cam, 5)
    tr = px.Tracer.of(gpu, s)
    ids = torch.empty(w * h, dtype=torch.int32, device="cuda")
    ts = torch.empty(w * h, dtype=torch.float32, device="cuda")
    tr.primary(cam, w, h, 5, ids, ts)
    gpu.wait()
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), want_ids)
    assert np.array_equal(ts.cpu().numpy(), want_t)
    assert np.mean(want_ids != 0xFFFFFFFF) > 0.3  # the mesh and ground fill much of the frame
    tr.close()


def test_c3_full_skin_boxes_refit_and_trace(gpu, orc):
    import torch

    s, rig = scenes.c3_skinned()
    assert len(s.verts) == 500_004 and len(s.faces) == 999_002 and rig.nbones == 64
    nv, nf = len(s.verts), len(s.faces)
    bones = rig.bones(3)
    dev = {k: torch.tensor(np.ascontiguousarray(a).view(np.uint8), device="cuda")
           for k, a in dict(rest=rig.rest, offsets=rig.offsets, pairs=rig.pairs, bones=bones,
                            faces=s.faces).items()}
    out = torch.empty((nv, 4), dtype=torch.float32, device="cuda")
    px.skin(gpu, dev["rest"], dev["offsets"], dev["pairs"], dev["bones"], rig.nbones, out, nv, 1e-4)
    gpu.wait()
    want_v = orc.skin(rig.rest, rig.offsets, rig.pairs, bones, 1e-4)
    assert np.array_equal(out.cpu().numpy(), want_v)  # Skin::cpu's operation order

    # face boxes of the pose, on the device
    boxes = torch.empty((nf, 8), dtype=torch.float32, device="cuda")
    px.face_boxes(gpu, out, dev["faces"], nf, boxes)
    gpu.wait()
    posed = scenes.Scene(**{**s.__dict__, "verts": want_v})
    want_boxes = posed.face_boxes()
    got_boxes = boxes.cpu().numpy()
    assert np.array_equal(got_boxes[:, [0, 1, 2, 4, 5, 6]], want_boxes[:, [0, 1, 2, 4, 5, 6]])

    # the rest pose's LBVH, then a refit to the pose
    rest_boxes = s.face_boxes()
    nodes, order, depth = orc.build(rest_boxes, 4)
    g = px.GpuBvh.build(gpu, rest_boxes, 4)
    b = g.download()
    assert b.depth == depth and np.array_equal(b.order, order)
    assert np.array_equal(b.nodes.view(np.uint32), nodes.view(np.uint32))
    assert g.update_device(boxes, nf)
    refit = orc.refit(nodes, order, want_boxes)
    got = g.download().nodes
    live = orc.reachable(nodes)
    assert np.array_equal(got[live].view(np.uint32), refit[live].view(np.uint32))
    g.close()

    # the posed frame, rebuilt on the device, on a band of rows
    w, h, spp = 1920, 1080, 1
    cam = cam_of(s, w, h)
    tr = px.Tracer.of(gpu, s)
    vptr, _ = tr.device_verts()
    px.skin(gpu, dev["rest"], dev["offsets"], dev["pairs"], dev["bones"], rig.nbones, vptr, nv, 1e-4)
    tr.repose_device(vptr, rebuild=True)
    tr.trace(cam, w, h, 0, spp)
    rows = np.linspace(0, h - 1, 24).round().astype(int).tolist()
    T = oracle_lib.TraceOracle(orc, posed)
    want = np.zeros(34 * w * h + 1, np.uint32)
    for r in rows:
        T.trace(cam, 0, spp, px=want, rows=(r, 1))
    rows_equal(tr.image(), want, w, w * h, rows)
    tr.close()
