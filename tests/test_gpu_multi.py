"""The frame split by tile rows on the device (phx_tracer_trace_rows,
phx_tracer_copy_rows), with two ranks emulated by two tracers in one
process (this pool runs one GPU a call): each traces its bands, its rows are
packed and unpacked into the other's image, and both images then equal one
whole-frame trace, every row plane bit for bit. The packed layout is the
host one phiray_b200.multi uses."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import multi, scenes
from phiray_b200 import _native as N
from tests.test_gpu_trace import cam_of

pytestmark = pytest.mark.gpu


def test_rows_split_and_exchanged_equal_a_whole_frame(gpu):
    import torch

    s = scenes.c2_mesh(levels=4, width=96, height=77, spp=2)
    w, h = s.width, s.height
    cam = cam_of(s, w, h)
    whole = px.Tracer.of(gpu, s)
    whole.trace(cam, w, h, 0, s.spp)
    want = whole.image()
    world, tile = 2, 16
    ranks = [px.Tracer.of(gpu, s) for _ in range(world)]
    lib = N.lib()
    block = multi.ROW_WORDS * multi.max_rows(h, world, tile) * w
    packed = []
    for r, tr in enumerate(ranks):
        for r0, rows in multi.bands(h, world, r, tile):
            N.check(lib.phx_tracer_trace_rows(tr.handle, cam.ctypes.data, w, h, 0, s.spp, r0, rows))
        tr.w, tr.h = w, h
        buf = torch.zeros(block, dtype=torch.int32, device="cuda")
        at = 0
        for r0, rows in multi.bands(h, world, r, tile):
            N.check(lib.phx_tracer_copy_rows(tr.handle, r0, rows, buf.data_ptr() + 4 * at, 0))
            at += multi.ROW_WORDS * rows * w
        gpu.wait()
        mine = multi.bands(h, world, r, tile)
        host = multi.pack_rows(tr.image(), w, h, mine)
        assert np.array_equal(buf.cpu().numpy().view(np.uint32)[: len(host)], host)  # the two layouts agree
        packed.append(buf)
    for r, tr in enumerate(ranks):
        for q in range(world):
            if q == r:
                continue
            at = 0
            for r0, rows in multi.bands(h, world, q, tile):
                N.check(lib.phx_tracer_copy_rows(tr.handle, r0, rows, packed[q].data_ptr() + 4 * at, 1))
                at += multi.ROW_WORDS * rows * w
        gpu.wait()
        got = tr.image()
        for plane, k in multi.ROW_PLANES:
            a, b = plane * w * h, (plane + k) * w * h
            assert np.array_equal(got[a:b], want[a:b]), (r, plane)
    for t in ranks + [whole]:
        t.close()


def test_trace_rows_rejects_rows_outside_the_frame(gpu):
    s = scenes.c1_plain(ntris=512, width=32, height=16, spp=1)
    tr = px.Tracer.of(gpu, s)
    cam = cam_of(s, 32, 16)
    rc = N.lib().phx_tracer_trace_rows(tr.handle, cam.ctypes.data, 32, 16, 0, 1, 10, 7)
    assert rc == N.PHX_ERR_INVALID
    tr.close()
