"""Trains the learned denoiser on the device, from pairs the tracer renders.

``python -m phiray_b200.train --scenes 160 --ref-spp 1024 --steps 4000
--out phiray_b200/weights/kpcn.phxu`` renders each seeded procedural scene
(`scenes.procedural`) once as one continuous accumulation: several short
segments (1-64 samples) whose px images, differenced from the running
total, are independent noisy inputs (each traced in two halves, the first
half's image giving the part-way snapshot of its sample spread), then
`ref-spp` further samples whose difference is the reference. Every px plane the network reads (sums,
albedo/normal/depth guides, sample and miss counts) accumulates linearly,
so a difference of two accumulations is the image of the samples between
them. The network then trains on random crops of those pairs with the
project's own forward and backward kernels (``Unet.train_step``).

Device memory for the data set and the crops is held in torch tensors on
the context's stream; torch does no arithmetic of the network.
"""

from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import kernels, scenes
from .denoiser import TILE, Unet, features, read_weights, snapshot_host
from .gpu import Gpu, GpuArray
from .tracer import PX_LEN, Tracer, camera

# planes that accumulate per sample: sums, guides, sample count, misses
_F32_PLANES = [(1, 4), (7, 14), (33, 34)]
_U32_PLANES = [(31, 32)]


def px_diff(a: np.ndarray, b: np.ndarray | None, n: int) -> np.ndarray:
    """The px image of the samples taken between accumulations b and a."""
    out = np.zeros(PX_LEN * n + 1, dtype=np.uint32)
    fo, fa = out.view(np.float32), a.view(np.float32)
    fb = None if b is None else b.view(np.float32)
    for lo, hi in _F32_PLANES:
        s = slice(lo * n, hi * n)
        fo[s] = fa[s] if fb is None else (fa[s].astype(np.float64) - fb[s]).astype(np.float32)
    for lo, hi in _U32_PLANES:
        s = slice(lo * n, hi * n)
        out[s] = a[s] if b is None else a[s] - b[s]
    return out


def radiance(px: np.ndarray, w: int, h: int) -> np.ndarray:
    """The linear mean over the samples that met something (util.wgsl's emit:
    light sum / max(k - gone, 1)) of a px image, (h, w, 3) float32 — the value
    the view transform shows; equal to Tracer::radiance (read.rs:240-251,
    sum / k) wherever every sample met something."""
    n = w * h
    f = px.view(np.float32)
    k = px[31 * n:32 * n].astype(np.float32)
    gone = f[33 * n:34 * n]
    return (f[n:4 * n].reshape(n, 3) / np.maximum(k - gone, 1.0)[:, None]).reshape(h, w, 3)


def relmse(x: np.ndarray, ref: np.ndarray) -> float:
    """mean over pixels and channels of (x - r)^2 / (r^2 + 0.01)."""
    x = x.astype(np.float64)
    r = ref.astype(np.float64)
    return float(np.mean((x - r) ** 2 / (r * r + 1e-2)))


def render_group(gpu: Gpu, scs, segments, ref_spp: int, chunk: int = 256):
    """Noisy images (one per segment, each with its part-way snapshot or None),
    and the reference image, of several scenes: one continuous accumulation
    per scene, every pass tracing all the scenes' frames in one persistent
    batch launch (a single 256 x 256 image cannot fill the GPU on its own)."""
    from .batch import Batch

    trs = [Tracer.of(gpu, sc) for sc in scs]
    cams = [camera(sc) for sc in scs]
    b = Batch(gpu)

    def run(first: int, spp: int) -> None:
        b.clear()
        for sc, tr, cam in zip(scs, trs, cams):
            b.add(tr, cam, sc.width, sc.height, first, spp)
        b.trace()

    frame = 0
    prev = [None] * len(scs)
    noisy = [[] for _ in scs]
    halves = [[] for _ in scs]
    for spp in segments:
        # a segment of two or more samples is traced in two halves: the first
        # half's image is its part-way snapshot (the pixels' sample spread)
        first = spp // 2
        mid = [None] * len(scs)
        if first > 0:
            run(frame, first)
            mid = [tr.image() for tr in trs]
        run(frame + first, spp - first)
        frame += spp
        for k, (sc, tr) in enumerate(zip(scs, trs)):
            n = sc.width * sc.height
            img = tr.image()
            noisy[k].append(px_diff(img, prev[k], n))
            halves[k].append(None if mid[k] is None else snapshot_host(px_diff(mid[k], prev[k], n), sc.width,
                                                                        sc.height))
            prev[k] = img
    left = ref_spp
    while left > 0:
        c = min(chunk, left)
        run(frame, c)
        frame += c
        left -= c
    refs = [px_diff(tr.image(), prev[k], sc.width * sc.height) for k, (sc, tr) in enumerate(zip(scs, trs))]
    b.close()
    for tr in trs:
        tr.close()
    return noisy, halves, refs


class DataSet:
    """Device-resident training pairs: features, demodulated radiance and
    remodulation planes of each noisy image, and its reference radiance."""

    def __init__(self, gpu: Gpu, count: int, size: int):
        import torch

        self.gpu, self.size, self.n = gpu, size, 0
        dev = "cuda"
        self.feat = torch.empty((count, size, size, 16), dtype=torch.bfloat16, device=dev)
        self.irr = torch.empty((count, size, size, 3), dtype=torch.float32, device=dev)
        self.alb = torch.empty((count, size, size, 3), dtype=torch.float32, device=dev)
        self.ref = torch.empty((count, size, size, 3), dtype=torch.float32, device=dev)
        self.spp = np.zeros(count, np.int32)
        self.bad = 0

    def add(self, noisy_px: np.ndarray, half: np.ndarray | None, ref_rad: np.ndarray, spp: int) -> None:
        """Appends one pair (`half`: the part-way snapshot, or None); a
        reference pixel that is not finite becomes 0 (counted in ``self.bad``)."""
        import torch

        fin = np.isfinite(ref_rad)
        if not fin.all():
            self.bad += int((~fin).sum())
            ref_rad = np.where(fin, ref_rad, 0.0)

        i, s = self.n, self.size
        buf = GpuArray.from_(self.gpu, noisy_px)
        hbuf = GpuArray.from_(self.gpu, np.ascontiguousarray(half, np.float32)) if half is not None else None
        features(self.gpu, buf, s, s, s, s, self.feat[i], self.irr[i], self.alb[i], half=hbuf)
        self.ref[i].copy_(torch.from_numpy(np.ascontiguousarray(ref_rad, dtype=np.float32)))
        self.gpu.wait()
        buf.free()
        if hbuf is not None:
            hbuf.free()
        self.spp[i] = spp
        self.n += 1

    def nonfinite(self) -> dict:
        """Count of values that are not finite in each device plane."""
        import torch

        return {k: int((~torch.isfinite(getattr(self, k)[:self.n].float())).sum().item())
                for k in ("feat", "irr", "alb", "ref")}

    def weights(self, spp_bias: float) -> np.ndarray | None:
        """Pair probabilities proportional to spp ** spp_bias (None: uniform).
        The loss of a low-spp pair is many times that of a high-spp one, so
        under uniform draws the few-sample images dominate the gradient; a
        positive bias draws the many-sample images more often."""
        if spp_bias == 0.0:
            return None
        w = self.spp[:self.n].astype(np.float64) ** spp_bias
        return w / w.sum()

    def batch(self, rng, B: int, crop: int, p: np.ndarray | None = None):
        """B random crops (random flips and transposes) as contiguous tensors;
        `p`: pair probabilities (``weights``), or None for uniform draws."""
        import torch

        idx = rng.integers(0, self.n, B) if p is None else rng.choice(self.n, B, p=p)
        s = self.size
        outs = [[], [], [], []]
        for i in idx:
            y0, x0 = (int(v) for v in rng.integers(0, s - crop + 1, 2))
            parts = [t[int(i), y0:y0 + crop, x0:x0 + crop] for t in (self.feat, self.irr, self.alb, self.ref)]
            if rng.random() < 0.5:
                parts = [torch.flip(p, (1,)) for p in parts]
            if rng.random() < 0.5:
                parts = [torch.flip(p, (0,)) for p in parts]
            if rng.random() < 0.5:
                parts = [p.transpose(0, 1) for p in parts]
            for o, p in zip(outs, parts):
                o.append(p)
        return [torch.stack(o).contiguous() for o in outs]


def _scene(i: int, size: int):
    return scenes.procedural(i, width=size, height=size)


def scene_stream(indices, size: int, workers: int):
    """Procedural scenes in order, generated ahead on `workers` host
    processes (spawned, so no CUDA state is inherited) while the GPU renders."""
    indices = list(indices)
    if workers <= 1:
        for i in indices:
            yield _scene(i, size)
        return
    import concurrent.futures as cf
    import multiprocessing as mp

    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        ahead = 2 * workers
        futs = [ex.submit(_scene, i, size) for i in indices[:ahead]]
        for k in range(len(indices)):
            if k + ahead < len(indices):
                futs.append(ex.submit(_scene, indices[k + ahead], size))
            yield futs[k].result()
            futs[k] = None


GROUP = 16  # scenes rendered together in one batch launch
DROP_HALF = 0.15  # share of training pairs given no part-way snapshot


def build_data(gpu: Gpu, indices, size: int, segments, ref_spp: int, log=print, workers: int = 0,
               keep: bool = True):
    """The data set of the scenes `indices`; with keep, also every scene's
    reference radiance and noisy px images on the host (8.9 MB an image at
    256 x 256: pass keep=False for large sets)."""
    indices = list(indices)
    ds = DataSet(gpu, len(indices) * len(segments), size)
    refs, noisy_all = [], []
    t0 = time.time()
    if workers <= 0:
        import os

        workers = max(1, min(8, (os.cpu_count() or 2) - 1))
    group = []

    drop = np.random.default_rng(12345)
    done = [0]

    def flush():
        noisy_g, halves_g, refs_g = render_group(gpu, group, segments, ref_spp)
        for noisy, halves, ref in zip(noisy_g, halves_g, refs_g):
            rr = radiance(ref, size, size)
            for spp, px, half in zip(segments, noisy, halves):
                # some pairs go without the snapshot, so the network also
                # serves callers that have none
                ds.add(px, None if drop.random() < DROP_HALF else half, rr, spp)
            if keep:
                refs.append(rr)
                noisy_all.append(noisy)
        done[0] += len(group)
        group.clear()
        log(f"rendered {done[0]}/{len(indices)} scenes ({time.time() - t0:.1f} s)")

    for sc in scene_stream(indices, size, workers):
        group.append(sc)
        if len(group) == GROUP:
            flush()
    if group:
        flush()
    return ds, refs, noisy_all


def world() -> tuple[int, int]:
    """(rank, world size) of the initialised process group, else (0, 1)."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(indices, rank: int, size: int) -> list:
    """The scenes one data-parallel rank renders: every size-th from its rank
    (disjoint, together all of them)."""
    return list(indices)[rank::size]


def average_grads(t, size: int) -> None:
    """In-place all-reduce average of a gradient tensor over the process
    group: NCCL's AVG where the backend has it, else a sum and a division."""
    import torch.distributed as dist

    if size <= 1:
        return
    if dist.get_backend() == "nccl":
        dist.all_reduce(t, op=dist.ReduceOp.AVG)
    else:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        t.div_(size)


def train(gpu: Gpu, ds: DataSet, steps: int, batch: int, crop: int, lr: float, seed: int = 1, log=print,
          err_weight: float = 0.1, init: np.ndarray | None = None, spp_bias: float = 0.0) -> tuple[Unet, list]:
    """Adam with a 200-step warm-up and a cosine decay; `init`: starting
    parameters (fine-tuning), else the seeded initialisation; `spp_bias`:
    see ``DataSet.weights``. Under an initialised process group each rank
    draws its crops from its own data set, and the gradient arena is
    averaged across ranks before every Adam step: every rank holds the same
    weights throughout (same start, same averaged gradients, same update)."""
    import torch

    rank, size = world()
    net = Unet(gpu, seed=seed, params=init)
    rng = np.random.default_rng(seed + 7919 * rank)
    p = ds.weights(spp_bias)
    loss = torch.zeros(1, dtype=torch.float32, device=f"cuda:{gpu.ordinal}")
    arena = net.grad_tensor() if size > 1 else None
    hist, acc, t0 = [], 0, time.time()
    for step in range(steps):
        warm = min(1.0, (step + 1) / 200)
        rate = lr * warm * 0.5 * (1.0 + math.cos(math.pi * step / steps))
        f, i, a, r = ds.batch(rng, batch, crop, p)
        if arena is None:
            net.train_step(f, i, a, r, batch, crop, crop, crop, crop, loss, rate, err_weight)
        else:
            # the network's stream is torch's current one, so the collective
            # follows the gradients and the Adam step follows the collective
            net.compute_grads(f, i, a, r, batch, crop, crop, crop, crop, loss, err_weight)
            average_grads(arena, size)
            net.adam(rate)
        acc += 1
        if (step + 1) % 100 == 0 or step + 1 == steps or (step < 100 and (step + 1) % 10 == 0):
            gpu.wait()
            v = float(loss.item()) / acc
            if not math.isfinite(v):
                raise FloatingPointError(f"training loss became {v} by step {step + 1}")
            hist.append((step + 1, v))
            log(f"step {step + 1}: loss {v:.5f} lr {rate:.2e} ({time.time() - t0:.1f} s)")
            loss.zero_()
            acc = 0
    gpu.wait()
    return net, hist


def evaluate(gpu: Gpu, net: Unet, noisy_px: np.ndarray, ref_rad: np.ndarray, w: int, h: int, half=None) -> dict:
    """relMSE against the reference of the noisy image, the a-trous Denoise,
    and the learned denoiser without and with the per-tile fallback at a few
    thresholds (with the share of tiles that kept the a-trous result)."""
    out = {"noisy": relmse(radiance(noisy_px, w, h), ref_rad)}
    buf = GpuArray.from_(gpu, noisy_px)
    hbuf = GpuArray.from_(gpu, np.ascontiguousarray(half, np.float32)) if half is not None else None
    kernels.denoise(gpu, buf, w, h)
    out["denoise"] = relmse(radiance(buf.read(np.uint32), w, h), ref_rad)
    tiles = ((w + TILE - 1) // TILE) * ((h + TILE - 1) // TILE)
    for name, thr in [("learned", 1e30)] + [(f"fallback_{t:g}", t) for t in (0.02, 0.05, 0.1, 0.2, 0.5)]:
        buf.write(noisy_px)
        kept = net.denoise_px(buf, w, h, half=hbuf, tile=TILE, threshold=thr, count=True)
        out[name] = relmse(radiance(buf.read(np.uint32), w, h), ref_rad)
        if name != "learned":
            out[name + "_tiles"] = kept / tiles
    buf.free()
    if hbuf is not None:
        hbuf.free()
    return out


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--scenes", type=int, default=160)
    ap.add_argument("--eval-scenes", type=int, default=8)
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--segments", default="1,2,4,4,8,16")
    ap.add_argument("--ref-spp", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--crop", type=int, default=128)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--first-scene", type=int, default=0, help="index of the first procedural scene")
    ap.add_argument("--init", default="", help="weights to fine-tune from (.phxu)")
    ap.add_argument("--spp-bias", type=float, default=0.0, help="draw pairs with probability ~ spp ** bias")
    ap.add_argument("--eval-ref-spp", type=int, default=4096, help="samples of the held-out references")
    ap.add_argument("--out", default="")
    ap.add_argument("--report", default="")
    args = ap.parse_args(argv)

    import os

    import torch

    size = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if size > 1:
        # data parallel, one process per GPU (torchrun): each rank renders its
        # share of the scenes; gradients are averaged over NCCL every step
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    rank, size = world()
    gpu = Gpu(local)
    gpu.set_stream(torch.cuda.current_stream().cuda_stream)
    segments = [int(s) for s in args.segments.split(",")]
    t0 = time.time()
    mine = shard(range(args.first_scene, args.first_scene + args.scenes), rank, size)
    ds, _, _ = build_data(gpu, mine, args.size, segments, args.ref_spp, keep=False,
                          log=print if rank == 0 else (lambda *a: None))
    t_data = time.time() - t0
    print("non-finite values in the data set:", ds.nonfinite(), "in references (zeroed):", ds.bad)
    t0 = time.time()
    init = read_weights(args.init) if args.init else None
    net, hist = train(gpu, ds, args.steps, args.batch, args.crop, args.lr, args.seed, init=init,
                      spp_bias=args.spp_bias)
    t_train = time.time() - t0
    lockstep = True
    if size > 1:
        # every rank must hold the same weights: compare a checksum of each
        import torch.distributed as dist

        mine_sum = torch.tensor([float(np.sum(net.params(), dtype=np.float64))], dtype=torch.float64,
                                device=f"cuda:{local}")
        sums = [torch.zeros_like(mine_sum) for _ in range(size)]
        dist.all_gather(sums, mine_sum)
        lockstep = all(float(x.item()) == float(sums[0].item()) for x in sums)
        if rank != 0:
            net.close()
            gpu.close()
            dist.destroy_process_group()
            return
    if args.out:
        net.save(args.out)
    held = range(100000, 100000 + args.eval_scenes)
    rows = []
    for i in held:
        sc = scenes.procedural(i, width=args.size, height=args.size)
        noisy, halves, refs = render_group(gpu, [sc], [4], args.eval_ref_spp)
        rows.append(evaluate(gpu, net, noisy[0][0], radiance(refs[0], args.size, args.size), args.size, args.size,
                             halves[0][0]))
    mean = {k: float(np.mean([r[k] for r in rows])) for k in rows[0]}
    report = {"scenes": args.scenes, "first_scene": args.first_scene, "ranks": size, "ranks_in_lockstep": lockstep,
              "pairs_rank0": ds.n, "nonfinite_ref_values": ds.bad,
              "segments": segments, "ref_spp": args.ref_spp, "eval_ref_spp": args.eval_ref_spp,
              "init": args.init or None, "spp_bias": args.spp_bias, "lr": args.lr, "steps": args.steps, "batch": args.batch, "crop": args.crop, "data_s": round(t_data, 1),
              "train_s": round(t_train, 1), "loss": hist, "heldout_4spp_relmse": mean, "heldout_rows": rows}
    print(json.dumps({k: v for k, v in report.items() if k not in ("loss", "heldout_rows")}))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    net.close()
    gpu.close()
    if size > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
