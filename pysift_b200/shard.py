"""Sharding a batch over the GPUs of one node (one process per GPU).

The path needs no exchange step: images (detection) and pairs (stitching)
are independent units.  A batch is dealt to the ranks by
longest-processing-time greedy (units sorted by cost, largest first, each
to the rank with the least load so far; equal loads go to the lower rank),
every rank runs its share through the single-GPU batched path, and the
results can be gathered once at the end: the counts first, then the rows
padded to the longest share, with one all_gather each (NCCL over NVLink on
GPUs, gloo on the CPU).  There is no collective during the compute.

The reference has no multi-GPU path (pysift/core.py runs one device); this
module is the scale-out of its per-image and per-pair calls.
"""
import numpy as np


def lpt_assign(costs, n_ranks):
    """Indices of `costs` per rank, longest-processing-time greedy: units in
    decreasing cost (ties by index), each to the least-loaded rank (ties to
    the lower rank).  Every index appears once; each rank's list is in
    increasing index order."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * n_ranks
    share = [[] for _ in range(n_ranks)]
    for i in order:
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        load[r] += float(costs[i])
        share[r].append(i)
    return [sorted(s) for s in share]


def image_cost(shape):
    """Detection cost of an image: its pixel count."""
    return float(shape[0]) * float(shape[1])


def pair_cost(shape1, shape2):
    """Stitching cost of a pair: the pixels of both views."""
    return image_cost(shape1) + image_cost(shape2)


def gather_rows(local, n_total, group=None, device=None):
    """All-gather variable-length per-unit results.

    local: {unit index: 2-D tensor (rows, cols)} of this rank (same dtype and
    column count everywhere).  Returns, on every rank, the list of n_total
    tensors in unit order.  Two collectives: the per-unit row counts, then
    this rank's rows padded to the largest share."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    items = sorted(local.items())
    ref = items[0][1] if items else None
    if ref is not None:
        device = ref.device if device is None else device
    cols = int(ref.shape[1]) if ref is not None else 0
    dtype = ref.dtype if ref is not None else torch.float32
    # counts: rows per unit (-1 = not this rank's), as a dense vector
    counts = torch.full((n_total,), -1, dtype=torch.int64, device=device)
    for i, t in items:
        counts[i] = int(t.shape[0])
    meta = torch.tensor([cols, sum(int(t.shape[0]) for _, t in items)], dtype=torch.int64, device=device)
    all_counts = [torch.empty_like(counts) for _ in range(world)]
    all_meta = [torch.empty_like(meta) for _ in range(world)]
    dist.all_gather(all_counts, counts, group=group)
    dist.all_gather(all_meta, meta, group=group)
    cols = max(int(m[0]) for m in all_meta)
    longest = max(int(m[1]) for m in all_meta)
    rows = torch.zeros((max(longest, 1), cols), dtype=dtype, device=device)
    at = 0
    for _, t in items:
        rows[at:at + t.shape[0]] = t
        at += t.shape[0]
    all_rows = [torch.empty_like(rows) for _ in range(world)]
    dist.all_gather(all_rows, rows, group=group)
    out = [None] * n_total
    for r in range(world):
        c = all_counts[r].cpu().numpy()
        at = 0
        for i in np.nonzero(c >= 0)[0]:
            n = int(c[i])
            out[int(i)] = all_rows[r][at:at + n]
            at += n
    missing = [i for i, t in enumerate(out) if t is None]
    if missing:
        raise RuntimeError(f"gather_rows: units {missing[:8]} were on no rank")
    return out


def detect_sharded(sift, images, rank, world, group=None, n_streams=8, gather=True):
    """PySIFT.detect_batch over `world` ranks: this rank detects its LPT share
    of `images`; with gather=True every rank returns the whole batch's
    (keypoints (N, 4), descriptors (N, 128)) CUDA tensors in input order,
    else {index: (keypoints, descriptors)} of its own share."""
    share = lpt_assign([image_cost(im.shape) for im in images], world)[rank]
    res = sift.detect_batch([images[i] for i in share], n_streams=n_streams, gpu_output=True) if share else []
    mine = {i: r for i, r in zip(share, res)}
    if not gather or world == 1:
        return mine if not gather else [mine[i] for i in range(len(images))]
    kps = gather_rows({i: r[0] for i, r in mine.items()}, len(images), group=group, device=sift.device)
    dsc = gather_rows({i: r[1] for i, r in mine.items()}, len(images), group=group, device=sift.device)
    return list(zip(kps, dsc))


def stitch_sharded(stitcher, pairs, rank, world, n_streams=8):
    """GPUPyStitch.stitch_batch over `world` ranks: {pair index: panorama}
    of this rank's LPT share (panoramas are host images; no gather)."""
    share = lpt_assign([pair_cost(a.shape, b.shape) for a, b in pairs], world)[rank]
    panos = stitcher.stitch_batch([pairs[i] for i in share], n_streams=n_streams) if share else []
    return dict(zip(share, panos))
