"""Multi-GPU form of the search: replicas.  Images are independent units and the search has no exchange step, so N
GPUs run N independent encoders (one process per GPU) and a host-side router assigns whole images to ranks by their
area (largest first onto the least-loaded rank, the reference's GP_ENCODERS batch split, encoder/src/batch.cpp:1005-1029,
across GPUs instead of streams).  torch.distributed carries only the routing metadata and the results' summaries."""
import heapq


def assign(areas, world):
    """Image indices per rank: longest-processing-time greedy on the areas (deterministic: ties by index)."""
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in sorted(range(len(areas)), key=lambda k: (-areas[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + areas[i], r))
    return [sorted(v) for v in out]


def run(images, encode, rank, world, group=None, areas=None):
    """Encode this rank's share of `images` with `encode(i, image) -> summary` and gather every summary on every rank
    (index -> summary).

    Either every rank passes the full list of images, or the caller passes `areas` (luma samples per image, the same
    list on every rank) and each rank loads only the images `assign(areas, world)[rank]` names, the other entries of
    `images` being None.  A rank given None for one of its own images raises ValueError."""
    import torch.distributed as dist
    if areas is None:
        areas = [0 if im is None else im[0].shape[0] * im[0].shape[1] for im in images]
        if world > 1:
            sizes = [None] * world
            dist.all_gather_object(sizes, areas, group=group)
            areas = [max(v) for v in zip(*sizes)]
    mine = assign(areas, world)[rank]
    missing = [i for i in mine if images[i] is None]
    if missing:
        raise ValueError("rank %d was not given its images %s (see assign())" % (rank, missing[:8]))
    res = {i: encode(i, images[i]) for i in mine}
    if world == 1:
        return res
    parts = [None] * world
    dist.all_gather_object(parts, res, group=group)
    merged = {}
    for p in parts:
        merged.update(p)
    return merged
