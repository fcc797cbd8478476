"""get_table over several GPUs, one process per GPU.

The grid's (size, wavelength) cells are independent until the shape
average, which reduces over the shapes of one cell (ShapeAveragingTask,
ShapeAveragingTask.hpp:127-166); CosTuuM's TaskManager builds one task
graph over the whole grid (TaskManager.hpp:445-1346). Here every rank
computes the full composition x wavelength x shape grid for its own subset
of the sizes, so each cell stays on one GPU and no exchange is needed until
the results are gathered. Sizes are dealt round robin over the ranks in
ascending order: the cost of a cell grows steeply with the size parameter,
and interleaving gives every rank a similar mix of small and large grains.

Each rank's cells are computed exactly as in a one-process get_table (the
per-grain schedule, kernels and reductions do not depend on the other
grains of a batch), so the gathered table equals the one-process table bit
for bit.
"""
import numpy as np

from . import CosTuuM


def size_shard(nsizes, world, rank):
    """Indices (into the ascending sizes) that rank computes."""
    return np.arange(rank, nsizes, world)


def merge_shards(parts, nsizes, world, size_axis):
    """Place each rank's sub-table (sizes along size_axis) at its sizes."""
    first = parts[0]
    shape = list(first.shape)
    shape[size_axis] = nsizes
    out = np.zeros(shape, first.dtype)
    for rank, part in enumerate(parts):
        idx = size_shard(nsizes, world, rank)
        sl = [slice(None)] * len(shape)
        sl[size_axis] = idx
        out[tuple(sl)] = part
    return out


def get_table(types, sizes, wavelengths, thetas, shape_distribution,
              alignment_distribution, dust_properties, group=None, **kwargs):
    """CosTuuM.get_table on every rank of torch.distributed's group, each on
    its own sizes; every rank returns the whole table (and, with
    return_status=True, the status array), unsqueezed: [type, size,
    wavelength, theta, k] and/or [type, size, wavelength, theta, 2 theta, 4,
    4]. The process group must be initialised (NCCL with one GPU per rank,
    or gloo); each rank computes on its current CUDA device's context
    (kwargs["context"], else the default context)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    types = np.atleast_1d(np.asarray(types))
    sizes = np.sort(np.atleast_1d(np.asarray(sizes, np.float64)))
    lams = np.atleast_1d(np.asarray(wavelengths, np.float64))
    thetas = np.atleast_1d(np.asarray(thetas, np.float64))
    mine = sizes[size_shard(len(sizes), world, rank)]
    want_status = bool(kwargs.pop("return_status", False))
    do_abs = kwargs.get("do_absorption", True)
    do_ext = kwargs.get("do_extinction", False)
    do_sca = kwargs.get("do_scattering", False)
    nq = (2 if do_abs else 0) + (3 if do_ext else 0)
    nt, nl, nth = len(types), len(lams), len(thetas)
    nsh = len(shape_distribution.shapes)
    parts = {}
    if len(mine):
        res = CosTuuM.get_table(types, mine, lams, thetas, shape_distribution,
                                alignment_distribution, dust_properties,
                                return_status=True, **kwargs)
        res = res if isinstance(res, tuple) else (res,)
        k = 0
        ns = len(mine)
        if nq:
            parts["q"] = np.asarray(res[k]).reshape(nt, ns, nl, nth, nq)
            k += 1
        if do_sca:
            parts["z"] = np.asarray(res[k]).reshape(nt, ns, nl, nth, 2 * nth, 4, 4)
            k += 1
        parts["status"] = np.asarray(res[k]).reshape(nt, ns, nl, nsh)
    else:
        if nq:
            parts["q"] = np.zeros((nt, 0, nl, nth, nq))
        if do_sca:
            parts["z"] = np.zeros((nt, 0, nl, nth, 2 * nth, 4, 4))
        parts["status"] = np.zeros((nt, 0, nl, nsh), np.int32)
    gathered = [None] * world
    dist.all_gather_object(gathered, parts, group=group)
    out = []
    if nq:
        out.append(merge_shards([g["q"] for g in gathered], len(sizes), world, 1))
    if do_sca:
        out.append(merge_shards([g["z"] for g in gathered], len(sizes), world, 1))
    if want_status:
        out.append(merge_shards([g["status"] for g in gathered], len(sizes), world, 1))
    return out[0] if len(out) == 1 else tuple(out)
