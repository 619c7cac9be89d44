"""Node-partitioned multi-process simulation, one process per GPU.

Restates the reference's data-parallel decomposition:

* FEMPhantom.distribute_mesh (python/feelmri/Phantom.py:194-239): the
  elements are split into `world` parts, each rank keeps its elements and the
  sorted unique nodes they use (nodes on part boundaries appear on several
  ranks), renumbered locally.  The reference partitions the dual graph with
  pymetis; here elements are split into contiguous blocks after sorting their
  centroids along the longest axis, which needs no external library.  Any
  element partition gives the same total k-space: each element's mass lands
  on exactly one rank, and Signal is linear in the mass weights.
* gather_data (python/feelmri/MPIUtilities.py:13-26): the partial k-spaces
  of all ranks are summed onto rank 0 -- here torch.distributed.reduce (NCCL
  between GPUs, gloo on CPU) of the complex array viewed as real pairs.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class LocalMesh:
    elems: np.ndarray          # (E_local, nb) int32, local numbering
    nodes: np.ndarray          # (N_local, 3)
    local_to_global: np.ndarray  # (N_local,) global node ids (sorted)
    element_ids: np.ndarray    # (E_local,) global element ids


def partition_elements(elems: np.ndarray, nodes: np.ndarray, world: int) -> np.ndarray:
    """Part index (0..world-1) of every element: contiguous blocks of
    elements ordered by centroid along the mesh's longest extent."""
    if world <= 1:
        return np.zeros(elems.shape[0], np.int64)
    cent = nodes[elems].mean(axis=1)
    axis = int(np.argmax(nodes.max(axis=0) - nodes.min(axis=0)))
    order = np.argsort(cent[:, axis], kind="stable")
    part = np.empty(elems.shape[0], np.int64)
    for r, idx in enumerate(np.array_split(order, world)):
        part[idx] = r
    return part


def distribute_mesh(elems: np.ndarray, nodes: np.ndarray, world: int, rank: int,
                    membership: np.ndarray | None = None) -> LocalMesh:
    """The local submesh of `rank` (Phantom.py:209-236)."""
    if membership is None:
        membership = partition_elements(elems, nodes, world)
    cells = np.flatnonzero(membership == rank)
    local = elems[cells]
    l2g = np.unique(local.ravel())
    g2l = -np.ones(nodes.shape[0], np.int64)
    g2l[l2g] = np.arange(l2g.size)
    local = g2l[local.ravel()].reshape(-1, elems.shape[1]).astype(np.int32)
    return LocalMesh(local, nodes[l2g], l2g, cells)


def reduce_device(backend: str, tensor, current_cuda: int | None = None):
    """Device the reduce buffer must live on: NCCL reduces CUDA tensors only,
    so host data goes to the current CUDA device; other backends reduce
    where the data is."""
    import torch
    if backend == "nccl" and tensor.device.type != "cuda":
        idx = torch.cuda.current_device() if current_cuda is None else current_cuda
        return torch.device("cuda", idx)
    return tensor.device


def gather_data(data, group=None, dst: int = 0):
    """Sum of `data` over all ranks, delivered on rank `dst` (other ranks
    get their input back unchanged, as MPI Reduce leaves them).  `data` is a
    numpy array or a torch tensor (host or device); complex values are
    reduced as (re, im) pairs.  With the NCCL backend host data is reduced
    through a buffer on the current CUDA device and returned on the host."""
    import torch
    import torch.distributed as dist
    is_np = isinstance(data, np.ndarray)
    t = torch.from_numpy(np.ascontiguousarray(data)) if is_np else data.contiguous()
    home = t.device
    buf = torch.view_as_real(t) if t.is_complex() else t
    buf = buf.to(reduce_device(dist.get_backend(group), buf), copy=True)
    dist.reduce(buf, dst=dst, op=dist.ReduceOp.SUM, group=group)
    if dist.get_rank(group) != dst:
        return data
    out = torch.view_as_complex(buf) if t.is_complex() else buf
    if out.device != home:
        out = out.to(home)
    return out.numpy() if is_np else out
