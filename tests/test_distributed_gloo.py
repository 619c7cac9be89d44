"""Multi-process node partition on CPU (gloo, world size 2): local submeshes,
local mass weights and partial k-spaces summed with gather_data equal the
single-process result.  The compute runs in the oracle (no GPU here); the
decomposition and the reduction are the product code under test."""
import os
import socket

import numpy as np
import pytest
import scipy.sparse as sp
import torch.multiprocessing as mp

from feelmri_b200 import workloads as W
from feelmri_b200.distributed import distribute_mesh, gather_data, partition_elements


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _local_kspace(mesh_elems, mesh_nodes, traj, Mxy_global, l2g=None):
    import oracle
    from oracle import fp64
    from feelmri_b200.Assemble import tabulate_at_quadrature
    from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
    qw, tab = tabulate_at_quadrature(FiniteElement(), QuadratureRule(order=2), np.float64)
    indptr, indices, data = oracle.mass_csc(mesh_elems, mesh_nodes, qw, tab)
    w = oracle.csc_rowsum(indptr, indices, data)
    N = mesh_nodes.shape[0]
    Mxy = Mxy_global if l2g is None else Mxy_global[l2g]
    T2 = np.full(N, 80.0)
    phi = np.zeros(N)
    return fp64.signal(sp.diags(w).tocsc(), *traj.points, traj.t, mesh_nodes, phi, T2, Mxy)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh = W.cylinder(1500)
        traj = W.cartesian(res=(6, 5, 2))
        rng = np.random.default_rng(0)
        Mxy = (rng.normal(size=(mesh.n_nodes, 2)) + 1j * rng.normal(size=(mesh.n_nodes, 2)))
        loc = distribute_mesh(mesh.elems, mesh.nodes, world, rank)
        K = _local_kspace(loc.elems, loc.nodes, traj, Mxy, loc.local_to_global)
        total = gather_data(K)
        if rank == 0:
            q.put(("total", total, loc.nodes.shape[0]))
        else:
            q.put(("local", None, loc.nodes.shape[0]))
    finally:
        dist.destroy_process_group()


def test_partition_covers_every_element_once():
    mesh = W.cylinder(2000)
    part = partition_elements(mesh.elems, mesh.nodes, 3)
    assert set(np.unique(part)) == {0, 1, 2}
    locs = [distribute_mesh(mesh.elems, mesh.nodes, 3, r, part) for r in range(3)]
    assert sum(l.elems.shape[0] for l in locs) == mesh.elems.shape[0]
    # nodes on part boundaries are shared (sum of local counts exceeds the total)
    assert sum(l.nodes.shape[0] for l in locs) > mesh.n_nodes
    for l in locs:
        np.testing.assert_array_equal(l.nodes, mesh.nodes[l.local_to_global])
        np.testing.assert_array_equal(mesh.elems[l.element_ids], l.local_to_global[l.elems])


@pytest.mark.timeout(240)
def test_two_rank_gather_equals_single_process():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=200) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    total = next(r[1] for r in results if r[0] == "total")
    mesh = W.cylinder(1500)
    traj = W.cartesian(res=(6, 5, 2))
    rng = np.random.default_rng(0)
    Mxy = (rng.normal(size=(mesh.n_nodes, 2)) + 1j * rng.normal(size=(mesh.n_nodes, 2)))
    ref = _local_kspace(mesh.elems, mesh.nodes, traj, Mxy)
    from oracle import fp64
    assert fp64.rel_l2(total, ref) < 1e-12
