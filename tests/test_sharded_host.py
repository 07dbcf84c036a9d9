"""Sharded plans on CPU: partition, local numbering, halo slots, the sharded apply and CG against
the unsharded oracle, in one process and as two gloo ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import grico_b200 as gb
from grico_b200.sharded import ShardedOperator, ShardGroup, ShardPlan, cell_ranks, gather_reduced, sharded_cg
from sharded_cases import HostOps, global_cg, poisson, reduced_apply


def _plan(*a, **k):
    return gb.compile(poisson(*a, **k), device=False)


def test_partition_is_contiguous_and_balanced():
    plan = _plan(2, (4, 4), 2, rounds=1)
    for parts in (1, 2, 3, 5):
        r = cell_ranks(plan, parts)
        assert np.all(np.diff(r) >= 0) and set(r.tolist()) == set(range(parts))
        counts = np.bincount(r)
        assert counts.max() - counts.min() <= 1  # uniform work: equal cell counts up to one
    with pytest.raises(ValueError):
        cell_ranks(plan, 65)


@pytest.mark.parametrize("parts", [2, 3, 4])
def test_shards_cover_each_reduced_dof_once(parts):
    plan = _plan(2, (4, 4), 2, rounds=1)
    shards = [ShardPlan(plan, r, parts, device=False) for r in range(parts)]
    owned = np.concatenate([s.global_reduced[: s.n_owned] for s in shards])
    assert np.array_equal(np.sort(owned), np.arange(plan.n_reduced))
    # every ghost is owned by a lower rank and sits in a halo slot; slots agree across shards
    slot_of = {}
    for s in shards:
        ghosts = s.global_reduced[s.n_owned:]
        for g in ghosts:
            owner = next(t for t in shards if g in set(t.global_reduced[: t.n_owned]))
            assert owner.rank < s.rank
        assert set(ghosts) <= set(s.global_reduced[s.halo_local])
        for loc, slot in zip(s.halo_local, s.halo_slot):
            g = int(s.global_reduced[loc])
            assert slot_of.setdefault(int(slot), g) == g
    assert len(slot_of) == shards[0].n_halo


def test_local_maps_match_global_maps_with_hanging_terms():
    """Multi-term (hanging-node) entries: every local cell's map, read through the local->global
    dof table, is the global map of that cell, tail rows included."""
    plan = _plan(2, (2, 1), 2, extent=(2.0, 1.0), refine=lambda g: g.refine(2, 2))
    assert any(b.tail_offsets is not None for b in plan.batches)

    def expanded(b, c, glob=None):
        nb = b.nbox
        out = []
        for i in range(nb):
            e = int(b.map_index[c * nb + i])
            if e >= 0:
                out.append([(int(e if glob is None else glob[e]), 1.0 if b.map_coef is None else b.map_coef[c * nb + i])])
            elif e == -1:
                out.append([])
            else:
                k = -e - 2
                rows = range(b.tail_offsets[k], b.tail_offsets[k + 1])
                out.append([(int(b.tail_index[t] if glob is None else glob[b.tail_index[t]]), float(b.tail_coef[t]))
                            for t in rows])
        return out

    for parts in (2, 3):
        for r in range(parts):
            s = ShardPlan(plan, r, parts, device=False)
            for lb in s.plan.batches:
                gb_ = next(b for b in plan.batches if b.degree == lb.degree and b.q == lb.q)
                pos = {int(c): k for k, c in enumerate(gb_.cells)}
                for lc, cell in enumerate(lb.cells):
                    assert expanded(lb, lc, s.global_full) == expanded(gb_, pos[int(cell)])


@pytest.mark.parametrize("D,roots,p,parts", [(2, (4, 4), 3, 3), (3, (2, 2, 2), 2, 2)])
def test_sharded_apply_matches_unsharded(D, roots, p, parts):
    plan = _plan(D, roots, p, rounds=1, mass=0.5)
    shards = [ShardPlan(plan, r, parts, device=False) for r in range(parts)]
    ops = HostOps()
    op = ShardedOperator(shards, ShardGroup(), ops)
    x = np.random.default_rng(3).standard_normal(plan.n_reduced)
    ref = reduced_apply(plan, x)
    ys = [ops.vector(s.n_reduced) for s in shards]
    op.apply([ops.upload(s.scatter(x)) for s in shards], ys)
    for s, y in zip(shards, ys):
        assert np.max(np.abs(y.numpy()[: s.n_reduced] - ref[s.global_reduced])) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("jacobi", [True, False])
def test_sharded_cg_in_one_process_matches_unsharded(jacobi):
    plan = _plan(2, (4, 4), 3, rounds=1)
    b = np.random.default_rng(5).standard_normal(plan.n_reduced)
    xr, iters = global_cg(plan, b, 1e-10, jacobi=jacobi)
    shards = [ShardPlan(plan, r, 3, device=False) for r in range(3)]
    ops = HostOps()
    op = ShardedOperator(shards, ShardGroup(), ops)
    xs, rep = sharded_cg(op, [ops.upload(s.scatter(b)) for s in shards], 1e-10, jacobi=jacobi)
    assert rep.status == 0
    assert abs(rep.iterations - iters) <= 1
    x = gather_reduced(shards, xs, plan.n_reduced, ops)
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)
    # ghosts hold the owners' values
    for s, xv in zip(shards, xs):
        assert np.allclose(xv.numpy()[: s.n_reduced], x[s.global_reduced], rtol=0, atol=1e-14 * np.abs(x).max())


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        plan = _plan(2, (4, 4), 3, rounds=1)
        b = np.random.default_rng(5).standard_normal(plan.n_reduced)
        shard = ShardPlan(plan, rank, world, device=False)
        ops = HostOps()
        op = ShardedOperator([shard], ShardGroup(), ops)
        xs, rep = sharded_cg(op, [ops.upload(shard.scatter(b))], 1e-10, jacobi=True)
        x = xs[0].numpy()[: shard.n_reduced]
        np.save(os.path.join(out, f"x{rank}.npy"), x)
        np.save(os.path.join(out, f"g{rank}.npy"), shard.global_reduced)
        np.save(os.path.join(out, f"it{rank}.npy"), np.array([rep.iterations, rep.status, shard.n_owned]))
    finally:
        dist.destroy_process_group()


def test_sharded_cg_two_gloo_ranks(tmp_path):
    """world_size 2 over gloo: each process holds one shard; the halo and scalar sums cross
    processes; the solution matches the unsharded oracle PCG."""
    world = 2
    mp.start_processes(_gloo_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    plan = _plan(2, (4, 4), 3, rounds=1)
    b = np.random.default_rng(5).standard_normal(plan.n_reduced)
    xr, iters = global_cg(plan, b, 1e-10, jacobi=True)
    x = np.zeros(plan.n_reduced)
    its = set()
    for r in range(world):
        xl = np.load(tmp_path / f"x{r}.npy")
        g = np.load(tmp_path / f"g{r}.npy")
        it, status, n_owned = np.load(tmp_path / f"it{r}.npy")
        assert status == 0
        its.add(int(it))
        x[g[:n_owned]] = xl[:n_owned]
        assert np.allclose(xl, xr[g], rtol=0, atol=1e-9 * np.abs(xr).max())
    assert len(its) == 1 and abs(its.pop() - iters) <= 1
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)


def test_sharded_plan_rejects_point_items():
    d = gb.Domain((0.0, 0.0), (1.0, 1.0), (4, 4))
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(2)))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(0.0, 1.0))
    gb.add_boundary(prob, gb.BoundaryFace(1, gb.LOWER), gb.Nitsche(10.0))
    plan = gb.compile(prob, device=False)
    assert plan.point_batches
    with pytest.raises(gb.GricoError):
        ShardPlan(plan, 0, 2, device=False)


@pytest.mark.parametrize("D,roots,p,parts", [(2, (4, 4), 3, 4), (3, (2, 2, 2), 2, 3)])
def test_neighbour_lists_are_symmetric(D, roots, p, parts):
    """Rank r lists rank q with the dofs they share exactly when q lists r with the same dofs,
    in the same (ascending global) order; every shared dof of a rank is listed with each other
    rank that touches it."""
    plan = _plan(D, roots, p, rounds=1)
    shards = [ShardPlan(plan, r, parts, device=False) for r in range(parts)]
    shared = {}
    for s in shards:
        g = s.global_reduced[s.halo_local]
        for q, pos in s.neighbours:
            assert q != s.rank and np.all(np.diff(g[pos]) > 0)
            shared[(s.rank, q)] = g[pos]
        listed = np.concatenate([g[pos] for _, pos in s.neighbours]) if s.neighbours else np.zeros(0)
        assert set(listed.tolist()) == set(g.tolist())
    for (r, q), ids in shared.items():
        assert np.array_equal(shared[(q, r)], ids)
    assert any(len(s.neighbours) >= 2 for s in shards)


def _gloo_halo_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        plan = _plan(2, (4, 4), 3, rounds=1, mass=0.5)
        x = np.random.default_rng(3).standard_normal(plan.n_reduced)
        shard = ShardPlan(plan, rank, world, device=False)
        ops = HostOps()
        for mode in ("neighbours", "allreduce"):
            op = ShardedOperator([shard], ShardGroup(halo=mode), ops)
            y = ops.vector(shard.n_reduced)
            op.apply([ops.upload(shard.scatter(x))], [y])
            np.save(os.path.join(out, f"y_{mode}{rank}.npy"), y.numpy()[: shard.n_reduced])
        np.save(os.path.join(out, f"g{rank}.npy"), shard.global_reduced)
    finally:
        dist.destroy_process_group()


def test_neighbour_halo_exchange_four_gloo_ranks(tmp_path):
    """world_size 4 over gloo (ranks with two and three neighbours): the point-to-point halo sum
    gives the unsharded apply, every rank holds the same bits for a dof it shares, and it agrees
    with the all-reduce halo to rounding."""
    world = 4
    mp.start_processes(_gloo_halo_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    plan = _plan(2, (4, 4), 3, rounds=1, mass=0.5)
    x = np.random.default_rng(3).standard_normal(plan.n_reduced)
    ref = reduced_apply(plan, x)
    scale = np.max(np.abs(ref))
    seen = {}
    for r in range(world):
        g = np.load(tmp_path / f"g{r}.npy")
        yn = np.load(tmp_path / f"y_neighbours{r}.npy")
        ya = np.load(tmp_path / f"y_allreduce{r}.npy")
        assert np.max(np.abs(yn - ref[g])) <= 1e-13 * scale
        assert np.max(np.abs(yn - ya)) <= 1e-14 * scale
        for gi, v in zip(g.tolist(), yn.tolist()):
            assert seen.setdefault(gi, v) == v   # bitwise the same on every rank holding it
