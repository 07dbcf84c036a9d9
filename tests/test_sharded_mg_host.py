"""Sharded hp-multigrid on CPU: the V-cycle over sharded levels (damped Jacobi V(2,2), transfers
through owned-entry sums, replicated coarse Cholesky) against the oracle's V-cycle
(multigrid.jl:858-889 restated), in one process and as two gloo ranks, and CG preconditioned by
it against the oracle's PCG."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import grico_oracle as go
import grico_b200 as gb
from grico_b200.sharded import ShardedMultigrid, ShardedOperator, ShardGroup, sharded_cg
from sharded_cases import HostOps
from test_multigrid_host import CASES, _oracle_levels, _product_plan


def _pair(name):
    origin, extent, roots, refine, p, faces = CASES[name]
    od, pdm = go.Domain(origin, extent, roots), gb.Domain(origin, extent, roots)
    refine(od.grid)
    refine(pdm.grid)
    return _oracle_levels(od, p, faces), _product_plan(pdm, p, faces=faces)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("name", ["2d_p4", "3d_p2"])
def test_unsplit_sharded_vcycle_matches_oracle(name):
    oplans, plan = _pair(name)
    mg = ShardedMultigrid(plan, 0, 1, ops=HostOps(), device=False)
    assert [s.n_reduced for s in mg.shards] == [len(o.solve_dofs) for o in oplans]
    r = np.random.default_rng(2).standard_normal(plan.n_reduced)
    z = mg.apply(torch.from_numpy(r.copy())).numpy()[: plan.n_reduced]
    zr = go.Multigrid(oplans).apply(r)
    assert np.linalg.norm(z - zr) <= 1e-11 * np.linalg.norm(zr)


def _gloo_rank(rank, world, port, out, name):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        _, plan = _pair(name)
        ops = HostOps()
        mg = ShardedMultigrid(plan, rank, world, ops=ops, device=False, group=ShardGroup())
        assert mg._links is not None and len(mg._links) == len(mg.shards) - 1  # point-to-point transfers
        fine = mg.shards[-1]
        r = np.random.default_rng(2).standard_normal(plan.n_reduced)
        z = mg.apply(ops.upload(fine.scatter(r))).numpy()[: fine.n_reduced]
        b = np.random.default_rng(5).standard_normal(plan.n_reduced)
        op = ShardedOperator([fine], ShardGroup(), ops)
        xs, rep = sharded_cg(op, [ops.upload(fine.scatter(b))], 1e-10, preconditioner=mg)
        np.save(os.path.join(out, f"z{rank}.npy"), z)
        np.save(os.path.join(out, f"x{rank}.npy"), xs[0].numpy()[: fine.n_reduced])
        np.save(os.path.join(out, f"g{rank}.npy"), fine.global_reduced)
        np.save(os.path.join(out, f"it{rank}.npy"), np.array([rep.iterations, rep.status, fine.n_owned]))
        np.save(os.path.join(out, f"levels{rank}.npy"), np.array([s.n_owned for s in mg.shards]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("2d_p4", 2), ("3d_p2", 2), ("2d_p4", 3)])
def test_sharded_vcycle_and_pcg_gloo_ranks(tmp_path, name, world):
    """world_size 2 and 3 over gloo: every level split across the ranks, halos and transfers
    exchanged point to point between the ranks that share entries; the V-cycle of a residual
    and the GMG-preconditioned CG solution match the oracle's; each level's owned dofs
    partition it."""
    mp.start_processes(_gloo_rank, args=(world, _free_port(), str(tmp_path), name), nprocs=world, join=True,
                       start_method="spawn")
    oplans, plan = _pair(name)
    omg = go.Multigrid(oplans)
    r = np.random.default_rng(2).standard_normal(plan.n_reduced)
    zr = omg.apply(r)
    b = np.random.default_rng(5).standard_normal(plan.n_reduced)
    xr, iters = go.cg_solve(oplans[-1].reduced_apply, b, precond=omg.apply, rtol=1e-10)
    sizes = [len(o.solve_dofs) for o in oplans]
    owned = np.zeros(len(sizes), dtype=np.int64)
    its = set()
    for k in range(world):
        g = np.load(tmp_path / f"g{k}.npy")
        z = np.load(tmp_path / f"z{k}.npy")
        x = np.load(tmp_path / f"x{k}.npy")
        it, status, _ = np.load(tmp_path / f"it{k}.npy")
        owned += np.load(tmp_path / f"levels{k}.npy")
        assert status == 0
        its.add(int(it))
        assert np.max(np.abs(z - zr[g])) <= 1e-11 * np.max(np.abs(zr))
        assert np.max(np.abs(x - xr[g])) <= 1e-9 * np.max(np.abs(xr))
    assert owned.tolist() == sizes
    # damped Jacobi on the modal basis is a weak smoother (~260 iterations to 1e-10 in 3-D), so
    # the order of the halo sums shifts the stopping iteration by a few percent
    assert len(its) == 1 and abs(its.pop() - iters) <= max(1, iters // 8)


@pytest.mark.parametrize("name,parts", [("2d_p4", 3), ("3d_p2", 2)])
def test_transfer_lists_agree_between_ranks(name, parts):
    """The point-to-point transfer lists: each rank's local coarse set is its shard's; what rank
    r sends rank q (restriction shares, prolongation values) is exactly what q expects from r;
    and the CSR row gather equals a loop over the rows."""
    from grico_b200.multigrid import GeometricMultigridPreconditioner, build_hierarchy
    from grico_b200.sharded import ShardPlan, _csr_take, _reduced_sets, _TransferLinks

    _, plan = _pair(name)
    plans, transfers = build_hierarchy(plan, GeometricMultigridPreconditioner(), device=False)
    shards = [[ShardPlan(p, r, parts, device=False) for p in plans] for r in range(parts)]
    sets = [_reduced_sets(p, shards[0][i].cell_rank, parts) for i, p in enumerate(plans)]
    for i, p in enumerate(plans):
        for r in range(parts):
            assert np.array_equal(np.sort(shards[r][i].global_reduced), sets[i][0][r])
    moved = 0
    for i, (off, col, _) in enumerate(transfers):
        rows = np.arange(0, len(off) - 1, 3)
        assert np.array_equal(_csr_take(off, rows), np.concatenate([np.arange(off[g], off[g + 1]) for g in rows]))
        links = [_TransferLinks(r, parts, off, col, sets[i][0], sets[i][1], sets[i + 1][0], sets[i + 1][1],
                                np.asarray(shards[r][i].global_reduced, dtype=np.int64), "cpu") for r in range(parts)]
        for r, lk in enumerate(links):
            for q, sel, sb in lk.r_send:
                ids = lk.cols_own[sel.numpy()]
                peer = next(x for x in links[q].r_recv if x[0] == r)
                got = shards[q][i].global_reduced[peer[1].numpy()]
                assert np.array_equal(ids, got) and sb.numel() == peer[2].numel()
                moved += ids.size
            for q, pos, sb in lk.p_send:
                ids = shards[r][i].global_reduced[pos.numpy()]
                peer = next(x for x in links[q].p_recv if x[0] == r)
                assert np.array_equal(ids, links[q].need[peer[1].numpy()])
                moved += ids.size
        for r, lk in enumerate(links):  # and every expected receive has its send
            assert all(any(x[0] == r for x in links[q].r_send) for q, _, _ in lk.r_recv)
            assert all(any(x[0] == r for x in links[q].p_send) for q, _, _ in lk.p_recv)
    assert moved > 0
