"""Multi-GPU batch sharding on the CPU: the longest-processing-time placement
(qsm_batch_partition, host only) and the split -> solve -> host gather of
qsmgpu.shard.tv_admm_sharded with two gloo ranks.  Inside these tests each rank's
per-volume solve is the float64 oracle TV-ADMM (src/inversion/tv.rs:63-97) on tiny
volumes, so the split and the gather run without a GPU; on GPUs the same function solves
each share with inversion.tv_admm_batch."""
import math
import multiprocessing as mp
import os
import socket
import traceback

import numpy as np
import pytest

from qsmgpu import Grid, QsmError, shard
from qsmgpu.inversion import TvParams
from oracle import qsm_oracle as O


def lpt(costs, m):
    order = sorted(range(len(costs)), key=lambda b: -costs[b])  # stable: ties in batch order
    load = [0.0] * m
    part = [0] * len(costs)
    for b in order:
        k = min(range(m), key=lambda i: (load[i], i))
        part[b] = k
        load[k] += costs[b]
    return part, load


def cost(g: Grid, iters=1):
    n = g.nx * g.ny * g.nz
    return n * math.log2(n + 2.0) * iters


def random_grids(seed, n):
    rng = np.random.default_rng(seed)
    return [Grid.new(int(rng.integers(64, 225)), int(rng.integers(64, 225)), int(rng.integers(48, 161)))
            for _ in range(n)]


@pytest.mark.parametrize("seed,n,m", [(0, 32, 2), (1, 32, 4), (2, 32, 8), (3, 5, 8), (4, 1, 3), (5, 17, 3)])
def test_partition_is_lpt(seed, n, m):
    grids = random_grids(seed, n)
    part, load = shard.partition(grids, m)
    want_part, want_load = lpt([cost(g) for g in grids], m)
    assert part == want_part
    np.testing.assert_allclose(load, want_load, rtol=1e-12)
    # the LPT bound: makespan <= (4/3 - 1/(3m)) OPT, with OPT >= max(mean load, largest volume)
    opt_lb = max(sum(load) / m, max(cost(g) for g in grids))
    assert max(load) <= (4.0 / 3.0 - 1.0 / (3 * m)) * opt_lb * (1 + 1e-12) or max(load) == max(cost(g) for g in grids)
    if n >= m:
        assert sorted(set(part)) == list(range(m))


def test_partition_weights_iterations_and_ties():
    g = Grid.new(32, 32, 32)
    part, load = shard.partition([g, g, g, g], 2)
    assert part == [0, 1, 0, 1]  # equal costs: batch order, lowest part first
    part, load = shard.partition([g, g, g], 2, iterations=[10, 250, 10])
    assert part == [1, 0, 1]
    assert shard.share([g, g, g], 1, 2, [10, 250, 10]) == [0, 2]


def test_partition_rejects_bad_arguments():
    with pytest.raises(QsmError):
        shard.partition([Grid.new(8, 8, 8)], 0)
    with pytest.raises(QsmError):
        shard.partition([Grid.new(8, 0, 8)], 2)
    assert shard.partition([], 3) == ([], [0.0, 0.0, 0.0])


def tiny_cases(seed=11, n=6):
    rng = np.random.default_rng(seed)
    cases = []
    for _ in range(n):
        dims = tuple(int(v) for v in rng.integers(6, 13, 3))
        grid = Grid.new(*dims)
        nz, ny, nx = grid.shape
        z, y, x = np.ogrid[:nz, :ny, :nx]
        mask = ((((x - (nx - 1) / 2) / (0.45 * nx)) ** 2 + ((y - (ny - 1) / 2) / (0.45 * ny)) ** 2 +
                 ((z - (nz - 1) / 2) / (0.45 * nz)) ** 2) < 1).astype(np.uint8)
        field = rng.normal(0.0, 0.02, grid.shape) * mask
        th = rng.uniform(0, 0.4)
        cases.append((np.ascontiguousarray(field), mask, grid, (math.sin(th), 0.0, math.cos(th))))
    return cases


def oracle_solve(sub, params):
    chis, iters = [], []
    for f, m, g, b in sub:
        chi, it = O.tv_admm(f, m, O.Grid(g.dims, g.voxel_size), b,
                            O.TvParams(params.lambda_, params.rho, params.tol, params.max_iter), return_iters=True)
        chis.append(chi)
        iters.append(it)
    return chis, iters


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir, fail_rank):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    res = {"rank": rank}
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=8))
        cases = tiny_cases()
        params = TvParams(2e-4, 2e-2, 1e-3, 40)

        def solve(sub, p):
            if rank == fail_rank:
                raise RuntimeError("injected solver failure")
            return oracle_solve(sub, p)

        chis, iters, mine = shard.tv_admm_sharded(cases, params, solve=solve)
        res["mine"] = mine
        if rank == 0:
            res["chis"] = chis
            res["iters"] = iters
        dist.destroy_process_group()
        res["status"] = "ok"
    except Exception as e:  # reported to the test, which decides
        res["status"] = "error"
        res["error"] = f"{type(e).__name__}: {e}"
        res["trace"] = traceback.format_exc()
    np.save(os.path.join(outdir, f"rank{rank}.npy"), np.array([res], dtype=object), allow_pickle=True)


def _run(world, tmp_path, fail_rank=-1, timeout=120):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path), fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
            pytest.fail("a rank did not finish")
    return [np.load(os.path.join(tmp_path, f"rank{r}.npy"), allow_pickle=True)[0] for r in range(world)]


def test_sharded_batch_two_gloo_ranks(tmp_path):
    res = _run(2, tmp_path)
    assert all(r["status"] == "ok" for r in res), [r.get("trace") for r in res]
    cases = tiny_cases()
    mine0, mine1 = res[0]["mine"], res[1]["mine"]
    assert sorted(mine0 + mine1) == list(range(len(cases))) and not set(mine0) & set(mine1)
    assert mine0 == shard.share([c[2] for c in cases], 0, 2, [40] * len(cases))
    want, want_it = oracle_solve(cases, TvParams(2e-4, 2e-2, 1e-3, 40))
    for got, ref in zip(res[0]["chis"], want):
        np.testing.assert_array_equal(got, ref)
    assert res[0]["iters"] == want_it


def test_sharded_batch_rank_failure_is_reported(tmp_path):
    """A rank whose solve raises leaves before the gather; the gathering rank's short
    process-group timeout turns the wait into an error instead of a hang."""
    res = _run(2, tmp_path, fail_rank=1)
    assert res[1]["status"] == "error" and "injected" in res[1]["error"]
    assert res[0]["status"] == "error"
