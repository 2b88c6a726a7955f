"""Multi-rank host logic on CPU (gloo, world size 2): sharded runs with global
particle ids reproduce the unsharded run particle by particle, and the observable
sums all-reduced over ranks equal the single-process sums."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_pkg

N_TOTAL, STEPS = 3001, 40


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _workload():
    pkg = load_pkg()
    wl = pkg.workloads.bjorken(N=N_TOTAL, precision="fp64", steps=STEPS)
    return pkg, wl


def _run_block(orc, pkg, wl, first, count):
    from helpers import oracle_medium
    P = orc.make_params(**dict(wl.params, particle_offset=first))
    md = oracle_medium(orc, wl)
    x0, p0 = orc.initial_lab_boost(P, md, wl.x[:, first:first + count], wl.p[:, first:first + count])
    out = orc.run(P, md, x0, p0, wl.first_step, wl.steps, threads=1)
    return out["x"], out["p"]


def _rank_main(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from oracle import oracle as orc
    pkg, wl = _workload()
    first, count = pkg.sharding.shard(N_TOTAL, rank, world)
    x, p = _run_block(orc, pkg, wl, first, count)
    np.save(os.path.join(outdir, f"p{rank}.npy"), p)
    sums = torch.from_numpy(pkg.sharding.observable_sums(p, x, wl.params["m"], 2.0, 0.2))
    dist.all_reduce(sums)
    if rank == 0:
        np.save(os.path.join(outdir, "sums.npy"), sums.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_shard_sizes(lmb):
    s = lmb.sharding
    for n, w in ((10, 3), (3001, 2), (7, 7), (5, 8)):
        blocks = [s.shard(n, r, w) for r in range(w)]
        assert sum(c for _, c in blocks) == n
        assert all(blocks[r][0] + blocks[r][1] == blocks[r + 1][0] for r in range(w - 1))
        assert max(c for _, c in blocks) - min(c for _, c in blocks) <= 1
    with pytest.raises(ValueError):
        s.shard(10, 2, 2)


def test_two_gloo_ranks_match_single_process(lmb, orc, tmp_path):
    pkg, wl = _workload()
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    x_all, p_all = _run_block(orc, pkg, wl, 0, N_TOTAL)
    p_sharded = np.concatenate([np.load(tmp_path / "p0.npy"), np.load(tmp_path / "p1.npy")], axis=1)
    assert np.array_equal(p_sharded, p_all)          # identical per-particle noise whatever the sharding
    ref = pkg.sharding.observable_sums(p_all, x_all, wl.params["m"], 2.0, 0.2)
    np.testing.assert_allclose(np.load(tmp_path / "sums.npy"), ref, rtol=1e-12)
