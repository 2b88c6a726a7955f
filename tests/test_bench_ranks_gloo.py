"""The benchmark's multi-rank host logic on CPU (gloo, world size 2): each rank takes
its block of global particle ids from sharding.shard (charm first, then bottom, as
bench.headline_workloads builds them), runs it (here on the CPU restatement in place
of the engine), and bench.reduce_over_ranks combines the ranks' figures: times by max,
executed particle-steps and observable sums by sum.  The result equals one process
running both ranks' shares."""
import os
import socket
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_TOTAL, STEPS = 2400, 60


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_figures(rank, world):
    sys.path.insert(0, ROOT)
    import bench
    pkg = bench.load_package()
    f = pkg.workloads.grid2p1_fields(nx=61, ny=61, nt=12, dx=0.3)
    wls = bench.headline_workloads(pkg, N_TOTAL, rank, world, precision="fp64", fields=f)
    for w in wls:
        w.steps = STEPS
    ids = [(int(w.params["particle_offset"]), w.n) for w in wls]
    _, executed, outs = bench.cpu_pass(wls, threads=1)
    sums = np.zeros(12)
    for w, o in zip(wls, outs):
        fo = o["fo_flag"] != 0
        sums += pkg.sharding.observable_sums(o["fo_mom"][:, fo], o["fo_pos"][:, fo], w.params["m"])
    return ids, {"pass_ms": 10.0 + rank, "executed": executed, "fo_sums": sums}


def _rank_main(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    ids, vals = _rank_figures(rank, world)
    agg = bench.reduce_over_ranks(vals, world, "cpu")
    np.save(os.path.join(outdir, f"ids{rank}.npy"), np.array(ids))
    if rank == 0:
        np.save(os.path.join(outdir, "agg.npy"), np.concatenate([[agg["pass_ms"], agg["executed"]], agg["fo_sums"]]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_and_reduce_like_one_process(tmp_path):
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    ids = [np.load(tmp_path / f"ids{r}.npy") for r in range(2)]
    blocks = sorted((int(a), int(n)) for r in ids for a, n in r)
    assert blocks[0][0] == 0 and sum(n for _, n in blocks) == N_TOTAL
    assert all(blocks[k][0] + blocks[k][1] == blocks[k + 1][0] for k in range(len(blocks) - 1))
    agg = np.load(tmp_path / "agg.npy")
    shares = [_rank_figures(r, 2) for r in range(2)]
    assert [list(map(tuple, i)) for i in ids] == [list(i) for i, _ in shares]
    assert agg[0] == 11.0                                  # max of the ranks' times
    assert agg[1] == sum(v["executed"] for _, v in shares)
    np.testing.assert_allclose(agg[2:], sum(v["fo_sums"] for _, v in shares), rtol=1e-12)
