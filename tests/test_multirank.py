"""Multi-rank host path on CPU (gloo, world size 2): each rank produces the
counts of its particle shard (p = rank mod nranks, as the reference strides
particles by MPI rank, src/RTMCphon.f90:1627), the counts are summed with
one all-reduce (the reference's MPI_Allreduce, :1587) and rank 0 assembles
kappa with ptg_kappa_from_counts.  The shard counts come from the oracle
(no GPU here); the all-reduced counts must equal the single-rank run's
exactly, because a trajectory depends only on its Philox counter."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import conftest  # noqa: F401  (loads the ptrans_b200 package in the spawned rank)
    import torch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from ptrans_b200 import abi as A
        from ptrans_b200 import synth
        from oracle import oracle as O
        m = synth.film_with_holes(lx=200.0, ly=200.0, lz=100.0, nholes=2, radius=30.0, seed=6)
        spec = synth.spectrum(8, seed=3, mfp_lo=5e-9, mfp_hi=2e-6)
        run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=5, np_=101, seed=9, rank=rank, nranks=world,
                         precision=A.PREC_FP64, nbins=4, bin_omega=(0.0, 15.0 * synth.THZ))
        counts, _, _ = O.Oracle(model=m, spectrum=spec).counts(run, threads=1)
        t = torch.from_numpy(counts.astype(np.int64))
        dist.all_reduce(t)
        if rank == 0:
            total = t.numpy().astype(np.uint64)
            full = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=5, np_=101, seed=9, precision=A.PREC_FP64,
                              nbins=4, bin_omega=(0.0, 15.0 * synth.THZ))
            k = A.kappa_from_counts(A.GeomBuf(m).view, spec, full, total)
            np.save(os.path.join(out_dir, "counts.npy"), total)
            np.save(os.path.join(out_dir, "kappa.npy"), np.array([k["kappa"], k["kappa_stderr"]]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_single_rank_run(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    from ptrans_b200 import abi as A
    from ptrans_b200 import synth
    from oracle import oracle as O
    m = synth.film_with_holes(lx=200.0, ly=200.0, lz=100.0, nholes=2, radius=30.0, seed=6)
    spec = synth.spectrum(8, seed=3, mfp_lo=5e-9, mfp_hi=2e-6)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=5, np_=101, seed=9, precision=A.PREC_FP64,
                     nbins=4, bin_omega=(0.0, 15.0 * synth.THZ))
    o = O.Oracle(model=m, spectrum=spec)
    single, _, _ = o.counts(run, threads=1)
    np.testing.assert_array_equal(np.load(tmp_path / "counts.npy"), single)
    ref = o.kappa(run, single)
    k = np.load(tmp_path / "kappa.npy")
    assert abs(k[0] - ref["kappa"]) <= 1e-12 * abs(ref["kappa"])


def test_bench_launcher_starts_the_ranks(tmp_path):
    """bench.py --gpus N, when no launcher set WORLD_SIZE, starts N ranks
    itself with the environment torchrun would give them; here the ranks are
    a gloo probe: they join one process group of N and all-reduce."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    out = tmp_path / "probe.json"
    probe = os.path.join(root, "tests", "rank_probe.py")
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    old = dict(os.environ)
    try:
        os.environ.clear()
        os.environ.update(env)
        rc = bench.spawn_ranks(3, probe, [str(out)], timeout_s=120)
    finally:
        os.environ.clear()
        os.environ.update(old)
    assert rc == 0
    import json
    got = json.load(open(out))
    assert got == {"world": 3, "sum": 6, "local_rank": 0, "master": "127.0.0.1"}
