"""N > 1 host logic on CPU with gloo (world_size 2): solves are sharded by
ParaRange with no exchange on the data path, each rank's results equal the
single-process results for the same solves, and timings aggregate as the
maximum over ranks.  The per-solve arithmetic here is the CPU oracle; the
GPU path shards the same way (bench.py)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from antelope_b200.dist import para_range


def test_para_range_partitions():
    for total in (0, 1, 7, 256):
        for size in (1, 2, 3, 8):
            blocks = [para_range(total, size, r) for r in range(size)]
            assert blocks[0][0] == 0 and blocks[-1][1] == total
            for (a, b), (c, d) in zip(blocks, blocks[1:]):
                assert b == c and a <= b
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _cases():
    from cases import variant
    return [variant(calc__Npoints=[5 + i, 4 + i], pulse__ncycles=1.0, pulse__cep=25.0 * i) for i in range(5)]


def _worker(rank, world, port, outdir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "tests", "golden")]
    import datetime

    import torch.distributed as dist

    from antelope_b200.dist import max_over_ranks, para_range, sum_over_ranks
    from oracle import pyoracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    cases = _cases()
    a, b = para_range(len(cases), world, rank)
    units = 0
    for i in range(a, b):
        out = pyoracle.run(cases[i])
        np.save(os.path.join(outdir, f"inter_{i}.npy"), out["inter"])
        units += out["dims"]["ntotal"] * out["dims"]["Nt"]
    t = max_over_ranks(1.0 + rank)
    total = sum_over_ranks(units)
    if rank == 0:
        np.save(os.path.join(outdir, "agg.npy"), np.array([t, total]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_matches_single_process(tmp_path):
    from oracle import pyoracle

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    cases = _cases()
    expect_units = 0
    for i, c in enumerate(cases):
        ref = pyoracle.run(c)
        got = np.load(tmp_path / f"inter_{i}.npy")
        assert np.array_equal(got, ref["inter"])
        expect_units += ref["dims"]["ntotal"] * ref["dims"]["Nt"]
    t, total = np.load(tmp_path / "agg.npy")
    assert t == 2.0            # max over ranks of 1 + rank
    assert total == expect_units


def _shard_cases():
    from cases import MATERIAL_CASES, variant
    return {"haldane_vg": variant(calc__Npoints=[7, 6], pulse__ncycles=1.0),
            "kanemele_w": MATERIAL_CASES["kanemele_w"]}


def _fake_sums(problem, rank):
    import antelope_b200 as ab
    width = ab.capi.lib.sbe_sums_width(problem._h)
    rng = np.random.default_rng(100 + rank)
    return rng.normal(size=(problem.dims.Nt + 1, width))


def _shard_worker(rank, world, port, outdir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "tests", "golden")]
    import datetime

    import torch.distributed as dist

    import antelope_b200 as ab
    from antelope_b200.dist import reduce_and_assemble

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    for name, case in _shard_cases().items():
        p = ab.Problem.from_dict(case)
        out = reduce_and_assemble(p, _fake_sums(p, rank))
        np.save(os.path.join(outdir, f"{name}_{rank}.npy"), np.concatenate([out.inter, out.intra, out.occ], 1))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_k_sharding_reduce_and_assemble(tmp_path):
    """k-sharded solves: each rank's (Nt + 1) x width k-sums are all-reduced
    and every rank assembles the same outputs, equal to assembling the sum of
    the ranks' sums in one process (sbe_assemble is host-only).  The sums are
    stand-ins here; the GPU test checks that slice sums add up to a full solve."""
    import antelope_b200 as ab

    port = _free_port()
    mp.start_processes(_shard_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    for name, case in _shard_cases().items():
        p = ab.Problem.from_dict(case)
        ref = ab.api.assemble(p, _fake_sums(p, 0) + _fake_sums(p, 1))
        expect = np.concatenate([ref.inter, ref.intra, ref.occ], 1)
        for r in range(2):
            got = np.load(tmp_path / f"{name}_{r}.npy")
            assert np.allclose(got, expect, rtol=1e-14, atol=0), (name, r)
