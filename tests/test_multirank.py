"""The N > 1 benchmark path on CPU with 2 gloo ranks: each rank maps its own
read shard (different seeds, same replicated index), and the only cross-rank
step is the max-over-ranks time and the sum of reads."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    import bench
    from msgseqtk_b200 import synth
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, n = bench.reduce_over_ranks(10.0 + 5.0 * rank, 100.0 + rank, "cpu")
        g = synth.small_genomes(seed=5, n_genomes=2, length=3000)
        m1, _ = synth.sample_pairs(g, 20, seed=bench.reads_seed(rank))
        out[rank] = (ms, n, m1.seqs.tobytes())
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_and_disjoint_shards():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    (ms0, n0, s0), (ms1, n1, s1) = out[0], out[1]
    assert ms0 == ms1 == 15.0          # max over ranks
    assert n0 == n1 == 201.0           # sum over ranks
    assert s0 != s1                    # each rank maps its own reads
    assert np.frombuffer(s0, np.uint8).size == np.frombuffer(s1, np.uint8).size


def test_single_rank_reduction_is_identity():
    import bench
    assert bench.reduce_over_ranks(3.5, 7.0, "cpu") == (3.5, 7.0)


def _clean_worker(rank, world, port, out):
    import argparse
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        args = argparse.Namespace(seed=2, genomes=2, median=2e4, pairs=40)
        g_ref, g_bg, v_ref, v_bg, s1, o1, s2, o2, _ = bench.clean_workload(args, rank, "cpu")
        ms, n = bench.reduce_over_ranks(1.0 + rank, 2.0 * (len(o1) - 1), "cpu")
        out[rank] = (v_ref.bwt.tobytes(), v_bg.bwt.tobytes(), s1.tobytes(), s2.tobytes(), len(o1) - 1, ms, n)
    finally:
        dist.destroy_process_group()


def test_two_rank_clean_shards():
    """The clean workload under 2 gloo ranks: both indexes replicated, each
    rank its own pairs (weak scaling), time max and reads summed."""
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_clean_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    a, b = out[0], out[1]
    assert a[0] == b[0] and a[1] == b[1]            # replicated indexes
    assert a[2] != b[2] and a[3] != b[3]            # disjoint read shards
    assert a[4] == b[4] == 40
    assert a[5] == b[5] == 2.0 and a[6] == b[6] == 160.0
