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
