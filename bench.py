"""Benchmark of the B200 read-mapping path on the scale workload.

Workload (one GPU): a synthetic metagenome of 200 genomes with log-normal
lengths (median 3 Mbp, sigma 0.5, ~600 Mbp, per-genome GC uniform 30-70%),
indexed as MSGseqTK's bidirectional FMD-index (~1.2 G BWT symbols), and 2 M
read pairs (2 x 150 bp, fragment ~ Normal(400, 50), 1% substitutions, 0.1%
indels of 1-3 bp, 5% random pairs). Mates are mapped as single reads, as the
reference's findSeedsPE does. A step maps one batch of reads (default 500 k
pairs = 1 M reads) end to end: SMEMs -> seed selection -> locate ->
redundant-seed removal -> chains -> DP + traceback -> CIGAR. Default parameters
(min seed 17, e-value 0.01, maxNSeed 500, GLOBAL NW, scores 1/3/5/2).

Both paths apply Alignment::filter on the device (-s 0.65, the reference's
default), so the records are the ones the reference keeps. The plain path
fills the reference's whole DP rectangles; the learned path lets a classifier
(trained on the GPU during setup, on chains of fresh reads from the same
generator) pick a band per chain, certified or recomputed, so its records
are identical (checked on the validation sample).

Reported line (rank 0): `value` = reads/s of the learned path over all ranks
with the reads already resident in HBM and results left on the device;
`plain_gpu` = the same for the plain path; `e2e` = the learned path
through msg_map_batches (msg_map_batch per batch, each batch's copies
overlapped with its neighbours' mapping) with pinned host reads in and host
alignment records out, copies inside the timed region; `e2e_sam` = to SAM
records, the host tail overlapped with the next batch's mapping (wall clock);
`roofline` for the dominant kernel;
`cpu_baseline` = the reference's own mapping path (compiled from its sources)
on a bounded sample of the same reads with all host threads.

`--impl reference` times that reference CPU path alone (rank 0; other ranks
exit without work).

`--workload clean` measures msgseqtk-clean's path instead: findMEMS of every
mate against a reference index (the scale metagenome) and a background index
(a second metagenome of half as many genomes, another seed), the two lists'
log-likelihoods and the log-odds keep decision per pair, on 2 x 150 bp pairs
drawn half from each genome set. `value` = reads/s (each mate counts) through
msg_clean_batch_device with the reads resident in HBM, `e2e` = the same
through msg_clean_batch from pinned host reads; the reference arm times the
reference's own clean task body (findMEMS_PE on both indexes) with all host
threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mapped reads/sec/GPU (2x150bp) + DP GCUPS, learned-band vs plain GPU, bit-exact SAM"
WORKLOADS = {
    "scale": "scale: 200 genomes ~600 Mbp (log-normal, GC 30-70%), 2x150 bp pairs, insert N(400,50), 1% sub, "
             "0.1% indel, 5% random pairs; mates mapped as single reads (findSeedsPE)",
    "uneven": "uneven: 200 genomes ~600 Mbp; single-end reads 60% 75-150 bp, 30% 250-300 bp, 10% 1-10 kbp, "
              "5% errors (70% substitutions, 30% indels); one batch",
    "repeats": "repeats: two ~750 Mbp metagenomes (log-normal lengths, GC 30-70%, 10% repeat families: 500-5000 bp "
               "units x 10-200 copies at 2-5% divergence) indexed together (~3.0 G BD symbols), 2x150 bp pairs, "
               "insert N(400,50), 1% sub, 0.1% indel, 5% random pairs",
    "clean": "clean: reference index = 200 genomes ~600 Mbp, background index = 100 genomes ~300 Mbp (other "
             "seed); 2x150 bp pairs, half from each set, insert N(400,50), 1% sub, 0.1% indel, 5% random pairs; "
             "findMEMS (min seed 17, e-value 0.01) on both indexes, log-odds > 0 keeps the pair",
}
CLEAN_METRIC = "cleaned reads/sec/GPU (2x150bp pairs, findMEMS on reference + background index, log-odds decision)"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes per SMEM extension, ncu on the 60-genome shape with 1 M-read
# batches (29.55 GB read + written for 449.5 M extensions)
SMEM_DRAM_BYTES_PER_EXT = 29.552e9 / 449.48e6
# DRAM bytes per MEM extension, ncu on the 60 + 30 genome clean shape
# (4.437 GB read + written for 57.32 M extensions)
MEM_DRAM_BYTES_PER_EXT = 4.437e9 / 57.32e6
HBM_FALLBACK = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pairs", type=int, default=None, help="read pairs per GPU (2 M; 10 M for repeats)")
    ap.add_argument("--batch-pairs", type=int, default=500_000)
    ap.add_argument("--genomes", type=int, default=200)
    ap.add_argument("--median", type=float, default=3e6)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU work of the baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--validate", type=int, default=2000, help="reads checked against the oracle after timing")
    ap.add_argument("--train-pairs", type=int, default=2_200_000,
                    help="read pairs (fresh seed) whose chains train the band classifier")
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--min-score", type=float, default=0.65, help="Alignment::filter rate (msgseqtk-align -s)")
    ap.add_argument("--repeat-mbp", type=float, default=750.0, help="size of each repeats metagenome (Mbp)")
    ap.add_argument("--workload", default="scale", choices=["scale", "uneven", "clean", "repeats"],
                    help="scale: 2x150 bp pairs; uneven: single-end reads of mixed lengths (one batch); "
                         "clean: msgseqtk-clean's MEM log-odds path on two indexes")
    ap.add_argument("--uneven-reads", type=int, default=500_000)
    ap.add_argument("--no-tune", action="store_true", help="keep the library's default kernel shapes (no autotuner)")
    ap.add_argument("--sb-contexts", type=int, default=4,
                    help="contexts mapping the 50 k-read batches side by side (1: one context only)")
    args = ap.parse_args()
    if args.pairs is None:
        args.pairs = 10_000_000 if args.workload == "repeats" else 2_000_000
    return args


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reads_seed(rank: int) -> int:
    """Each rank maps its own pairs (weak scaling; the index is replicated)."""
    return 1000 + rank


def reduce_over_ranks(ms: float, n_reads: float, device) -> tuple[float, float]:
    """Max of the timed region over ranks and total reads over ranks; the only
    cross-rank communication of the benchmark (no data-path collective)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return ms, n_reads
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    n = torch.tensor([n_reads], dtype=torch.float64, device=device)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(t.item()), float(n.item())


def uneven_reads(genomes, n, seed):
    """Single-end reads of mixed lengths: 60% U{75..150}, 30% U{250..300},
    10% U{1000..10000} bp, all with 5% errors (70% substitutions, 30% indels
    of 1-3 bp), shuffled. Each group is sampled at its longest length and every
    read cut to its own length (a prefix of a read is a read of the same error
    model)."""
    from msgseqtk_b200 import synth
    rng = np.random.default_rng(seed)
    groups = [(int(0.6 * n), 75, 150), (int(0.3 * n), 250, 300), (n - int(0.6 * n) - int(0.3 * n), 1000, 10000)]
    seqs, quals = [], []
    for k, (m, lo, hi) in enumerate(groups):
        if m <= 0:
            continue
        rs = synth.sample_reads(genomes, m, L=hi, seed=seed * 10 + k, sub_rate=0.035, indel_rate=0.015)
        lens = rng.integers(lo, hi + 1, m)
        for i in range(m):
            seqs.append(rs.read(i)[:lens[i]])
            quals.append(rs.quals[rs.offs[i]:rs.offs[i] + lens[i]])
    order = rng.permutation(len(seqs))
    seqs = [seqs[k] for k in order]
    quals = [quals[k] for k in order]
    offs = np.zeros(len(seqs) + 1, dtype=np.int64)
    np.cumsum([len(x) for x in seqs], out=offs[1:])
    return synth.ReadSet(np.concatenate(seqs).astype(np.uint8), offs, np.concatenate(quals).astype(np.uint8),
                         np.zeros((len(seqs), 3), dtype=np.int64))


def make_workload(args, rank, device):
    from msgseqtk_b200 import index_build, synth
    t0 = time.time()
    if args.workload == "repeats":
        genomes = (synth.repeat_metagenome(seed=args.seed + 300, total_bp=args.repeat_mbp * 1e6, median=args.median) +
                   synth.repeat_metagenome(seed=args.seed + 400, total_bp=args.repeat_mbp * 1e6, median=args.median))
    else:
        genomes = synth.scale_genomes(seed=args.seed, n_genomes=args.genomes, median=args.median)
    t1 = time.time()
    view = index_build.build_view(genomes, device=device)
    t2 = time.time()
    if args.workload == "uneven":
        reads = uneven_reads(genomes, args.uneven_reads, seed=reads_seed(rank))
    else:
        m1, m2 = synth.sample_pairs(genomes, args.pairs, seed=reads_seed(rank))
        reads = synth.interleave(m1, m2)
    t3 = time.time()
    setup = {"genome_s": round(t1 - t0, 1), "index_s": round(t2 - t1, 1), "reads_s": round(t3 - t2, 1)}
    return genomes, view, reads, setup


def cpu_baseline(genomes, view, reads, target_s, impl_line=False):
    """The reference's mapping path (oracle/_ref, compiled from its sources)
    on a bounded sample of the reads, all host threads."""
    from oracle.bind import REF_SO, Reference
    if not os.path.exists(REF_SO):
        return None
    t0 = time.time()
    ref = Reference(genomes, view=view)
    build_s = time.time() - t0
    threads = ref.lib.ref_max_threads()
    n_cal = min(len(reads), 200 * threads)
    _, _, sec = ref.map_batch(reads.seqs[:reads.offs[n_cal]], reads.quals[:reads.offs[n_cal]],
                              reads.offs[:n_cal + 1], n_threads=threads)
    rate = n_cal / max(sec, 1e-9)
    n = int(min(len(reads), max(n_cal, rate * target_s)))
    a, b = reads.offs[0], reads.offs[n]
    mapped, n_aln, sec = ref.map_batch(reads.seqs[a:b], reads.quals[a:b], reads.offs[:n + 1] - a, n_threads=threads)
    return {"value": n / sec, "unit": "reads/s", "cores": threads, "kind": "reference",
            "sample": f"first {n} reads of the workload (of {len(reads)}), reference findSeeds->getChains->"
                      f"buildAlignments->filter->evaluate->calcMapQ->sort per read, OpenMP {threads} threads",
            "seconds": round(sec, 2), "mapped_reads": int(mapped), "index_build_s": round(build_s, 1)}, ref


def sam_validation(ref, view, ctx, reads, n, params, min_score):
    """SAM fields of the first n reads (whole pairs), mapped on the GPU and
    passed through the library's paired-end tail, against the reference's
    whole paired-end path (findSeedsPE -> ... -> AlignmentPE -> output) with
    -m 400 -d 50, compiled from its sources."""
    from msgseqtk_b200 import lib
    from oracle.sam_fields import ours_as_fields, ref_as_fields
    n = min(n, len(reads))
    n -= n % 2
    if n <= 0:
        return None
    try:
        seq, qual, off = reads.seqs[:reads.offs[n]], reads.quals[:reads.offs[n]], reads.offs[:n + 1]
        exp = ref_as_fields(ref.sam_pe_batch(seq, qual, off, min_score_rate=min_score, max_report=1,
                                             pairing=dict(mean=400.0, sd=50.0, min=-100.0, max=900.0)))
        res = ctx.map(seq, off, params)
        recs, md = lib.tail(view, seq, off, qual, res["aln"], res["cigar"], res["read_aln_off"],
                            lib.tail_params(min_score_rate=min_score, max_report=1),
                            pairing=lib.pair_params(mean=400.0, sd=50.0, min_ins=-100.0, max_ins=900.0))
        got = ours_as_fields(recs, md, seq, qual, off, res["cigar"], pairs=True)
        bad = sum(1 for g, e in zip(got, exp) if g != e) + abs(len(got) - len(exp))
        return {"pairs": n // 2, "records": len(exp), "mismatching_records": bad,
                "compared": "SAM fields (flag, tid, pos, MAPQ, CIGAR, SEQ, QUAL, TLEN, AS, MD, XH, NH, XN, XP; "
                            "float tags to the bit) of the learned-band path + msg_tail_pe_batch against the "
                            "reference's paired-end path, -m 400 -d 50 -s %g" % min_score}
    except Exception as exc:  # reported in the line, not fatal to the measurement
        return {"error": f"{type(exc).__name__}: {exc}"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    genomes, view, reads, setup = make_workload(args, rank, dev)
    from oracle.bind import REF_SO, Reference
    if not os.path.exists(REF_SO):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmsgref.so was not built"}))
        return
    ref = Reference(genomes, view=view)
    threads = ref.lib.ref_max_threads()
    n_cal = min(len(reads), 200 * threads)
    _, _, sec = ref.map_batch(reads.seqs[:reads.offs[n_cal]], reads.quals[:reads.offs[n_cal]],
                              reads.offs[:n_cal + 1], n_threads=threads)
    rate = n_cal / max(sec, 1e-9)
    per_step = int(min(len(reads) // max(1, args.steps + args.warmup), max(1000, rate * args.cpu_seconds / 2)))
    times = []
    for s in range(args.warmup + args.steps):
        a_r = (s * per_step) % max(1, len(reads) - per_step)
        a, b = reads.offs[a_r], reads.offs[a_r + per_step]
        _, _, sec = ref.map_batch(reads.seqs[a:b], reads.quals[a:b], reads.offs[a_r:a_r + per_step + 1] - a,
                                  n_threads=threads)
        if s >= args.warmup:
            times.append(sec)
    total = sum(times)
    value = per_step * len(times) / total
    line = {"metric": METRIC, "value": value, "unit": "reads/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * total / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOADS[args.workload],
                       "reads_per_step": per_step, "bd_symbols": view.n, "parallelism": f"omp{threads}"},
            "cpu_baseline": {"value": value, "unit": "reads/s", "cores": threads, "kind": "reference",
                             "sample": f"{per_step} reads per step from the workload"},
            "e2e": {"value": value, "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "setup": setup}
    print(json.dumps(line), flush=True)


def clean_workload(args, rank, device):
    """Reference and background metagenomes, their index views, and pairs
    drawn half from each (shuffled): (g_ref, g_bg, v_ref, v_bg, mates1,
    offs1, mates2, offs2, setup)."""
    from msgseqtk_b200 import index_build, synth
    t0 = time.time()
    g_ref = synth.scale_genomes(seed=args.seed, n_genomes=args.genomes, median=args.median)
    g_bg = synth.scale_genomes(seed=args.seed + 100, n_genomes=max(1, args.genomes // 2), median=args.median)
    t1 = time.time()
    v_ref = index_build.build_view(g_ref, device=device)
    v_bg = index_build.build_view(g_bg, device=device)
    t2 = time.time()
    half = args.pairs // 2
    a1, a2 = synth.sample_pairs(g_ref, half, seed=reads_seed(rank))
    b1, b2 = synth.sample_pairs(g_bg, args.pairs - half, seed=reads_seed(rank) + 500)
    order = np.random.default_rng(reads_seed(rank)).permutation(args.pairs)
    mates = []
    for x, y in ((a1, b1), (a2, b2)):
        lens = np.concatenate([np.diff(x.offs), np.diff(y.offs)])[order]
        starts = np.concatenate([x.offs[:-1], len(x.seqs) + y.offs[:-1]])[order]
        flat = np.concatenate([x.seqs, y.seqs])
        offs = np.zeros(args.pairs + 1, dtype=np.int64)
        np.cumsum(lens, out=offs[1:])
        idx = np.repeat(starts - offs[:-1], lens) + np.arange(offs[-1])
        mates += [flat[idx], offs]
    t3 = time.time()
    setup = {"genome_s": round(t1 - t0, 1), "index_s": round(t2 - t1, 1), "reads_s": round(t3 - t2, 1)}
    return (g_ref, g_bg, v_ref, v_bg, *mates, setup)


def main_clean(args, world, rank, local):
    import torch
    import torch.distributed as dist
    from msgseqtk_b200 import lib
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://")
    g_ref, g_bg, v_ref, v_bg, s1, o1, s2, o2, setup = clean_workload(args, rank, f"cuda:{local}")
    torch.cuda.empty_cache()
    ref, bg = lib.Context(local), lib.Context(local)
    t0 = time.time()
    ref.load_index(v_ref)
    bg.load_index(v_bg)
    setup["load_s"] = round(time.time() - t0, 1)
    setup["index_gb"] = round((ref.index_bytes() + bg.index_bytes()) / 1e9, 2)
    params = lib.mem_params()
    bp = min(args.batch_pairs, args.pairs)
    n_batches = max(1, args.pairs // bp)
    d1, d2 = torch.from_numpy(s1).cuda(), torch.from_numpy(s2).cuda()
    offd = []
    for k in range(n_batches):
        offd.append((torch.from_numpy(o1[k * bp:(k + 1) * bp + 1] - o1[k * bp]).cuda(),
                     torch.from_numpy(o2[k * bp:(k + 1) * bp + 1] - o2[k * bp]).cuda()))
    stream = torch.cuda.ExternalStream(ref.stream_handle())

    def run_device(k):
        a1, a2 = int(o1[k * bp]), int(o2[k * bp])
        return ref.clean_device(bg, d1.data_ptr() + a1, offd[k][0].data_ptr(), bp, d2.data_ptr() + a2,
                                offd[k][1].data_ptr(), params)

    for s in range(args.warmup):
        run_device(s % n_batches)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    agg = {"n_ext": 0, "n_launch": 0, "ms_mem": 0.0, "kept": 0}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for s in range(args.steps):
        res = run_device((args.warmup + s) % n_batches)
        st = ref.stats()
        agg["n_ext"] += st["n_ext"]; agg["n_launch"] += st["n_launch"]; agg["ms_mem"] += st["ms_smem"]
        agg["kept"] += int(res[3].sum())
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms, total_reads = reduce_over_ranks(ev0.elapsed_time(ev1), 2.0 * bp * args.steps, "cuda")
    value = total_reads / (ms / 1000.0)

    # end to end: pinned host mates in, host decisions out
    h1 = torch.from_numpy(s1).pin_memory().numpy()
    h2 = torch.from_numpy(s2).pin_memory().numpy()
    hoff = [(torch.from_numpy(o1[k * bp:(k + 1) * bp + 1] - o1[k * bp]).pin_memory().numpy(),
             torch.from_numpy(o2[k * bp:(k + 1) * bp + 1] - o2[k * bp]).pin_memory().numpy())
            for k in range(n_batches)]

    def run_host(k):
        a1, b1 = int(o1[k * bp]), int(o1[(k + 1) * bp])
        a2, b2 = int(o2[k * bp]), int(o2[(k + 1) * bp])
        return ref.clean(bg, h1[a1:b1], hoff[k][0], h2[a2:b2], hoff[k][1], params), (b1 - a1) + (b2 - a2)

    run_host(0)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    h2d = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s in range(args.steps):
        k = (args.warmup + s) % n_batches
        _, nbytes = run_host(k)
        h2d += nbytes + hoff[k][0].nbytes + hoff[k][1].nbytes
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e, e2e_reads = reduce_over_ranks(e0.elapsed_time(e1), 2.0 * bp * args.steps, "cuda")
    e2e = {"value": e2e_reads / (ms_e2e / 1000.0), "unit": "reads/s", "h2d_bytes_per_step": int(h2d // args.steps),
           "d2h_bytes_per_step": int(25 * bp)}

    peaks = json.load(open(PEAKS)) if os.path.exists(PEAKS) else {}
    hbm = peaks.get("hbm_gbs")
    peak_note = "measured" if hbm else "fallback"
    hbm = hbm or HBM_FALLBACK
    # two 32 B occurrence buckets per extension, plus each mate's bases once per index
    alg = 64.0 * agg["n_ext"] + 2.0 * float(o1[bp] + o2[bp]) * args.steps
    achieved = alg / (agg["ms_mem"] / 1000.0) / 1e9 if agg["ms_mem"] > 0 else 0.0
    roofline = {"kernel": "k_mems (MEM forward extension, both indexes)", "bound": "hbm", "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": MEM_DRAM_BYTES_PER_EXT * agg["n_ext"] / args.steps,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_mems launch on the "
                                  "60 + 30 genome shape, per extension, times this launch's extensions",
                "peak_source": peak_note, "alg_bytes_per_launch": alg / args.steps,
                "kernel_ms_per_step": agg["ms_mem"] / args.steps,
                "extensions_per_step": agg["n_ext"] / args.steps}

    valid = None
    if rank == 0 and args.validate > 0:
        from oracle.bind import Oracle
        orc_r, orc_b = Oracle(v_ref), Oracle(v_bg)
        n = min(args.validate, bp)
        r, g, lod, keep = ref.clean(bg, s1[:o1[n]], o1[:n + 1], s2[:o2[n]], o2[:n + 1], params)
        bad = 0
        for i in range(n):
            m1, m2 = s1[o1[i]:o1[i + 1]], s2[o2[i]:o2[i + 1]]
            er = orc_r.mems(m1)[1] + orc_r.mems(m2)[1]
            eb = orc_b.mems(m1)[1] + orc_b.mems(m2)[1]
            if not (np.float64(er).view(np.int64) == np.float64(r[i]).view(np.int64)
                    and np.float64(eb).view(np.int64) == np.float64(g[i]).view(np.int64)
                    and bool(keep[i]) == bool(-er + eb > 0)):
                bad += 1
        valid = {"pairs": n, "mismatching_pairs": bad, "compared": "refLoglik, bgLoglik bit patterns and keep"}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = clean_cpu_rate(g_ref, g_bg, v_ref, v_bg, s1, o1, s2, o2, args.cpu_seconds)

    if rank == 0:
        line = {"metric": CLEAN_METRIC, "value": value, "unit": "reads/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOADS["clean"], "pairs_per_step": bp, "reads_per_step": 2 * bp,
                           "bd_symbols": [v_ref.n, v_bg.n],
                           "l2": ("inputs larger than L2 (indexes %.1f GB; %d batches of %.0f MB of mates cycled, "
                                  "each larger than L2)" % (setup["index_gb"], n_batches,
                                                            (o1[bp] + o2[bp]) / 1e6)),
                           "parallelism": f"dp{world}" if world > 1 else "single GPU"},
                "kept_fraction": agg["kept"] / (bp * args.steps),
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
                "gpu_launches": agg["n_launch"], "validation": valid, "setup": setup}
        print(json.dumps(line), flush=True)
    ref.close()
    bg.close()
    if world > 1:
        dist.destroy_process_group()


def clean_cpu_rate(g_ref, g_bg, v_ref, v_bg, s1, o1, s2, o2, target_s, steps=1, warmup=0):
    """The reference's clean task body (oracle/_ref) on bounded samples of the
    pairs with all host threads: reads/s and the sample description."""
    from oracle.bind import REF_SO, Reference
    if not os.path.exists(REF_SO):
        return None
    ref, bg = Reference(g_ref, view=v_ref), Reference(g_bg, view=v_bg)
    threads = ref.lib.ref_max_threads()
    n_pairs = len(o1) - 1

    def run(a, n):
        return ref.clean_batch(bg, s1[o1[a]:o1[a + n]], o1[a:a + n + 1] - o1[a], s2[o2[a]:o2[a + n]],
                               o2[a:a + n + 1] - o2[a], n_threads=threads)[4]

    n_cal = min(n_pairs, 500 * threads)
    rate = n_cal / max(run(0, n_cal), 1e-9)
    n = int(min(n_pairs // max(1, steps), max(n_cal, rate * target_s)))
    times = [run((k * n) % max(1, n_pairs - n + 1), n) for k in range(steps)]
    timed = times[-1:] if steps == 1 else times[warmup:]
    value = 2.0 * n * len(timed) / sum(timed)
    return {"value": value, "unit": "reads/s", "cores": threads, "kind": "reference",
            "sample": f"{n} pairs per step of the workload (of {n_pairs}), the reference's findMEMS_PE on both "
                      f"indexes + loglik + log-odds per pair, OpenMP {threads} threads",
            "seconds": round(sum(timed), 2), "ms_per_step": 1000.0 * sum(timed) / len(timed)}


def run_reference_clean(args, world, rank):
    if rank != 0:
        return
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    g_ref, g_bg, v_ref, v_bg, s1, o1, s2, o2, setup = clean_workload(args, rank, dev)
    from oracle.bind import REF_SO
    if not os.path.exists(REF_SO):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmsgref.so was not built"}))
        return
    per = max(1.0, args.cpu_seconds / 2)
    cpu = clean_cpu_rate(g_ref, g_bg, v_ref, v_bg, s1, o1, s2, o2, per, steps=args.warmup + args.steps,
                         warmup=args.warmup)
    value = cpu["value"]
    line = {"metric": CLEAN_METRIC, "value": value, "unit": "reads/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cpu.pop("ms_per_step"), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOADS["clean"], "bd_symbols": [v_ref.n, v_bg.n],
                       "parallelism": f"omp{cpu['cores']}"},
            "cpu_baseline": cpu, "e2e": {"value": value, "unit": "reads/s", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}, "setup": setup}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference" and args.workload == "clean":
        return run_reference_clean(args, world, rank)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.workload == "clean":
        return main_clean(args, world, rank, local)
    import torch
    import torch.distributed as dist
    from msgseqtk_b200 import lib
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://")
    genomes, view, reads, setup = make_workload(args, rank, f"cuda:{local}")
    torch.cuda.empty_cache()
    ctx = lib.Context(local)
    t0 = time.time()
    ctx.load_index(view)
    setup["load_s"] = round(time.time() - t0, 1)
    setup["index_gb"] = round(ctx.index_bytes() / 1e9, 2)
    # plain: the reference's whole flank rectangles; learned: per-chain band
    # from the classifier, certified or recomputed (same records)
    plain_params = lib.default_params(min_score_rate=args.min_score)
    params = lib.default_params(min_score_rate=args.min_score, band_mode=2)

    # train the band classifier on chains of fresh reads from the same generator
    from msgseqtk_b200 import synth
    t0 = time.time()
    tm1, tm2 = synth.sample_pairs(genomes, args.train_pairs, seed=reads_seed(rank) + 5000)
    treads = synth.interleave(tm1, tm2)
    t1 = time.time()
    feats, labels = [], []
    tb = 2 * args.batch_pairs

    def collect(a, b):
        """Certificates of reads a..b, in halves when the batch's rectangles
        exceed the context's DP storage (one collection fills them all)."""
        try:
            f, l = ctx.band_collect(treads.seqs[treads.offs[a]:treads.offs[b]],
                                    treads.offs[a:b + 1] - treads.offs[a], plain_params)
        except lib.MsgError as e:
            if b - a < 2 or "too large" not in str(e):
                raise
            collect(a, (a + b) // 2)
            collect((a + b) // 2, b)
            return
        feats.append(f)
        labels.append(l)

    for a in range(0, len(treads), tb):
        collect(a, min(len(treads), a + tb))
    feats = np.concatenate(feats)
    labels = np.concatenate(labels)
    n_all = len(labels)
    keep = labels >= 0  # chains a band can apply to
    feats, labels = feats[keep], labels[keep]
    t2 = time.time()
    bparams, bloss = ctx.band_train(feats, labels, epochs=args.epochs, batch=4096, lr=2e-3, seed=11)
    torch.cuda.synchronize()
    t3 = time.time()
    from oracle import band_mlp
    train_acc = float(np.mean(band_mlp.classify(bparams, feats) == labels))
    band_info = {"train_chains": int(len(labels)), "collected_chains": int(n_all),
                 "label_counts": np.bincount(labels, minlength=4).tolist(),
                 "classes": "band half-width 7, 15, 31, whole rectangles", "epochs": args.epochs,
                 "loss_first_last": [float(bloss[0]), float(bloss[-1])], "train_accuracy": round(train_acc, 4),
                 "collect_s": round(t2 - t1, 2), "train_s": round(t3 - t2, 2), "reads_s": round(t1 - t0, 1)}
    del treads, tm1, tm2

    # batches: reads resident on the device, and pinned host copies for e2e
    bp = 2 * args.batch_pairs if args.workload in ("scale", "repeats") else len(reads)
    n_batches = max(1, len(reads) // bp)
    d_seq = torch.from_numpy(reads.seqs).cuda()
    offs_d = []
    for k in range(n_batches):
        o = reads.offs[k * bp:(k + 1) * bp + 1]
        offs_d.append(torch.from_numpy(o - o[0]).cuda())
    h_seq = torch.from_numpy(reads.seqs).pin_memory().numpy()
    h_offs = [torch.from_numpy(reads.offs[k * bp:(k + 1) * bp + 1] - reads.offs[k * bp]).pin_memory().numpy()
              for k in range(n_batches)]
    stream = torch.cuda.ExternalStream(ctx.stream_handle())

    # the library's autotuner picks the SMEM and DP kernel shapes on the
    # first batch, whole (untimed; records do not depend on the shapes; a
    # smaller sample leaves the DP launches too short to rank the shapes as
    # the full batch does)
    ns = min(bp, len(reads))
    if args.no_tune:
        dp_shape = {"tuned": False, "note": "library default shapes"}
    else:
        dp_shape = ctx.autotune(reads.seqs[:reads.offs[ns]], reads.offs[:ns + 1], params)
        dp_shape["sample_reads"] = ns

    def offs_sb(first, count):
        """Device offsets of reads first .. first + count, rebased to 0."""
        o = reads.offs[first:first + count + 1]
        return torch.from_numpy(o - o[0]).cuda()

    def run_device(k, prm):
        base = int(reads.offs[k * bp])
        return ctx.map_device(d_seq.data_ptr() + base, offs_d[k].data_ptr(), len(offs_d[k]) - 1, prm)

    counters = ("n_ext", "dp_cells", "dp_cells_done", "n_reads", "n_launch", "n_aln", "host_sorted", "n_sa",
                "n_chain", "n_band_exact", "n_band_drop", "n_band_fallback", "n_filtered", "n_dp_warp",
                "n_smem_rerun", "smem_retries", "n_ext_ff", "n_ff_steps")

    def timed(prm, clocks=None):
        """W warm-up steps, then K timed steps on new batches (inputs larger
        than L2), device-timed on the library's stream, max over ranks."""
        for s in range(args.warmup):
            run_device(s % n_batches, prm)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        if clocks:
            clocks.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        agg = {"smem": 0.0, "locate": 0.0, "chain": 0.0, "dp": 0.0}
        agg.update({k: 0 for k in counters})
        agg["n_dp_class"] = [0] * 5
        agg["dp_class_cells"] = [0] * 5
        agg["ms_dp_part"] = [0.0] * 4
        torch.cuda.synchronize()
        ev0.record(stream)
        for s in range(args.steps):
            run_device((args.warmup + s) % n_batches, prm)
            st = ctx.stats()
            agg["smem"] += st["ms_smem"]; agg["locate"] += st["ms_locate"]; agg["chain"] += st["ms_chain"]
            agg["dp"] += st["ms_dp"]
            for k in counters:
                agg[k] += st[k]
            for k in ("n_dp_class", "dp_class_cells", "ms_dp_part"):
                agg[k] = [x + y for x, y in zip(agg[k], st[k])]
        ev1.record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop() if clocks else None
        ms, total_reads = reduce_over_ranks(ev0.elapsed_time(ev1), float(agg["n_reads"]), "cuda")
        return ms, total_reads, agg, clk

    ms_p, reads_p, agg_p, _ = timed(plain_params)
    ms, total_reads, agg, clk = timed(params, Clocks(local))
    value = total_reads / (ms / 1000.0)

    # the same path in batches of 50 k reads (an interactive caller's batch
    # size): fixed per-batch costs show against the 1 M-read batches above
    small_batch = None
    sb = 50_000
    n_sb = min(40, bp // sb, len(reads) // sb - 3)  # 3 untimed batches first
    if args.workload in ("scale", "repeats") and n_sb >= 1:
        for s in range(3):
            ctx.map_device(d_seq.data_ptr() + int(reads.offs[s * sb]), offs_sb(s * sb, sb).data_ptr(), sb, params)
        torch.cuda.synchronize()
        sb_offs = [offs_sb((3 + s) * sb, sb) for s in range(n_sb)]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        sb_stage = {"smem": 0.0, "locate": 0.0, "chain": 0.0, "dp": 0.0, "total": 0.0}
        e0.record(stream)
        for s in range(n_sb):
            ctx.map_device(d_seq.data_ptr() + int(reads.offs[(3 + s) * sb]), sb_offs[s].data_ptr(), sb, params)
            st = ctx.stats()
            for k in ("smem", "locate", "chain", "dp", "total"):
                sb_stage[k] += st["ms_" + k] / n_sb
        e1.record(stream)
        torch.cuda.synchronize()
        sb_value = n_sb * sb / (e0.elapsed_time(e1) / 1000.0)
        small_batch = {"value": sb_value, "unit": "reads/s", "batch_reads": sb, "batches": n_sb,
                       "fraction_of_value": sb_value / value, "stage_ms_per_batch": sb_stage}
        # the same batches on several contexts that share the index
        # (msg_ctx_share_index), one host thread each: a batch's slowest
        # reads and chains overlap the other batches' work on their streams
        P = args.sb_contexts
        if P > 1:
            side = []
            for _ in range(P - 1):
                c2 = lib.Context(local)
                c2.share_index(ctx)
                if not args.no_tune:
                    c2.apply_shapes(dp_shape)
                c2.band_model_set(bparams)
                side.append(c2)
            cs = [ctx] + side
            sts = [stream] + [torch.cuda.ExternalStream(c.stream_handle()) for c in side]

            def sb_map(c, s):
                c.map_device(d_seq.data_ptr() + int(reads.offs[(3 + s) * sb]), sb_offs[s].data_ptr(), sb, params)

            for c in side:  # each context sizes its buffers untimed
                for s in range(3):
                    sb_map(c, s)
            torch.cuda.synchronize()
            errs = []

            def sb_worker(j):
                try:
                    for s in range(j, n_sb, P):
                        sb_map(cs[j], s)
                except Exception as exc:  # re-raised below
                    errs.append(exc)

            e0.record(stream)
            for st_ in sts[1:]:
                st_.wait_event(e0)
            workers = [threading.Thread(target=sb_worker, args=(j,)) for j in range(P)]
            for w in workers:
                w.start()
            for w in workers:
                w.join()
            if errs:
                raise errs[0]
            for st_ in sts[1:]:
                ev = torch.cuda.Event()
                ev.record(st_)
                stream.wait_event(ev)
            e1.record(stream)
            torch.cuda.synchronize()
            cv = n_sb * sb / (e0.elapsed_time(e1) / 1000.0)
            small_batch["contexts"] = {"value": cv, "unit": "reads/s", "contexts": P, "batches": n_sb,
                                       "fraction_of_value": cv / value,
                                       "note": "one host thread per context, index shared (msg_ctx_share_index); "
                                               "device time from the first launch to the last stream's end"}
            for c in side:
                c.close()
    banded = agg["n_band_exact"] + agg["n_band_drop"] + agg["n_band_fallback"]

    def gcups(a):
        return {"reference_cells": a["dp_cells"] / (a["dp"] / 1000.0) / 1e9 if a["dp"] > 0 else 0.0,
                "computed_cells": a["dp_cells_done"] / (a["dp"] / 1000.0) / 1e9 if a["dp"] > 0 else 0.0}

    plain = {"value": reads_p / (ms_p / 1000.0), "unit": "reads/s", "ms_per_step": ms_p / args.steps,
             "dp_ms_per_step": agg_p["dp"] / args.steps, "gcups": gcups(agg_p),
             "dp_cells_computed": agg_p["dp_cells_done"], "warp_path_chains": agg_p["n_dp_warp"]}
    band_info.update({"dp_ms_per_step": agg["dp"] / args.steps, "gcups": gcups(agg),
                      "dp_cells_computed": agg["dp_cells_done"], "dp_cells_reference": agg["dp_cells"],
                      "warp_path_chains": agg["n_dp_warp"],
                      "banded_chains": banded, "certified_exact": agg["n_band_exact"],
                      "certified_filtered": agg["n_band_drop"], "fallback": agg["n_band_fallback"],
                      "fallback_rate": agg["n_band_fallback"] / banded if banded else 0.0,
                      "speedup_vs_plain": value / plain["value"] if plain["value"] > 0 else None})

    # end to end through the public API: pinned host reads in, records out
    # into pinned host buffers
    def pinned(n, dtype):
        dt = np.dtype(dtype)
        return torch.empty(n * dt.itemsize, dtype=torch.uint8).pin_memory().numpy().view(dt)

    aln_buf = pinned(8 * bp, lib.ALN_DTYPE)
    cig_buf = pinned(64 * bp, np.uint32)
    roff_buf = pinned(bp + 1, np.int64)
    obufs = [(aln_buf, cig_buf, roff_buf), (pinned(8 * bp, lib.ALN_DTYPE), pinned(64 * bp, np.uint32),
                                            pinned(bp + 1, np.int64))]

    def host_batch(k):
        a, b = int(reads.offs[k * bp]), int(reads.offs[min(len(reads), (k + 1) * bp)])
        return h_seq[a:b], h_offs[k]

    # msg_map_batches: batch k+1's upload and batch k-1's download overlap
    # batch k's mapping (two pinned record buffers, alternating)
    ctx.map_batches([host_batch(s % n_batches) for s in range(min(args.warmup, 2))], obufs[:min(args.warmup, 2)],
                    params)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    steps_b = [host_batch((args.warmup + s) % n_batches) for s in range(args.steps)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    counts = ctx.map_batches(steps_b, [obufs[s % 2] for s in range(args.steps)], params)
    e1.record(stream)
    torch.cuda.synchronize()
    h2d = sum(q.nbytes + o.nbytes for q, o in steps_b)
    d2h = sum(na * lib.ALN_DTYPE.itemsize + nc * 4 + o.nbytes for (na, nc), (_, o) in zip(counts, steps_b))
    e2e_reads = sum(len(o) - 1 for _, o in steps_b)
    ms_e2e, e2e_reads = reduce_over_ranks(e0.elapsed_time(e1), float(e2e_reads), "cuda")
    e2e = {"value": e2e_reads / (ms_e2e / 1000.0), "unit": "reads/s", "h2d_bytes_per_step": int(h2d // args.steps),
           "d2h_bytes_per_step": int(d2h // args.steps)}

    # to SAM records: the same calls, with the library's host tail of batch k
    # on host threads while the GPU maps batch k + 1 (wall clock, since the
    # host work counts). Pairs (scale workload): msgseqtk-align's paired-end
    # tail with -m 400 -d 50 (insert range [-100, 900]); single reads: the
    # single-end tail.
    from concurrent.futures import ThreadPoolExecutor
    tail_threads = max(1, (os.cpu_count() or 2) - 1)
    tprm = lib.tail_params(min_score_rate=args.min_score, max_report=1, n_threads=tail_threads)
    pairing = lib.pair_params(mean=400.0, sd=50.0, min_ins=-100.0, max_ins=900.0) if args.workload in ("scale", "repeats") \
        else None
    bufs = [(aln_buf, cig_buf, roff_buf), (pinned(8 * bp, lib.ALN_DTYPE), pinned(64 * bp, np.uint32),
                                            pinned(bp + 1, np.int64))]
    n_sam = 0

    def sam_step(s, pool, fut):
        k = s % n_batches
        a, b = int(reads.offs[k * bp]), int(reads.offs[min(len(reads), (k + 1) * bp)])
        al, cg, ro = bufs[s % 2]
        na, nc = ctx.map_into(h_seq[a:b], h_offs[k], al, cg, ro, params)
        if fut is not None:
            fut.result()
        return pool.submit(lib.tail, view, h_seq[a:b], h_offs[k], reads.quals[a:b], al[:na], cg[:nc], ro, tprm,
                           pairing)

    with ThreadPoolExecutor(1) as pool:
        fut = sam_step(0, pool, None)
        fut.result()
        fut = None
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in range(args.steps):
            fut = sam_step(args.warmup + s, pool, fut)
            n_sam += len(h_offs[(args.warmup + s) % n_batches]) - 1
        recs, _ = fut.result()
        t1 = time.perf_counter()
    ms_sam, n_sam = reduce_over_ranks(1000.0 * (t1 - t0), float(n_sam), "cuda")
    e2e_sam = {"value": n_sam / (ms_sam / 1000.0), "unit": "reads/s", "tail_threads": tail_threads,
               "timing": "wall clock: msg_map_batch from pinned host reads, then the host tail of that batch "
                         "(msg_tail_pe_batch for pairs, -m 400 -d 50; msg_tail_batch for single reads) on host "
                         "threads overlapped with the next batch's mapping; ends with every SAM record built",
               "tail": "paired-end" if pairing is not None else "single-end",
               "records_last_step": int(len(recs))}

    # roofline of the dominant stage
    peaks = json.load(open(PEAKS)) if os.path.exists(PEAKS) else {}
    hbm = peaks.get("hbm_gbs")
    peak_note = "measured" if hbm else "fallback"
    hbm = hbm or HBM_FALLBACK
    stage_ms = {k: agg[k] for k in ("smem", "locate", "chain", "dp")}
    dom = max(stage_ms, key=stage_ms.get)
    read_bytes = float(reads.offs[min(len(reads), n_batches * bp)]) / n_batches * args.steps
    # two 32 B occurrence buckets per bi-interval extension, one 32 B sector
    # per fast-forward step (a suffix-array word, a 16-byte text chunk or an
    # inverse-suffix-array word), plus the read bytes
    smem_bytes = 64.0 * agg["n_ext"] + 32.0 * agg["n_ff_steps"] + read_bytes
    achieved = smem_bytes / (agg["smem"] / 1000.0) / 1e9 if agg["smem"] > 0 else 0.0
    # DRAM bytes per extension measured by ncu on the 60-genome workload shape
    # with 1 M-read batches, scaled to this launch
    traffic = SMEM_DRAM_BYTES_PER_EXT * agg["n_ext"] / args.steps
    smem_roof = {"kernel": "k_smem_thread (SMEM bi-interval extension)", "bound": "hbm", "achieved": achieved,
                 "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                 "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_smem_thread launch "
                                   "on the 60-genome shape, per extension, times this launch's extensions",
                 "peak_source": peak_note, "alg_bytes_per_launch": smem_bytes / args.steps}
    # DP: integer-pipe bound; 11 algorithmic integer ops per reference cell
    # (NW: M 3 adds + 2 max, I 2 adds + 1 max, D 2 adds + 1 max) over the DP
    # stage's time, against the INT32 issue rate of the GPU: SMs x 128 lanes
    # x the SM clock sampled under load (no measured integer peak exists)
    props = torch.cuda.get_device_properties(local)
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    int_peak = props.multi_processor_count * 128 * sm_mhz * 1e6 / 1e12
    dp_ops = 11.0 * agg["dp_cells"]
    dp_achieved = dp_ops / (agg["dp"] / 1000.0) / 1e12 if agg["dp"] > 0 else 0.0
    dp_roof = {"kernel": "k_dp_stripe (seed-guided affine DP, register stripes)", "bound": "int32 pipe",
               "achieved": dp_achieved, "peak": int_peak, "unit": "Tops/s", "frac": dp_achieved / int_peak,
               "traffic": None,
               "peak_source": "derived: %d SMs x 128 INT32 lanes x %.0f MHz (median SM clock under load)"
                              % (props.multi_processor_count, sm_mhz),
               "ops_per_cell": 11, "reference_cells_per_step": agg["dp_cells"] / args.steps,
               "cells_evaluated_per_step": agg["dp_cells_done"] / args.steps}
    roofline = dict(dp_roof if dom == "dp" else smem_roof)
    roofline.update({"dominant_stage": dom, "stage_ms_per_step": {k: v / args.steps for k, v in stage_ms.items()},
                     "stages": {"smem": smem_roof, "dp": dp_roof}})

    # validation: a sample of the timed reads through the oracle
    valid = None
    if rank == 0 and args.validate > 0:
        from oracle.bind import Oracle
        orc = Oracle(view)
        n = min(args.validate, len(reads))
        res = ctx.map(reads.seqs[:reads.offs[n]], reads.offs[:n + 1], params)
        res_p = ctx.map(reads.seqs[:reads.offs[n]], reads.offs[:n + 1], plain_params)
        same = all(np.array_equal(res[k], res_p[k]) for k in ("aln", "cigar", "read_aln_off"))
        bad = 0
        checked = 0
        for i in range(n):
            L = len(reads.read(i))
            if L > 2000:
                continue  # the oracle fills whole double matrices: long reads are checked by the tests
            checked += 1
            exp = [e for e in orc.align_read(reads.read(i)) if not (e["aln_score"] < L * args.min_score)]
            got = res["aln"][res["read_aln_off"][i]:res["read_aln_off"][i + 1]]
            if len(exp) != len(got):
                bad += 1
                continue
            for g, e in zip(got, exp):
                f = [int(g[x]) for x in ("tid", "strand", "t_start", "t_end", "aln_from", "aln_to", "aln_start",
                                         "aln_end", "aln_score")]
                ef = [e["tid"], e["strand"], e["t_start"], e["t_end"], e["aln_from"], e["aln_to"], e["aln_start"],
                      e["aln_end"], int(e["aln_score"])]
                w = [int(x) for x in res["cigar"][g["cigar_off"]:g["cigar_off"] + g["n_cigar"]]]
                if f != ef or w != e["cigar"]:
                    bad += 1
                    break
        valid = {"reads": checked, "mismatching_reads": bad, "learned_equals_plain": bool(same),
                 "compared": "records after Alignment::filter (alnScore >= L * %g)" % args.min_score}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline and args.workload in ("scale", "repeats"):
        r = cpu_baseline(genomes, view, reads, args.cpu_seconds)
        cpu = r[0] if r else None
        if r and valid is not None:
            valid["sam"] = sam_validation(r[1], view, ctx, reads, args.validate, params, args.min_score)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "reads/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "config": {"workload": WORKLOADS[args.workload],
                           "reads_per_step": bp, "pairs_per_gpu": args.pairs, "bd_symbols": view.n,
                           "l2": ("inputs larger than L2 (index %.1f GB; %d batches of %.0f MB of reads cycled, "
                                  "each larger than L2)" % (setup["index_gb"], n_batches,
                                                            reads.offs[-1] / n_batches / 1e6)
                                  if n_batches > 1 else "inputs larger than L2 (index %.1f GB, %.0f MB of reads "
                                  "per step)" % (setup["index_gb"], reads.offs[-1] / 1e6)),
                           "parallelism": f"dp{world}" if world > 1 else "single GPU"},
                "gcups": gcups(agg), "plain_gpu": plain, "learned_band": band_info,
                "e2e": e2e, "e2e_sam": e2e_sam, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
                "gpu_launches": agg["n_launch"], "validation": valid, "setup": setup, "tuned_shapes": dp_shape, "small_batch": small_batch,
                "stats": dict({k: agg[k] for k in counters},
                              dp_classes={"names": ["row-by-row", "stripes", "banded stripes", "warp", "banded warp"],
                                          "chains": agg["n_dp_class"], "cells": agg["dp_class_cells"]},
                              dp_ms_per_step_by_part={"prepare_and_size": agg["ms_dp_part"][0] / args.steps,
                                                      "classes_and_sort": agg["ms_dp_part"][1] / args.steps,
                                                      "fills_and_tracebacks": agg["ms_dp_part"][2] / args.steps,
                                                      "filter_and_cigars": agg["ms_dp_part"][3] / args.steps})}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
