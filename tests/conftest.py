import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


class Case:
    """A committed fixture: genome, reads, the reference's index view and its
    per-read results for one or more parameter sets."""

    def __init__(self, name):
        from msgseqtk_b200.index_build import FmdView
        d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
        self.name = name
        self.d = d
        go = d["genome_off"]
        self.genomes = [d["genome"][go[k]:go[k + 1]] for k in range(len(go) - 1)]
        self.reads = d["reads"]
        self.read_off = d["read_off"]
        lens = np.diff(go).astype(np.int64)
        chr_off = go.astype(np.int64)
        self.view = FmdView(len(d["bwt"]), d["bwt"], d["B"], d["sample_rows"], d["sample_vals"], d["bd_start"],
                            d["bd_end"], lens, d["genome"], chr_off)
        self.n_params = sum(1 for k in d.files if k.endswith("_params"))

    def read(self, i):
        return self.reads[self.read_off[i]:self.read_off[i + 1]]

    def params(self, k):
        p = self.d[f"p{k}_params"]
        return dict(min_len=int(p[0]), max_evalue=float(p[1]), max_nseed=int(p[2]), mode=int(p[3]))

    def expected(self, k):
        d = self.d
        md = bytes(d[f"p{k}_md"]).decode().split("\n") if len(d[f"p{k}_md"]) else []
        return dict(smem=d[f"p{k}_smem"], smem_off=d[f"p{k}_smem_off"], seed=d[f"p{k}_seed"],
                    seed_off=d[f"p{k}_seed_off"], aln=d[f"p{k}_aln"], aln_off=d[f"p{k}_aln_off"],
                    cigar=d[f"p{k}_cigar"], md=md)


@pytest.fixture(scope="session")
def cases():
    return {n: Case(n) for n in ("uniform", "repeats")}


@pytest.fixture(scope="session")
def oracle_built():
    from oracle.bind import build_oracle
    return build_oracle()
