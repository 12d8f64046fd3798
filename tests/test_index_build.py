"""Host-side FMD view builder: suffix array by prefix doubling equals a naive
sort, and the view equals the reference's committed one."""
import numpy as np

from msgseqtk_b200 import index_build, synth


def naive_sa(text):
    t = bytes(text.tolist())
    return np.array(sorted(range(len(t)), key=lambda i: t[i:]), dtype=np.int64)


def test_suffix_array_small_random_multi_sentinel():
    rng = np.random.default_rng(3)
    for trial in range(20):
        chroms = [synth._BASES[rng.integers(0, 4, size=int(rng.integers(1, 40)))] for _ in range(int(rng.integers(1, 5)))]
        text = index_build.bd_text(chroms)
        sa = index_build.suffix_array(text).numpy()
        assert np.array_equal(sa, naive_sa(text)), trial


def test_suffix_array_repetitive():
    chroms = [np.full(50, 1, np.uint8), np.tile(np.array([1, 2], np.uint8), 30)]
    text = index_build.bd_text(chroms)
    assert np.array_equal(index_build.suffix_array(text).numpy(), naive_sa(text))


def test_suffix_array_partitioned_sort():
    """Texts longer than one sort call takes (3 G symbols in the repeat-rich
    workload) sort their keys in partitions; forced here with tiny limits,
    on repetitive and random texts alike."""
    rng = np.random.default_rng(11)
    for trial in range(4):
        chroms = [synth._BASES[rng.integers(0, 4, size=int(rng.integers(200, 900)))] for _ in range(3)]
        chroms.append(np.tile(chroms[0][:37], 9))  # a repeat family
        text = index_build.bd_text(chroms)
        sa = index_build.suffix_array(text, chunk=97, sort_limit=701).numpy()
        assert np.array_equal(sa, naive_sa(text)), trial


def test_view_equals_reference_fixture(cases):
    for c in cases.values():
        v = index_build.build_view(c.genomes)
        assert v.n == c.view.n
        assert np.array_equal(v.bwt, c.view.bwt)
        assert np.array_equal(v.B, c.view.B)
        assert np.array_equal(v.sample_rows, c.view.sample_rows)
        assert np.array_equal(v.sample_vals, c.view.sample_vals)
        assert np.array_equal(v.bd_start, c.view.bd_start) and np.array_equal(v.bd_end, c.view.bd_end)
        assert np.array_equal(v.chr_len + 1, c.d["chr_len_ref"])  # getChromLength counts the terminator
