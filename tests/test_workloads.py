"""The seeded synthetic workloads behind the bench configurations: sizes,
alphabets and structure as documented, and the same bytes for the same seed."""
import numpy as np

from distributed_suffix_sorting_evaluation_b200 import workloads as W


def test_batch_lengths_of_the_batched_configuration():
    lens = W.batch_lengths(20000, 1 << 10, 16 << 20, seed=5)
    assert lens.size == 20000
    assert int(lens.sum()) == 34_194_858_181  # the realised total the bench reports
    assert lens.min() >= 1 << 10 and lens.max() <= 16 << 20
    # log-uniform: about half the texts below the geometric midpoint (128 KiB)
    assert 0.45 < float(np.mean(lens < (128 << 10))) < 0.55


def test_markov_dna_alphabet_and_determinism():
    a = W.markov_dna(1 << 20, seed=2)
    b = W.markov_dna(1 << 20, seed=2)
    assert np.array_equal(a, b)
    assert set(np.unique(a).tolist()) == set(b"ACGT")
    assert not np.array_equal(a, W.markov_dna(1 << 20, seed=3))


def test_pangenome_copies_and_separators():
    n, base = 1 << 22, 1 << 18
    t = W.pangenome(n, seed=3, base_len=base)
    assert t.size == n
    assert set(np.unique(t).tolist()) <= set(b"ACGT$")
    seps = np.flatnonzero(t == ord("$"))
    assert 12 <= seps.size <= 16  # one '$' after every ~base-long copy
    # consecutive copies agree position by position until the first indel shifts
    # them (0.1% substitutions, 0.01% indels): check a short stretch
    first, second = t[: seps[0]], t[seps[0] + 1: seps[1]]
    assert float(np.mean(first[:256] == second[:256])) > 0.95


def test_zipf256_uses_every_byte_value():
    z = W.zipf256(1 << 22, seed=4)
    counts = np.bincount(z, minlength=256)
    assert (counts > 0).all()  # sigma = 256: the reference cli refuses this text
    assert 0.15 < counts.max() / z.size < 0.3  # the most frequent symbol under s = 1.1


def test_profiling_size_keeps_the_copy_count():
    """bench.py --text-mib 256 --base-kib 1280 shrinks the 2 GiB pangenome to 256
    MiB with the full-size copy count (the tie groups of ~204 elements that the
    profiling captures of the group sorts need)."""
    import argparse
    import importlib.util
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    args = argparse.Namespace(workload="cfg3a_dc39_pangenome_2GiB", text_mib=256, base_kib=1280)
    w, gen_kw, label = bench._single_workload(args)
    assert w["n"] == 256 << 20 and gen_kw == {"base_len": 1280 << 10}
    assert label == "cfg3a_dc39_pangenome_2GiB@256MiB,base1280KiB"
    t = getattr(W, w["gen"])(w["n"], seed=w["seed"], **gen_kw)
    full_copies = (2 << 30) // ((10 << 20) + 1)
    assert abs(int(np.count_nonzero(t == ord("$"))) - full_copies) <= 2
    # the base option applies to the pangenome generator only
    w2, gen_kw2, _ = bench._single_workload(argparse.Namespace(workload="cfg2_dc39_markov_dna_1GiB",
                                                               text_mib=0, base_kib=1280))
    assert gen_kw2 == {} and w2["n"] == 1 << 30
