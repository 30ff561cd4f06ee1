"""Launch-mapping variants (care_b200_tuning) leave every result unchanged:
LPT anchor order, the persistent work-queue MSA kernel, 8 warps per anchor,
256-thread alignment CTAs, length-packed alignment pairs, mirrored pairs
sharing their scans and CUDA-graph replay of each batch are byte-identical
to the default mapping, through the C ABI, on an uneven workload (candidate
counts from 1 to thousands), on equal-length paired-end reads and in several
batches."""
import os

import numpy as np
import pytest

import care_b200
from care_b200 import datagen, learned

pytestmark = pytest.mark.gpu

VARIANTS = [
    {"msa_order": 1},
    {"msa_queue": 1},
    {"msa_order": 1, "msa_queue": 1},
    {"msa_warps": 8},
    {"align_block": 256},
    {"pair_order": 1},
    {"graph": 1},
    {"pair_mirror": 1},
    {"pair_mirror": 1, "pair_order": 1},
    {"cand_set_log2": 8},
    {"cand_set_log2": 12},
    {"align_warp": 1},
    {"align_warp": 1, "pair_mirror": 1, "align_block": 256},
    {"align_warp": 1, "pair_mirror": 1, "pair_order": 1},
    {"align_classes": 1},
    {"align_classes": 1, "pair_order": 1, "align_block": 256},
    {"msa_order": 1, "msa_queue": 1, "msa_warps": 8, "align_block": 256, "pair_order": 1, "graph": 1,
     "pair_mirror": 1},
]

UNEVEN_ARGS = "-c 40 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode SE --candidateCorrection"


@pytest.fixture(scope="module")
def uneven(tmp_path_factory):
    rs = datagen.single_end_uneven(seed=61, genome_size=400_000, coverage=40)
    d = tmp_path_factory.mktemp("tune")
    inp = str(d / "in.fq")
    rs.write_fastq(inp)
    return rs, inp, d


def _run(inp, args, tuning=None, out=None, batch_size=0, **kw):
    with care_b200.Corrector(care_b200.options_from_args(args, batch_size=batch_size, **kw)) as c:
        c.load_files([inp])
        c.build_tables()
        if tuning:
            c.tuning = dict(care_b200.Tuning.from_dict({}).as_dict(), **tuning)
            assert all(c.tuning[k] == v for k, v in tuning.items())
        res = c.correct_range()
        if out:
            c.write_output(out)
    return res


def _same(a, b):
    assert np.array_equal(a.status, b.status)
    assert np.array_equal(a.num_edits, b.num_edits)
    corr = (a.status & 1) == 1
    assert np.array_equal(a.sequences[corr], b.sequences[corr])
    key = lambda r: sorted(zip(r.cand_read_ids.tolist(), r.cand_anchor_ids.tolist(), r.cand_shifts.tolist(),
                               r.cand_use_edits.tolist(), [bytes(x) for x in r.cand_sequences]))
    assert key(a) == key(b)


def test_uneven_candidate_counts(uneven):
    """The fixture is uneven: anchors with a handful and with hundreds of candidates."""
    rs, inp, d = uneven
    with care_b200.Corrector(care_b200.options_from_args(UNEVEN_ARGS)) as c:
        c.load_files([inp])
        c.build_tables()
        c.correct_range()
        st = c.last_stats()
    assert st["pairs"] / st["anchors"] > 20


@pytest.mark.parametrize("variant", VARIANTS, ids=lambda v: "+".join(sorted(v)))
def test_variant_byte_identical(uneven, variant):
    rs, inp, d = uneven
    base_out, var_out = str(d / "base.fq"), str(d / "var.fq")
    base = _run(inp, UNEVEN_ARGS, out=base_out)
    var = _run(inp, UNEVEN_ARGS, variant, out=var_out)
    _same(base, var)
    assert open(base_out, "rb").read() == open(var_out, "rb").read()


@pytest.mark.parametrize("variant", [VARIANTS[-1], {"graph": 1}], ids=["all", "graph"])
def test_variant_in_several_batches(uneven, variant):
    """Batches of 4,096 anchors: the instantiated graph is updated in place
    from batch to batch (last batch smaller)."""
    rs, inp, d = uneven
    _same(_run(inp, UNEVEN_ARGS), _run(inp, UNEVEN_ARGS, variant, batch_size=4096))


@pytest.mark.parametrize("batch_size", [0, 1536], ids=["one-batch", "batches"])
def test_mirror_pairs_paired_end(tmp_path, batch_size):
    """Equal-length paired-end reads of a repeat-rich genome (many tied
    shifts): with pair_mirror most pairs are answered by their mirror's scan,
    and records, pair flags and the written file are unchanged. With small
    batches only pairs whose reads are anchors of the same batch mirror."""
    rs = datagen.paired_end_repeats(seed=63, genome_size=150_000, repeat_unit=600, repeat_copies=8)
    inp = str(tmp_path / "pe.fq")
    rs.write_fastq(inp)
    args = "-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE --candidateCorrection"
    outs, stats = [], []
    for tuning in (None, {"pair_mirror": 1}):
        with care_b200.Corrector(care_b200.options_from_args(args, batch_size=batch_size)) as c:
            c.load_files([inp])
            c.build_tables()
            if tuning:
                c.tuning = dict(care_b200.Tuning.from_dict({}).as_dict(), **tuning)
            res = c.correct_range()
            stats.append(c.last_stats())
            out = str(tmp_path / f"out{len(outs)}.fq")
            c.write_output(out)
        outs.append((res, out))
    _same(outs[0][0], outs[1][0])
    assert open(outs[0][1], "rb").read() == open(outs[1][1], "rb").read()
    assert stats[0]["pairs"] == stats[1]["pairs"]
    # the scans run: about half of all pairs in one batch, fewer saved in many
    ratio = stats[1]["word_compares"] / stats[0]["word_compares"]
    assert ratio < (0.6 if batch_size == 0 else 1.0)


@pytest.mark.parametrize("log2", [6, 7])
def test_candidate_spill_pass(uneven, log2):
    """A main-pass set of 64 or 128 entries sends every anchor with more than
    32 or 64 unique candidates to the second, full-set pass: the candidate
    lists, and so every result, equal the default mapping's."""
    rs, inp, d = uneven
    base_out, var_out = str(d / "base_sp.fq"), str(d / "var_sp.fq")
    base = _run(inp, UNEVEN_ARGS, out=base_out)
    with care_b200.Corrector(care_b200.options_from_args(UNEVEN_ARGS)) as c:
        c.load_files([inp])
        c.build_tables()
        c.tuning = dict(care_b200.Tuning.from_dict({}).as_dict(), cand_set_log2=log2)
        var = c.correct_range()
        st = c.last_stats()
        c.write_output(var_out)
    assert 0.05 * st["anchors"] < st["spilled_anchors"] < st["anchors"]
    _same(base, var)
    assert open(base_out, "rb").read() == open(var_out, "rb").read()


def test_variants_with_the_learned_decision(tmp_path):
    rs = datagen.paired_end_repeats(seed=62, genome_size=200_000, repeat_unit=1000, repeat_copies=6)
    inp = str(tmp_path / "pe.fq")
    rs.write_fastq(inp)
    args = "-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE"
    params = learned.load_params(os.path.join(os.path.dirname(care_b200.__file__), "data", "mlp_pe30x.bin"))

    def rows(tuning):
        with care_b200.Corrector(care_b200.options_from_args(args, correction_type=1)) as c:
            c.load_files([inp])
            c.build_tables()
            c.set_mlp(params)
            if tuning:
                c.tuning = dict(care_b200.Tuning.from_dict({}).as_dict(), **tuning)
            f = c.collect_features()
            res = c.correct_range()
        o = np.lexsort((f["pos"], f["read_id"]))
        return res, {k: v[o] for k, v in f.items()}

    base, fb = rows(None)
    var, fv = rows(VARIANTS[-1])
    _same(base, var)
    for k in ("read_id", "pos", "orig", "cons"):
        assert np.array_equal(fb[k], fv[k])
    assert np.array_equal(fb["x"].view(np.uint32), fv["x"].view(np.uint32))
    assert np.array_equal(fb["logit"], fv["logit"])


def test_autotuner_on_a_sample(uneven):
    """The tuner walks the knobs, checks every variant's results against the
    default's and returns a valid mapping no slower than the default."""
    from care_b200 import autotune
    rs, inp, d = uneven
    with care_b200.Corrector(care_b200.options_from_args(UNEVEN_ARGS)) as c:
        c.load_files([inp])
        c.build_tables()
        best, info = autotune.tune(c, c.num_reads, sweeps=1, steps=1, log=lambda m: None)
        c.tuning = best                                       # accepted by the library
    assert set(best) == set(autotune.DEFAULT)
    assert info["best_ms"] <= info["default_ms"]
    assert len(info["measured"]) >= 1 + sum(len(v) - 1 for v in autotune.KNOBS.values())


def test_counted_word_compares(uneven):
    """The alignment's statistics form changes no result and counts between
    one and all of the un-pruned word compares of the same scans."""
    rs, inp, d = uneven
    with care_b200.Corrector(care_b200.options_from_args(UNEVEN_ARGS)) as c:
        c.load_files([inp])
        c.build_tables()
        base = c.correct_range()
        st0 = c.last_stats()
        c.count_word_compares(True)
        counted = c.correct_range()
        st1 = c.last_stats()
        c.count_word_compares(False)
        c.correct_range()
        st2 = c.last_stats()
    _same(base, counted)
    assert st0["word_compares_run"] == 0 and st2["word_compares_run"] == 0
    assert st1["word_compares"] == st0["word_compares"]
    assert 0 < st1["word_compares_run"] < st1["word_compares"]
