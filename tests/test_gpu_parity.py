"""Parity of the CUDA path (called through the C ABI) with the CPU oracle and
the reference's care-cpu outputs. Integer/byte work is bit-exact; the float
column sums follow the reference's order, so outputs are byte-identical."""
import ctypes
import os
import struct

import numpy as np
import pytest

import _oracle
import care_b200
from care_b200 import datagen

pytestmark = pytest.mark.gpu

CASES = sorted(__import__("conftest").manifest()["cases"])


def run_gpu(files, args, out=None, stats=None, tuning=None, **kw):
    o = care_b200.options_from_args(args, **kw)
    with care_b200.Corrector(o) as c:
        if tuning:
            c.tuning = tuning
        c.load_files(files)
        c.build_tables()
        res = c.correct_range()
        if stats is not None:
            stats.update(c.last_stats())
        if out:
            c.write_output(out)
        tables = [c.get_table(m) for m in range(c.num_maps)]
    return res, tables


@pytest.mark.parametrize("case", CASES)
def test_golden_file_byte_identical(golden, tmp_path, case):
    m = golden.cases[case]
    out = str(tmp_path / "gpu.fq")
    run_gpu([golden.input(m["input"])], m["args"], out=out)
    assert open(out, "rb").read() == golden.expected(case)


def compare_with_oracle(files, args, res, tables, threads=8):
    o = _oracle.opts_from_args(args)
    orc = _oracle.OracleRun(files, o, threads=threads)
    try:
        for m, (k, off, v) in enumerate(tables):
            ok, ooff, ov = orc.table(m)
            assert np.array_equal(k, ok) and np.array_equal(off, ooff) and np.array_equal(v, ov), f"table {m}"
        status, hq, ue, ne, seq = orc.anchors()
        lens = orc.lengths()
        g_corr = (res.status & 1).astype(np.uint8)
        g_hq = ((res.status >> 1) & 1).astype(np.uint8)
        g_ue = ((res.status >> 2) & 1).astype(np.uint8)
        assert np.array_equal(g_corr, status)
        corr = status == 1
        assert np.array_equal(g_hq[corr], hq[corr])
        assert np.array_equal(g_ue[corr], ue[corr])
        assert np.array_equal(res.num_edits[corr & (ue == 1)], ne[corr & (ue == 1)])
        for i in np.nonzero(corr)[0]:
            L = lens[i]
            assert bytes(res.sequences[i, :L]) == bytes(seq[i, :L]), f"anchor {i}"
        cands, cseq = orc.candidates()
        exp = sorted((c[0], c[1], c[2], c[3], bytes(cseq[j, :lens[c[0]]])) for j, c in enumerate(cands))
        got = sorted((int(res.cand_read_ids[j]), int(res.cand_anchor_ids[j]), int(res.cand_shifts[j]),
                      int(res.cand_use_edits[j]), bytes(res.cand_sequences[j, :lens[res.cand_read_ids[j]]]))
                     for j in range(len(res.cand_read_ids)))
        assert got == exp
    finally:
        orc.close()


@pytest.mark.parametrize("case", ["pe_q2_cand", "un_excl_cand", "se_cand", "pe_q1"])
def test_stage_outputs_match_oracle(golden, case):
    m = golden.cases[case]
    files = [golden.input(m["input"])]
    res, tables = run_gpu(files, m["args"])
    compare_with_oracle(files, m["args"], res, tables)


@pytest.mark.parametrize("mapping", ["default", "tuned"])
@pytest.mark.parametrize("workload,args", [
    ("pe", "-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE --candidateCorrection"),
    ("se", "-c 30 -k 20 -h 16 --pairmode SE"),
    ("un", "-c 40 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode SE --candidateCorrection"),
    ("large", "-c 50 -k 20 -h 48 -q --qualityScoreBits 2 --pairmode PE --excludeAmbiguous --candidateCorrection"),
])
def test_medium_sets_match_oracle(tmp_path, workload, args, mapping):
    """Medium sets of each workload model against the oracle, with the default
    launch mapping and with the committed tuning of that workload."""
    from care_b200 import autotune
    tuning = autotune.load({"pe": "pe", "se": "pe", "un": "uneven", "large": "large"}[workload]) \
        if mapping == "tuned" else None
    if workload == "large":
        # the large set's model: 50x, indels, N bases (ambiguous reads excluded)
        rs = datagen.paired_end_large(seed=24, genome_size=300_000, chunk_pairs=20_000)
    elif workload == "pe":
        rs = datagen.paired_end_repeats(seed=21, genome_size=300_000, repeat_unit=2000, repeat_copies=6)
    elif workload == "se":
        rs = datagen.single_end_uniform(seed=22, genome_size=200_000, num_reads=60_000)
    else:
        rs = datagen.single_end_uneven(seed=23, genome_size=200_000, coverage=40)
    inp = str(tmp_path / "in.fq")
    rs.write_fastq(inp)
    res, tables = run_gpu([inp], args, tuning=tuning)
    compare_with_oracle([inp], args, res, tables)


def test_upload_path_equals_file_path(golden):
    """Read storage and tables handed over through the upload entry points
    (the integration route for an existing CpuReadStorage / minhasher)."""
    m = golden.cases["pe_q2_cand"]
    files = [golden.input(m["input"])]
    res_a, tables = run_gpu(files, m["args"])
    orc = _oracle.OracleRun(files, _oracle.opts_from_args(m["args"]), threads=4)
    try:
        seq, qual, amb = orc.storage()
        lens = orc.lengths()
        with care_b200.Corrector(care_b200.options_from_args(m["args"])) as c:
            c.upload_reads(seq, lens, qual, amb)
            c.upload_tables([orc.table(i) for i in range(len(tables))])
            res_b = c.correct_range()
    finally:
        orc.close()
    assert np.array_equal(res_a.status, res_b.status)
    assert np.array_equal(res_a.sequences, res_b.sequences)
    assert sorted(res_a.cand_read_ids.tolist()) == sorted(res_b.cand_read_ids.tolist())


def test_batch_size_invariance(golden):
    m = golden.cases["pe_q2_cand"]
    files = [golden.input(m["input"])]
    res_a, _ = run_gpu(files, m["args"])
    res_b, _ = run_gpu(files, m["args"], batch_size=64)
    assert np.array_equal(res_a.status, res_b.status)
    assert np.array_equal(res_a.num_edits, res_b.num_edits)
    assert np.array_equal(res_a.sequences, res_b.sequences)
    key = lambda r: sorted(zip(r.cand_read_ids.tolist(), r.cand_anchor_ids.tolist()))
    assert key(res_a) == key(res_b)


def test_sub_range_equals_full_range(golden):
    m = golden.cases["se_plain"]
    files = [golden.input(m["input"])]
    o = care_b200.options_from_args(m["args"])
    with care_b200.Corrector(o) as c:
        c.load_files(files)
        c.build_tables()
        full = c.correct_range()
        part = c.correct_range(1000, 700)
    assert np.array_equal(full.status[1000:1700], part.status)
    corr = (part.status & 1) == 1          # rows of uncorrected anchors are unspecified
    assert corr.sum() > 0
    assert np.array_equal(full.sequences[1000:1700][corr], part.sequences[corr])


def test_serialized_records(golden):
    """EncodedTempCorrectedSequence byte records (correctedsequence.hpp:148-340)."""
    m = golden.cases["pe_q2_cand"]
    files = [golden.input(m["input"])]
    o = care_b200.options_from_args(m["args"])
    with care_b200.Corrector(o) as c:
        c.load_files(files)
        c.build_tables()
        raw = c.correct_range_raw(0, c.num_reads)
        blob = c.serialize(raw)
        status = np.ctypeslib.as_array(raw.anchor_status, shape=(raw.num_anchors,)).copy()
        nedits = np.ctypeslib.as_array(raw.anchor_num_edits, shape=(raw.num_anchors,)).copy()
        ncand = raw.num_candidates
    pos = 0
    anchors = cands = 0
    while pos < len(blob):
        rid, flags = struct.unpack_from("<II", blob, pos)
        nbytes = flags & ((1 << 29) - 1)
        typ = (flags >> 29) & 1
        hq = flags >> 31
        ue = (flags >> 30) & 1
        if typ == 0:
            anchors += 1
            assert status[rid] & 1 and bool(hq) == bool(status[rid] & 2) and bool(ue) == bool(status[rid] & 4)
            if ue:
                assert struct.unpack_from("<i", blob, pos + 8)[0] == nedits[rid]
        else:
            cands += 1
        pos += 8 + nbytes
    assert pos == len(blob)
    stored = ((status & 1) == 1) & ~(((status & 6) == 6) & (nedits == 0))
    assert anchors == int(stored.sum())
    assert cands == ncand


def test_short_reads_and_empty_anchors(tmp_path):
    """Reads shorter than k get no candidates (determineNumValues skips them)
    and are still emitted unchanged."""
    rs = datagen.single_end_uniform(seed=31, genome_size=5000, num_reads=1500, L=100)
    rs.lengths[::7] = 15          # shorter than k = 20
    inp = str(tmp_path / "in.fq")
    rs.write_fastq(inp)
    args = "-c 30 -k 20 -h 16 --pairmode SE"
    res, tables = run_gpu([inp], args, out=str(tmp_path / "gpu.fq"))
    assert not (res.status[::7] & 1).any()
    compare_with_oracle([inp], args, res, tables)
    r = __import__("subprocess").run([_oracle.CLI, "-i", inp, "-d", str(tmp_path), "-o", "or.fq"] + args.split(),
                                     capture_output=True)
    assert r.returncode == 0
    assert open(tmp_path / "gpu.fq", "rb").read() == open(tmp_path / "or.fq", "rb").read()
