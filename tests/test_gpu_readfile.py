"""The binary read-storage and minhash-table files on the GPU: storage and
tables loaded from the files care-cpu saved (tests/golden/make_preprocessed.py)
correct exactly like storage parsed from the same FASTQ and tables built on the
GPU, saves reproduce the reference's files, the CLI's load flags give the same
output, and a file with other quality bits is rejected as in the reference."""
import gzip
import os
import struct
import subprocess

import numpy as np
import pytest

import care_b200

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {"pre_pe": "-c 50 -k 20 -h 16 -q --qualityScoreBits 2 --pairmode PE --candidateCorrection",
         "pre_un": "-c 10 -k 20 -h 16 -q --qualityScoreBits 8 --pairmode SE --candidateCorrection"}


def unpack(tmp, name):
    out = {}
    for ext in ("fq", "bin"):
        p = os.path.join(tmp, f"{name}.{ext}")
        with open(p, "wb") as f:
            f.write(gzip.decompress(open(os.path.join(GOLD, f"{name}.{ext}.gz"), "rb").read()))
        out[ext] = p
    return out


def run(args, fq=None, binf=None, out=None):
    with care_b200.Corrector(care_b200.options_from_args(args)) as c:
        if fq:
            c.load_files([fq])
        if binf:
            c.load_preprocessed_reads(binf)
        c.build_tables()
        res = c.correct_range()
        if out:
            c.write_output(out)
    return res


def same(a, b):
    assert np.array_equal(a.status, b.status)
    assert np.array_equal(a.num_edits, b.num_edits)
    corr = (a.status & 1) == 1
    assert np.array_equal(a.sequences[corr], b.sequences[corr])
    key = lambda r: sorted(zip(r.cand_read_ids.tolist(), r.cand_anchor_ids.tolist(), r.cand_shifts.tolist(),
                               r.cand_use_edits.tolist(), [bytes(x) for x in r.cand_sequences]))
    assert key(a) == key(b)


@pytest.mark.parametrize("name", sorted(CASES))
def test_loaded_storage_corrects_like_fastq(tmp_path, name):
    p = unpack(str(tmp_path), name)
    a = run(CASES[name], fq=p["fq"])
    b = run(CASES[name], binf=p["bin"])
    assert (a.status & 1).sum() > 0
    same(a, b)


@pytest.mark.parametrize("name", sorted(CASES))
def test_save_reproduces_reference_file(tmp_path, name):
    p = unpack(str(tmp_path), name)
    out = str(tmp_path / "saved.bin")
    with care_b200.Corrector(care_b200.options_from_args(CASES[name])) as c:
        c.load_files([p["fq"]])
        c.save_preprocessed_reads(out)
    ref, ours = open(p["bin"], "rb").read(), open(out, "rb").read()
    end = lambda b: 53 + sum(struct.unpack_from("<3Q", b, 21))       # start of the ambiguous ids
    assert len(ref) == len(ours) and end(ref) == end(ours)
    assert ref[:end(ref)] == ours[:end(ours)]
    ids = lambda b: sorted(struct.unpack_from(f"<{struct.unpack_from('<Q', b, end(b))[0]}I", b, end(b) + 8))
    assert ids(ref) == ids(ours)


def test_cli_load_flag(tmp_path):
    p = unpack(str(tmp_path), "pre_pe")
    outs = []
    for extra in ([], ["--load-preprocessedreads-from", p["bin"]]):
        d = tmp_path / f"o{len(outs)}"
        d.mkdir()
        cmd = [care_b200.CLI_PATH, "-i", p["fq"], "-d", str(d), "-o", "out.fq"] + CASES["pre_pe"].split() + extra
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        outs.append((d / "out.fq").read_bytes())
    assert outs[0] == outs[1] and len(outs[0]) > 0


def test_quality_bits_mismatch_rejected(tmp_path):
    p = unpack(str(tmp_path), "pre_un")                 # saved with 8-bit qualities
    with care_b200.Corrector(care_b200.options_from_args(CASES["pre_un"].replace("Bits 8", "Bits 2"))) as c:
        with pytest.raises(care_b200.CareError, match="bits per quality"):
            c.load_preprocessed_reads(p["bin"])


H4 = "-c 50 -k 20 -h 4 -q --qualityScoreBits 2 --pairmode PE --candidateCorrection"


def tables_file(tmp):
    p = os.path.join(tmp, "pre_pe_h4.tables")
    with open(p, "wb") as f:
        f.write(gzip.decompress(open(os.path.join(GOLD, "pre_pe_h4.tables.gz"), "rb").read()))
    return p


def test_loaded_tables_correct_like_built_tables(tmp_path):
    p = unpack(str(tmp_path), "pre_pe")
    tab = tables_file(str(tmp_path))
    with care_b200.Corrector(care_b200.options_from_args(H4)) as c:
        c.load_files([p["fq"]])
        c.build_tables()
        built = [c.get_table(m) for m in range(c.num_maps)]
        a = c.correct_range()
    with care_b200.Corrector(care_b200.options_from_args(H4)) as c:
        c.load_preprocessed_reads(p["bin"])
        c.load_hashtables(tab)
        assert c.num_maps == 4
        loaded = [c.get_table(m) for m in range(c.num_maps)]
        b = c.correct_range()
    for x, y in zip(built, loaded):
        for u, v in zip(x, y):
            assert np.array_equal(u, v)
    assert (a.status & 1).sum() > 0
    same(a, b)


def test_save_tables_reproduces_reference_file(tmp_path):
    p = unpack(str(tmp_path), "pre_pe")
    out = str(tmp_path / "saved.tables")
    with care_b200.Corrector(care_b200.options_from_args(H4)) as c:
        c.load_files([p["fq"]])
        c.build_tables()
        c.save_hashtables(out)
    assert open(out, "rb").read() == open(tables_file(str(tmp_path)), "rb").read()


def test_cli_load_both_files(tmp_path):
    p = unpack(str(tmp_path), "pre_pe")
    tab = tables_file(str(tmp_path))
    outs = []
    for extra in ([], ["--load-preprocessedreads-from", p["bin"], "--load-hashtables-from", tab]):
        d = tmp_path / f"t{len(outs)}"
        d.mkdir()
        cmd = [care_b200.CLI_PATH, "-i", p["fq"], "-d", str(d), "-o", "out.fq"] + H4.split() + extra
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        outs.append((d / "out.fq").read_bytes())
    assert outs[0] == outs[1] and len(outs[0]) > 0
