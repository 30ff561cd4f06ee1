"""STEP1 parsed and encoded on the device (care_b200_load_reads_from_files_device)
against the host parse (care_b200_load_reads_from_files), through the C ABI.

The whole read storage is compared through care-cpu's read-storage file
(care_b200_save_preprocessed_reads: packed sequences, encoded qualities,
lengths, ambiguous ids), byte for byte, and the corrected output of every
golden case must equal care-cpu's. Covered: N bases and lower case
(include/chunkedreadstorageconstruction.hpp:67-92), the N-rotation counter
across 65,536-read parser batches (:106, :259) and across two single-end
files, two files of mates, --excludeAmbiguous, 1/2/8-bit qualities
(include/qualityscorecompression.hpp:90-119), CRLF line ends, a missing last
line end, FASTA; and a file whose layout is not strict 4-line FASTQ is
refused with the storage left to the host parse."""
import os

import numpy as np
import pytest

import care_b200
from care_b200 import datagen

pytestmark = pytest.mark.gpu
CASES = sorted(__import__("conftest").manifest()["cases"])


def storage_bytes(files, args, device, tmp_path, tag):
    with care_b200.Corrector(care_b200.options_from_args(args)) as c:
        c.load_files(files, device=device)
        out = str(tmp_path / f"{tag}_{int(device)}.bin")
        c.save_preprocessed_reads(out)
    data = open(out, "rb").read()
    os.unlink(out)
    return data


def assert_same_storage(files, args, tmp_path, tag="s"):
    host = storage_bytes(files, args, False, tmp_path, tag)
    dev = storage_bytes(files, args, True, tmp_path, tag)
    assert len(dev) == len(host)
    assert dev == host


@pytest.mark.parametrize("case", CASES)
def test_golden_case_storage_and_output(golden, tmp_path, case):
    m = golden.cases[case]
    files = [golden.input(m["input"])]
    assert_same_storage(files, m["args"], tmp_path)
    out = str(tmp_path / "dev.fq")
    with care_b200.Corrector(care_b200.options_from_args(m["args"])) as c:
        c.load_files(files, device=True)
        c.build_tables()
        c.correct_range()
        c.write_output(out)
    assert open(out, "rb").read() == golden.expected(case)


def test_rotation_over_parser_batches(tmp_path):
    """More than two 65,536-read batches with N bases (0.1 % per base) and
    lower-case reads: the turn counter restarts at every batch."""
    rs = datagen.paired_end_large(seed=71, genome_size=400_000, chunk_pairs=20_000)
    lower = np.zeros(rs.num_reads, bool)
    lower[::97] = True
    rs.seqs[lower] = np.where(rs.seqs[lower] == ord("N"), ord("n"), rs.seqs[lower] + 32)
    assert rs.num_reads > 2 * 65536
    inp = str(tmp_path / "n.fq")
    rs.write_fastq(inp)
    args = "-c 50 -k 20 -h 16 -q --qualityScoreBits 2 --pairmode PE --excludeAmbiguous"
    assert_same_storage([inp], args, tmp_path)


def test_two_files_of_mates_and_two_single_end_files(tmp_path):
    rs = datagen.paired_end_large(seed=72, genome_size=200_000, chunk_pairs=20_000)
    lines = open_fastq_records(rs)
    m1, m2 = str(tmp_path / "r1.fq"), str(tmp_path / "r2.fq")
    with open(m1, "wb") as f:
        f.write(b"".join(lines[0::2]))
    with open(m2, "wb") as f:
        f.write(b"".join(lines[1::2]))
    assert_same_storage([m1, m2], "-c 50 -k 20 -h 16 -q --qualityScoreBits 8 --pairmode PE", tmp_path, "pe")
    # single-end: the second file restarts the turn counter
    assert_same_storage([m1, m2], "-c 50 -k 20 -h 16 -q --qualityScoreBits 1 --pairmode SE", tmp_path, "se")


def open_fastq_records(rs):
    out = []
    for i in range(rs.num_reads):
        L = int(rs.lengths[i])
        out.append(b"@r%d x\n%s\n+\n%s\n" % (i, rs.seqs[i, :L].tobytes(), rs.quals[i, :L].tobytes()))
    return out


def test_crlf_missing_last_line_end_and_fasta(tmp_path):
    rs = datagen.single_end_uneven(seed=73, genome_size=60_000, coverage=20)
    recs = open_fastq_records(rs)
    crlf = str(tmp_path / "crlf.fq")
    with open(crlf, "wb") as f:
        f.write(b"".join(recs).replace(b"\n", b"\r\n"))
    args = "-c 20 -k 20 -h 16 -q --qualityScoreBits 2 --pairmode SE"
    assert_same_storage([crlf], args, tmp_path, "crlf")
    cut = str(tmp_path / "cut.fq")
    with open(cut, "wb") as f:
        f.write(b"".join(recs)[:-1])
    assert_same_storage([cut], args, tmp_path, "cut")
    fa = str(tmp_path / "r.fa")
    with open(fa, "wb") as f:
        for i in range(rs.num_reads):
            f.write(b">r%d\n%s\n" % (i, rs.seqs[i, :int(rs.lengths[i])].tobytes()))
    assert_same_storage([fa], "-c 20 -k 20 -h 16 --pairmode SE", tmp_path, "fa")


def test_irregular_layout_is_left_to_the_host_parse(tmp_path):
    rs = datagen.single_end_uniform(seed=74, genome_size=20_000, num_reads=3000)
    recs = open_fastq_records(rs)
    bad = str(tmp_path / "blank.fq")
    with open(bad, "wb") as f:
        f.write(b"".join(recs[:100]) + b"\n" + b"".join(recs[100:]))
    args = "-c 30 -k 20 -h 16 --pairmode SE"
    with care_b200.Corrector(care_b200.options_from_args(args)) as c:
        with pytest.raises(care_b200.CareError, match=r"\(-1\)"):
            c.load_files([bad], device=True)
        c.load_files([bad])
        assert c.num_reads == 3000
