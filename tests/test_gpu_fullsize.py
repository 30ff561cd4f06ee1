"""Byte identity with the reference's care-cpu at the full sizes of the two
headline workloads, through the C ABI:

- single-end: 1 Mbp uniform genome, 300,000 x 100 bp reads, 1% substitutions,
  Q30/Q10; -c 30 -k 20 -h 16 --pairmode SE;
- paired-end: the benchmark's own read set (5 Mbp genome with 2% repeats,
  1,000,000 x 150 bp interleaved reads, position-dependent substitutions and
  Phred model, seed 2); -c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE.

and, on smaller genomes, the large workload's model (5 Mbp, 1.67M PE reads
with indels and N bases; -c 50 -k 20 -h 48 -q --qualityScoreBits 2 --pairmode
PE --excludeAmbiguous) and the uneven workload's model (2 Mbp, 50-250 bp SE
reads from repeat families; -c 40 -k 20 -h 32 -q --qualityScoreBits 2
--pairmode SE). All are corrected with the default launch mapping and with
the committed tuned mapping of their workload (one device batch for the whole
set), and each corrected FASTQ must equal care-cpu's by SHA-256. care-cpu's output path
is the reference's own (src/dispatch_care_correct_cpu.cpp:157-170, then the
merge and write of src/correctionresultoutput.cpp:1023-1060).
"""
import hashlib
import os
import subprocess

import pytest

import _oracle
import care_b200
from care_b200 import autotune, datagen

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(_oracle.CARE_CPU), reason="reference care-cpu not built")]

SE_ARGS = "-c 30 -k 20 -h 16 --pairmode SE"
PE_ARGS = "-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE"
# the large and the uneven workload models on smaller genomes
LARGE_ARGS = "-c 50 -k 20 -h 48 -q --qualityScoreBits 2 --pairmode PE --excludeAmbiguous"
UNEVEN_ARGS = "-c 40 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode SE"
TUNING = {"se": "pe", "pe": "pe", "large": "large", "uneven": "uneven"}


def sha256(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for block in iter(lambda: f.read(1 << 24), b""):
            h.update(block)
    return h.hexdigest()


@pytest.fixture(scope="module")
def workdir(tmp_path_factory):
    return tmp_path_factory.mktemp("fullsize")


_cache = {}


def reference_output(workdir, name: str, args: str) -> tuple[str, str]:
    """(input FASTQ, care-cpu's output) of a workload, generated once per module."""
    if name in _cache:
        return _cache[name]
    if name == "se":
        rs = datagen.single_end_uniform(seed=1, genome_size=1_000_000, num_reads=300_000, L=100)
        assert rs.num_reads == 300_000
    elif name == "pe":
        rs = datagen.paired_end_repeats(seed=2, genome_size=5_000_000, repeat_unit=5000)
        assert rs.num_reads == 1_000_000
    elif name == "large":       # 5 Mbp: 1.67M reads with indels and N bases
        rs = datagen.paired_end_large(seed=5, genome_size=5_000_000)
    else:                       # 2 Mbp: ~530k reads of 50-250 bases, repeat families
        rs = datagen.single_end_uneven(seed=3, genome_size=2_000_000, coverage=40.0)
    fq = str(workdir / f"{name}.fq")
    datagen.write_fastq_fast(rs, fq)
    del rs
    threads = len(os.sched_getaffinity(0))
    r = subprocess.run([_oracle.CARE_CPU, "-i", fq, "-d", str(workdir), "-o", f"{name}_cpu.fq",
                        "-t", str(threads)] + args.split(), capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-2000:]
    _cache[name] = (fq, str(workdir / f"{name}_cpu.fq"))
    return _cache[name]


@pytest.mark.parametrize("mapping", ["default", "tuned"])
@pytest.mark.parametrize("name,args", [("se", SE_ARGS), ("pe", PE_ARGS), ("large", LARGE_ARGS),
                                       ("uneven", UNEVEN_ARGS)])
def test_full_size_output_equals_care_cpu(workdir, name, args, mapping):
    fq, ref = reference_output(workdir, name, args)
    out = str(workdir / f"{name}_{mapping}_gpu.fq")
    with care_b200.Corrector(care_b200.options_from_args(args)) as c:
        if mapping == "tuned":
            c.tuning = autotune.load(TUNING[name])
        c.load_files([fq])
        c.build_tables()
        c.correct_range_raw(0, c.num_reads)
        stats = c.last_stats()
        c.write_output(out)
    if mapping == "tuned":
        assert stats["batches"] == 1            # the whole set is one device batch
    assert os.path.getsize(out) == os.path.getsize(ref)
    assert sha256(out) == sha256(ref)
    os.unlink(out)
