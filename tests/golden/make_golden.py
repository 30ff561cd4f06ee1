"""Regenerates the golden fixtures from the reference's own care-cpu.

    make -C oracle ref && python tests/golden/make_golden.py

Inputs are seeded synthetic read sets (care_b200.datagen) small enough to
commit; each expected output is care-cpu (built from the reference sources by
oracle/Makefile) run with the option set named in CASES. The reference is
only needed to regenerate; the tests read the committed .gz files.
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from care_b200 import datagen  # noqa: E402

CARE_CPU = os.path.join(ROOT, "oracle", "_ref", "care-cpu")


def write_gz(path: str, data: bytes) -> None:
    """Deterministic gzip (no timestamp, no file name)."""
    with open(path, "wb") as raw, gzip.GzipFile(fileobj=raw, mode="wb", compresslevel=9, mtime=0, filename="") as g:
        g.write(data)


def make_delta(original: bytes, output: bytes) -> bytes:
    """Records whose header or sequence changed: "index\theader\tsequence" lines."""
    a = original.split(b"\n")
    b = output.split(b"\n")
    assert len(a) == len(b), "record count changed"
    lines = []
    for i in range(0, len(a) - 1, 4):
        if a[i] != b[i] or a[i + 1] != b[i + 1]:
            lines.append(b"%d\t%s\t%s" % (i // 4, b[i][1:], b[i + 1]))
    return b"\n".join(lines) + b"\n"


def apply_delta(original: bytes, delta: bytes) -> bytes:
    """Inverse of make_delta: the full expected output file."""
    a = original.split(b"\n")
    for line in delta.split(b"\n"):
        if not line:
            continue
        idx, head, seq = line.split(b"\t")
        i = 4 * int(idx)
        a[i] = b"@" + head
        a[i + 1] = seq
    return b"\n".join(a)


def make_inputs():
    out = {}
    # single-end, uniform genome, 100 bp (the 1 Mbp / 300k-read workload, scaled down)
    out["se"] = datagen.single_end_uniform(seed=11, genome_size=10_000, num_reads=3000)
    # paired-end with a repeat family, position-dependent errors, Phred qualities
    out["pe"] = datagen.paired_end_repeats(seed=12, genome_size=12_000, repeat_unit=500,
                                           repeat_copies=4)
    # single-end, lengths 50..250, repeats, N bases and lower-case bases
    rs = datagen.single_end_uneven(seed=13, genome_size=12_000, coverage=30)
    rng = np.random.default_rng(14)
    for i in rng.choice(rs.num_reads, max(1, rs.num_reads // 30), replace=False):
        rs.seqs[i, rng.integers(0, rs.lengths[i])] = ord("N")
    for i in rng.choice(rs.num_reads, max(1, rs.num_reads // 60), replace=False):
        p = rng.integers(0, rs.lengths[i])
        rs.seqs[i, p] = rs.seqs[i, p] + 32
    out["un"] = rs
    return out


# case name -> (input, care-cpu arguments)
CASES = {
    "se_plain": ("se", "-c 30 -k 20 -h 16 --pairmode SE"),
    "se_cand": ("se", "-c 30 -k 20 -h 16 --pairmode SE --candidateCorrection"),
    "pe_q2": ("pe", "-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE"),
    "pe_q2_cand": ("pe", "-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE --candidateCorrection"),
    "pe_q8_cand": ("pe", "-c 30 -k 20 -h 32 -q --qualityScoreBits 8 --pairmode PE --candidateCorrection"),
    "pe_q1": ("pe", "-c 30 -k 20 -h 24 -q --qualityScoreBits 1 --pairmode PE"),
    "un_q2": ("un", "-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode SE"),
    "un_excl_cand": ("un", "-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode SE --excludeAmbiguous --candidateCorrection"),
    "un_q8_labels": ("un", "-c 30 -k 16 -h 20 -q --qualityScoreBits 8 --pairmode SE --correctionQualityLabels"),
}


def main():
    if not os.path.exists(CARE_CPU):
        sys.exit("build the reference first: make -C oracle ref")
    inputs = make_inputs()
    manifest = {"cases": {}, "inputs": {}}
    with tempfile.TemporaryDirectory() as tmp:
        for name, rs in inputs.items():
            path = os.path.join(tmp, name + ".fq")
            rs.write_fastq(path)
            with open(path, "rb") as f:
                write_gz(os.path.join(HERE, name + ".fq.gz"), f.read())
            manifest["inputs"][name] = {"reads": rs.num_reads, "paired": rs.paired}
        for case, (inp, args) in CASES.items():
            outdir = os.path.join(tmp, case)
            cmd = [CARE_CPU, "-i", os.path.join(tmp, inp + ".fq"), "-d", outdir, "-o", "out.fq", "-t", "4"] + args.split()
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                sys.exit(f"care-cpu failed for {case}:\n{r.stdout}\n{r.stderr}")
            data = open(os.path.join(outdir, "out.fq"), "rb").read()
            original = open(os.path.join(tmp, inp + ".fq"), "rb").read()
            write_gz(os.path.join(HERE, case + ".delta.gz"), make_delta(original, data))
            manifest["cases"][case] = {"input": inp, "args": args,
                                       "sha256": hashlib.sha256(data).hexdigest()}
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print(json.dumps(manifest, indent=1))


if __name__ == "__main__":
    main()
