"""Regenerates the preprocessed-read fixtures from the reference's own care-cpu.

    make -C oracle ref && python tests/golden/make_preprocessed.py

Each case is a seeded synthetic read set (care_b200.datagen) written as FASTQ
and the binary read storage that `care-cpu --save-preprocessedreads-to` writes
for it (ChunkedReadStorage::saveToFile, include/chunkedreadstorage.hpp). For
the paired-end set also the minhash tables that `care-cpu --save-hashtables-to`
writes with 4 maps (OrdinaryCpuMinhasher::writeToStream,
include/ordinaryminhasher.hpp:303-316). All are committed gzip-compressed; the
tests read only the committed files.
"""
from __future__ import annotations

import gzip
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from care_b200 import datagen  # noqa: E402

CARE_CPU = os.path.join(ROOT, "oracle", "_ref", "care-cpu")

# name -> (read set, care-cpu options)
# tables of a case's reads: name -> (case, care-cpu options)
TABLES = {"pre_pe_h4": ("pre_pe", "-c 50 -k 20 -h 4 -q --qualityScoreBits 2 --pairmode PE")}

CASES = {
    # equal lengths (no length bits), 2-bit qualities, reads with N bases
    "pre_pe": (lambda: datagen.paired_end_large(seed=91, genome_size=6_000, chunk_pairs=2_000),
               "-c 50 -k 20 -h 16 -q --qualityScoreBits 2 --pairmode PE"),
    # lengths 50..250 (bit-packed lengths), 8-bit qualities
    "pre_un": (lambda: datagen.single_end_uneven(seed=92, genome_size=4_000, coverage=10),
               "-c 10 -k 20 -h 16 -q --qualityScoreBits 8 --pairmode SE"),
}


def main() -> int:
    for name, (make, args) in CASES.items():
        rs = make()
        with tempfile.TemporaryDirectory() as d:
            fq = os.path.join(d, name + ".fq")
            rs.write_fastq(fq)
            binf = os.path.join(d, name + ".bin")
            cmd = [CARE_CPU, "-i", fq, "-d", d, "-o", "out.fq", "-t", "4",
                   "--save-preprocessedreads-to", binf] + args.split()
            subprocess.run(cmd, check=True, capture_output=True, text=True)
            for src, dst in ((fq, name + ".fq.gz"), (binf, name + ".bin.gz")):
                with open(src, "rb") as f, open(os.path.join(HERE, dst), "wb") as g:
                    g.write(gzip.compress(f.read(), mtime=0))
            for tname, (case, targs) in TABLES.items():
                if case != name:
                    continue
                tab = os.path.join(d, tname + ".tables")
                cmd = [CARE_CPU, "-i", fq, "-d", d, "-o", "out2.fq", "-t", "4",
                       "--save-hashtables-to", tab] + targs.split()
                subprocess.run(cmd, check=True, capture_output=True, text=True)
                with open(tab, "rb") as f, open(os.path.join(HERE, tname + ".tables.gz"), "wb") as g:
                    g.write(gzip.compress(f.read(), mtime=0))
        print(name, len(rs.lengths), "reads")
    return 0


if __name__ == "__main__":
    sys.exit(main())
