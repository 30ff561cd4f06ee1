"""The CPU oracle against the reference itself.

Every golden case (tests/golden/, outputs of the reference's care-cpu built
from its sources) must be reproduced byte for byte by the oracle. When the
reference binary is present (oracle/_ref/care-cpu), a freshly generated
input is also compared directly.
"""
import ctypes
import hashlib
import os
import subprocess

import pytest

import _oracle
from care_b200 import datagen


@pytest.mark.parametrize("case", sorted(__import__("conftest").manifest()["cases"]))
def test_oracle_reproduces_golden(golden, tmp_path, case):
    m = golden.cases[case]
    inp = golden.input(m["input"])
    expected = golden.expected(case)
    assert hashlib.sha256(expected).hexdigest() == m["sha256"]
    opts = _oracle.opts_from_args(m["args"])
    opts.threads = 4
    out = str(tmp_path / "oracle.fq")
    files = (ctypes.c_char_p * 1)(inp.encode())
    step2 = ctypes.c_double()
    rc = _oracle.lib().co_run(files, 1, out.encode(), ctypes.byref(opts), ctypes.byref(step2))
    assert rc == 0
    got = open(out, "rb").read()
    assert got == expected


@pytest.mark.skipif(not os.path.exists(_oracle.CARE_CPU), reason="reference care-cpu not built")
@pytest.mark.parametrize("args", [
    "-c 25 -k 18 -h 20 --pairmode PE -q --qualityScoreBits 2 --candidateCorrection",
    "-c 35 -k 24 -h 12 --pairmode SE",
])
def test_oracle_matches_reference_binary(tmp_path, args):
    if "PE" in args:
        rs = datagen.paired_end_repeats(seed=101, genome_size=8000, repeat_unit=400, repeat_copies=3)
    else:
        rs = datagen.single_end_uniform(seed=102, genome_size=6000, num_reads=2000, L=120)
    inp = str(tmp_path / "in.fq")
    rs.write_fastq(inp)
    r = subprocess.run([_oracle.CARE_CPU, "-i", inp, "-d", str(tmp_path), "-o", "ref.fq", "-t", "2"] + args.split(),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([_oracle.CLI, "-i", inp, "-d", str(tmp_path), "-o", "or.fq", "-t", "2"] + args.split(),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert open(tmp_path / "ref.fq", "rb").read() == open(tmp_path / "or.fq", "rb").read()
