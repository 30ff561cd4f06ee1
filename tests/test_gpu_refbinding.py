"""The reference's own care-cpu program with its STEP2 bound to this library
(care_b200/binding/correct_b200.cpp in place of src/correct_cpu.cpp, built by
`make -C oracle ref-b200`): the reference's STEP1 builds its read storage and
minhasher, the binding hands them to the device and returns the serialized
records, and the reference's STEP3 (SerializedObjectStorage sort, merge,
write) produces the output file. It must equal care-cpu's own output on every
golden case, byte for byte."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BOUND = os.path.join(ROOT, "oracle", "_ref", "care-cpu-b200")
CASES = sorted(__import__("conftest").manifest()["cases"])

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(BOUND), reason="care-cpu-b200 not built (make -C oracle ref-b200)")]


@pytest.mark.parametrize("case", CASES)
def test_reference_program_with_bound_step2(golden, tmp_path, case):
    m = golden.cases[case]
    inp = golden.input(m["input"])
    r = subprocess.run([BOUND, "-i", inp, "-d", str(tmp_path), "-o", "bound.fq", "-t", "4"] + m["args"].split(),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Correction throughput" in r.stdout
    assert open(tmp_path / "bound.fq", "rb").read() == golden.expected(case)


def test_bound_program_with_tables_loaded_from_a_file(tmp_path):
    """Tables care-cpu saved with -c 50 loaded under -c 30: the reference
    keeps the file's per-map threshold, so the binding hands its minhasher to
    the device through the table file instead of rebuilding the tables."""
    import gzip
    gold = os.path.join(ROOT, "tests", "golden")
    inp, tab = str(tmp_path / "pre_pe.fq"), str(tmp_path / "pre_pe_h4.tables")
    for src, dst in (("pre_pe.fq.gz", inp), ("pre_pe_h4.tables.gz", tab)):
        with open(dst, "wb") as f:
            f.write(gzip.decompress(open(os.path.join(gold, src), "rb").read()))
    care_cpu = os.path.join(ROOT, "oracle", "_ref", "care-cpu")
    args = ["-c", "30", "-k", "20", "-h", "4", "-q", "--qualityScoreBits", "2", "--pairmode", "PE",
            "--load-hashtables-from", tab]
    outs = []
    for exe, name in ((care_cpu, "ref.fq"), (BOUND, "bound.fq")):
        r = subprocess.run([exe, "-i", inp, "-d", str(tmp_path), "-o", name, "-t", "4"] + args,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(open(tmp_path / name, "rb").read())
    assert outs[0] == outs[1]
