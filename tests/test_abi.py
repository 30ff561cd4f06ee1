"""The C-ABI library loads and exports every entry point include/care_b200.h
declares (no compute without a GPU)."""
import os
import re
import subprocess

import care_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "care_b200.h")).read()
    return sorted(set(re.findall(r"\b(care_b200_\w+)\s*\(", text)))


def test_header_matches_python_binding():
    assert declared() == sorted(care_b200.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = care_b200.load_library()
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", care_b200.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (care_b200_\w+)", out))
    assert set(declared()) <= exported


def test_default_options_match_reference_defaults():
    o = care_b200.default_options()
    assert (o.kmerlength, o.num_maps, o.min_overlap, o.new_columns_to_correct, o.quality_bits) == (20, 48, 30, 15, 8)
    assert abs(o.max_error_rate - 0.2) < 1e-7 and abs(o.min_overlap_ratio - 0.3) < 1e-7
    assert abs(o.estimated_errorrate - 0.06) < 1e-7 and abs(o.m_coverage - 0.6) < 1e-7
    assert abs(o.paired_filter_threshold - 0.06) < 1e-7


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    try:
        care_b200.Corrector(estimated_coverage=30.0)
    except care_b200.CareError as e:
        assert "create" in str(e)
    else:
        raise AssertionError("context creation must fail loudly without a GPU")


def test_tuning_struct_and_default():
    """care_b200_tuning: the header's fields in order are the binding's, the
    library's default mapping is the autotuner's starting point, and every
    knob the tuner walks is a field."""
    text = open(os.path.join(ROOT, "include", "care_b200.h")).read()
    body = re.search(r"typedef struct care_b200_tuning \{(.*?)\} care_b200_tuning;", text, re.S).group(1)
    fields = re.findall(r"^\s*int\s+(\w+);", body, re.M)
    assert fields == [k for k, _ in care_b200.Tuning._fields_]
    from care_b200 import autotune
    assert care_b200.Tuning.from_dict({}).as_dict() == autotune.DEFAULT
    assert set(autotune.KNOBS) <= set(fields)


def test_cli_lists_care_cpu_options():
    """The drop-in binary accepts care-cpu's option names (the usage text, no
    GPU needed) and rejects unknown options."""
    out = subprocess.run([care_b200.CLI_PATH, "--help"], capture_output=True, text=True)
    assert out.returncode == 0
    text = out.stdout + out.stderr
    for opt in ("--kmerlength", "--hashmaps", "--useQualityScores", "--qualityScoreBits", "--excludeAmbiguous",
                "--candidateCorrection", "--candidateCorrectionNewColumns", "--minalignmentoverlap",
                "--maxmismatchratio", "--minalignmentoverlapratio", "--errorfactortuning", "--coveragefactortuning",
                "--pairedFilterThreshold", "--correctionQualityLabels", "--correctionType",
                "--save-preprocessedreads-to", "--load-preprocessedreads-from", "--save-hashtables-to",
                "--load-hashtables-from"):
        assert opt in text, opt
    bad = subprocess.run([care_b200.CLI_PATH, "--no-such-option"], capture_output=True, text=True)
    assert bad.returncode != 0 and "unknown option" in bad.stderr
