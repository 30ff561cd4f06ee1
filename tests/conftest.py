import gzip
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def golden_input(tmp_path, name: str) -> str:
    """Decompresses a committed golden input into tmp_path; returns the path."""
    out = os.path.join(str(tmp_path), name + ".fq")
    if not os.path.exists(out):
        with gzip.open(os.path.join(GOLDEN, name + ".fq.gz"), "rb") as g, open(out, "wb") as f:
            f.write(g.read())
    return out


def golden_expected(tmp_path, case: str) -> bytes:
    """The reference care-cpu output of a golden case (input + stored delta)."""
    from golden.make_golden import apply_delta  # noqa: E402
    m = manifest()["cases"][case]
    original = open(golden_input(tmp_path, m["input"]), "rb").read()
    with gzip.open(os.path.join(GOLDEN, case + ".delta.gz"), "rb") as g:
        delta = g.read()
    return apply_delta(original, delta)


@pytest.fixture
def golden(tmp_path):
    class G:
        cases = manifest()["cases"]

        def input(self, name):
            return golden_input(tmp_path, name)

        def expected(self, case):
            return golden_expected(tmp_path, case)

    return G()
