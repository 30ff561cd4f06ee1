"""Sharded correction through the C ABI on one GPU: the record streams of
the shards of a read set, merged, equal the whole range's records; the
Python record encoder (care_b200.shard) equals the library's serializer."""
import numpy as np
import pytest

import _oracle
import care_b200
from care_b200 import shard

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["pe_q2_cand", "se_cand", "un_excl_cand"])
@pytest.mark.parametrize("world", [2, 3])
def test_shards_merge_to_full_range(golden, case, world):
    m = golden.cases[case]
    with care_b200.Corrector(care_b200.options_from_args(m["args"])) as c:
        c.load_files([golden.input(m["input"])])
        c.build_tables()
        full = c.serialize(c.correct_range_raw(0, c.num_reads))
        parts = []
        for r in range(world):
            first, count = shard.shard_range(c.num_reads, r, world, bool(c.opts.paired_end))
            parts.append(c.serialize(c.correct_range_raw(first, count)))
    merged = shard.merge_records(parts)
    assert shard.record_multiset(merged) == shard.record_multiset(full)


def test_python_encoder_equals_library(golden):
    m = golden.cases["pe_q2_cand"]
    inp = golden.input(m["input"])
    orc = _oracle.OracleRun([inp], _oracle.opts_from_args(m["args"]), threads=4)
    try:
        with care_b200.Corrector(care_b200.options_from_args(m["args"])) as c:
            c.load_files([inp])
            c.build_tables()
            raw = c.correct_range_raw(0, c.num_reads)
            lib_blob = c.serialize(raw)
            res = c.correct_range()
        lens = orc.lengths()
        py_blob = shard.encode_records(range(res.first, res.first + len(res.status)), res.status, res.num_edits,
                                       res.sequences, res.cand_read_ids, res.cand_shifts, res.cand_use_edits,
                                       res.cand_sequences, lens, orc.original)
        assert shard.record_multiset(py_blob) == shard.record_multiset(lib_blob)
        assert shard.record_multiset(orc.records()) == shard.record_multiset(lib_blob)
    finally:
        orc.close()
