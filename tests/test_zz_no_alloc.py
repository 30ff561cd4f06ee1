"""The allocation-free entry point (care_b200_correct_range_noalloc).

It serves callers that cannot call cudaMalloc -- their device buffers come
from a framework's own pool or are mapped from elsewhere -- so every input
and output here is a device buffer this test owns (allocated with torch,
outside the entry point), and the entry point's working memory is the
library's fixed device array. Its results must equal those of the regular
entry point on the same anchors, on two calls in a row (the second call
reuses the array the first one left behind). Outputs are integer and byte
data: compared exactly. The file is collected last, so a run that stops at
its first failure has run every other test before it.
"""
import gzip
import os

import numpy as np
import pytest

import _oracle
import care_b200
from care_b200 import datagen

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


class DeviceStorage:
    """Read storage and tables of a Corrector copied into caller-owned
    (torch) device buffers, in the layouts of care_b200_device_reads and
    care_b200_device_tables."""

    def __init__(self, c: care_b200.Corrector, files, args, lengths=None):
        import torch
        tables = [c.get_table(i) for i in range(c.num_maps)]
        orc = _oracle.OracleRun(files, _oracle.opts_from_args(args), threads=4)
        try:
            seq, qual, amb = orc.storage()
            lens = orc.lengths() if lengths is None else lengths
        finally:
            orc.close()
        self.n = seq.shape[0]
        self.max_len = c.max_length
        dev = torch.device("cuda:0")
        if qual is None:                      # no qualities in use: a placeholder the entry point ignores
            qual = np.zeros((1, 1), np.uint32)
        self.t = [torch.from_numpy(seq.view(np.int32)).to(dev), torch.from_numpy(qual.view(np.int32)).to(dev),
                  torch.from_numpy(np.asarray(lens, np.int32)).to(dev)]
        flags = np.zeros(self.n, np.uint8)
        flags[amb] = 1
        self.t.append(torch.from_numpy(flags).to(dev))
        descs, slots, values = care_b200.table_device_layout(tables)
        self.t += [torch.from_numpy(np.frombuffer(descs, np.uint8).copy()).to(dev),
                   torch.from_numpy(np.frombuffer(slots, np.uint8).copy()).to(dev),
                   torch.from_numpy(values.view(np.int32)).to(dev)]
        s, q, ln, am, d, sl, v = self.t
        self.reads = care_b200.DeviceReads(s.data_ptr(), seq.shape[1], ln.data_ptr(), q.data_ptr(), qual.shape[1],
                                           am.data_ptr(), self.n, self.max_len)
        self.tables = care_b200.DeviceTables(len(tables), d.data_ptr(), sl.data_ptr(), v.data_ptr(),
                                             c.result_threshold)

    def outputs(self, count):
        import torch
        dev = torch.device("cuda:0")
        return (torch.full((count,), 255, dtype=torch.uint8, device=dev),
                torch.full((count,), -1, dtype=torch.int32, device=dev),
                torch.full((count, self.max_len), 7, dtype=torch.uint8, device=dev))

    def correct(self, opts, first, count, outs=None):
        import torch
        st, ne, sq = outs if outs is not None else self.outputs(count)
        care_b200.correct_range_noalloc(opts, self.reads, self.tables, first, count, st.data_ptr(), ne.data_ptr(),
                                        sq.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        return st.cpu().numpy(), ne.cpu().numpy(), sq.cpu().numpy()


def assert_equal_to_main_path(ref, first, count, got, min_corrected=0.5):
    g_st, g_ne, g_sq = got
    r_st = ref.status[first:first + count]
    assert np.array_equal(g_st, r_st)
    corr = (r_st & 1) == 1
    assert corr.sum() > count * min_corrected
    assert np.array_equal(g_ne[corr], ref.num_edits[first:first + count][corr])
    assert np.array_equal(g_sq[corr], ref.sequences[first:first + count][corr])
    assert not g_sq[~corr].any()


def test_noalloc_matches_correct_range(golden):
    m = golden.cases["pe_q2"]
    files = [golden.input(m["input"])]
    opts = care_b200.options_from_args(m["args"])
    with care_b200.Corrector(opts) as c:
        c.load_files(files)
        c.build_tables()
        ref = c.correct_range()
        ds = DeviceStorage(c, files, m["args"])
    n = ds.n
    for first, count in [(0, n), (200, n - 400)]:
        assert_equal_to_main_path(ref, first, count, ds.correct(opts, first, count))


def test_noalloc_uses_the_threshold_of_tables_loaded_from_a_file(tmp_path):
    """Tables care-cpu saved with -c 50 (per-map threshold 125) queried under
    options with -c 10 (which would derive 25): the main path adopts the
    file's threshold, and so does this entry point when the tables say so."""
    inp = str(tmp_path / "pre_pe.fq")
    tab = str(tmp_path / "pre_pe_h4.tables")
    for src, dst in (("pre_pe.fq.gz", inp), ("pre_pe_h4.tables.gz", tab)):
        with open(dst, "wb") as f:
            f.write(gzip.decompress(open(os.path.join(GOLD, src), "rb").read()))
    args = "-c 10 -k 20 -h 4 -q --qualityScoreBits 2 --pairmode PE"
    opts = care_b200.options_from_args(args)
    with care_b200.Corrector(opts) as c:
        c.load_files([inp])
        c.load_hashtables(tab)
        assert c.result_threshold == 125
        ref = c.correct_range()
        ds = DeviceStorage(c, [inp], args)
    assert_equal_to_main_path(ref, 0, ds.n, ds.correct(opts, 0, ds.n), min_corrected=0.0)


def test_noalloc_pair_overflow_then_normal_call(tmp_path):
    """More candidate pairs than the array holds: CARE_B200_ELIMIT, and the
    next call (fewer anchors) still equals the main path."""
    rs = datagen.single_end_uniform(seed=41, genome_size=20_000, num_reads=care_b200.NOALLOC_MAX_ANCHORS, L=100)
    inp = str(tmp_path / "dense.fq")
    rs.write_fastq(inp)
    args = "-c 80 -k 20 -h 16 --pairmode SE"
    opts = care_b200.options_from_args(args)
    with care_b200.Corrector(opts) as c:
        c.load_files([inp])
        c.build_tables()
        ref = c.correct_range()
        assert c.last_stats()["pairs"] > care_b200.NOALLOC_MAX_PAIRS
        ds = DeviceStorage(c, [inp], args)
    with pytest.raises(care_b200.CareError, match=r"\(-6\)"):
        ds.correct(opts, 0, ds.n)
    assert_equal_to_main_path(ref, 1000, 4000, ds.correct(opts, 1000, 4000))


def test_noalloc_rejects_lengths_beyond_max_length(golden):
    m = golden.cases["pe_q2"]
    files = [golden.input(m["input"])]
    opts = care_b200.options_from_args(m["args"])
    with care_b200.Corrector(opts) as c:
        c.load_files(files)
        c.build_tables()
        ref = c.correct_range()
        lens = np.full(c.num_reads, c.max_length, np.int32)
        lens[777] = c.max_length + 1
        bad = DeviceStorage(c, files, m["args"], lengths=lens)
        ok = DeviceStorage(c, files, m["args"])
    with pytest.raises(care_b200.CareError, match=r"\(-1\)"):
        bad.correct(opts, 0, 64)
    assert_equal_to_main_path(ref, 0, ok.n, ok.correct(opts, 0, ok.n))


def test_noalloc_leaves_free_device_memory_unchanged(golden):
    """After the first call on the device (which places the array), further
    calls change nothing in the device's free memory."""
    import torch
    m = golden.cases["pe_q2"]
    files = [golden.input(m["input"])]
    opts = care_b200.options_from_args(m["args"])
    with care_b200.Corrector(opts) as c:
        c.load_files(files)
        c.build_tables()
        ref = c.correct_range()
        ds = DeviceStorage(c, files, m["args"])
    outs = ds.outputs(ds.n)
    ds.correct(opts, 0, ds.n, outs)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        got = ds.correct(opts, 0, ds.n, outs)
        assert torch.cuda.mem_get_info()[0] == free0
    assert_equal_to_main_path(ref, 0, ds.n, got)


def test_noalloc_rejects_sizes_beyond_its_array():
    import torch
    opts = care_b200.options_from_args("-c 30 -k 20 -h 4 --pairmode SE")
    dev = torch.device("cuda:0")
    n = care_b200.NOALLOC_MAX_ANCHORS + 2
    buf = torch.zeros(n * 16, dtype=torch.int32, device=dev)
    dreads = care_b200.DeviceReads(buf.data_ptr(), 10, buf.data_ptr(), 0, 0, buf.data_ptr(), n, 150)
    dtables = care_b200.DeviceTables(4, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 0)
    with pytest.raises(care_b200.CareError, match=r"\(-6\)"):
        care_b200.correct_range_noalloc(opts, dreads, dtables, 0, n, buf.data_ptr(), buf.data_ptr(),
                                        buf.data_ptr(), 0)
