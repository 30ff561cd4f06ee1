"""The allocation-free entry point (care_b200_correct_range_noalloc).

It serves callers that cannot call cudaMalloc -- their device buffers come
from a framework's own pool or are mapped from elsewhere -- so every input
and output here is a device buffer this test owns (allocated with torch,
outside the entry point), and the entry point's working memory is the
library's fixed device array. Its results must equal those of the regular
entry point on the same anchors, on two calls in a row (the second call
reuses the array the first one left behind). Outputs are integer and byte
data: compared exactly.
"""
import numpy as np
import pytest

import _oracle
import care_b200

pytestmark = pytest.mark.gpu


def test_noalloc_matches_correct_range(golden):
    import torch

    m = golden.cases["pe_q2"]
    files = [golden.input(m["input"])]
    opts = care_b200.options_from_args(m["args"])
    with care_b200.Corrector(opts) as c:
        c.load_files(files)
        c.build_tables()
        ref = c.correct_range()
        tables = [c.get_table(i) for i in range(c.num_maps)]
        max_len = c.max_length

    orc = _oracle.OracleRun(files, _oracle.opts_from_args(m["args"]), threads=4)
    try:
        seq, qual, amb = orc.storage()
        lens = orc.lengths()
    finally:
        orc.close()
    n = seq.shape[0]
    dev = torch.device("cuda:0")
    t_seq = torch.from_numpy(seq.view(np.int32)).to(dev)
    t_qual = torch.from_numpy(qual.view(np.int32)).to(dev)
    t_len = torch.from_numpy(lens.astype(np.int32)).to(dev)
    flags = np.zeros(n, np.uint8)
    flags[amb] = 1
    t_amb = torch.from_numpy(flags).to(dev)
    descs, slots, values = care_b200.table_device_layout(tables)
    t_descs = torch.from_numpy(np.frombuffer(descs, np.uint8).copy()).to(dev)
    t_slots = torch.from_numpy(np.frombuffer(slots, np.uint8).copy()).to(dev)
    t_vals = torch.from_numpy(values.view(np.int32)).to(dev)

    dreads = care_b200.DeviceReads(t_seq.data_ptr(), seq.shape[1], t_len.data_ptr(), t_qual.data_ptr(),
                                   qual.shape[1], t_amb.data_ptr(), n, max_len)
    dtables = care_b200.DeviceTables(len(tables), t_descs.data_ptr(), t_slots.data_ptr(), t_vals.data_ptr())
    stream = torch.cuda.current_stream().cuda_stream

    for first, count in [(0, n), (200, n - 400)]:
        st = torch.full((count,), 255, dtype=torch.uint8, device=dev)
        ne = torch.full((count,), -1, dtype=torch.int32, device=dev)
        sq = torch.full((count, max_len), 7, dtype=torch.uint8, device=dev)
        care_b200.correct_range_noalloc(opts, dreads, dtables, first, count, st.data_ptr(), ne.data_ptr(),
                                        sq.data_ptr(), stream)
        torch.cuda.synchronize()
        g_st = st.cpu().numpy()
        g_ne = ne.cpu().numpy()
        g_sq = sq.cpu().numpy()
        r_st = ref.status[first:first + count]
        assert np.array_equal(g_st, r_st)
        corr = (r_st & 1) == 1
        assert corr.sum() > count // 2
        assert np.array_equal(g_ne[corr], ref.num_edits[first:first + count][corr])
        assert np.array_equal(g_sq[corr], ref.sequences[first:first + count][corr])
        assert not g_sq[~corr].any()


def test_noalloc_rejects_sizes_beyond_its_array():
    import torch
    opts = care_b200.options_from_args("-c 30 -k 20 -h 4 --pairmode SE")
    dev = torch.device("cuda:0")
    n = care_b200.NOALLOC_MAX_ANCHORS + 2
    buf = torch.zeros(n * 16, dtype=torch.int32, device=dev)
    dreads = care_b200.DeviceReads(buf.data_ptr(), 10, buf.data_ptr(), 0, 0, buf.data_ptr(), n, 150)
    dtables = care_b200.DeviceTables(4, buf.data_ptr(), buf.data_ptr(), buf.data_ptr())
    with pytest.raises(care_b200.CareError, match=r"\(-6\)"):
        care_b200.correct_range_noalloc(opts, dreads, dtables, 0, n, buf.data_ptr(), buf.data_ptr(),
                                        buf.data_ptr(), 0)
