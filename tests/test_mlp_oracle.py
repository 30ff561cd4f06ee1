"""Pins of the learned-decision oracles (CPU only): bfloat16 rounding,
the analytic gradient against finite differences, Adam against torch, the
C forward pass against the numpy one, and the decision-column rows of the C
oracle on a small genome."""
import ctypes
import os
import sys

import numpy as np
import pytest
import torch

import _oracle
from care_b200 import datagen

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as mo  # noqa: E402


def test_bf16_round_matches_torch():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.standard_normal(20000).astype(np.float32) * 10.0 ** rng.integers(-20, 20, 20000),
                        np.array([0.0, -0.0, 1.0, 65504.0, 3.0e38, -1e-40, np.inf, -np.inf], np.float32)])
    x = x.astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(mo.bf16(x), ref)
    L = _oracle.lib()
    c = np.array([L.co_bf16_round(float(v)) for v in x[:2000]], np.float32)
    assert np.array_equal(c, ref[:2000])


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((12, mo.NFEAT))
    y = (rng.random(12) < 0.5).astype(np.float64)
    p = mo.random_params(3, x).astype(np.float64)
    _, g = mo.loss_and_grad(p, x, y, emulate=False)
    eps = 1e-6
    idx = np.concatenate([rng.choice(np.arange(mo.W1, mo.B1), 12), rng.choice(np.arange(mo.B1, mo.W2), 6),
                          rng.choice(np.arange(mo.W2, mo.B2), 12), rng.choice(np.arange(mo.B2, mo.W3), 6),
                          rng.choice(np.arange(mo.W3, mo.B3), 6), [mo.B3]])
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (mo.loss_and_grad(pp, x, y, emulate=False)[0] - mo.loss_and_grad(pm, x, y, emulate=False)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-8, (i, fd, g[i])


def test_emulated_gradient_close_to_exact():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((4096, mo.NFEAT)).astype(np.float32)
    y = (rng.random(4096) < 0.3).astype(np.float32)
    p = mo.random_params(5, x)
    l0, g0 = mo.loss_and_grad(p, x, y, emulate=False)
    l1, g1 = mo.loss_and_grad(p, x, y, emulate=True)
    assert abs(l0 - l1) < 1e-2 * abs(l0)
    cos = g0 @ g1 / np.linalg.norm(g0) / np.linalg.norm(g1)
    assert cos > 0.999
    assert np.linalg.norm(g0 - g1) < 2e-2 * np.linalg.norm(g0)


def test_adam_matches_torch():
    rng = np.random.default_rng(6)
    p = mo.random_params(7)
    w = torch.nn.Parameter(torch.from_numpy(p[:mo.NPARAM].copy()))
    opt = torch.optim.Adam([w], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    m = np.zeros(mo.NPARAM, np.float32)
    v = np.zeros(mo.NPARAM, np.float32)
    for t in range(1, 6):
        g = (rng.standard_normal(mo.NPARAM) * 10.0 ** rng.uniform(-6, -1)).astype(np.float32)
        w.grad = torch.from_numpy(g.copy())
        opt.step()
        mo.adam(p, g, m, v, t)
        np.testing.assert_allclose(p[:mo.NPARAM], w.detach().numpy(), rtol=2e-6, atol=1e-9)


def test_c_forward_matches_numpy():
    rng = np.random.default_rng(8)
    x = rng.standard_normal((3000, mo.NFEAT)).astype(np.float32) * 2 + 0.5
    p = mo.random_params(9, x)
    ref = mo.forward(p, x, emulate=True)["logit"]
    L = _oracle.lib()
    pp = p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    got = np.array([L.co_mlp_logit(pp, np.ascontiguousarray(r).ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
                    for r in x], np.float32)
    d = np.abs(got - ref)
    assert np.quantile(d, 0.999) < 1e-4
    assert d.max() < 2e-2


@pytest.fixture(scope="module")
def small_pe(tmp_path_factory):
    rs = datagen.paired_end_repeats(seed=41, genome_size=60_000, repeat_unit=500, repeat_copies=6)
    d = tmp_path_factory.mktemp("clf")
    inp = str(d / "in.fq")
    rs.write_fastq(inp)
    return rs, inp


ARGS = "-c 30 -k 20 -h 16 -q --qualityScoreBits 2 --pairmode PE"


def _run(inp, mode, params=None, min_cov=3):
    o = _oracle.opts_from_args(ARGS)
    o.clf_mode = mode
    o.clf_min_coverage = min_cov
    keep = None
    if params is not None:
        keep = np.ascontiguousarray(params, np.float32)
        o.mlp = keep.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    run = _oracle.OracleRun([inp], o, threads=4)
    run._keep = keep
    return run


def test_decision_rows_are_the_non_hq_mismatch_columns(small_pe):
    rs, inp = small_pe
    run = _run(inp, 1)
    try:
        f = run.features()
        status, hq, ue, ne, seq = run.anchors()
        assert len(f["read_id"]) > 100
        # only corrected non-HQ anchors own rows
        assert np.all(status[f["read_id"]] == 1) and not np.any(hq[f["read_id"]])
        # rows are in anchor order, then position order
        key = f["read_id"].astype(np.int64) * 1000 + f["pos"]
        assert np.all(np.diff(key) > 0)
        assert np.all(f["orig"] != f["cons"])
        # original base of the row matches the read
        codes = {ord("A"): 0, ord("C"): 1, ord("G"): 2, ord("T"): 3}
        for rid, pos, ob in zip(f["read_id"][:500], f["pos"][:500], f["orig"][:500]):
            assert codes[int(rs.seqs[rid, pos])] == ob
        x = f["x"]
        assert np.all(np.isfinite(x))
        assert np.all((x[:, 4] > 0) & (x[:, 4] <= 1))                    # support
        assert set(np.unique(x[:, 21])) <= {0.0, 1.0} and set(np.unique(x[:, 22])) <= {0.0, 1.0}
        assert np.all(x[:, 7] * 30 >= 3 - 1e-4)                           # coverage >= min coverage
        # plain output is unchanged by reporting rows
        plain = _run(inp, 0)
        try:
            assert np.array_equal(plain.anchors()[4], seq)
            assert plain.features()["read_id"].size == 0
        finally:
            plain.close()
    finally:
        run.close()


def test_constant_networks_bracket_the_plain_rule(small_pe):
    """b3 = +20 writes the consensus at every decision column, b3 = -20 keeps
    every original base; all other bases equal the plain rule's."""
    rs, inp = small_pe
    plain = _run(inp, 1)
    try:
        f = plain.features()
        base = plain.anchors()[4]
        for b3, pick in ((20.0, "cons"), (-20.0, "orig")):
            p = np.zeros(mo.NFLOATS, np.float32)
            p[mo.ISTD:] = 1.0
            p[mo.B3] = b3
            run = _run(inp, 2, p)
            try:
                g = run.features()
                assert np.array_equal(g["read_id"], f["read_id"]) and np.array_equal(g["pos"], f["pos"])
                assert np.all(g["logit"] == np.float32(b3))
                seq = run.anchors()[4]
                exp = base.copy()
                exp[f["read_id"], f["pos"]] = np.frombuffer(b"ACGT", np.uint8)[f[pick]]
                assert np.array_equal(seq, exp)
            finally:
                run.close()
    finally:
        plain.close()
