"""The learned decision on the GPU, called through the C ABI.

- forward, gradient and Adam of the tensor-core kernels against the numpy
  oracle (oracle/mlp_oracle.py), which applies the same bfloat16 roundings;
- the decision-column rows of the CUDA path against the C oracle (bit-exact);
- the network-decided correction against the C oracle's network mode;
- training on seeded genomes and the base-level gain over the classic rule
  on a held-out genome.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

import _oracle
import care_b200
from care_b200 import datagen

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu

# Tolerances. Device and oracle apply identical bfloat16 roundings, so they
# differ only by FP32 accumulation order inside the tensor cores (~1e-6
# relative) and by the last bit of erff/expf, which can move a bfloat16
# rounding by one unit in rare elements.
LOGIT_Q999 = 1e-4          # 99.9 % of logits within this (absolute, on |logit| <= ~10)
LOGIT_MAX = 2e-2           # every logit within this
GRAD_REL = 2e-3            # ||g_gpu - g_oracle|| / ||g_oracle|| per parameter block
ADAM_RTOL = 2e-6           # one Adam update of the same gradient


def _rows(seed, n, scale=1.0):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal((n, mo.NFEAT)) * scale + rng.uniform(-1, 1, mo.NFEAT)).astype(np.float32)
    w = rng.standard_normal(mo.NFEAT)
    y = ((x @ w + 0.5 * rng.standard_normal(n)) > 0).astype(np.float32)
    return x, y


@pytest.mark.parametrize("n", [1, 127, 128, 10_001, 200_000])
def test_forward_matches_oracle(n):
    x, _ = _rows(1, n, 2.0)
    p = mo.random_params(2, x)
    with care_b200.Mlp() as m:
        m.params = p
        got = m.forward(x)
    ref = mo.forward(p, x, emulate=True)["logit"]
    d = np.abs(got.astype(np.float64) - ref)
    assert np.all(np.isfinite(got))
    assert np.quantile(d, 0.999) <= LOGIT_Q999
    assert d.max() <= LOGIT_MAX


BLOCKS = {"W1": (mo.W1, mo.B1), "b1": (mo.B1, mo.W2), "W2": (mo.W2, mo.B2), "b2": (mo.B2, mo.W3),
          "w3": (mo.W3, mo.B3), "b3": (mo.B3, mo.NPARAM)}


@pytest.mark.parametrize("n,weighted", [(100, False), (3000, False), (70_000, False), (3000, True), (70_000, True)])
def test_gradient_matches_oracle(n, weighted):
    x, y = _rows(3, n)
    w = np.random.default_rng(9).choice(np.array([1.0, 30.0], np.float32), n, p=[0.9, 0.1]) if weighted else None
    p = mo.random_params(4, x)
    with care_b200.Mlp() as m:
        m.params = p
        loss, g = m.gradient(x, y, w)
    l_ref, g_ref = mo.loss_and_grad(p, x, y, emulate=True, w=w)
    assert abs(loss - l_ref) <= 1e-4 * abs(l_ref) + 1e-6
    for name, (a, b) in BLOCKS.items():
        num = np.linalg.norm(g[a:b] - g_ref[a:b])
        den = np.linalg.norm(g_ref[a:b])
        assert num <= GRAD_REL * den + 1e-9, (name, num / max(den, 1e-30))
    # the device gradient is the exact network's gradient up to bfloat16
    _, g_exact = mo.loss_and_grad(p, x, y, emulate=False, w=w)
    cos = float(g @ g_exact / np.linalg.norm(g) / np.linalg.norm(g_exact))
    assert cos > 0.999


def test_adam_step_matches_oracle():
    x, y = _rows(5, 20_000)
    p = mo.random_params(6, x)
    with care_b200.Mlp() as m:
        m.params = p                                   # also resets the moments
        pm, mm, vv = p.copy(), np.zeros(mo.NPARAM, np.float32), np.zeros(mo.NPARAM, np.float32)
        for t in range(1, 4):
            _, g = m.gradient(x, y)                    # the gradient the step will use
            m.train_step(x, y, lr=1e-3)
            mo.adam(pm, g, mm, vv, t, lr=1e-3)
            np.testing.assert_allclose(m.params[:mo.NPARAM], pm[:mo.NPARAM], rtol=ADAM_RTOL, atol=1e-9)


def test_training_graph_reduces_loss():
    x, y = _rows(7, 300_000)
    with care_b200.Mlp(seed=3) as m:
        m.set_data(x, y)
        p0 = m.params
        mu, istd = mo.normalisation(x)
        np.testing.assert_allclose(p0[mo.MEAN:mo.ISTD], mu, rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(p0[mo.ISTD:], istd, rtol=1e-5)
        losses = m.train(epochs=4, batch=8192, lr=3e-3, seed=5)
        p1 = m.params
    assert losses.shape == (4 * 37,)
    assert np.all(np.isfinite(losses)) and np.all(np.isfinite(p1))
    assert losses[-8:].mean() < 0.7 * losses[:2].mean()
    l0 = mo.loss_and_grad(p0, x[:20000], y[:20000])[0]
    l1 = mo.loss_and_grad(p1, x[:20000], y[:20000])[0]
    assert l1 < 0.7 * l0


# ---- decision columns of the correction path ----

ARGS = "-c 30 -k 20 -h 16 -q --qualityScoreBits 2 --pairmode PE"


@pytest.fixture(scope="module")
def pe_small(tmp_path_factory):
    rs = datagen.paired_end_repeats(seed=51, genome_size=150_000, repeat_unit=1000, repeat_copies=6)
    d = tmp_path_factory.mktemp("mlp")
    inp = str(d / "in.fq")
    rs.write_fastq(inp)
    return rs, inp


def _oracle_run(inp, mode, params=None):
    o = _oracle.opts_from_args(ARGS)
    o.clf_mode = mode
    keep = None
    if params is not None:
        keep = np.ascontiguousarray(params, np.float32)
        o.mlp = keep.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    run = _oracle.OracleRun([inp], o, threads=8)
    run._keep = keep
    return run


def _sorted(f):
    order = np.lexsort((f["pos"], f["read_id"]))
    return {k: (None if v is None else v[order]) for k, v in f.items()}


def test_decision_rows_match_oracle(pe_small):
    rs, inp = pe_small
    with care_b200.Corrector(care_b200.options_from_args(ARGS)) as c:
        c.load_files([inp])
        c.build_tables()
        g = _sorted(c.collect_features())
        plain = c.correct_range()
    run = _oracle_run(inp, 1)
    try:
        f = run.features()
        seq = run.anchors()[4]
    finally:
        run.close()
    assert len(f["read_id"]) > 500
    assert np.array_equal(g["read_id"], f["read_id"])
    assert np.array_equal(g["pos"], f["pos"].astype(np.int32))
    assert np.array_equal(g["orig"], f["orig"]) and np.array_equal(g["cons"], f["cons"])
    assert np.array_equal(g["x"].view(np.uint32), f["x"].view(np.uint32))     # bit-exact
    assert g["logit"] is None
    corr = (plain.status & 1) == 1
    assert np.array_equal(plain.sequences[corr], seq[corr])


def _labels(rs, f):
    truth = rs.truth[f["read_id"], f["pos"]]
    return (truth == np.frombuffer(b"ACGT", np.uint8)[f["cons"]]).astype(np.float32)


def test_network_mode_matches_oracle(pe_small):
    rs, inp = pe_small
    with care_b200.Corrector(care_b200.options_from_args(ARGS)) as c:
        c.load_files([inp])
        c.build_tables()
        f = c.collect_features()
    p = mo.random_params(8, f["x"])
    # a network fitted a little, its output shifted so that a fifth of the
    # rows keep the original base
    with care_b200.Mlp() as m:
        m.params = p
        m.set_data(f["x"], _labels(rs, f))
        m.train(epochs=2, batch=4096, lr=3e-3, seed=1)
        p = m.params
        p[mo.B3] -= np.quantile(m.forward(f["x"]), 0.2)
    with care_b200.Corrector(care_b200.options_from_args(ARGS, correction_type=1)) as c:
        c.load_files([inp])
        c.build_tables()
        c.set_mlp(p)
        g = _sorted(c.collect_features())
        res = c.correct_range()
    run = _oracle_run(inp, 2, p)
    try:
        o = run.features()
        status, hq, ue, ne, seq = run.anchors()
    finally:
        run.close()
    assert np.array_equal(g["read_id"], o["read_id"]) and np.array_equal(g["pos"], o["pos"].astype(np.int32))
    d = np.abs(g["logit"].astype(np.float64) - o["logit"])
    assert np.quantile(d, 0.999) <= LOGIT_Q999 and d.max() <= LOGIT_MAX
    pos = o["logit"] > 0
    assert 0.05 < pos.mean() < 0.95
    # a verdict can differ only where |logit| is within the largest device -
    # oracle difference; those reads are set aside
    unsure = np.unique(o["read_id"][np.abs(o["logit"]) <= d.max()])
    assert len(unsure) <= 0.02 * len(np.unique(o["read_id"])) + 5
    keep = (status == 1)
    keep[unsure] = False
    assert np.array_equal((res.status & 1) == 1, status == 1)
    assert np.array_equal(res.sequences[keep], seq[keep])
    assert np.array_equal(((res.status >> 2) & 1)[keep], ue[keep])
    assert np.array_equal(res.num_edits[keep], ne[keep])


# ---- the gain of the trained network ----

def _f1_of(rs, path):
    _, seqs, _ = datagen.read_fastq(path)
    n, L = rs.seqs.shape
    corr = np.zeros((n, L), np.uint8)
    for i, s in enumerate(seqs):
        corr[i, :len(s)] = np.frombuffer(s, np.uint8)
    return datagen.base_level_counts(rs.seqs, corr, rs.truth, rs.lengths)


def _genome(seed, G):
    return datagen.paired_end_repeats(seed=seed, genome_size=G, repeat_unit=max(100, G // 1000))


def test_trained_network_gains_over_classic_rule(tmp_path):
    """Train on the decision columns of three seeded genomes (labels from the
    true sequence), evaluate on a held-out genome with candidate correction:
    base-level F1 above the classic rule's with fewer false positives."""
    from care_b200 import learned
    G = 1_000_000
    x, y, w = learned.training_set([_genome(s, G) for s in (201, 202, 203)], workdir=str(tmp_path))
    assert x.shape[0] > 100_000 and y.mean() > 0.95 and (w > 1).sum() > 50
    params, losses = learned.train(x, y, w, epochs=30, batch=16384, lr=1e-3, seed=3)
    assert np.all(np.isfinite(params)) and losses[-20:].mean() < losses[:5].mean()
    pfile = str(tmp_path / "mlp.bin")
    learned.save_params(pfile, params)
    assert np.array_equal(learned.load_params(pfile), params)
    rs = _genome(204, G)
    inp = str(tmp_path / "held.fq")
    rs.write_fastq(inp)
    out = {}
    for ct in (0, 1):
        with care_b200.Corrector(care_b200.options_from_args(learned.DEFAULT_ARGS, correction_type=ct)) as c:
            c.load_files([inp])
            c.build_tables()
            if ct:
                c.set_mlp(params)
            c.correct_range()
            path = str(tmp_path / f"out{ct}.fq")
            c.write_output(path)
        out[ct] = _f1_of(rs, path)
    (tp0, fp0, fn0, _), (tp1, fp1, fn1, _) = out[0], out[1]
    f0, f1 = datagen.f1(tp0, fp0, fn0), datagen.f1(tp1, fp1, fn1)
    print(f"classic TP {tp0} FP {fp0} FN {fn0} F1 {f0:.5f} | network TP {tp1} FP {fp1} FN {fn1} F1 {f1:.5f}")
    assert f1 > f0
    assert fp1 < fp0


def test_cli_learned_decision_equals_library(pe_small, tmp_path):
    """care-b200 --correctionType 1 --ml-mlpfile writes what the library path writes."""
    import subprocess
    from care_b200 import learned
    rs, inp = pe_small
    params = learned.load_params(os.path.join(os.path.dirname(care_b200.__file__), "data", "mlp_pe30x.bin"))
    with care_b200.Corrector(care_b200.options_from_args(ARGS, correction_type=1)) as c:
        c.load_files([inp])
        c.build_tables()
        c.set_mlp(params)
        c.correct_range()
        lib_out = str(tmp_path / "lib.fq")
        c.write_output(lib_out)
    pfile = str(tmp_path / "p.bin")
    learned.save_params(pfile, params)
    r = subprocess.run([care_b200.CLI_PATH, "-i", inp, "-d", str(tmp_path), "-o", "cli.fq", "--correctionType", "1",
                        "--ml-mlpfile", pfile] + ARGS.split(), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert open(tmp_path / "cli.fq", "rb").read() == open(lib_out, "rb").read()
    # without a parameter file the driver refuses type 1
    r = subprocess.run([care_b200.CLI_PATH, "-i", inp, "-d", str(tmp_path), "-o", "x.fq", "--correctionType", "1"]
                       + ARGS.split(), capture_output=True, text=True)
    assert r.returncode != 0


def test_decision_rows_over_several_batches(pe_small):
    rs, inp = pe_small

    def rows(batch):
        with care_b200.Corrector(care_b200.options_from_args(ARGS, batch_size=batch)) as c:
            c.load_files([inp])
            c.build_tables()
            return _sorted(c.collect_features())

    a, b = rows(0), rows(2048)
    for k in ("read_id", "pos", "orig", "cons"):
        assert np.array_equal(a[k], b[k])
    assert np.array_equal(a["x"].view(np.uint32), b["x"].view(np.uint32))
