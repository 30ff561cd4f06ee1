"""Training of the learned decision (correction_type 1).

The network answers the reference's classifier question (correctAnchorClf,
include/corrector.hpp:1448-1472): at an anchor position of a non-HQ MSA whose
base differs from the consensus, is the consensus base written? Its training
rows are the decision columns the classic rule itself passes over
(care_b200_collect_features under correction_type 0) on seeded synthetic
genomes, labelled from the known true sequence:

- label 1 when the consensus base is the true base (writing it is right);
- label 0 otherwise.

Writing the consensus where the original base was already right is a false
positive correction; those rows weigh ``fp_weight`` in the loss (every other
row weighs 1), so the network trades a few true corrections for fewer false
ones at the plain logit > 0 cut.

    python -m care_b200.learned -o mlp.bin            # 3 genomes of 5 Mbp, PE 30x
    care-b200 ... --correctionType 1 --ml-mlpfile mlp.bin
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
import time

import numpy as np

from . import Corrector, Mlp, MLP_FLOATS, options_from_args
from . import datagen

FP_WEIGHT = 30.0
DEFAULT_ARGS = "-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE --candidateCorrection"
# training set models: read generator and the care-cpu options of the runs
MODELS = {
    "pe30": ("paired_end_repeats", DEFAULT_ARGS),
    "large50": ("paired_end_large",
                "-c 50 -k 20 -h 48 -q --qualityScoreBits 2 --pairmode PE --excludeAmbiguous --candidateCorrection"),
}
ACGT = np.frombuffer(b"ACGT", np.uint8)


def label_rows(rows: dict, truth: np.ndarray):
    """(label, orig_right) per row: consensus base == true base, original
    base == true base. truth is (num_reads, max_len) ASCII."""
    t = truth[rows["read_id"], rows["pos"]]
    return (t == ACGT[rows["cons"]]).astype(np.float32), (t == ACGT[rows["orig"]]).astype(np.float32)


def row_weights(label: np.ndarray, orig_right: np.ndarray, fp_weight: float = FP_WEIGHT) -> np.ndarray:
    w = np.ones(label.shape[0], np.float32)
    w[(label == 0) & (orig_right == 1)] = fp_weight
    return w


def collect_rows(fastq: str, args: str = DEFAULT_ARGS, device: int = 0) -> dict:
    """Decision-column rows of the classic rule on one input file."""
    with Corrector(options_from_args(args, correction_type=0, device=device)) as c:
        c.load_files([fastq])
        c.build_tables()
        return c.collect_features()


def training_set(readsets, args: str = DEFAULT_ARGS, workdir: str | None = None, device: int = 0,
                 fp_weight: float = FP_WEIGHT):
    """Rows, labels and weights over several datagen.ReadSet objects."""
    xs, ys, ws = [], [], []
    with tempfile.TemporaryDirectory(dir=workdir) as d:
        for i, rs in enumerate(readsets):
            path = os.path.join(d, f"train{i}.fq")
            rs.write_fastq(path)
            rows = collect_rows(path, args, device)
            y, ok = label_rows(rows, rs.truth)
            xs.append(rows["x"])
            ys.append(y)
            ws.append(row_weights(y, ok, fp_weight))
    return np.concatenate(xs), np.concatenate(ys), np.concatenate(ws)


def train(x, y, w=None, epochs: int = 30, batch: int = 65536, lr: float = 1e-3, seed: int = 1,
          init_seed: int = 7, device: int = 0):
    """Adam on the device (one CUDA graph per run); returns (params, losses)."""
    with Mlp(device=device, seed=init_seed) as m:
        m.set_data(x, y, w)
        losses = m.train(epochs=epochs, batch=batch, lr=lr, seed=seed)
        return m.params, losses


def save_params(path: str, params: np.ndarray) -> None:
    p = np.ascontiguousarray(params, dtype="<f4")
    if p.shape != (MLP_FLOATS,):
        raise ValueError(f"expected {MLP_FLOATS} parameters")
    p.tofile(path)


def load_params(path: str) -> np.ndarray:
    p = np.fromfile(path, dtype="<f4")
    if p.shape != (MLP_FLOATS,):
        raise ValueError(f"{path}: expected {MLP_FLOATS} float32 values")
    return p


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("-o", "--output", required=True, help="parameter file (float32 little-endian)")
    ap.add_argument("--genomes", type=int, default=3)
    ap.add_argument("--genome-size", type=int, default=5_000_000)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--model", choices=sorted(MODELS), default="pe30",
                    help="pe30: the 30x benchmark model; large50: 50x, h48, indels and N bases")
    ap.add_argument("--args", default=None, help="care-cpu options of the training runs (default: the model's)")
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--fp-weight", type=float, default=FP_WEIGHT)
    ap.add_argument("-g", "--gpu", type=int, default=0)
    a = ap.parse_args(argv)
    t0 = time.time()
    G = a.genome_size
    gen, margs = MODELS[a.model]
    if gen == "paired_end_large":
        sets = [datagen.paired_end_large(seed=a.seed + i, genome_size=G) for i in range(a.genomes)]
    else:
        sets = [datagen.paired_end_repeats(seed=a.seed + i, genome_size=G, repeat_unit=max(100, G // 1000))
                for i in range(a.genomes)]
    x, y, w = training_set(sets, a.args or margs, device=a.gpu, fp_weight=a.fp_weight)
    print(f"{x.shape[0]} rows, {float(y.mean()):.4f} consensus right, {int((w > 1).sum())} false-positive rows",
          file=sys.stderr)
    params, losses = train(x, y, w, a.epochs, a.batch, a.lr, device=a.gpu)
    save_params(a.output, params)
    print(f"loss {losses[0]:.4f} -> {losses[-1]:.4f} over {len(losses)} steps, {time.time() - t0:.1f} s",
          file=sys.stderr)
    return 0


if __name__ == "__main__":
    sys.exit(main())
