"""Autotuner of the launch mapping (care_b200_tuning) for one workload.

The knobs change how a batch is laid onto the GPU, never what it computes:

- msa_order   anchors in longest-processing-time order (most candidates first)
- msa_queue   persistent MSA CTAs pulling anchors from a device work queue
- msa_warps   warps per anchor in the MSA stage (4 or 8)
- align_block threads per CTA of the alignment stage (128 or 256)
- pair_order  alignment pairs packed by candidate length within each anchor
- graph       each batch's launches replayed as one CUDA graph
- pair_mirror (a, c) and (c, a) of equal-length anchors of a batch share one scan
- cand_set_log2  capacity of the main candidate pass's de-duplication set
  (occupancy against anchors redone by the full-set pass)
- align_warp  a warp per alignment work item (lanes take shifts) instead of
  a thread per work item
- align_classes  pairs partitioned by the plane width of their longer read,
  one alignment launch per width

Coordinate descent from the default: each knob in turn takes the value with
the lowest device time (CUDA events of the pipeline, mean of timed passes
after a warm-up); two sweeps. Every variant's results (anchor status, edit
counts, corrected rows, candidate corrections) must equal the default's, or
the tuner stops with an error. The choice is written as JSON, committed per
workload under care_b200/tuning/, and loaded by bench.py.

    python -m care_b200.autotune --workload uneven -o care_b200/tuning/se_uneven.json
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile
import time

import numpy as np

from . import Corrector, options_from_args

HERE = os.path.dirname(os.path.abspath(__file__))
TUNING_DIR = os.path.join(HERE, "tuning")

KNOBS = {
    "msa_order": [0, 1],
    "msa_queue": [0, 1],
    "msa_warps": [4, 8],
    "align_block": [128, 256],
    "pair_order": [0, 1],
    "graph": [0, 1],
    "pair_mirror": [0, 1],
    "cand_set_log2": [9, 10, 11],
    "align_warp": [0, 1],
    "align_classes": [0, 1],
}
DEFAULT = {"msa_order": 0, "msa_queue": 0, "msa_warps": 4, "align_block": 128, "pair_order": 0, "graph": 0,
           "pair_mirror": 0, "cand_set_log2": 10, "align_warp": 0, "align_classes": 0}

WORKLOADS = {
    "pe": ("-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE", 5_000_000),
    "uneven": ("-c 40 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode SE", 10_000_000),
    "large": ("-c 50 -k 20 -h 48 -q --qualityScoreBits 2 --pairmode PE --excludeAmbiguous", 10_000_000),
}


TUNING_FILES = {"pe": "pe_5Mbp_30x.json", "uneven": "se_uneven_40x.json", "large": "pe_large_50x.json"}


def tuning_file(workload: str) -> str:
    return os.path.join(TUNING_DIR, TUNING_FILES.get(workload, workload + ".json"))


def load(workload: str) -> dict | None:
    """The committed tuning of a workload, or None (the default mapping)."""
    p = tuning_file(workload)
    if not os.path.exists(p):
        return None
    return json.load(open(p))["tuning"]


def _fingerprint(res) -> tuple:
    corr = (res.status & 1) == 1
    cands = sorted(zip(res.cand_read_ids.tolist(), res.cand_anchor_ids.tolist(), res.cand_shifts.tolist(),
                       res.cand_use_edits.tolist(), [bytes(r) for r in res.cand_sequences]))
    return (res.status.tobytes(), res.num_edits.tobytes(), res.sequences[corr].tobytes(), hash(tuple(cands)))


def measure(c: Corrector, tuning: dict, n: int, steps: int = 3) -> float:
    c.tuning = tuning
    c.correct_range_device(0, n)                 # warm-up (and graph instantiation)
    ms = []
    for _ in range(steps):
        c.correct_range_device(0, n)
        ms.append(c.last_timing()[0])
    return float(np.mean(ms))


def tune(c: Corrector, n: int, sweeps: int = 2, steps: int = 3, log=print) -> tuple[dict, dict]:
    c.tuning = DEFAULT
    ref = _fingerprint(c.correct_range(0, n))
    seen = {}

    def timed(t):
        key = json.dumps(t, sort_keys=True)
        if key not in seen:
            c.tuning = t
            if _fingerprint(c.correct_range(0, n)) != ref:
                raise RuntimeError(f"tuning {t} changed the results")
            seen[key] = measure(c, t, n, steps)
            log(f"  {t} -> {seen[key]:.2f} ms")
        return seen[key]

    best = dict(DEFAULT)
    best_ms = timed(best)
    for _ in range(sweeps):
        for k, values in KNOBS.items():
            for v in values:
                if v == best[k]:
                    continue
                t = dict(best, **{k: v})
                ms = timed(t)
                if ms < best_ms:
                    best, best_ms = t, ms
    return best, {"best_ms": best_ms, "default_ms": seen[json.dumps(DEFAULT, sort_keys=True)],
                  "measured": {k: round(v, 3) for k, v in seen.items()}}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="uneven")
    ap.add_argument("--genome", type=int, default=None, help="bp of the sample genome (default: the workload's)")
    ap.add_argument("--seed", type=int, default=77)
    ap.add_argument("-o", "--output", default=None)
    ap.add_argument("-g", "--gpu", type=int, default=0)
    a = ap.parse_args(argv)
    from . import datagen
    args, G = WORKLOADS[a.workload]
    G = a.genome or G
    t0 = time.time()
    if a.workload == "uneven":
        rs = datagen.single_end_uneven(seed=a.seed, genome_size=G, coverage=40.0)
    elif a.workload == "large":
        rs = datagen.paired_end_large(seed=a.seed, genome_size=G)
    else:
        rs = datagen.paired_end_repeats(seed=a.seed, genome_size=G, repeat_unit=max(100, G // 1000))
    with tempfile.TemporaryDirectory() as d:
        fq = os.path.join(d, "sample.fq")
        rs.write_fastq(fq)
        with Corrector(options_from_args(args, device=a.gpu)) as c:
            c.load_files([fq])
            c.build_tables()
            n = c.num_reads
            print(f"sample: {n} reads, {G} bp genome ({time.time() - t0:.0f} s)", file=sys.stderr)
            best, info = tune(c, n, log=lambda m: print(m, file=sys.stderr))
    out = {"workload": a.workload, "args": args, "sample_genome_bp": G, "sample_reads": n, "seed": a.seed,
           "tuning": best, **info}
    path = a.output or tuning_file(a.workload)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps({"tuning": best, "best_ms": info["best_ms"], "default_ms": info["default_ms"]}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
