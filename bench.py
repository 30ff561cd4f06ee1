#!/usr/bin/env python
"""Reads corrected per second on B200: CARE's per-anchor correction path.

Workload (default): the 5 Mbp / 30x paired-end set -- seeded random genome
with 2% of its length in 20 copies of a 5 kbp repeat at 1% divergence,
1,000,000 interleaved 150 bp reads, fragments ~N(400, 40), substitution rate
rising linearly 0.2% -> 1.5% along the read, Phred qualities from the rate
+ N(0, 3); options -c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE.

One step = correcting every read of the set once (the reference's STEP2,
src/dispatch_care_correct_cpu.cpp:157-168; reads/s = reads / STEP2 time).

  value : device time of the pipeline with reads and tables resident in HBM
          (CUDA events on the library's stream), L2 flushed between steps.
  e2e   : the same through the C ABI from host buffers -- upload of the read
          storage (care_b200_upload_reads) + correction with the results
          copied back to host memory (care_b200_correct_range), wall clock.
  --impl reference : the reference's care-cpu (built from its sources by
          oracle/Makefile) on all host cores, on the same read set and
          options; one care-cpu run per step (~15 s on 16 cores).
  parity : the plain method's corrected FASTQ (untimed, after the timed
          steps) against care-cpu's output of the same file, by SHA-256.
  learned : the same steps with the learned decision (correction_type 1,
          network parameters care_b200/data/mlp_pe30x.bin, trained by
          `python -m care_b200.learned` on three other seeded genomes), and
          base-level TP/FP/FN/F1 of both forms against the true reads.

--workload large : 50 Mbp genome with 5% repeats, 150 bp PE at 50x (~16.7M
          reads), position-dependent substitutions plus 0.01% single-base
          indels and 0.1% N bases; -c 50 -k 20 -h 48 -q --qualityScoreBits 2
          --pairmode PE --excludeAmbiguous; plain and learned forms with
          base-level counts (network care_b200/data/mlp_pe50x_h48.bin).
--workload uneven : the batched uneven set instead -- 10 Mbp genome with 8%
          repeats in families of 5-500 copies (0.5-2% divergence), single-end
          reads of 50-250 bp at 40x (~2.7M reads), same error and quality
          model; -c 40 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode SE.

Blocks of the default run (pe, one GPU; --no-extra skips them): `uneven` and
`large`, the two other workloads below with their committed tunings, a few
steps each (min(steps, 5) after min(warmup, 3)), timed like `value`; the large
block also carries plain and learned base-level counts.

Multi-GPU: one process per GPU; each rank corrects its own read set
(independent genome partitions, no data-path collective) -> weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ARGS = "-c 30 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode PE"
ARGS_UNEVEN = "-c 40 -k 20 -h 32 -q --qualityScoreBits 2 --pairmode SE"
ARGS_LARGE = "-c 50 -k 20 -h 48 -q --qualityScoreBits 2 --pairmode PE --excludeAmbiguous"
MLP_FILE_LARGE = os.path.join(ROOT, "care_b200", "data", "mlp_pe50x_h48.bin")
METRIC = "reads corrected/s on 1 B200: plain vs MLP-classifier form at matched base F1"
MLP_FILE = os.path.join(ROOT, "care_b200", "data", "mlp_pe30x.bin")
# k_msa DRAM bytes per anchor: dram__bytes_read.sum + dram__bytes_write.sum of
# one ncu capture of 100,000 anchors of this workload model (68.24 MB read +
# 4.75 MB written)
MSA_DRAM_BYTES_PER_ANCHOR = 730.0
CARE_CPU = os.path.join(ROOT, "oracle", "_ref", "care-cpu")
L2_BYTES = 126 * 1024 * 1024


def workload(rank: int, genome_size: int, kind: str = "pe"):
    from care_b200 import datagen
    if kind == "large":
        return datagen.paired_end_large(seed=5 + 1000 * rank, genome_size=genome_size)
    if kind == "uneven":
        return datagen.single_end_uneven(seed=3 + 1000 * rank, genome_size=genome_size, coverage=40.0)
    # 2% of the genome in 20 copies of one repeat unit (5 kbp at 5 Mbp)
    rs = datagen.paired_end_repeats(seed=2 + 1000 * rank, genome_size=genome_size,
                                    repeat_unit=max(100, genome_size // 1000))
    return rs


def encode_quality_2bit(quals: np.ndarray) -> np.ndarray:
    """qualityscorecompression.hpp:95-119 with 2 bits: bins Q<=4,13,20,>20."""
    q = quals.astype(np.int32) - 33
    code = np.where(q <= 4, 0, np.where(q <= 13, 1, np.where(q <= 20, 2, 3))).astype(np.uint32)
    n, L = code.shape
    per = 16
    pitch = (2 * L + 31) // 32
    padded = np.zeros((n, pitch * per), np.uint32)
    padded[:, :L] = code
    padded = padded.reshape(n, pitch, per)
    shifts = (30 - 2 * np.arange(per, dtype=np.uint32))
    return (padded << shifts).sum(axis=2, dtype=np.uint64).astype(np.uint32)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        exe = shutil.which("nvidia-smi")
        if exe:
            self.proc = subprocess.Popen([exe, "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def host_cores() -> int:
    """Cores this process may use: the affinity mask, capped by a cgroup CPU
    quota (a container can see more CPUs than it is allowed to run on)."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        quota, period = open("/sys/fs/cgroup/cpu.max").read().split()[:2]
        if quota != "max":
            n = min(n, max(1, int(float(quota) / float(period) + 0.5)))
    except (OSError, ValueError):
        try:
            q = int(open("/sys/fs/cgroup/cpu/cpu.cfs_quota_us").read())
            p = int(open("/sys/fs/cgroup/cpu/cpu.cfs_period_us").read())
            if q > 0:
                n = min(n, max(1, round(q / p)))
        except (OSError, ValueError):
            pass
    return max(1, n)


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def care_cpu_run(fq: str, tmpdir: str, threads: int, args: str, out: str = "cpu_out.fq"):
    """One care-cpu run on the FASTQ `fq` with `threads` threads; returns
    (reads/s of its STEP2 throughput line, path of its corrected output)."""
    cmd = [CARE_CPU, "-i", fq, "-d", tmpdir, "-o", out, "-t", str(threads)] + args.split()
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=1200)
    if r.returncode != 0:
        raise RuntimeError("care-cpu failed: " + r.stderr[-500:])
    m = re.search(r"Correction throughput : ~([0-9.e+]+) reads/second", r.stdout)
    return float(m.group(1)), os.path.join(tmpdir, out)


def care_cpu_sample(tmpdir: str, threads: int, genome: int = 250_000):
    """care-cpu on a small sample of the paired-end model (`genome`-bp genome,
    50,000 reads at the default size): the one-thread rate."""
    from care_b200 import datagen
    path = os.path.join(tmpdir, f"sample_{genome}.fq")
    if not os.path.exists(path):
        rs = datagen.paired_end_repeats(seed=7, genome_size=genome, repeat_unit=max(250, genome // 1000))
        datagen.write_fastq_fast(rs, path)
    return care_cpu_run(path, tmpdir, threads, ARGS, out="sample_out.fq")[0]


def workload_config(args) -> dict:
    """The `config` keys both arms share: the workload, its reads and options."""
    run_args = {"uneven": ARGS_UNEVEN, "large": ARGS_LARGE}.get(args.workload, ARGS)
    g = args.genome
    size = f"{g // 1_000_000}Mbp" if g % 1_000_000 == 0 else f"{g // 1000}kbp"
    name = {"uneven": "se_uneven_%s_40x_50-250bp", "large": "pe_large_%s_50x_150bp_indels_N"}.get(
        args.workload, "pe_%s_30x_150bp") % size
    return {"workload": name, "args": run_args, "genome_bp": args.genome}


def run_reference(args, rank, world):
    """The reference's own care-cpu on all host cores, on the same read set
    and options as the GPU arm (rank 0's set); one care-cpu run per step,
    its STEP2 throughput line (src/dispatch_care_correct_cpu.cpp:168)."""
    if rank != 0:
        return
    threads = host_cores()
    cfg = workload_config(args)
    if not os.path.exists(CARE_CPU):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/care-cpu not built (make -C oracle ref)"}))
        return
    from care_b200 import datagen
    with tempfile.TemporaryDirectory() as tmp:
        progress("generating reads")
        rs = workload(0, args.genome, args.workload)
        n = rs.num_reads
        fq = os.path.join(tmp, "reads.fq")
        datagen.write_fastq_fast(rs, fq)
        del rs
        cfg["reads_per_gpu"] = n
        for w in range(args.warmup):
            care_cpu_run(fq, tmp, threads, cfg["args"])
            progress(f"care-cpu warm-up run {w} done")
        vals = []
        for s in range(args.steps):
            vals.append(care_cpu_run(fq, tmp, threads, cfg["args"])[0])
            progress(f"care-cpu timed run {s}: {vals[-1]:.0f} reads/s")
    v = float(np.median(vals))                    # median of the timed runs
    sample = f"the whole workload ({n} reads), care-cpu -t {threads}, one run per step; median of {len(vals)} runs"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "reads/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": n / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded)", "config": cfg,
            "cpu_baseline": {"value": v, "unit": "reads/s", "cores": threads, "kind": "reference",
                             "sample": sample, "runs": vals, "cpu_model": cpu_model()},
            "e2e": {"value": v, "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


T0 = time.time()


def progress(msg: str) -> None:
    """Phase marks on stderr (the JSON line stays the only stdout output)."""
    print(f"[bench {time.time() - T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def int_peaks():
    """Integer-pipe peaks of this GPU from care-b200-peaks (POPC alone and
    the alignment's word-compare instruction mix, registers only)."""
    exe = os.path.join(ROOT, "care_b200", "care-b200-peaks")
    if not os.path.exists(exe):
        return None
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    return json.loads(r.stdout) if r.returncode == 0 else None


def base_counts(rs, path):
    """TP/FP/FN/TN of a corrected FASTQ against the true reads."""
    from care_b200 import datagen
    n, L = rs.seqs.shape
    data = open(path, "rb").read().split(b"\n")
    corr = np.frombuffer(b"".join(data[1:4 * n:4]), np.uint8).reshape(n, L)
    return datagen.base_level_counts(rs.seqs, corr, rs.truth, rs.lengths)


def sha256_file(path: str) -> str:
    import hashlib
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for block in iter(lambda: f.read(1 << 24), b""):
            h.update(block)
    return h.hexdigest()


def timed_steps(corr, n, steps, flush):
    """Device ms and per-stage ms (mean over steps), wall ms per step."""
    import torch
    dev_ms, stage, t_wall = [], np.zeros(4), 0.0
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        corr.correct_range_device(0, n)
        t_wall += time.perf_counter() - w0
        tot, st = corr.last_timing()
        dev_ms.append(tot)
        stage += np.array(st)
    return float(np.mean(dev_ms)), stage / steps, t_wall / steps * 1e3


def workload_block(kind: str, steps: int, warmup: int, flush, local: int, tmp: str, learned: bool) -> dict:
    """Another workload of the same metric as a block of the line: its own
    seeded read set and options, the committed tuning, the same timing as
    `value` (device time of whole passes, L2 flushed between steps); for the
    large set also base-level counts of the plain and learned forms."""
    import care_b200
    from care_b200 import autotune, datagen
    genome = {"uneven": 10_000_000, "large": 50_000_000}[kind]
    run_args = {"uneven": ARGS_UNEVEN, "large": ARGS_LARGE}[kind]
    progress(f"{kind} block: generating reads")
    rs = workload(0, genome, kind)
    n = rs.num_reads
    fq = os.path.join(tmp, f"{kind}.fq")
    datagen.write_fastq_fast(rs, fq)
    tuned = autotune.load(kind)
    forms = [("plain", 0)] + ([("learned", 1)] if learned and kind == "large" and os.path.exists(MLP_FILE_LARGE) else [])
    out = {"workload": workload_config(argparse.Namespace(workload=kind, genome=genome))["workload"],
           "reads": n, "args": run_args, "steps": steps, "warmup": warmup, "tuning": tuned,
           "timing": "as value: device time of whole passes, inputs resident, L2 flushed between steps"}
    for name, ctype in forms:
        c = care_b200.Corrector(care_b200.options_from_args(run_args, device=local, correction_type=ctype))
        if ctype:
            from care_b200 import learned as lrn
            c.set_mlp(lrn.load_params(MLP_FILE_LARGE))
        if tuned:
            c.tuning = tuned
        t0 = time.perf_counter()
        c.load_files([fq])
        c.build_tables()
        step1 = time.perf_counter() - t0
        for _ in range(warmup):
            c.correct_range_device(0, n)
        import torch
        torch.cuda.synchronize()
        ms, stage, _ = timed_steps(c, n, steps, flush)
        st = c.last_stats()
        blk = {"value": n / (ms / 1e3), "unit": "reads/s", "ms_per_step": ms,
               "stage_ms": {"candidates": stage[0], "align": stage[1], "msa": stage[2], "classifier": stage[3]},
               "pairs_per_step": st["pairs"], "step1_s": step1, "gpu_launches": st["launches"] * steps}
        if kind == "large":
            progress(f"{kind} block: {name} base-level counts")
            c.correct_range(0, n)
            o = os.path.join(tmp, f"{kind}_{name}.fq")
            c.write_output(o)
            tp, fp, fn, tn = base_counts(rs, o)
            blk["base_level"] = {"tp": tp, "fp": fp, "fn": fn, "f1": datagen.f1(tp, fp, fn)}
            os.unlink(o)
        c.close()
        out[name] = blk
        progress(f"{kind} block: {name} {blk['value'] / 1e6:.2f}M reads/s")
    if "learned" in out:
        out["learned"]["ratio_vs_plain"] = out["learned"]["value"] / out["plain"]["value"]
    os.unlink(fq)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="care_b200", choices=["care_b200", "reference"])
    ap.add_argument("--workload", default="pe", choices=["pe", "uneven", "large"])
    ap.add_argument("--genome", type=int, default=None, help="bp (default 5 Mbp, uneven 10 Mbp, large 50 Mbp)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the uneven and large workload blocks of the default (pe, 1 GPU) run")
    ap.add_argument("--tuning", default="auto", choices=["auto", "default"],
                    help="auto: the committed launch mapping of the workload (care_b200/tuning/)")
    args = ap.parse_args()
    if args.genome is None:
        args.genome = {"uneven": 10_000_000, "large": 50_000_000}.get(args.workload, 5_000_000)
    uneven = args.workload == "uneven"
    large = args.workload == "large"
    run_args = ARGS_UNEVEN if uneven else (ARGS_LARGE if large else ARGS)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    import care_b200

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    tmp = tempfile.mkdtemp(prefix=f"careb200_bench_{rank}_")
    progress("generating reads")
    rs = workload(rank, args.genome, args.workload)
    n = rs.num_reads
    fq = os.path.join(tmp, "reads.fq")
    from care_b200 import datagen
    datagen.write_fastq_fast(rs, fq)

    opts = care_b200.options_from_args(run_args, device=local)
    corr = care_b200.Corrector(opts)
    from care_b200 import autotune
    tuned = autotune.load(args.workload) if args.tuning == "auto" else None
    if tuned:
        corr.tuning = tuned
    t0 = time.perf_counter()
    progress("STEP1: load + tables")
    corr.load_files([fq])
    corr.build_tables()
    progress("STEP1 done")
    step1_s = time.perf_counter() - t0
    sig_ms = corr.signatures_ms()            # once per read storage, outside the timed steps

    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    for w in range(args.warmup):
        corr.correct_range_device(0, n)
        progress(f"warm-up step {w} done")
    barrier()
    with ClockSampler(local) as clk:
        ms, stage, wall_ms = timed_steps(corr, n, args.steps, flush)
        barrier()
    stats = corr.last_stats()
    # one untimed pass of the alignment's statistics form: the word compares
    # its scans actually run after the early exits
    corr.count_word_compares(True)
    corr.correct_range_device(0, n)
    run_words = corr.last_stats()["word_compares_run"]
    corr.count_word_compares(False)
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n / (ms / 1e3)

    # the corrected FASTQ of the plain method (untimed): its digest for the
    # comparison with care-cpu's output of the same file, and its base counts
    progress("plain output")
    corr.correct_range(0, n)
    plain_out = os.path.join(tmp, "plain.fq")
    corr.write_output(plain_out)
    plain_sha = sha256_file(plain_out)

    # the learned decision on the same reads: device time of the same steps,
    # then base-level counts of both forms against the true reads
    learned = None
    mlp_file = MLP_FILE_LARGE if large else MLP_FILE
    if not args.no_learned and not uneven and os.path.exists(mlp_file):
        from care_b200 import learned as lrn, datagen
        params = lrn.load_params(mlp_file)
        progress("learned form: load + tables")
        mcorr = care_b200.Corrector(care_b200.options_from_args(run_args, device=local, correction_type=1))
        mcorr.set_mlp(params)
        if tuned:
            mcorr.tuning = tuned
        mcorr.load_files([fq])
        mcorr.build_tables()
        for _ in range(args.warmup):
            mcorr.correct_range_device(0, n)
        barrier()
        mms, mstage, _ = timed_steps(mcorr, n, args.steps, flush)
        mlaunches = mcorr.last_stats()["launches"]
        barrier()
        if world > 1:
            t = torch.tensor([mms], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            mms = float(t.item())
        progress("learned form timed; base-level counts")
        counts = {}
        for name, c in (("plain", corr), ("learned", mcorr)):
            out = plain_out
            if c is mcorr:
                c.correct_range(0, n)
                out = os.path.join(tmp, f"{name}.fq")
                c.write_output(out)
            tp, fp, fn, tn = base_counts(rs, out)
            counts[name] = {"tp": tp, "fp": fp, "fn": fn, "f1": datagen.f1(tp, fp, fn)}
            if c is mcorr:
                os.unlink(out)
        mcorr.close()
        mvalue = world * n / (mms / 1e3)
        learned = {"value": mvalue, "unit": "reads/s", "ms_per_step": mms, "ratio_vs_plain": mvalue / value,
                   "stage_ms": {"candidates": mstage[0], "align": mstage[1], "msa": mstage[2],
                                "classifier": mstage[3]},
                   "network": "24-64-64-1 GELU, bf16 tcgen05 GEMMs, fp32 accumulate",
                   "params": os.path.relpath(mlp_file, ROOT),
                   "base_level": counts, "gpu_launches": mlaunches * args.steps}

    progress("timed steps done")
    # e2e through the C ABI from host buffers
    from care_b200 import encode_reads
    packed = np.ascontiguousarray(encode_reads(rs.seqs, rs.lengths))
    quals = np.ascontiguousarray(encode_quality_2bit(rs.quals))
    lens = np.ascontiguousarray(rs.lengths.astype(np.int32))
    h2d = packed.nbytes + quals.nbytes + lens.nbytes
    for _ in range(max(1, args.warmup)):
        corr.upload_reads(packed, lens, quals)
        corr.correct_range_raw(0, n)
    barrier()
    e2e_s, up_s = [], []
    for _ in range(args.steps):
        w0 = time.perf_counter()
        corr.upload_reads(packed, lens, quals)
        w1 = time.perf_counter()
        raw = corr.correct_range_raw(0, n)
        e2e_s.append(time.perf_counter() - w0)
        up_s.append(w1 - w0)
    barrier()
    d2h = raw.num_anchors * (1 + 4 + raw.max_length) + int(raw.num_candidates) * (13 + raw.max_length)
    e2e_t = float(np.mean(e2e_s))
    if world > 1:
        t = torch.tensor([e2e_t], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = float(t.item())

    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    # MSA stage, HBM roofline: per pair the packed read (4*ceil(L/16) B, 40 B
    # at L=150) + 2-bit qualities (same) + 4 B id + 13 B alignment tuple; per
    # anchor its own row and qualities and the corrected row (L B); L taken
    # as the mean of the set's rows
    row_b = float(np.mean(8 * ((rs.lengths.astype(np.int64) + 15) // 16)))
    mean_len = float(np.mean(rs.lengths))
    per_pair = row_b + 17
    msa_bytes = stats["pairs"] * per_pair + n * (row_b + mean_len)
    msa_gbs = msa_bytes / (stage[2] / 1e3) / 1e9
    # alignment stage: un-pruned 32-bit word compares counted by k_align
    # (1486 per pair at L=150)
    align_words = stats["word_compares"]
    align_rate = align_words / (stage[1] / 1e3)
    ip = int_peaks()
    line = {
        "metric": METRIC, "value": value, "unit": "reads/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded), " + rs.name,
        "config": {**workload_config(args), "reads_per_gpu": n,
                   "l2": "flushed between steps (252 MB write); working set > L2",
                   "parallelism": f"replicas x{world} (independent read sets)",
                   "stage_ms": {"candidates": stage[0], "align": stage[1], "msa": stage[2]},
                   "pairs_per_step": stats["pairs"], "wall_ms_per_step": wall_ms,
                   "value_excludes": "the minhash signatures of the reads (k_signatures, once per read storage "
                                     "at upload/load; every step's candidate lookup reuses them): signatures_ms",
                   "signatures_ms": sig_ms,
                   "tuning": corr.tuning, "tuning_source": "care_b200/tuning (autotuned)" if tuned else "default",
                   "step1_s": step1_s},
        "roofline": {"kernel": "k_msa", "bound": "hbm", "achieved": msa_gbs, "peak": hbm_peak,
                     "bytes_per_pair": per_pair,
                     "unit": "GB/s", "frac": msa_gbs / hbm_peak,
                     "traffic": None if (uneven or large) else MSA_DRAM_BYTES_PER_ANCHOR * n,
                     "traffic_source": "ncu capture of 100,000 anchors scaled by anchors per launch",
                     "peak_source": "measured" if peaks else "fallback"},
        "roofline_alignment": {"kernel": "k_align", "bound": "int", "unit": "word compares/s",
                               "achieved": align_rate, "ms": stage[1],
                               "peak": ip["word_compares_per_s"] if ip else None,
                               "frac": align_rate / ip["word_compares_per_s"] if ip else None,
                               "popc_per_s": ip["popc_per_s"] if ip else None,
                               "work": "un-pruned: 2 orientations x sum over shifts of ceil(overlap/32), counted per "
                                       "scanned pair by k_align (1486 per pair at L=150)", "work_per_step": align_words,
                               "ms_includes": "k_pair_mirror and k_pair_order when the mapping uses them",
                               "run_per_step": run_words,
                               "run_achieved": run_words / (stage[1] / 1e3),
                               "run_frac": run_words / (stage[1] / 1e3) / ip["word_compares_per_s"] if ip else None,
                               "run_work": "word compares the scans actually run after their early exits "
                                           "(statistics form of k_align, one untimed pass)",
                               "peak_source": "care-b200-peaks (measured, registers only)" if ip else None},
        "roofline_msa_compute": {"kernel": "k_msa", "bound": "alu", "unit": "element updates/s",
                                 "achieved": stats["msa_elements"] / (stage[2] / 1e3),
                                 "peak": ip["msa_elements_per_s"] if ip else None,
                                 "frac": (stats["msa_elements"] / (stage[2] / 1e3) / ip["msa_elements_per_s"])
                                 if ip else None,
                                 "work": "bases added to column sums (anchor and candidates, every build), "
                                         "counted by k_msa",
                                 "work_per_step": stats["msa_elements"],
                                 "rebuild_elements_per_step": stats["msa_rebuild_elements"],
                                 "rebuilt_anchors_per_step": stats["msa_rebuilt_anchors"],
                                 "peak_source": "care-b200-peaks k_peak_msa (the per-element update mix in "
                                                "registers)" if ip else None},
        "e2e": {"value": world * n / e2e_t, "unit": "reads/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "upload_ms": float(np.mean(up_s)) * 1e3,
                "correct_ms": (e2e_t - float(np.mean(up_s))) * 1e3,
                "includes": "upload of the read storage and its minhash signatures (signatures_ms), "
                            "correction, results copied back",
                "signatures_ms": corr.signatures_ms(),
                "value_is": "mean over the timed steps (host wall clock of this rank)",
                "median_value": world * n / float(np.median(e2e_s)),
                "step_ms": [round(x * 1e3, 3) for x in e2e_s]},
        "gpu_launches": stats["launches"] * args.steps,         # counted by the library per call
        "clocks": clk.summary(),
    }
    if learned is not None:
        line["learned"] = learned
    line["parity"] = {"checked": False, "gpu_sha256": plain_sha}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(CARE_CPU):
        # care-cpu on all host cores on the same FASTQ with the same options:
        # the reported baseline, and the byte comparison of the two outputs
        threads = host_cores()
        progress(f"e2e done; care-cpu on the same {n} reads, {threads} threads")
        runs, cpu_sha = [], None
        for r in range(3):
            v, out = care_cpu_run(fq, tmp, threads, run_args)
            runs.append(v)
            if cpu_sha is None:
                cpu_sha = sha256_file(out)
            os.unlink(out)
        v = float(np.median(runs))
        line["parity"] = {"checked": True, "identical": cpu_sha == plain_sha, "gpu_sha256": plain_sha,
                          "care_cpu_sha256": cpu_sha,
                          "what": "corrected FASTQ of the plain method (tuned mapping) vs care-cpu's, same input"}
        progress("care-cpu sample on 1 thread")
        one = care_cpu_sample(tmp, 1)
        line["cpu_baseline"] = {"value": v, "unit": "reads/s", "cores": threads, "kind": "reference",
                                "sample": f"the whole workload ({n} reads), care-cpu -t {threads}; median of 3 runs",
                                "runs": runs, "per_core_reads_s": one,
                                "per_core_sample": "care-cpu -t 1 on 250 kbp genome, 50,000 reads, PE model",
                                "cpu_model": cpu_model()}
    corr.close()
    if rank == 0 and world == 1 and args.workload == "pe" and not args.no_extra:
        # the batched uneven set and the large set, a few steps each
        del rs
        ks, kw = min(args.steps, 5), min(args.warmup, 3)
        for kind in ("uneven", "large"):
            try:
                line[kind] = workload_block(kind, ks, kw, flush, local, tmp, learned=not args.no_learned)
            except Exception as e:           # the main line is still printed
                line[kind] = {"error": f"{type(e).__name__}: {e}"}
                progress(f"{kind} block failed: {e}")
    shutil.rmtree(tmp, ignore_errors=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
