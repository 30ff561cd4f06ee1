"""Seeded synthetic read sets for the correction path.

CARE ships no benchmark data; the workloads it is measured on are defined
only by shape: genome size, repeat content, read length, coverage, error and
quality model. This module produces those read sets from a seed, together
with the error-free ("true") read sequences in read orientation, which the
base-level TP/FP/FN metric of the reference's evaluation tool
(evaluationtool/arteval.cpp:183-201) needs.

Encoding: bases are uint8 codes 0..3 for A,C,G,T (the 2-bit code of
include/sequencehelpers.hpp:86-100 of the reference).
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

ASCII = np.frombuffer(b"ACGT", dtype=np.uint8)


@dataclasses.dataclass
class ReadSet:
    seqs: np.ndarray          # (n, Lmax) uint8 ASCII, padded with 0 past length
    quals: np.ndarray         # (n, Lmax) uint8 ASCII Phred+33
    truth: np.ndarray         # (n, Lmax) uint8 ASCII error-free sequence
    lengths: np.ndarray       # (n,) int32
    paired: bool
    name: str

    @property
    def num_reads(self) -> int:
        return int(self.lengths.shape[0])

    def write_fastq(self, path: str, truth: bool = False) -> None:
        """Write interleaved FASTQ (mates adjacent for paired sets)."""
        src = self.truth if truth else self.seqs
        with open(path, "wb") as f:
            n = self.num_reads
            chunk = 200_000
            for b in range(0, n, chunk):
                e = min(n, b + chunk)
                parts = []
                for i in range(b, e):
                    L = int(self.lengths[i])
                    parts.append(b"@r%d\n" % i)
                    parts.append(src[i, :L].tobytes())
                    parts.append(b"\n+\n")
                    parts.append(self.quals[i, :L].tobytes())
                    parts.append(b"\n")
                f.write(b"".join(parts))


def write_fastq_fast(rs: ReadSet, path: str) -> None:
    """Interleaved FASTQ of the reads ("@r<id>" headers, as ReadSet.write_fastq);
    sets of more than 2M fixed-length reads take the bulk writer instead."""
    n, W = rs.num_reads, rs.seqs.shape[1]
    if (rs.lengths == W).all() and n > 2_000_000:
        return write_fastq_fixed(rs, path)
    lens = rs.lengths
    seqs = rs.seqs.tobytes()
    quals = rs.quals.tobytes()
    with open(path, "wb") as f:
        chunk = 100_000
        for b in range(0, n, chunk):
            parts = []
            for i in range(b, min(n, b + chunk)):
                o, L = i * W, int(lens[i])
                parts += [b"@r%d\n" % i, seqs[o:o + L], b"\n+\n", quals[o:o + L], b"\n"]
            f.write(b"".join(parts))


def write_fastq_fixed(rs: ReadSet, path: str, chunk: int = 1_000_000) -> None:
    """Fixed-length reads as 4-line FASTQ records built in bulk: header
    "@r<id, 10 digits>", sequence, "+", qualities."""
    n, L = rs.seqs.shape
    rec = 17 + 2 * L
    with open(path, "wb") as f:
        for b in range(0, n, chunk):
            e = min(n, b + chunk)
            m = e - b
            buf = np.empty((m, rec), np.uint8)
            ids = np.arange(b, e, dtype=np.int64)
            buf[:, 0] = ord("@")
            buf[:, 1] = ord("r")
            for d in range(10):
                buf[:, 11 - d] = ord("0") + (ids // 10 ** d) % 10
            buf[:, 12] = ord("\n")
            buf[:, 13:13 + L] = rs.seqs[b:e]
            buf[:, 13 + L] = ord("\n")
            buf[:, 14 + L] = ord("+")
            buf[:, 15 + L] = ord("\n")
            buf[:, 16 + L:16 + 2 * L] = rs.quals[b:e]
            buf[:, 16 + 2 * L] = ord("\n")
            f.write(buf.tobytes())


def random_genome(rng: np.random.Generator, size: int) -> np.ndarray:
    return rng.integers(0, 4, size=size, dtype=np.uint8)


def mutate(rng: np.random.Generator, seq: np.ndarray, rate: float) -> np.ndarray:
    """Substitute each base with probability `rate` by one of the other three."""
    out = seq.copy()
    hit = rng.random(seq.shape[0]) < rate
    out[hit] = (out[hit] + rng.integers(1, 4, size=int(hit.sum()), dtype=np.uint8)) & 3
    return out


def place_repeats(rng: np.random.Generator, genome: np.ndarray,
                  families: list[tuple[int, int, float]]) -> None:
    """Write repeat copies into the genome at non-overlapping positions.

    families: list of (unit_length, copies, divergence). Each copy is the unit
    with independent substitutions at the family's divergence.
    """
    G = genome.shape[0]
    total = sum(u * c for u, c, _ in families)
    if total > G:
        raise ValueError("repeats do not fit in the genome")
    # random non-overlapping layout: distribute the free space as random gaps
    pieces = []
    for fi, (u, c, d) in enumerate(families):
        pieces.extend([(fi, u)] * c)
    order = rng.permutation(len(pieces))
    free = G - total
    cuts = np.sort(rng.integers(0, free + 1, size=len(pieces)))
    gaps = np.diff(np.concatenate([[0], cuts]))
    units = [random_genome(rng, u) for (u, _, _) in families]
    pos = 0
    for k, idx in enumerate(order):
        fi, u = pieces[idx]
        pos += int(gaps[k])
        genome[pos:pos + u] = mutate(rng, units[fi], families[fi][2])
        pos += u


def revcomp_codes(a: np.ndarray) -> np.ndarray:
    return (3 - a)[..., ::-1]


def _extract(genome: np.ndarray, starts: np.ndarray, L: int) -> np.ndarray:
    idx = starts[:, None] + np.arange(L)[None, :]
    return genome[idx]


def _pos_dependent_errors(rng, truth_codes, lengths, lo=0.002, hi=0.015,
                          qsd=3.0, qmin=2, qmax=40):
    """Substitution rate rising linearly along the read; Q from the rate."""
    n, Lmax = truth_codes.shape
    pos = np.arange(Lmax)[None, :].astype(np.float64)
    # rate and -10 log10(rate) per distinct read length, then per read
    ulen, inv = np.unique(lengths, return_inverse=True)
    denom = np.maximum(ulen[:, None] - 1, 1).astype(np.float64)
    pu = lo + (hi - lo) * np.minimum(pos / denom, 1.0)
    p = pu[inv.reshape(-1)]
    qbase = (-10.0 * np.log10(pu))[inv.reshape(-1)]
    err = rng.random((n, Lmax)) < p
    valid = pos < lengths[:, None]
    err &= valid
    codes = truth_codes.copy()
    codes[err] = (codes[err] + rng.integers(1, 4, size=int(err.sum()), dtype=np.uint8)) & 3
    q = np.rint(qbase + rng.normal(0.0, qsd, size=(n, Lmax)))
    q = np.clip(q, qmin, qmax).astype(np.uint8)
    return codes, q, valid


def _finish(codes, truth_codes, q, valid, lengths, paired, name):
    seqs = np.where(valid, ASCII[codes], 0).astype(np.uint8)
    truth = np.where(valid, ASCII[truth_codes], 0).astype(np.uint8)
    quals = np.where(valid, q + 33, 0).astype(np.uint8)
    return ReadSet(seqs, quals, truth, lengths.astype(np.int32), paired, name)


def single_end_uniform(seed: int = 1, genome_size: int = 1_000_000,
                       num_reads: int = 300_000, L: int = 100,
                       error_rate: float = 0.01) -> ReadSet:
    """Uniform-random genome, fixed-length SE reads on a random strand, i.i.d.
    substitutions, Q30 on correct and Q10 on erroneous bases."""
    rng = np.random.default_rng(seed)
    genome = random_genome(rng, genome_size)
    starts = rng.integers(0, genome_size - L + 1, size=num_reads)
    truth = _extract(genome, starts, L)
    rc = rng.random(num_reads) < 0.5
    truth[rc] = revcomp_codes(truth[rc])
    err = rng.random((num_reads, L)) < error_rate
    codes = truth.copy()
    codes[err] = (codes[err] + rng.integers(1, 4, size=int(err.sum()), dtype=np.uint8)) & 3
    q = np.where(err, 10, 30).astype(np.uint8)
    valid = np.ones((num_reads, L), dtype=bool)
    lengths = np.full(num_reads, L, dtype=np.int32)
    return _finish(codes, truth, q, valid, lengths, False, "se_uniform")


def paired_end_repeats(seed: int = 2, genome_size: int = 5_000_000,
                       coverage: float = 30.0, L: int = 150,
                       frag_mean: float = 400.0, frag_sd: float = 40.0,
                       repeat_unit: int = 5000, repeat_copies: int = 20,
                       repeat_div: float = 0.01) -> ReadSet:
    """Genome with one repeat family, interleaved PE reads (R2 is the reverse
    complement of the fragment end), position-dependent substitutions."""
    rng = np.random.default_rng(seed)
    genome = random_genome(rng, genome_size)
    if repeat_copies > 0:
        place_repeats(rng, genome, [(repeat_unit, repeat_copies, repeat_div)])
    num_pairs = int(round(coverage * genome_size / (2 * L)))
    frag = np.clip(np.rint(rng.normal(frag_mean, frag_sd, size=num_pairs)), L, None).astype(np.int64)
    starts = (rng.random(num_pairs) * (genome_size - frag + 1)).astype(np.int64)
    r1 = _extract(genome, starts, L)
    r2 = revcomp_codes(_extract(genome, starts + frag - L, L))
    flip = rng.random(num_pairs) < 0.5          # fragment from the other strand
    r1f = np.where(flip[:, None], r2, r1)
    r2f = np.where(flip[:, None], r1, r2)
    truth = np.empty((2 * num_pairs, L), dtype=np.uint8)
    truth[0::2] = r1f
    truth[1::2] = r2f
    lengths = np.full(2 * num_pairs, L, dtype=np.int32)
    codes, q, valid = _pos_dependent_errors(rng, truth, lengths)
    return _finish(codes, truth, q, valid, lengths, True, "pe_repeats")


def paired_end_large(seed: int = 5, genome_size: int = 50_000_000, coverage: float = 50.0, L: int = 150,
                     frag_mean: float = 400.0, frag_sd: float = 40.0, repeat_fraction: float = 0.05,
                     indel_rate: float = 1e-4, n_rate: float = 1e-3, chunk_pairs: int = 500_000) -> ReadSet:
    """The large set: repeat families (5 kbp units, 20 copies, 0.5-2%
    divergence) over `repeat_fraction` of the genome, interleaved 150 bp PE
    reads, position-dependent substitutions and qualities as in
    paired_end_repeats, plus single-base insertions and deletions
    (`indel_rate` per base) and N bases (`n_rate` per base, quality kept).
    Generated in chunks of pairs, each from its own seeded stream, so memory
    stays bounded. truth holds the error-free read (the genome without the
    indel), so an indel counts as residual errors past its position."""
    rng = np.random.default_rng(seed)
    genome = random_genome(rng, genome_size)
    unit, copies = 5000, 20
    nfam = int(repeat_fraction * genome_size) // (unit * copies)
    if nfam > 0:
        place_repeats(rng, genome, [(unit, copies, float(rng.uniform(0.005, 0.02))) for _ in range(nfam)])
    num_pairs = int(round(coverage * genome_size / (2 * L)))
    n = 2 * num_pairs
    seqs = np.empty((n, L), np.uint8)
    quals = np.empty((n, L), np.uint8)
    truth = np.empty((n, L), np.uint8)
    j = np.arange(L)[None, :]

    def chunk(c: int) -> None:
        b = c * chunk_pairs
        m = min(chunk_pairs, num_pairs - b)
        cr = np.random.default_rng([seed, 1 + c])
        frag = np.clip(np.rint(cr.normal(frag_mean, frag_sd, size=m)), L + 1, None).astype(np.int64)
        starts = (cr.random(m) * (genome_size - frag + 1)).astype(np.int64)
        s1 = _extract(genome, starts, L + 1)                          # read orientation, one spare base
        s2 = revcomp_codes(_extract(genome, starts + frag - L - 1, L + 1))
        flip = cr.random(m) < 0.5
        a = np.where(flip[:, None], s2, s1)
        bseg = np.where(flip[:, None], s1, s2)
        seg = np.empty((2 * m, L + 1), np.uint8)
        seg[0::2] = a
        seg[1::2] = bseg
        tr = seg[:, :L].copy()
        # single-base indels: the read takes the segment with one base
        # dropped (deletion) or one random base inserted
        rd = seg[:, :L].copy()
        hit = np.nonzero(cr.random(2 * m) < 1.0 - (1.0 - indel_rate) ** L)[0]
        if hit.size:
            pos = cr.integers(1, L, size=hit.size)[:, None]
            ins = cr.random(hit.size) < 0.5
            src = np.where(ins[:, None], j - (j > pos), j + (j >= pos))
            rows = np.take_along_axis(seg[hit], src, axis=1)
            extra = cr.integers(0, 4, size=hit.size, dtype=np.uint8)
            rows[ins, pos[ins, 0]] = extra[ins]
            rd[hit] = rows
        # the substitution and quality model of _pos_dependent_errors for
        # fixed-length reads, drawn in float32
        pr = (0.002 + 0.013 * np.arange(L, dtype=np.float32) / np.float32(L - 1)).astype(np.float32)
        err = cr.random((2 * m, L), dtype=np.float32) < pr[None, :]
        codes = rd
        codes[err] = (codes[err] + cr.integers(1, 4, size=int(err.sum()), dtype=np.uint8)) & 3
        qb = (-10.0 * np.log10(pr)).astype(np.float32)
        q = np.clip(np.rint(qb[None, :] + cr.standard_normal((2 * m, L), dtype=np.float32) * np.float32(3.0)),
                    2, 40).astype(np.uint8)
        sq = ASCII[codes]
        sq[cr.random((2 * m, L)) < n_rate] = ord("N")
        seqs[2 * b:2 * (b + m)] = sq
        quals[2 * b:2 * (b + m)] = q + 33
        truth[2 * b:2 * (b + m)] = ASCII[tr]

    # chunks are independent streams writing disjoint rows: run them on threads
    import concurrent.futures
    import os
    nchunks = (num_pairs + chunk_pairs - 1) // chunk_pairs
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(nchunks, os.cpu_count() or 1)) as ex:
        list(ex.map(chunk, range(nchunks)))
    return ReadSet(seqs, quals, truth, np.full(n, L, dtype=np.int32), True, "pe_large")


def single_end_uneven(seed: int = 3, genome_size: int = 10_000_000,
                      coverage: float = 40.0, Lmin: int = 50, Lmax: int = 250,
                      repeat_fraction: float = 0.08) -> ReadSet:
    """Genome with many repeat families (5-500 copies, 0.5-2% divergence) and
    variable-length SE reads, so per-anchor candidate counts are very uneven."""
    rng = np.random.default_rng(seed)
    genome = random_genome(rng, genome_size)
    fams = []
    budget = int(repeat_fraction * genome_size)
    while budget > 0:
        u = int(rng.integers(300, 3001))
        c = int(np.exp(rng.uniform(np.log(5), np.log(500))))
        c = max(5, min(c, budget // u))
        if c < 5:
            break
        fams.append((u, c, float(rng.uniform(0.005, 0.02))))
        budget -= u * c
    place_repeats(rng, genome, fams)
    mean_len = 0.5 * (Lmin + Lmax)
    n = int(round(coverage * genome_size / mean_len))
    lengths = rng.integers(Lmin, Lmax + 1, size=n).astype(np.int32)
    starts = (rng.random(n) * (genome_size - lengths + 1)).astype(np.int64)
    idx = starts[:, None] + np.arange(Lmax)[None, :]
    idx = np.minimum(idx, genome_size - 1)
    truth = genome[idx]
    rc = rng.random(n) < 0.5
    # reverse-complement the first L bases of the rows drawn for the minus strand
    j = np.arange(Lmax)[None, :]
    rows = np.nonzero(rc)[0]
    for b in range(0, rows.shape[0], 100_000):
        r = rows[b:b + 100_000]
        Lr = lengths[r][:, None]
        src = np.where(j < Lr, Lr - 1 - j, j)
        sub = np.take_along_axis(truth[r], src, axis=1)
        truth[r] = np.where(j < Lr, 3 - sub, sub)
    codes, q, valid = _pos_dependent_errors(rng, truth, lengths)
    return _finish(codes, truth, q, valid, lengths, False, "se_uneven")


WORKLOADS = {
    "se_uniform": single_end_uniform,
    "pe_repeats": paired_end_repeats,
    "se_uneven": single_end_uneven,
    "pe_large": paired_end_large,
}


def base_level_counts(original: np.ndarray, corrected: np.ndarray,
                      truth: np.ndarray, lengths: np.ndarray):
    """TP/FP/FN/TN per base as in evaluationtool/arteval.cpp:183-201:
    TP orig!=true & corr==true; FP orig==true & corr!=true;
    FN orig!=true & corr!=true; TN orig==true & corr==true."""
    valid = np.arange(original.shape[1])[None, :] < lengths[:, None]
    o_ok = (original == truth) & valid
    c_ok = (corrected == truth) & valid
    o_bad = (~(original == truth)) & valid
    c_bad = (~(corrected == truth)) & valid
    tp = int((o_bad & c_ok).sum())
    fp = int((o_ok & c_bad).sum())
    fn = int((o_bad & c_bad).sum())
    tn = int((o_ok & c_ok).sum())
    return tp, fp, fn, tn


def f1(tp: int, fp: int, fn: int) -> float:
    d = 2 * tp + fp + fn
    return 0.0 if d == 0 else 2 * tp / d


def read_fastq(path: str):
    """Minimal 4-line FASTQ reader -> (headers, list of sequence bytes, list of quals)."""
    heads, seqs, quals = [], [], []
    with open(path, "rb") as f:
        lines = f.read().split(b"\n")
    for i in range(0, len(lines) - 3, 4):
        if not lines[i].startswith(b"@"):
            break
        heads.append(lines[i][1:])
        seqs.append(lines[i + 1])
        quals.append(lines[i + 3])
    return heads, seqs, quals


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("workload", choices=sorted(WORKLOADS))
    ap.add_argument("out")
    ap.add_argument("--seed", type=int, default=None)
    ap.add_argument("--scale", type=float, default=1.0,
                    help="multiply the genome size (coverage stays)")
    ap.add_argument("--truth", default=None, help="also write error-free reads here")
    a = ap.parse_args(argv)
    fn = WORKLOADS[a.workload]
    kw = {}
    if a.seed is not None:
        kw["seed"] = a.seed
    if a.scale != 1.0:
        import inspect
        gs = inspect.signature(fn).parameters["genome_size"].default
        kw["genome_size"] = int(gs * a.scale)
        if a.workload == "se_uniform":
            kw["num_reads"] = int(300_000 * a.scale)
    rs = fn(**kw)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    rs.write_fastq(a.out)
    if a.truth:
        rs.write_fastq(a.truth, truth=True)
    print(f"{rs.name}: {rs.num_reads} reads, Lmax {rs.seqs.shape[1]}")


if __name__ == "__main__":
    main()
