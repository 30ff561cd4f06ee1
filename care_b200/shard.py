"""Correcting one read set on several GPUs (one process per GPU).

Anchors are independent given the read-only read storage and tables, so the
path shards by anchor: every rank holds the whole storage and tables, corrects
one contiguous anchor range (pair-aligned for paired-end input, as
CpuErrorCorrector::processMulti requires, corrector.hpp:328) and serializes
its results in the reference's record format (EncodedTempCorrectedSequence,
correctedsequence.hpp:148-340). The records are gathered once at the end
(no collective on the data path); the reference's STEP3 orders records by
read id itself (sortserializedresults.hpp), so the merged stream is the
concatenation in rank order.
"""
from __future__ import annotations

import struct

import numpy as np


def shard_range(num_reads: int, rank: int, world: int, paired: bool) -> tuple[int, int]:
    """(first, count) of this rank's anchors: contiguous, balanced, covering
    [0, num_reads) exactly once; pair-aligned for paired-end storage."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    unit = 2 if paired else 1
    if paired and num_reads % 2:
        raise ValueError("paired-end storage has an even number of reads")
    units = num_reads // unit
    b = units * rank // world * unit
    e = units * (rank + 1) // world * unit
    return b, e - b


def merge_records(blobs) -> bytes:
    """Record streams of the ranks, in rank order."""
    return b"".join(blobs)


def iter_records(blob: bytes):
    """(read_id, hq, use_edits, type, payload bytes) of each record."""
    pos = 0
    while pos < len(blob):
        rid, flags = struct.unpack_from("<II", blob, pos)
        n = flags & ((1 << 29) - 1)
        yield rid, flags >> 31, (flags >> 30) & 1, (flags >> 29) & 1, blob[pos + 8:pos + 8 + n]
        pos += 8 + n
    if pos != len(blob):
        raise ValueError("truncated record stream")


def record_multiset(blob: bytes):
    return sorted(iter_records(blob))


def gather_records(blob: bytes, group=None) -> bytes:
    """All ranks' record streams, merged in rank order (on every rank): the
    sizes first, then one all-gather of byte tensors padded to the largest
    stream (CUDA tensors over NCCL, host tensors over gloo; no pickling)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    size = torch.tensor([len(blob)], dtype=torch.int64, device=dev)
    sizes = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(sizes, size, group=group)
    sizes = [int(x.item()) for x in sizes]
    cap = max(max(sizes), 1)
    mine = torch.zeros(cap, dtype=torch.uint8, device=dev)
    if blob:
        mine[:len(blob)] = torch.frombuffer(bytearray(blob), dtype=torch.uint8).to(dev)
    parts = [torch.empty(cap, dtype=torch.uint8, device=dev) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    return merge_records(p[:n].cpu().numpy().tobytes() for p, n in zip(parts, sizes))


def correct_sharded(corrector, rank: int, world: int, group=None) -> bytes:
    """This rank's share of the correction on its GPU, then the merged record
    stream of the whole read set (identical on every rank)."""
    paired = bool(corrector.opts.paired_end)
    first, count = shard_range(corrector.num_reads, rank, world, paired)
    raw = corrector.correct_range_raw(first, count)
    blob = corrector.serialize(raw)
    return gather_records(blob, group) if world > 1 else blob


def encode_records(anchor_ids, status, num_edits, anchor_seqs, cand_ids, cand_shifts, cand_use_edits,
                   cand_seqs, lengths, original) -> bytes:
    """The record stream of a result set, as care_b200_serialize_results
    writes it: anchors (save filter: corrected and not an HQ anchor with zero
    edits, correct_cpu.cpp:255-273), then candidate corrections. `original`
    maps a read id to its uncorrected sequence bytes (for edit lists)."""
    out = bytearray()

    def rec(rid, hq, ue, typ, shift, seq, L):
        if ue:
            orig = original(rid)
            epos = [p for p in range(L) if seq[p] != orig[p]]
            nbytes = 4 + 5 * len(epos) + (4 if typ else 0)
            out.extend(struct.pack("<II", rid, (hq << 31) | (ue << 30) | (typ << 29) | nbytes))
            out.extend(struct.pack("<i", len(epos)))
            for p in epos:
                out.extend(struct.pack("<i", p))
            out.extend(bytes(seq[p] for p in epos))
        else:
            nbytes = 4 + L + (4 if typ else 0)
            out.extend(struct.pack("<II", rid, (hq << 31) | (ue << 30) | (typ << 29) | nbytes))
            out.extend(struct.pack("<i", L))
            out.extend(bytes(seq[:L]))
        if typ:
            out.extend(struct.pack("<i", shift))

    for k, rid in enumerate(anchor_ids):
        st = int(status[k])
        if not st & 1:
            continue
        hq, ue = (st >> 1) & 1, (st >> 2) & 1
        if hq and ue and int(num_edits[k]) == 0:
            continue
        rec(int(rid), hq, ue, 0, 0, anchor_seqs[k], int(lengths[rid]))
    for j, rid in enumerate(cand_ids):
        rec(int(rid), 0, int(cand_use_edits[j]), 1, int(cand_shifts[j]), cand_seqs[j], int(lengths[rid]))
    return bytes(out)
