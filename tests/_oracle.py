"""ctypes bindings of the CPU oracle (oracle/care_oracle.h) for the tests.

Test infrastructure only: the oracle is the checker, never the product.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE_DIR, "_ref", "libcareoracle.so")
CLI = os.path.join(ORACLE_DIR, "_ref", "care-oracle")
CARE_CPU = os.path.join(ORACLE_DIR, "_ref", "care-cpu")


class CoOpts(ctypes.Structure):
    _fields_ = [
        ("kmerlength", ctypes.c_int), ("num_maps", ctypes.c_int), ("min_overlap", ctypes.c_int),
        ("max_error_rate", ctypes.c_float), ("min_overlap_ratio", ctypes.c_float),
        ("estimated_errorrate", ctypes.c_float), ("estimated_coverage", ctypes.c_float),
        ("m_coverage", ctypes.c_float), ("paired_filter_threshold", ctypes.c_float),
        ("new_columns_to_correct", ctypes.c_int), ("use_quality", ctypes.c_int),
        ("quality_bits", ctypes.c_int), ("exclude_ambiguous", ctypes.c_int),
        ("correct_candidates", ctypes.c_int), ("paired_end", ctypes.c_int), ("threads", ctypes.c_int),
        ("quality_labels", ctypes.c_int), ("clf_mode", ctypes.c_int), ("clf_min_coverage", ctypes.c_int),
        ("mlp", ctypes.POINTER(ctypes.c_float)),
    ]


class CoReads(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint32), ("min_len", ctypes.c_int), ("max_len", ctypes.c_int),
        ("seq_pitch", ctypes.c_int), ("qual_pitch", ctypes.c_int), ("quality_bits", ctypes.c_int),
        ("has_quality", ctypes.c_int), ("seq", ctypes.POINTER(ctypes.c_uint32)),
        ("qual", ctypes.POINTER(ctypes.c_uint32)), ("len", ctypes.POINTER(ctypes.c_int32)),
        ("ambig", ctypes.POINTER(ctypes.c_uint8)), ("text", ctypes.c_char_p),
        ("rec_off", ctypes.POINTER(ctypes.c_size_t)), ("fasta", ctypes.c_int),
    ]


class CoTable(ctypes.Structure):
    _fields_ = [("keys", ctypes.POINTER(ctypes.c_uint64)), ("offsets", ctypes.POINTER(ctypes.c_uint32)),
                ("values", ctypes.POINTER(ctypes.c_uint32)), ("nkeys", ctypes.c_size_t)]


class CoTables(ctypes.Structure):
    _fields_ = [("num_maps", ctypes.c_int), ("k", ctypes.c_int), ("threshold", ctypes.c_int),
                ("t", ctypes.POINTER(CoTable))]


class CoAnchor(ctypes.Structure):
    _fields_ = [("status", ctypes.c_uint8), ("hq", ctypes.c_uint8), ("use_edits", ctypes.c_uint8),
                ("pad", ctypes.c_uint8), ("num_edits", ctypes.c_int32)]


class CoCand(ctypes.Structure):
    _fields_ = [("read_id", ctypes.c_uint32), ("anchor_id", ctypes.c_uint32), ("shift", ctypes.c_int32),
                ("length", ctypes.c_int32), ("use_edits", ctypes.c_uint8), ("pad", ctypes.c_uint8 * 3)]


NFEAT = 24
MLP_FLOATS = 5873


class CoFeature(ctypes.Structure):
    _fields_ = [("read_id", ctypes.c_uint32), ("pos", ctypes.c_int16), ("orig", ctypes.c_uint8),
                ("cons", ctypes.c_uint8), ("logit", ctypes.c_float), ("x", ctypes.c_float * NFEAT)]


class CoResults(ctypes.Structure):
    _fields_ = [("first", ctypes.c_uint32), ("count", ctypes.c_uint32), ("max_len", ctypes.c_int),
                ("anchors", ctypes.POINTER(CoAnchor)), ("anchor_seq", ctypes.POINTER(ctypes.c_char)),
                ("cands", ctypes.POINTER(CoCand)), ("cand_seq", ctypes.POINTER(ctypes.c_char)),
                ("num_cands", ctypes.c_size_t), ("cap_cands", ctypes.c_size_t),
                ("feats", ctypes.POINTER(CoFeature)), ("num_feats", ctypes.c_size_t),
                ("cap_feats", ctypes.c_size_t)]


class CoAlign(ctypes.Structure):
    _fields_ = [("score", ctypes.c_int), ("overlap", ctypes.c_int), ("shift", ctypes.c_int),
                ("nops", ctypes.c_int), ("valid", ctypes.c_int)]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", ORACLE_DIR], check=True, capture_output=True)
    L = ctypes.CDLL(LIB)
    P = ctypes.POINTER
    L.co_default_opts.argtypes = [P(CoOpts)]
    L.co_reads_from_files.argtypes = [P(ctypes.c_char_p), ctypes.c_int, P(CoOpts)]
    L.co_reads_from_files.restype = P(CoReads)
    L.co_reads_free.argtypes = [P(CoReads)]
    L.co_build_tables.argtypes = [P(CoReads), P(CoOpts)]
    L.co_build_tables.restype = P(CoTables)
    L.co_tables_free.argtypes = [P(CoTables)]
    L.co_correct.argtypes = [P(CoReads), P(CoTables), P(CoOpts), ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
    L.co_correct.restype = P(CoResults)
    L.co_results_free.argtypes = [P(CoResults)]
    L.co_write_output.argtypes = [P(CoReads), P(CoResults), P(CoOpts), ctypes.c_char_p]
    L.co_run.argtypes = [P(ctypes.c_char_p), ctypes.c_int, ctypes.c_char_p, P(CoOpts), P(ctypes.c_double)]
    L.co_bf16_round.argtypes = [ctypes.c_float]
    L.co_bf16_round.restype = ctypes.c_float
    L.co_mlp_logit.argtypes = [P(ctypes.c_float), P(ctypes.c_float)]
    L.co_mlp_logit.restype = ctypes.c_float
    L.co_encode_2bit.argtypes = [ctypes.c_char_p, ctypes.c_int, P(ctypes.c_uint32)]
    L.co_decode_2bit.argtypes = [P(ctypes.c_uint32), ctypes.c_int, ctypes.c_char_p]
    L.co_revcomp_2bit.argtypes = [P(ctypes.c_uint32), ctypes.c_int, P(ctypes.c_uint32)]
    L.co_to_hilo.argtypes = [P(ctypes.c_uint32), ctypes.c_int, P(ctypes.c_uint32)]
    L.co_murmur64.argtypes = [ctypes.c_uint64]
    L.co_murmur64.restype = ctypes.c_uint64
    L.co_signature.argtypes = [P(ctypes.c_uint32), ctypes.c_int, ctypes.c_int, ctypes.c_int, P(ctypes.c_uint64)]
    L.co_threshold.argtypes = [ctypes.c_float]
    L.co_encode_quality.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, P(ctypes.c_uint32)]
    L.co_decode_quality.argtypes = [P(ctypes.c_uint32), ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
    L.co_quality_weights.argtypes = [P(ctypes.c_float)]
    L.co_shd.argtypes = [P(ctypes.c_uint32), ctypes.c_int, P(ctypes.c_uint32), ctypes.c_int, ctypes.c_int,
                         ctypes.c_float, ctypes.c_float, P(CoAlign)]
    L.co_orientation.argtypes = [P(CoAlign), P(CoAlign), ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                 ctypes.c_int, ctypes.c_float]
    L.co_pair_flags.argtypes = [P(ctypes.c_uint32), ctypes.c_int, P(ctypes.c_uint32), ctypes.c_int,
                                P(ctypes.c_uint8), P(ctypes.c_uint8)]
    _lib = L
    return L


def opts_from_args(args: str) -> CoOpts:
    """care-cpu style argument string -> CoOpts."""
    o = CoOpts()
    lib().co_default_opts(ctypes.byref(o))
    toks = args.split()
    i = 0
    while i < len(toks):
        t = toks[i]
        v = toks[i + 1] if i + 1 < len(toks) else None
        if t in ("-c", "--coverage"):
            o.estimated_coverage = float(v); i += 1
        elif t in ("-k", "--kmerlength"):
            o.kmerlength = int(v); i += 1
        elif t in ("-h", "--hashmaps"):
            o.num_maps = int(v); i += 1
        elif t == "--pairmode":
            o.paired_end = v in ("PE", "pe"); i += 1
        elif t in ("-q", "--useQualityScores"):
            o.use_quality = 1
        elif t == "--qualityScoreBits":
            o.quality_bits = int(v); i += 1
        elif t == "--excludeAmbiguous":
            o.exclude_ambiguous = 1
        elif t == "--candidateCorrection":
            o.correct_candidates = 1
        elif t == "--correctionQualityLabels":
            o.quality_labels = 1
        elif t in ("-t", "--threads"):
            o.threads = int(v); i += 1
        else:
            raise ValueError(t)
        i += 1
    return o


class OracleRun:
    """Reads + tables + per-anchor results of the oracle for one input."""

    def __init__(self, files, opts: CoOpts, threads: int = 4, first: int = 0, count: int | None = None):
        L = lib()
        self.opts = opts
        arr = (ctypes.c_char_p * len(files))(*[f.encode() for f in files])
        self.reads = L.co_reads_from_files(arr, len(files), ctypes.byref(opts))
        if not self.reads:
            raise RuntimeError("oracle could not read input")
        self.tables = L.co_build_tables(self.reads, ctypes.byref(opts))
        r = self.reads.contents
        self.first = first
        self.res = L.co_correct(self.reads, self.tables, ctypes.byref(opts), first,
                                r.n - first if count is None else count, threads)

    def close(self):
        L = lib()
        L.co_results_free(self.res)
        L.co_tables_free(self.tables)
        L.co_reads_free(self.reads)

    def table(self, m: int):
        t = self.tables.contents.t[m]
        nk = t.nkeys
        keys = np.ctypeslib.as_array(t.keys, shape=(nk,)).copy() if nk else np.zeros(0, np.uint64)
        offs = np.ctypeslib.as_array(t.offsets, shape=(nk + 1,)).copy()
        nv = int(offs[-1])
        vals = np.ctypeslib.as_array(t.values, shape=(nv,)).copy() if nv else np.zeros(0, np.uint32)
        return keys, offs, vals

    def anchors(self):
        res = self.res.contents
        n = res.count
        a = np.ctypeslib.as_array(ctypes.cast(res.anchors, ctypes.POINTER(ctypes.c_uint8)), shape=(n * 8,))
        a = a.reshape(n, 8)
        status = a[:, 0].astype(np.uint8)
        hq = a[:, 1].astype(np.uint8)
        ue = a[:, 2].astype(np.uint8)
        ne = a[:, 4:8].copy().view(np.int32).reshape(n)
        L = res.max_len
        seq = np.ctypeslib.as_array(ctypes.cast(res.anchor_seq, ctypes.POINTER(ctypes.c_uint8)), shape=(n, L)).copy()
        return status, hq, ue, ne, seq

    def candidates(self):
        res = self.res.contents
        nc = res.num_cands
        L = res.max_len
        if nc == 0:
            return [], np.zeros((0, L), np.uint8)
        c = [(res.cands[i].read_id, res.cands[i].anchor_id, res.cands[i].shift, res.cands[i].use_edits)
             for i in range(nc)]
        seq = np.ctypeslib.as_array(ctypes.cast(res.cand_seq, ctypes.POINTER(ctypes.c_uint8)), shape=(nc, L)).copy()
        return c, seq

    def features(self):
        """Decision-column rows: dict of read_id, pos, orig, cons (2-bit
        codes), logit and x (n, 24), in anchor then position order."""
        res = self.res.contents
        n = res.num_feats
        if n == 0:
            return {"read_id": np.zeros(0, np.uint32), "pos": np.zeros(0, np.int16),
                    "orig": np.zeros(0, np.uint8), "cons": np.zeros(0, np.uint8),
                    "logit": np.zeros(0, np.float32), "x": np.zeros((0, NFEAT), np.float32)}
        raw = np.ctypeslib.as_array(ctypes.cast(res.feats, ctypes.POINTER(ctypes.c_uint8)),
                                    shape=(n * ctypes.sizeof(CoFeature),)).copy()
        dt = np.dtype([("read_id", "<u4"), ("pos", "<i2"), ("orig", "u1"), ("cons", "u1"),
                       ("logit", "<f4"), ("x", "<f4", (NFEAT,))])
        a = raw.view(dt)
        return {k: a[k].copy() for k in dt.names}

    def original(self, rid: int) -> bytes:
        """Uncorrected (2-bit decoded) sequence of a read."""
        r = self.reads.contents
        L = int(r.len[rid])
        buf = ctypes.create_string_buffer(max(L, 1) + 1)
        words = ctypes.cast(ctypes.addressof(r.seq.contents) + rid * r.seq_pitch * 4, ctypes.POINTER(ctypes.c_uint32))
        lib().co_decode_2bit(words, L, buf)
        return buf.raw[:L]

    def records(self) -> bytes:
        """The results as the library's record stream (care_b200.shard.encode_records)."""
        from care_b200.shard import encode_records
        status, hq, ue, ne, seq = self.anchors()
        st = (status & 1) | (hq << 1) | (ue << 2)
        cands, cseq = self.candidates()
        n = status.shape[0]
        return encode_records(range(self.first, self.first + n), st, ne, seq,
                              [c[0] for c in cands], [c[2] for c in cands], [c[3] for c in cands], cseq,
                              self.lengths(), self.original)

    def lengths(self):
        r = self.reads.contents
        return np.ctypeslib.as_array(r.len, shape=(r.n,)).copy()

    def storage(self):
        """Packed rows, encoded quality rows (or None) and ambiguous ids."""
        r = self.reads.contents
        seq = np.ctypeslib.as_array(r.seq, shape=(r.n, r.seq_pitch)).copy()
        qual = (np.ctypeslib.as_array(r.qual, shape=(r.n, r.qual_pitch)).copy()
                if r.has_quality else None)
        amb = np.nonzero(np.ctypeslib.as_array(r.ambig, shape=(r.n,)))[0].astype(np.uint32)
        return seq, qual, amb
