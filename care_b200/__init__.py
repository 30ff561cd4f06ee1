"""care_b200 -- B200 (sm_100a) read-error correction, CARE's per-anchor path.

Python view of the C ABI in include/care_b200.h (the library itself is C++
and CUDA; this module only loads it with ctypes). The shared library must be
built first (`python -m care_b200.build`); importing never falls back to any
other implementation.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcareb200.so")
CLI_PATH = os.path.join(HERE, "care-b200")


class CareError(RuntimeError):
    pass


class Options(ctypes.Structure):
    """care_b200_options; defaults of include/options.hpp:37-98 (reference)."""
    _fields_ = [
        ("kmerlength", ctypes.c_int),
        ("num_maps", ctypes.c_int),
        ("min_overlap", ctypes.c_int),
        ("max_error_rate", ctypes.c_float),
        ("min_overlap_ratio", ctypes.c_float),
        ("estimated_errorrate", ctypes.c_float),
        ("estimated_coverage", ctypes.c_float),
        ("m_coverage", ctypes.c_float),
        ("paired_filter_threshold", ctypes.c_float),
        ("new_columns_to_correct", ctypes.c_int),
        ("use_quality", ctypes.c_int),
        ("quality_bits", ctypes.c_int),
        ("exclude_ambiguous", ctypes.c_int),
        ("correct_candidates", ctypes.c_int),
        ("paired_end", ctypes.c_int),
        ("correction_type", ctypes.c_int),
        ("quality_labels", ctypes.c_int),
        ("threads", ctypes.c_int),
        ("device", ctypes.c_int),
        ("batch_size", ctypes.c_int),
        ("clf_min_coverage", ctypes.c_int),
    ]


class Results(ctypes.Structure):
    _fields_ = [
        ("first_anchor", ctypes.c_uint32),
        ("num_anchors", ctypes.c_uint32),
        ("max_length", ctypes.c_int32),
        ("anchor_status", ctypes.POINTER(ctypes.c_uint8)),
        ("anchor_num_edits", ctypes.POINTER(ctypes.c_int32)),
        ("anchor_sequences", ctypes.POINTER(ctypes.c_char)),
        ("num_candidates", ctypes.c_uint64),
        ("cand_read_ids", ctypes.POINTER(ctypes.c_uint32)),
        ("cand_anchor_ids", ctypes.POINTER(ctypes.c_uint32)),
        ("cand_shifts", ctypes.POINTER(ctypes.c_int32)),
        ("cand_use_edits", ctypes.POINTER(ctypes.c_uint8)),
        ("cand_sequences", ctypes.POINTER(ctypes.c_char)),
    ]


# every entry point of include/care_b200.h
EXPORTS = [
    "care_b200_default_options", "care_b200_create", "care_b200_destroy",
    "care_b200_last_error", "care_b200_upload_reads", "care_b200_upload_tables",
    "care_b200_build_tables", "care_b200_get_table", "care_b200_correct_range",
    "care_b200_correct_range_device", "care_b200_serialize_results",
    "care_b200_load_reads_from_files", "care_b200_load_reads_from_files_device", "care_b200_write_output", "care_b200_last_timing",
    "care_b200_last_stats", "care_b200_count_word_compares", "care_b200_load_preprocessed_reads",
    "care_b200_save_preprocessed_reads", "care_b200_load_hashtables", "care_b200_save_hashtables", "care_b200_num_reads", "care_b200_max_length", "care_b200_num_maps",
    "care_b200_result_threshold",
    "care_b200_correct_range_noalloc",
    "care_b200_set_mlp", "care_b200_collect_features", "care_b200_mlp_default_train_options",
    "care_b200_mlp_create", "care_b200_mlp_destroy", "care_b200_mlp_last_error", "care_b200_mlp_set_params",
    "care_b200_mlp_get_params", "care_b200_mlp_init", "care_b200_mlp_set_data", "care_b200_mlp_train",
    "care_b200_mlp_gradient", "care_b200_mlp_train_step", "care_b200_mlp_forward",
    "care_b200_default_tuning", "care_b200_set_tuning", "care_b200_get_tuning",
]


class Tuning(ctypes.Structure):
    """care_b200_tuning: launch mapping of a batch (results do not depend on it)."""
    _fields_ = [("msa_order", ctypes.c_int), ("msa_queue", ctypes.c_int), ("msa_warps", ctypes.c_int),
                ("align_block", ctypes.c_int), ("pair_order", ctypes.c_int), ("graph", ctypes.c_int),
                ("pair_mirror", ctypes.c_int), ("cand_set_log2", ctypes.c_int), ("align_warp", ctypes.c_int),
                ("align_classes", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}

    @classmethod
    def from_dict(cls, d):
        t = cls()
        load_library().care_b200_default_tuning(ctypes.byref(t))
        for k, v in d.items():
            if not hasattr(t, k):
                raise TypeError(f"unknown tuning field {k}")
            setattr(t, k, int(v))
        return t

MLP_FEATURES = 24
MLP_HIDDEN = 64
MLP_PARAMS = 5825
MLP_FLOATS = 5873


class Features(ctypes.Structure):
    """care_b200_features: decision-column rows of the last collect call."""
    _fields_ = [("count", ctypes.c_uint64), ("x", ctypes.POINTER(ctypes.c_float)),
                ("read_ids", ctypes.POINTER(ctypes.c_uint32)), ("meta", ctypes.POINTER(ctypes.c_uint32)),
                ("logits", ctypes.POINTER(ctypes.c_float))]


class TrainOptions(ctypes.Structure):
    """care_b200_mlp_train_options."""
    _fields_ = [("epochs", ctypes.c_int), ("batch", ctypes.c_int), ("lr", ctypes.c_double),
                ("beta1", ctypes.c_double), ("beta2", ctypes.c_double), ("eps", ctypes.c_double),
                ("seed", ctypes.c_uint64)]

NOALLOC_MAX_ANCHORS = 16384
NOALLOC_MAX_PAIRS = 1048576


class DeviceReads(ctypes.Structure):
    """care_b200_device_reads: caller-owned device read storage."""
    _fields_ = [
        ("packed", ctypes.c_void_p), ("pitch_ints", ctypes.c_size_t), ("lengths", ctypes.c_void_p),
        ("quals", ctypes.c_void_p), ("qual_pitch_ints", ctypes.c_size_t), ("ambiguous", ctypes.c_void_p),
        ("num_reads", ctypes.c_uint32), ("max_length", ctypes.c_int),
    ]


class DeviceTables(ctypes.Structure):
    """care_b200_device_tables: caller-owned device minhash tables."""
    _fields_ = [("num_maps", ctypes.c_int), ("descs", ctypes.c_void_p), ("slots", ctypes.c_void_p),
                ("values", ctypes.c_void_p), ("threshold", ctypes.c_int)]

_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libcareb200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise CareError(f"{path} is missing: build it with `python -m care_b200.build`")
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    c_ctx = ctypes.c_void_p
    lib.care_b200_default_options.argtypes = [P(Options)]
    lib.care_b200_create.argtypes = [P(Options), P(c_ctx)]
    lib.care_b200_destroy.argtypes = [c_ctx]
    lib.care_b200_last_error.argtypes = [c_ctx]
    lib.care_b200_last_error.restype = ctypes.c_char_p
    lib.care_b200_upload_reads.argtypes = [c_ctx, P(ctypes.c_uint32), ctypes.c_size_t, P(ctypes.c_int32),
                                           P(ctypes.c_uint32), ctypes.c_size_t, P(ctypes.c_uint32),
                                           ctypes.c_size_t, ctypes.c_uint32]
    lib.care_b200_upload_tables.argtypes = [c_ctx, ctypes.c_int, P(P(ctypes.c_uint64)), P(P(ctypes.c_uint32)),
                                            P(P(ctypes.c_uint32)), P(ctypes.c_size_t)]
    lib.care_b200_build_tables.argtypes = [c_ctx]
    lib.care_b200_get_table.argtypes = [c_ctx, ctypes.c_int, P(P(ctypes.c_uint64)), P(P(ctypes.c_uint32)),
                                        P(P(ctypes.c_uint32)), P(ctypes.c_size_t)]
    lib.care_b200_correct_range.argtypes = [c_ctx, ctypes.c_uint32, ctypes.c_uint32, P(Results)]
    lib.care_b200_correct_range_device.argtypes = [c_ctx, ctypes.c_uint32, ctypes.c_uint32]
    lib.care_b200_serialize_results.argtypes = [c_ctx, P(Results), P(ctypes.c_uint8), ctypes.c_size_t,
                                                P(ctypes.c_size_t)]
    lib.care_b200_load_reads_from_files.argtypes = [c_ctx, P(ctypes.c_char_p), ctypes.c_int]
    lib.care_b200_load_reads_from_files_device.argtypes = [c_ctx, P(ctypes.c_char_p), ctypes.c_int]
    lib.care_b200_write_output.argtypes = [c_ctx, ctypes.c_char_p]
    lib.care_b200_last_timing.argtypes = [c_ctx, P(ctypes.c_float), P(ctypes.c_float), ctypes.c_int]
    lib.care_b200_last_stats.argtypes = [c_ctx, P(ctypes.c_uint64), ctypes.c_int]
    lib.care_b200_count_word_compares.argtypes = [c_ctx, ctypes.c_int]
    lib.care_b200_load_preprocessed_reads.argtypes = [c_ctx, ctypes.c_char_p]
    lib.care_b200_save_preprocessed_reads.argtypes = [c_ctx, ctypes.c_char_p]
    lib.care_b200_load_hashtables.argtypes = [c_ctx, ctypes.c_char_p]
    lib.care_b200_save_hashtables.argtypes = [c_ctx, ctypes.c_char_p]
    lib.care_b200_correct_range_noalloc.argtypes = [P(Options), P(DeviceReads), P(DeviceTables), ctypes.c_uint32,
                                                     ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                                     ctypes.c_void_p, ctypes.c_void_p]
    c_mlp = ctypes.c_void_p
    fp = P(ctypes.c_float)
    lib.care_b200_set_mlp.argtypes = [c_ctx, fp]
    lib.care_b200_collect_features.argtypes = [c_ctx, ctypes.c_uint32, ctypes.c_uint32, P(Results), P(Features)]
    lib.care_b200_mlp_default_train_options.argtypes = [P(TrainOptions)]
    lib.care_b200_mlp_default_train_options.restype = None
    lib.care_b200_mlp_create.argtypes = [ctypes.c_int, P(c_mlp)]
    lib.care_b200_mlp_destroy.argtypes = [c_mlp]
    lib.care_b200_mlp_last_error.argtypes = [c_mlp]
    lib.care_b200_mlp_last_error.restype = ctypes.c_char_p
    lib.care_b200_mlp_set_params.argtypes = [c_mlp, fp]
    lib.care_b200_mlp_get_params.argtypes = [c_mlp, fp]
    lib.care_b200_mlp_init.argtypes = [c_mlp, ctypes.c_uint64]
    lib.care_b200_mlp_set_data.argtypes = [c_mlp, fp, fp, fp, ctypes.c_uint64, ctypes.c_int]
    lib.care_b200_mlp_train.argtypes = [c_mlp, P(TrainOptions), fp, ctypes.c_uint64, P(ctypes.c_uint64)]
    lib.care_b200_mlp_gradient.argtypes = [c_mlp, fp, fp, fp, ctypes.c_uint64, fp, fp]
    lib.care_b200_mlp_train_step.argtypes = [c_mlp, fp, fp, fp, ctypes.c_uint64, P(TrainOptions), fp]
    lib.care_b200_mlp_forward.argtypes = [c_mlp, fp, ctypes.c_uint64, fp]
    lib.care_b200_default_tuning.argtypes = [P(Tuning)]
    lib.care_b200_set_tuning.argtypes = [c_ctx, P(Tuning)]
    lib.care_b200_get_tuning.argtypes = [c_ctx, P(Tuning)]
    lib.care_b200_num_reads.argtypes = [c_ctx]
    lib.care_b200_num_reads.restype = ctypes.c_uint32
    lib.care_b200_max_length.argtypes = [c_ctx]
    lib.care_b200_num_maps.argtypes = [c_ctx]
    lib.care_b200_result_threshold.argtypes = [c_ctx]
    _lib = lib
    return lib


def default_options(**kw) -> Options:
    lib = load_library()
    o = Options()
    lib.care_b200_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


@dataclasses.dataclass
class CorrectionResults:
    first: int
    status: np.ndarray            # uint8 per anchor: 1 corrected, 2 hq, 4 edit list
    num_edits: np.ndarray
    sequences: np.ndarray         # (num_anchors, max_len) uint8 ASCII
    cand_read_ids: np.ndarray
    cand_anchor_ids: np.ndarray
    cand_shifts: np.ndarray
    cand_use_edits: np.ndarray
    cand_sequences: np.ndarray    # (num_candidates, max_len)


class Corrector:
    """One device context: read storage + minhash tables + correction."""

    def __init__(self, options: Options | None = None, **kw):
        self.lib = load_library()
        self.opts = options if options is not None else default_options(**kw)
        self._ctx = ctypes.c_void_p()
        rc = self.lib.care_b200_create(ctypes.byref(self.opts), ctypes.byref(self._ctx))
        if rc != 0:
            msg = self.lib.care_b200_last_error(self._ctx) if self._ctx else b""
            raise CareError(f"care_b200_create failed ({rc}) {msg!r}")
        self._keep = []

    def close(self):
        if self._ctx:
            self.lib.care_b200_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise CareError(f"{what} failed ({rc}): {self.lib.care_b200_last_error(self._ctx).decode()}")

    # -- read storage / tables -------------------------------------------------
    def upload_reads(self, packed: np.ndarray, lengths: np.ndarray, quals: np.ndarray | None = None,
                     ambiguous: np.ndarray | None = None):
        packed = np.ascontiguousarray(packed, dtype=np.uint32)
        lengths = np.ascontiguousarray(lengths, dtype=np.int32)
        amb = np.ascontiguousarray(ambiguous if ambiguous is not None else np.zeros(0, np.uint32), dtype=np.uint32)
        qp = None
        qpitch = 0
        if quals is not None:
            quals = np.ascontiguousarray(quals, dtype=np.uint32)
            qp = _ptr(quals, ctypes.c_uint32)
            qpitch = quals.shape[1]
        self._check(self.lib.care_b200_upload_reads(
            self._ctx, _ptr(packed, ctypes.c_uint32), packed.shape[1], _ptr(lengths, ctypes.c_int32),
            qp, qpitch, _ptr(amb, ctypes.c_uint32), amb.shape[0], packed.shape[0]), "upload_reads")

    def load_files(self, files: Sequence[str], device: bool = False):
        """STEP1 from FASTQ/FASTA files; device=True parses and encodes on the
        GPU (strict 4-line FASTQ / 2-line FASTA; CareError otherwise)."""
        arr = (ctypes.c_char_p * len(files))(*[f.encode() for f in files])
        if device:
            self._check(self.lib.care_b200_load_reads_from_files_device(self._ctx, arr, len(files)),
                        "load_reads_from_files_device")
        else:
            self._check(self.lib.care_b200_load_reads_from_files(self._ctx, arr, len(files)), "load_reads_from_files")

    def load_preprocessed_reads(self, path: str):
        """Read storage from a file written by care-cpu --save-preprocessedreads-to
        (or by save_preprocessed_reads), in place of parsing FASTQ."""
        self._check(self.lib.care_b200_load_preprocessed_reads(self._ctx, path.encode()), "load_preprocessed_reads")

    def save_preprocessed_reads(self, path: str):
        """The uploaded read storage in care-cpu's binary read-storage layout."""
        self._check(self.lib.care_b200_save_preprocessed_reads(self._ctx, path.encode()), "save_preprocessed_reads")

    def load_hashtables(self, path: str):
        """Tables from a file written by care-cpu --save-hashtables-to (or by
        save_hashtables), in place of build_tables."""
        self._check(self.lib.care_b200_load_hashtables(self._ctx, path.encode()), "load_hashtables")

    def save_hashtables(self, path: str):
        """The tables in care-cpu's minhash-table layout."""
        self._check(self.lib.care_b200_save_hashtables(self._ctx, path.encode()), "save_hashtables")

    def build_tables(self):
        self._check(self.lib.care_b200_build_tables(self._ctx), "build_tables")

    def upload_tables(self, tables: Sequence[tuple[np.ndarray, np.ndarray, np.ndarray]]):
        m = len(tables)
        ks = [np.ascontiguousarray(t[0], dtype=np.uint64) for t in tables]
        os_ = [np.ascontiguousarray(t[1], dtype=np.uint32) for t in tables]
        vs = [np.ascontiguousarray(t[2], dtype=np.uint32) for t in tables]
        P = ctypes.POINTER
        kp = (P(ctypes.c_uint64) * m)(*[_ptr(k, ctypes.c_uint64) for k in ks])
        op = (P(ctypes.c_uint32) * m)(*[_ptr(o, ctypes.c_uint32) for o in os_])
        vp = (P(ctypes.c_uint32) * m)(*[_ptr(v, ctypes.c_uint32) for v in vs])
        nk = (ctypes.c_size_t * m)(*[k.shape[0] for k in ks])
        self._check(self.lib.care_b200_upload_tables(self._ctx, m, kp, op, vp, nk), "upload_tables")

    def get_table(self, m: int):
        P = ctypes.POINTER
        k = P(ctypes.c_uint64)()
        o = P(ctypes.c_uint32)()
        v = P(ctypes.c_uint32)()
        n = ctypes.c_size_t()
        self._check(self.lib.care_b200_get_table(self._ctx, m, ctypes.byref(k), ctypes.byref(o),
                                                 ctypes.byref(v), ctypes.byref(n)), "get_table")
        nk = n.value
        keys = np.ctypeslib.as_array(k, shape=(nk,)).copy() if nk else np.zeros(0, np.uint64)
        offs = np.ctypeslib.as_array(o, shape=(nk + 1,)).copy()
        nv = int(offs[-1]) if nk else 0
        vals = np.ctypeslib.as_array(v, shape=(nv,)).copy() if nv else np.zeros(0, np.uint32)
        return keys, offs, vals

    @property
    def num_reads(self) -> int:
        return int(self.lib.care_b200_num_reads(self._ctx))

    @property
    def max_length(self) -> int:
        return int(self.lib.care_b200_max_length(self._ctx))

    @property
    def num_maps(self) -> int:
        return int(self.lib.care_b200_num_maps(self._ctx))

    @property
    def result_threshold(self) -> int:
        """Per-map result threshold of the tables (buckets with more ids are dropped)."""
        return int(self.lib.care_b200_result_threshold(self._ctx))

    # -- correction ------------------------------------------------------------
    def correct_range_raw(self, first: int, count: int) -> Results:
        res = Results()
        self._check(self.lib.care_b200_correct_range(self._ctx, first, count, ctypes.byref(res)), "correct_range")
        return res

    def correct_range(self, first: int = 0, count: int | None = None) -> CorrectionResults:
        if count is None:
            count = self.num_reads - first
        res = self.correct_range_raw(first, count)
        L = res.max_length
        na = res.num_anchors
        nc = int(res.num_candidates)

        def arr(p, shape, dt):
            if int(np.prod(shape)) == 0:
                return np.zeros(shape, dt)
            return np.ctypeslib.as_array(p, shape=shape).view(dt).copy()

        return CorrectionResults(
            first=res.first_anchor,
            status=arr(res.anchor_status, (na,), np.uint8),
            num_edits=arr(res.anchor_num_edits, (na,), np.int32),
            sequences=arr(ctypes.cast(res.anchor_sequences, ctypes.POINTER(ctypes.c_uint8)), (na, L), np.uint8),
            cand_read_ids=arr(res.cand_read_ids, (nc,), np.uint32),
            cand_anchor_ids=arr(res.cand_anchor_ids, (nc,), np.uint32),
            cand_shifts=arr(res.cand_shifts, (nc,), np.int32),
            cand_use_edits=arr(res.cand_use_edits, (nc,), np.uint8),
            cand_sequences=arr(ctypes.cast(res.cand_sequences, ctypes.POINTER(ctypes.c_uint8)), (nc, L), np.uint8),
        )

    def correct_range_device(self, first: int = 0, count: int | None = None):
        if count is None:
            count = self.num_reads - first
        self._check(self.lib.care_b200_correct_range_device(self._ctx, first, count), "correct_range_device")

    def serialize(self, res: Results) -> bytes:
        need = ctypes.c_size_t()
        self._check(self.lib.care_b200_serialize_results(self._ctx, ctypes.byref(res), None, 0,
                                                         ctypes.byref(need)), "serialize")
        buf = np.zeros(need.value, np.uint8)
        self._check(self.lib.care_b200_serialize_results(self._ctx, ctypes.byref(res), _ptr(buf, ctypes.c_uint8),
                                                         need.value, ctypes.byref(need)), "serialize")
        return buf.tobytes()

    def write_output(self, path: str):
        self._check(self.lib.care_b200_write_output(self._ctx, path.encode()), "write_output")

    # -- launch mapping --------------------------------------------------------
    @property
    def tuning(self) -> dict:
        t = Tuning()
        self._check(self.lib.care_b200_get_tuning(self._ctx, ctypes.byref(t)), "get_tuning")
        return t.as_dict()

    @tuning.setter
    def tuning(self, d: dict):
        t = Tuning.from_dict(d)
        self._check(self.lib.care_b200_set_tuning(self._ctx, ctypes.byref(t)), "set_tuning")

    # -- learned decision ------------------------------------------------------
    def set_mlp(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.shape != (MLP_FLOATS,):
            raise ValueError(f"expected {MLP_FLOATS} parameters")
        self._check(self.lib.care_b200_set_mlp(self._ctx, _ptr(p, ctypes.c_float)), "set_mlp")

    def collect_features(self, first: int = 0, count: int | None = None):
        """Correction of the range plus its decision-column rows: dict of
        read_id, pos, orig, cons (2-bit codes), x (n, 24) and logit (None
        under the classic rule)."""
        if count is None:
            count = self.num_reads - first
        res = Results()
        f = Features()
        self._check(self.lib.care_b200_collect_features(self._ctx, first, count, ctypes.byref(res),
                                                        ctypes.byref(f)), "collect_features")
        n = int(f.count)
        if n == 0:
            return {"read_id": np.zeros(0, np.uint32), "pos": np.zeros(0, np.int32), "orig": np.zeros(0, np.uint8),
                    "cons": np.zeros(0, np.uint8), "x": np.zeros((0, MLP_FEATURES), np.float32),
                    "logit": None if not f.logits else np.zeros(0, np.float32)}
        meta = np.ctypeslib.as_array(f.meta, shape=(n,)).copy()
        return {
            "read_id": np.ctypeslib.as_array(f.read_ids, shape=(n,)).copy(),
            "pos": (meta & 0xFFFF).astype(np.int32),
            "orig": ((meta >> 16) & 3).astype(np.uint8),
            "cons": ((meta >> 18) & 3).astype(np.uint8),
            "x": np.ctypeslib.as_array(f.x, shape=(n, MLP_FEATURES)).copy(),
            "logit": np.ctypeslib.as_array(f.logits, shape=(n,)).copy() if f.logits else None,
        }

    def last_stats(self):
        st = (ctypes.c_uint64 * 11)()
        self._check(self.lib.care_b200_last_stats(self._ctx, st, 11), "last_stats")
        return {"anchors": st[0], "pairs": st[1], "candidate_corrections": st[2], "word_compares": st[3],
                "msa_elements": st[4], "batches": st[5], "launches": st[6], "spilled_anchors": st[7],
                "word_compares_run": st[8], "msa_rebuild_elements": st[9], "msa_rebuilt_anchors": st[10]}

    def count_word_compares(self, on: bool = True):
        """Run the alignment's statistics form in the following calls: it also
        counts the word compares actually run (last_stats()["word_compares_run"])."""
        self._check(self.lib.care_b200_count_word_compares(self._ctx, int(bool(on))), "count_word_compares")

    def last_timing(self):
        """(total ms, [candidates, alignment, MSA, classifier] ms) of the last call."""
        t = ctypes.c_float()
        st = (ctypes.c_float * 4)()
        self._check(self.lib.care_b200_last_timing(self._ctx, ctypes.byref(t), st, 4), "last_timing")
        return t.value, list(st)

    def signatures_ms(self) -> float:
        """Device ms of the last minhash-signature pass over the read storage
        (once per uploaded or loaded storage; the correction calls reuse it)."""
        t = ctypes.c_float()
        st = (ctypes.c_float * 5)()
        self._check(self.lib.care_b200_last_timing(self._ctx, ctypes.byref(t), st, 5), "last_timing")
        return float(st[4])


def train_options(**kw) -> TrainOptions:
    o = TrainOptions()
    load_library().care_b200_mlp_default_train_options(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown training option {k}")
        setattr(o, k, v)
    return o


class Mlp:
    """The decision network on one device: parameters, resident training
    rows, Adam training (one CUDA graph per run), gradients and logits."""

    def __init__(self, device: int = 0, seed: int = 1):
        self.lib = load_library()
        self._h = ctypes.c_void_p()
        rc = self.lib.care_b200_mlp_create(device, ctypes.byref(self._h))
        if rc != 0:
            raise CareError(f"care_b200_mlp_create failed ({rc})")
        if seed != 1:
            self._check(self.lib.care_b200_mlp_init(self._h, seed), "mlp_init")

    def close(self):
        if self._h:
            self.lib.care_b200_mlp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise CareError(f"{what} failed ({rc}): {self.lib.care_b200_mlp_last_error(self._h).decode()}")

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(MLP_FLOATS, np.float32)
        self._check(self.lib.care_b200_mlp_get_params(self._h, _ptr(p, ctypes.c_float)), "mlp_get_params")
        return p

    @params.setter
    def params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (MLP_FLOATS,):
            raise ValueError(f"expected {MLP_FLOATS} parameters")
        self._check(self.lib.care_b200_mlp_set_params(self._h, _ptr(p, ctypes.c_float)), "mlp_set_params")

    @staticmethod
    def _rows(x, y=None, w=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        if x.ndim != 2 or x.shape[1] != MLP_FEATURES:
            raise ValueError("rows must be (n, 24)")
        out = [x]
        for v in (y, w):
            if v is not None:
                v = np.ascontiguousarray(v, dtype=np.float32)
                if v.shape != (x.shape[0],):
                    raise ValueError("one label and one weight per row")
            out.append(v)
        return out

    @staticmethod
    def _fp(a):
        return None if a is None else _ptr(a, ctypes.c_float)

    def set_data(self, x, y, weights=None, normalise: bool = True):
        x, y, w = self._rows(x, y, weights)
        self._check(self.lib.care_b200_mlp_set_data(self._h, _ptr(x, ctypes.c_float), _ptr(y, ctypes.c_float),
                                                    self._fp(w), x.shape[0], 1 if normalise else 0), "mlp_set_data")

    def train(self, **kw) -> np.ndarray:
        o = train_options(**kw)
        n = ctypes.c_uint64()
        cap = 1 << 20
        losses = np.zeros(cap, np.float32)
        self._check(self.lib.care_b200_mlp_train(self._h, ctypes.byref(o), _ptr(losses, ctypes.c_float), cap,
                                                 ctypes.byref(n)), "mlp_train")
        return losses[:min(n.value, cap)].copy()

    def gradient(self, x, y, weights=None):
        x, y, w = self._rows(x, y, weights)
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = ctypes.c_float()
        self._check(self.lib.care_b200_mlp_gradient(self._h, _ptr(x, ctypes.c_float), _ptr(y, ctypes.c_float),
                                                    self._fp(w), x.shape[0], _ptr(g, ctypes.c_float),
                                                    ctypes.byref(loss)), "mlp_gradient")
        return float(loss.value), g

    def train_step(self, x, y, weights=None, **kw) -> float:
        x, y, w = self._rows(x, y, weights)
        o = train_options(**kw)
        loss = ctypes.c_float()
        self._check(self.lib.care_b200_mlp_train_step(self._h, _ptr(x, ctypes.c_float), _ptr(y, ctypes.c_float),
                                                      self._fp(w), x.shape[0], ctypes.byref(o), ctypes.byref(loss)),
                    "mlp_train_step")
        return float(loss.value)

    def forward(self, x) -> np.ndarray:
        x = self._rows(x)[0]
        out = np.zeros(x.shape[0], np.float32)
        self._check(self.lib.care_b200_mlp_forward(self._h, _ptr(x, ctypes.c_float), x.shape[0],
                                                   _ptr(out, ctypes.c_float)), "mlp_forward")
        return out


def fmix64(x: np.ndarray) -> np.ndarray:
    """MurmurHash3's 64-bit finalizer over a uint64 array."""
    x = x.copy()
    with np.errstate(over="ignore"):
        x ^= x >> np.uint64(33)
        x *= np.uint64(0xff51afd7ed558ccd)
        x ^= x >> np.uint64(33)
        x *= np.uint64(0xc4ceb9fe1a85ec53)
        x ^= x >> np.uint64(33)
    return x


def table_device_layout(tables):
    """Host arrays in the device table layout of care_b200_device_tables:
    (descs bytes, slots bytes, values uint32) from per-map (keys, offsets,
    values). Slots: power-of-two capacity >= 2 keys, linear probing from the
    MurmurHash3 fmix64 of the key."""
    descs, slots, vals = [], [], []
    slot_base = value_base = 0
    sdt = np.dtype([("key", "<u8"), ("offset", "<u4"), ("count", "<u4")])
    ddt = np.dtype([("slot_base", "<u8"), ("value_base", "<u8"), ("mask", "<u4"), ("pad", "<u4")])
    for keys, offs, values in tables:
        n = keys.shape[0]
        cap = 16
        while cap < 2 * n:
            cap <<= 1
        s = np.zeros(cap, sdt)
        h = fmix64(keys.astype(np.uint64)) & np.uint64(cap - 1)
        for i in range(n):
            pos = int(h[i])
            while s["count"][pos] != 0:
                pos = (pos + 1) & (cap - 1)
            s[pos] = (keys[i], offs[i], offs[i + 1] - offs[i])
        d = np.zeros(1, ddt)
        d[0] = (slot_base, value_base, cap - 1, 0)
        descs.append(d)
        slots.append(s)
        vals.append(values.astype(np.uint32))
        slot_base += cap
        value_base += values.shape[0]
    return (np.concatenate(descs).tobytes(), np.concatenate(slots).tobytes(),
            np.concatenate(vals) if vals else np.zeros(0, np.uint32))


def correct_range_noalloc(options: Options, reads: DeviceReads, tables: DeviceTables, first: int, count: int,
                          status_ptr: int, num_edits_ptr: int, sequences_ptr: int, stream: int = 0) -> None:
    """care_b200_correct_range_noalloc: anchor correction into caller-owned
    device buffers, for callers that cannot allocate device memory; the
    library allocates nothing here either."""
    lib = load_library()
    rc = lib.care_b200_correct_range_noalloc(ctypes.byref(options), ctypes.byref(reads), ctypes.byref(tables),
                                             first, count, status_ptr, num_edits_ptr, sequences_ptr, stream)
    if rc != 0:
        raise CareError(f"care_b200_correct_range_noalloc failed ({rc})")


def encode_reads(seqs: np.ndarray, lengths: np.ndarray):
    """ASCII reads (n, Lmax) -> packed 2-bit rows (n, ceil(Lmax/16)) uint32, MSB-first,
    zero padded; non-ACGT characters become A (caller handles N rotation)."""
    n, Lmax = seqs.shape
    code = np.zeros((n, Lmax), np.uint32)
    code[seqs == ord("C")] = 1
    code[seqs == ord("G")] = 2
    code[seqs == ord("T")] = 3
    valid = np.arange(Lmax)[None, :] < lengths[:, None]
    code[~valid] = 0
    pitch = (Lmax + 15) // 16
    padded = np.zeros((n, pitch * 16), np.uint32)
    padded[:, :Lmax] = code
    padded = padded.reshape(n, pitch, 16)
    shifts = (30 - 2 * np.arange(16, dtype=np.uint32))
    return (padded << shifts).sum(axis=2, dtype=np.uint64).astype(np.uint32)


def options_from_args(args: str | Sequence[str], **kw) -> Options:
    """care-cpu command-line options (src/options.cpp:54-383) -> Options."""
    toks = args.split() if isinstance(args, str) else list(args)
    o = default_options()
    flags = {"-q": "use_quality", "--useQualityScores": "use_quality",
             "--excludeAmbiguous": "exclude_ambiguous", "--candidateCorrection": "correct_candidates",
             "--correctionQualityLabels": "quality_labels"}
    valued = {"-c": ("estimated_coverage", float), "--coverage": ("estimated_coverage", float),
              "-k": ("kmerlength", int), "--kmerlength": ("kmerlength", int),
              "-h": ("num_maps", int), "--hashmaps": ("num_maps", int),
              "-t": ("threads", int), "--threads": ("threads", int),
              "--qualityScoreBits": ("quality_bits", int),
              "--minalignmentoverlap": ("min_overlap", int),
              "--maxmismatchratio": ("max_error_rate", float),
              "--minalignmentoverlapratio": ("min_overlap_ratio", float),
              "--errorfactortuning": ("estimated_errorrate", float),
              "--coveragefactortuning": ("m_coverage", float),
              "--pairedFilterThreshold": ("paired_filter_threshold", float),
              "--candidateCorrectionNewColumns": ("new_columns_to_correct", int),
              "--batchsize": ("batch_size", int), "-g": ("device", int), "--gpu": ("device", int),
              "--correctionType": ("correction_type", int)}
    i = 0
    while i < len(toks):
        t = toks[i]
        if t in flags:
            setattr(o, flags[t], 1)
        elif t == "--pairmode":
            o.paired_end = 1 if toks[i + 1] in ("PE", "pe") else 0
            i += 1
        elif t in valued:
            name, typ = valued[t]
            setattr(o, name, typ(toks[i + 1]))
            i += 1
        else:
            raise ValueError(f"unsupported option {t}")
        i += 1
    for k, v in kw.items():
        setattr(o, k, v)
    return o
