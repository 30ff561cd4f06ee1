"""care-cpu's binary read-storage and minhash-table files
(--save-preprocessedreads-to, --save-hashtables-to), without a GPU: the files
the reference wrote for seeded read sets (tests/golden/make_preprocessed.py)
hold exactly the read storage this library's own preprocessing builds from the
same FASTQ and the tables the oracle builds, and the writers reproduce the
reference's bytes (the ambiguous ids, which the reference writes in the order
of a hash set, as a set)."""
import ctypes
import gzip
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
SRC = [os.path.join(ROOT, "tests", "harness", "readfile_harness.cpp"),
       os.path.join(ROOT, "care_b200", "csrc", "readfile.cpp"),
       os.path.join(ROOT, "care_b200", "csrc", "hostio.cpp")]
DEPS = SRC + [os.path.join(ROOT, "care_b200", "csrc", f) for f in ("readfile.hpp", "hostio.hpp")]
OUT = os.path.join(ROOT, "tests", "_build", "libreadfile.so")
CASES = {"pre_pe": (True, 2), "pre_un": (False, 8)}      # paired end, quality bits
U64 = ctypes.c_ulonglong


def harness():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    if not os.path.exists(OUT) or any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in DEPS):
        tmp = f"{OUT}.{os.getpid()}.tmp"
        subprocess.run(["g++", "-shared", "-fPIC", "-O2", "-std=c++17", "-o", tmp] + SRC + ["-lpthread"],
                       check=True, capture_output=True)
        os.replace(tmp, OUT)
    lib = ctypes.CDLL(OUT)
    lib.rf_load.restype = ctypes.c_void_p
    lib.rf_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(U64), ctypes.c_char_p, ctypes.c_int]
    lib.rf_parse.restype = ctypes.c_void_p
    lib.rf_parse.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(U64), ctypes.c_char_p,
                             ctypes.c_int]
    for f in (lib.rf_arrays, lib.rf_parse_arrays):
        f.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4
    lib.rf_free.argtypes = lib.rf_parse_free.argtypes = [ctypes.c_void_p]
    lib.rf_parse_digest.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                                    ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.c_char_p, ctypes.c_int]
    lib.rt_load.restype = ctypes.c_void_p
    lib.rt_load.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(U64), ctypes.c_char_p, ctypes.c_int]
    lib.rt_map_size.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(U64), ctypes.POINTER(U64)]
    lib.rt_map.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.rt_write.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
    lib.rt_free.argtypes = [ctypes.c_void_p]
    lib.rf_write.argtypes = [ctypes.c_char_p, U64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, U64, U64,
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, U64, ctypes.c_char_p,
                             ctypes.c_int]
    return lib


H = harness()


def unpack(tmp, name):
    out = {}
    for ext in ("fq", "bin"):
        p = os.path.join(tmp, f"{name}.{ext}")
        with open(p, "wb") as f:
            f.write(gzip.decompress(open(os.path.join(GOLD, f"{name}.{ext}.gz"), "rb").read()))
        out[ext] = p
    return out


def storage(handle_fn, arrays_fn, free_fn, *args):
    info = (U64 * 8)()
    err = ctypes.create_string_buffer(256)
    h = handle_fn(*args, info, err, 256)
    assert h, err.value.decode()
    n, mn, mx, hasq, qbits, sp, qp, na = list(info)
    seq = np.zeros(n * sp, np.uint32)
    ln = np.zeros(n, np.int32)
    qual = np.zeros(max(n * qp, 1), np.uint32)
    amb = np.zeros(max(na, 1), np.uint32)
    arrays_fn(h, seq.ctypes.data, ln.ctypes.data, qual.ctypes.data, amb.ctypes.data)
    free_fn(h)
    return dict(n=n, min=mn, max=mx, hasq=hasq, qbits=qbits, sp=sp, qp=qp, seq=seq, len=ln,
                qual=qual[:n * qp], amb=amb[:na])


def load(path):
    return storage(H.rf_load, H.rf_arrays, H.rf_free, path.encode())


def section_end(path):
    """Offset where the ambiguous-id section starts."""
    b = open(path, "rb").read()
    lb, sb, qb, ab = struct.unpack_from("<4Q", b, 21)
    return 53 + lb + sb + qb, b


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_file_holds_our_preprocessing(tmp_path, name):
    pe, qbits = CASES[name]
    p = unpack(str(tmp_path), name)
    ref = load(p["bin"])
    ours = storage(H.rf_parse, H.rf_parse_arrays, H.rf_parse_free, p["fq"].encode(), int(pe), qbits)
    for k in ("n", "min", "max", "sp", "qp", "qbits"):
        assert ref[k] == ours[k], k
    assert ref["hasq"] == 1
    assert np.array_equal(ref["len"], ours["len"])
    assert np.array_equal(ref["seq"], ours["seq"])
    assert np.array_equal(ref["qual"], ours["qual"])
    assert sorted(ref["amb"].tolist()) == sorted(ours["amb"].tolist())
    if name == "pre_pe":
        assert len(ref["amb"]) > 0                   # reads with N bases
    else:
        assert ref["min"] < ref["max"]               # bit-packed lengths


@pytest.mark.parametrize("name", sorted(CASES))
def test_writer_reproduces_reference_bytes(tmp_path, name):
    p = unpack(str(tmp_path), name)
    ref = load(p["bin"])
    amb = np.sort(ref["amb"])
    out = str(tmp_path / "ours.bin")
    err = ctypes.create_string_buffer(256)
    rc = H.rf_write(out.encode(), ref["n"], ref["min"], ref["max"], ref["hasq"], ref["qbits"], ref["sp"], ref["qp"],
                    ref["seq"].ctypes.data, ref["len"].ctypes.data, ref["qual"].ctypes.data, amb.ctypes.data,
                    len(amb), err, 256)
    assert rc == 0, err.value.decode()
    end_ref, b_ref = section_end(p["bin"])
    end_out, b_out = section_end(out)
    assert end_ref == end_out and b_ref[:end_ref] == b_out[:end_out]
    assert len(b_ref) == len(b_out)
    ids = lambda b, e: sorted(struct.unpack_from(f"<{struct.unpack_from('<Q', b, e)[0]}I", b, e + 8))
    assert ids(b_ref, end_ref) == ids(b_out, end_out)
    back = load(out)
    for k in ("seq", "len", "qual"):
        assert np.array_equal(back[k], ref[k])


def test_truncated_file_is_rejected(tmp_path):
    p = unpack(str(tmp_path), "pre_un")
    b = open(p["bin"], "rb").read()
    for cut in (10, 60, len(b) // 2, len(b) - 3):
        q = tmp_path / f"cut{cut}.bin"
        q.write_bytes(b[:cut])
        info = (U64 * 8)()
        err = ctypes.create_string_buffer(256)
        assert not H.rf_load(str(q).encode(), info, err, 256)
        assert b"truncated" in err.value or b"inconsistent" in err.value


def load_tables(path, max_maps=64):
    info = (U64 * 4)()
    err = ctypes.create_string_buffer(256)
    h = H.rt_load(path.encode(), max_maps, info, err, 256)
    assert h, err.value.decode()
    maps = []
    for m in range(info[2]):
        nk, nv = U64(), U64()
        H.rt_map_size(h, m, ctypes.byref(nk), ctypes.byref(nv))
        keys = np.zeros(max(nk.value, 1), np.uint64)
        offs = np.zeros(nk.value + 1, np.uint32)
        vals = np.zeros(max(nv.value, 1), np.uint32)
        H.rt_map(h, m, keys.ctypes.data, offs.ctypes.data, vals.ctypes.data)
        maps.append((keys[:nk.value], offs, vals[:nv.value]))
    return h, list(info), maps


def test_reference_tables_equal_the_oracle(tmp_path):
    import _oracle
    p = unpack(str(tmp_path), "pre_pe")
    tab = tmp_path / "pre_pe_h4.tables"
    tab.write_bytes(gzip.decompress(open(os.path.join(GOLD, "pre_pe_h4.tables.gz"), "rb").read()))
    h, info, maps = load_tables(str(tab))
    H.rt_free(h)
    k, thr, nmaps, _ = info
    assert (k, thr, nmaps) == (20, 125, 4)
    run = _oracle.OracleRun([p["fq"]], _oracle.opts_from_args("-c 50 -k 20 -h 4 -q --qualityScoreBits 2 --pairmode PE"),
                            threads=4)
    try:
        for m in range(4):
            ok, oo, ov = run.table(m)
            rk, ro, rv = maps[m]
            assert len(rk) > 50
            assert np.array_equal(rk, ok) and np.array_equal(ro, oo) and np.array_equal(rv, ov), m
    finally:
        run.close()


def test_table_writer_reproduces_reference_bytes(tmp_path):
    ref = tmp_path / "ref.tables"
    ref.write_bytes(gzip.decompress(open(os.path.join(GOLD, "pre_pe_h4.tables.gz"), "rb").read()))
    h, info, maps = load_tables(str(ref))
    out = tmp_path / "ours.tables"
    err = ctypes.create_string_buffer(256)
    assert H.rt_write(h, str(out).encode(), err, 256) == 0, err.value.decode()
    H.rt_free(h)
    assert out.read_bytes() == ref.read_bytes()
    h2, _, _ = load_tables(str(ref), max_maps=2)              # the reference loads min(file, requested) maps
    nk = U64(); nv = U64()
    H.rt_map_size(h2, 1, ctypes.byref(nk), ctypes.byref(nv))
    assert nk.value == len(maps[1][0])
    H.rt_free(h2)


def digest(f0, f1=None, pe=False, qbits=2, threads=1):
    d, n = U64(), U64()
    err = ctypes.create_string_buffer(256)
    rc = H.rf_parse_digest(f0.encode(), f1.encode() if f1 else None, int(pe), qbits, threads, ctypes.byref(d),
                           ctypes.byref(n), err, 256)
    assert rc == 0, err.value.decode()
    return d.value, n.value


def _records(rng, n, L=120, at_quality=False, fasta=False, crlf=False, n_bases=False):
    eol = "\r\n" if crlf else "\n"
    out = []
    for i in range(n):
        s = "".join(rng.choice("ACGT") for _ in range(L))
        if n_bases and i % 7 == 0:
            s = s[:5] + "N" + s[6:]
        if fasta:
            out.append(f">r{i}{eol}{s}{eol}")
        else:
            q = "".join(rng.choice("#+5?@AEI") for _ in range(L))
            if at_quality:
                q = "@" + q[1:]                        # quality lines that begin like a header
            out.append(f"@r{i} x{eol}{s}{eol}+{eol}{q}{eol}")
    return out


@pytest.mark.parametrize("kind", ["fastq", "at_quality", "fasta", "crlf", "pe2", "se2"])
def test_parallel_scan_equals_sequential(tmp_path, kind):
    """The threaded record scan gives exactly the single-threaded result."""
    import random
    rng = random.Random(hash(kind) & 0xffff)
    recs = _records(rng, 12000, at_quality=(kind == "at_quality"), fasta=(kind == "fasta"),
                    crlf=(kind == "crlf"), n_bases=True)
    f0 = tmp_path / "a.fq"
    f1 = None
    if kind in ("pe2", "se2"):
        f1 = tmp_path / "b.fq"
        f0.write_text("".join(recs[0::2]))
        f1.write_text("".join(recs[1::2] + (recs[-1:] if kind == "se2" else [])))
    else:
        f0.write_text("".join(recs))
    pe = kind in ("pe2", "fastq", "at_quality", "crlf")
    args = (str(f0), str(f1) if f1 else None, pe)
    ref = digest(*args, threads=1)
    assert ref[1] > 0
    for t in (2, 3, 8, 16):
        assert digest(*args, threads=t) == ref, t


def test_parallel_scan_falls_back_on_irregular_files(tmp_path):
    """A file whose records do not chain at the segment starts (here: records
    with a missing quality line) is scanned sequentially, with the same result."""
    import random
    rng = random.Random(5)
    recs = _records(rng, 8000)
    broken = [r if i % 997 else "@bad{}\nACGT\n".format(i) for i, r in enumerate(recs)]
    f = tmp_path / "irregular.fq"
    f.write_text("".join(broken))
    ref = digest(str(f), threads=1)
    assert digest(str(f), threads=8) == ref


def test_sizes_beyond_the_file_are_rejected(tmp_path):
    """Counts in a damaged header that the file cannot hold are rejected
    before anything is allocated."""
    p = unpack(str(tmp_path), "pre_un")
    b = bytearray(open(p["bin"], "rb").read())
    for off, val in ((0, 2 ** 32 - 1), (0, 10 ** 9)):                 # read count
        bad = bytearray(b)
        struct.pack_into("<Q", bad, off, val)
        q = tmp_path / "bad.bin"
        q.write_bytes(bytes(bad))
        info = (U64 * 8)()
        err = ctypes.create_string_buffer(256)
        assert not H.rf_load(str(q).encode(), info, err, 256)
    t = bytearray(gzip.decompress(open(os.path.join(GOLD, "pre_pe_h4.tables.gz"), "rb").read()))
    nv = struct.unpack_from("<Q", t, 16)[0]
    slots_at = 16 + 8 + 4 * nv + 4 + 8 * 4                             # u64 slots of map 0's index
    struct.pack_into("<Q", t, slots_at, 2 ** 40)
    struct.pack_into("<Q", t, slots_at - 8, 2 ** 40)                   # capacity to match
    q = tmp_path / "bad.tables"
    q.write_bytes(bytes(t))
    info = (U64 * 4)()
    err = ctypes.create_string_buffer(256)
    assert not H.rt_load(str(q).encode(), 64, info, err, 256)
    assert b"inconsistent key index" in err.value
