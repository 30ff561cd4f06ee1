"""The per-thread device helpers (care_b200/csrc/device.cuh), built for the
host, against the CPU oracle: shifted Hamming both strands + orientation,
canonical k-mers, MurmurHash finalizer. Runs without a GPU."""
import ctypes
import os
import random
import subprocess

import numpy as np
import pytest

import _oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "harness", "device_math.cu")
OUT = os.path.join(ROOT, "tests", "_build", "libdevice_math.so")
DEPS = [SRC, os.path.join(ROOT, "care_b200", "csrc", "device.cuh")]


def harness():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    if not os.path.exists(OUT) or any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in DEPS):
        # built under a process-private name and renamed into place: test
        # workers that start together never load a half-written library
        tmp = f"{OUT}.{os.getpid()}.tmp"
        subprocess.run(["nvcc", "-shared", "-Xcompiler", "-fPIC,-ffp-contract=off", "-O2", "-std=c++17",
                        "-o", tmp, SRC], check=True, capture_output=True)
        os.replace(tmp, OUT)
    lib = ctypes.CDLL(OUT)
    P = ctypes.POINTER
    lib.hd_shd.argtypes = [P(ctypes.c_uint32), ctypes.c_int, P(ctypes.c_uint32), ctypes.c_int, ctypes.c_int,
                           ctypes.c_float, ctypes.c_float, ctypes.c_int, P(ctypes.c_int)]
    lib.hd_canonical_kmers.argtypes = [P(ctypes.c_uint32), ctypes.c_int, ctypes.c_int, P(ctypes.c_uint64)]
    lib.hd_murmur64.argtypes = [ctypes.c_uint64]
    lib.hd_murmur64.restype = ctypes.c_uint64
    lib.hd_unpruned_words.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.hd_shd_pair.argtypes = [P(ctypes.c_uint32), P(ctypes.c_uint32), ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                ctypes.c_float, P(ctypes.c_int)]
    return lib


H = harness()
O = _oracle.lib()


def enc(s):
    n = (len(s) + 15) // 16
    out = (ctypes.c_uint32 * max(n, 1))()
    O.co_encode_2bit(s.encode(), len(s), out)
    return out


def rc(s):
    return s[::-1].translate(str.maketrans("ACGT", "TGCA"))


def mutate(rng, s, k):
    s = list(s)
    for _ in range(k):
        i = rng.randrange(len(s))
        s[i] = rng.choice([b for b in "ACGT" if b != s[i]])
    return "".join(s)


@pytest.mark.parametrize("seed", range(300))
def test_alignment_matches_oracle(seed):
    rng = random.Random(1000 + seed)
    La = rng.randint(20, 256)
    Lc = rng.randint(20, 256)
    g = "".join(rng.choice("ACGT") for _ in range(800))
    a0 = rng.randrange(0, 500)
    a = g[a0:a0 + La]
    c0 = max(0, a0 + rng.randrange(-Lc + 10, La - 10))
    c = mutate(rng, g[c0:c0 + Lc], rng.randrange(0, 10))
    c = (c + "".join(rng.choice("ACGT") for _ in range(Lc)))[:Lc]
    if seed % 2:
        c = rc(c)
    if seed % 7 == 0:
        c = "".join(rng.choice("ACGT") for _ in range(Lc))          # unrelated read
    mo = rng.choice([30, 30, 20, 45])
    mer = rng.choice([0.2, 0.2, 0.1, 0.3])
    ratio = rng.choice([0.3, 0.3, 0.2])
    nw = {4: 4, 5: 5, 6: 6, 7: 8, 8: 8}[max(4, (max(La, Lc) + 31) // 32)]
    out = (ctypes.c_int * 11)()
    assert H.hd_shd(enc(a), La, enc(c), Lc, mo, mer, ratio, nw, out) == 0
    f, r = _oracle.CoAlign(), _oracle.CoAlign()
    O.co_shd(enc(a), La, enc(c), Lc, mo, ctypes.c_float(mer), ctypes.c_float(ratio), ctypes.byref(f))
    O.co_shd(enc(a), La, enc(rc(c)), Lc, mo, ctypes.c_float(mer), ctypes.c_float(ratio), ctypes.byref(r))
    assert list(out[0:5]) == [f.score, f.overlap, f.shift, f.nops, f.valid]
    assert list(out[5:10]) == [r.score, r.overlap, r.shift, r.nops, r.valid]
    assert out[10] == O.co_orientation(ctypes.byref(f), ctypes.byref(r), La, Lc, ctypes.c_float(ratio), mo,
                                       ctypes.c_float(0.06))


@pytest.mark.parametrize("k", [11, 16, 20, 24, 31, 32])
def test_canonical_kmers(k):
    rng = random.Random(k)
    s = "".join(rng.choice("ACGT") for _ in range(250))
    out = (ctypes.c_uint64 * 250)()
    H.hd_canonical_kmers(enc(s), 250, k, out)
    code = {"A": 0, "C": 1, "G": 2, "T": 3}
    for p in range(250 - k + 1):
        km = s[p:p + k]
        f = int("".join(str(code[x]) for x in km), 4)
        r = int("".join(str(code[x]) for x in rc(km)), 4)
        assert out[p] == min(f, r)


def test_murmur():
    for x in [0, 1, 7, 2 ** 40 + 3, 2 ** 64 - 1]:
        assert H.hd_murmur64(x) == O.co_murmur64(x)


def test_unpruned_word_count_closed_form():
    """The work counter of k_align (un-pruned 32-bit word compares of one
    orientation) against a loop over the scanned shifts."""
    def brute(la, lc, mo):
        w = sum(-(-min(la - t, lc) // 32) for t in range(0, la - mo + 1) if min(la - t, lc) > 0)
        w += sum(-(-min(la, lc - t) // 32) for t in range(1, lc - mo + 1) if min(la, lc - t) > 0)
        return w
    assert H.hd_unpruned_words(150, 150, 45) == 743
    assert H.hd_unpruned_words(100, 100, 30) == 354
    rng = random.Random(5)
    for _ in range(3000):
        la, lc = rng.randint(1, 256), rng.randint(1, 256)
        mo = max(rng.randint(1, 80), int(la * 0.3))
        assert H.hd_unpruned_words(la, lc, mo) == brute(la, lc, mo), (la, lc, mo)


def _oracle_shd(a, c, mo, mer, ratio):
    res = _oracle.CoAlign()
    O.co_shd(enc(a), len(a), enc(c), len(c), mo, mer, ratio, ctypes.byref(res))
    return [res.score, res.overlap, res.shift, res.nops, res.valid]


@pytest.mark.parametrize("seed", range(200))
def test_pair_scan_equals_both_directions(seed):
    """One tie-aware scan of an equal-length pair gives the reference's
    alignment of (a, c) and of (c, a): random pairs, overlapping pairs with
    errors, and low-complexity pairs whose scores tie at several shifts."""
    rng = random.Random(7000 + seed)
    L = rng.choice([50, 64, 100, 101, 150, 160, 200, 250])
    kind = seed % 4
    if kind == 0:
        a = "".join(rng.choice("ACGT") for _ in range(L))
        c = "".join(rng.choice("ACGT") for _ in range(L))
    elif kind == 1:
        g = "".join(rng.choice("ACGT") for _ in range(2 * L))
        sh = rng.randint(0, L // 2)
        a, c = mutate(rng, g[:L], rng.randint(0, 6)), mutate(rng, g[sh:sh + L], rng.randint(0, 6))
    else:
        unit = "".join(rng.choice("ACGT") for _ in range(rng.randint(1, 4)))
        g = (unit * (2 * L))[:2 * L]
        sh = rng.randint(0, L // 2)
        a, c = mutate(rng, g[:L], rng.randint(0, 3)), mutate(rng, g[sh:sh + L], rng.randint(0, 3))
    mo, mer, ratio = 30, 0.2, 0.30
    out = (ctypes.c_int * 10)()
    assert H.hd_shd_pair(enc(a), enc(c), L, mo, mer, ratio, out) == 0
    assert list(out[:5]) == _oracle_shd(a, c, mo, mer, ratio), (a, c)
    assert list(out[5:]) == _oracle_shd(c, a, mo, mer, ratio), (a, c)
