"""Known-answer tests of the oracle's stage functions against independent
Python statements of the same definitions (small cases, pure Python)."""
import ctypes
import random

import numpy as np
import pytest

import _oracle

L = _oracle.lib()
M64 = (1 << 64) - 1


def enc(s: str):
    n = (len(s) + 15) // 16
    out = (ctypes.c_uint32 * max(n, 1))()
    L.co_encode_2bit(s.encode(), len(s), out)
    return out


def py_encode(s):
    code = {"A": 0, "C": 1, "G": 2, "T": 3}
    n = (len(s) + 15) // 16
    words = []
    for w in range(n):
        x = 0
        for p in range(16):
            i = 16 * w + p
            x = (x << 2) | (code.get(s[i], 0) if i < len(s) else 0)
        words.append(x)
    return words


def fmix64(x):
    x ^= x >> 33
    x = (x * 0xff51afd7ed558ccd) & M64
    x ^= x >> 33
    x = (x * 0xc4ceb9fe1a85ec53) & M64
    x ^= x >> 33
    return x


def rc(s):
    return s[::-1].translate(str.maketrans("ACGT", "TGCA"))


def rand_seq(rng, n):
    return "".join(rng.choice("ACGT") for _ in range(n))


def test_murmur_finalizer():
    for x in [0, 1, 2, 12345, M64, 0xDEADBEEFCAFEBABE]:
        assert L.co_murmur64(x) == fmix64(x)


@pytest.mark.parametrize("n", [1, 15, 16, 17, 31, 32, 33, 100, 150, 250])
def test_encode_decode_revcomp(n):
    rng = random.Random(n)
    s = rand_seq(rng, n)
    e = enc(s)
    assert list(e)[: (n + 15) // 16] == py_encode(s)
    buf = ctypes.create_string_buffer(n + 1)
    L.co_decode_2bit(e, n, buf)
    assert buf.raw[:n].decode() == s
    out = (ctypes.c_uint32 * ((n + 15) // 16))()
    L.co_revcomp_2bit(e, n, out)
    assert list(out) == py_encode(rc(s))


@pytest.mark.parametrize("n", [1, 16, 31, 32, 33, 64, 100, 150, 250])
def test_hilo_layout(n):
    rng = random.Random(100 + n)
    s = rand_seq(rng, n)
    e = enc(s)
    words = 2 * ((n + 31) // 32)
    out = (ctypes.c_uint32 * words)()
    L.co_to_hilo(e, n, out)
    code = {"A": 0, "C": 1, "G": 2, "T": 3}
    half = words // 2
    for w in range(half):
        hi = lo = 0
        for p in range(32):
            i = 32 * w + p
            c = code[s[i]] if i < n else 0
            hi = (hi << 1) | (c >> 1)
            lo = (lo << 1) | (c & 1)
        assert out[w] == hi and out[half + w] == lo


def py_signature(s, k, maps):
    code = {"A": 0, "C": 1, "G": 2, "T": 3}
    mask = M64 >> (2 * (32 - k))
    res = [M64] * maps
    if len(s) >= k:
        for p in range(len(s) - k + 1):
            km = s[p:p + k]
            f = 0
            for ch in km:
                f = (f << 2) | code[ch]
            r = 0
            for ch in rc(km):
                r = (r << 2) | code[ch]
            c = min(f, r)
            for h in range(maps):
                res[h] = min(res[h], fmix64((c + h) & M64))
    return [x & mask for x in res]


@pytest.mark.parametrize("n,k,maps", [(100, 20, 16), (150, 20, 32), (40, 32, 4), (19, 20, 3), (37, 11, 5)])
def test_signature(n, k, maps):
    rng = random.Random(n * 7 + k)
    s = rand_seq(rng, n)
    out = (ctypes.c_uint64 * maps)()
    L.co_signature(enc(s), n, k, maps, out)
    assert list(out) == py_signature(s, k, maps)


def py_shd(a, c, min_overlap, mer, ratio):
    """Shifted Hamming as the argmin formulation: the first shift, in the
    reference's scan order, among those with mismatches < int(ov*mer), that
    minimises mismatches + La + Lc - 2*ov."""
    La, Lc = len(a), len(c)
    minov = max(min_overlap, int(np.float32(La) * np.float32(ratio)))
    total = La + Lc
    order = list(range(0, La - minov + 1)) + [-t for t in range(1, Lc - minov + 1)]
    best, bshift = total, -Lc
    for s in order:
        if s >= 0:
            ov = min(La - s, Lc)
            mm = sum(1 for i in range(ov) if a[s + i] != c[i])
        else:
            t = -s
            ov = min(La, Lc - t)
            mm = sum(1 for i in range(ov) if c[t + i] != a[i])
        lim = int(np.float32(ov) * np.float32(mer))
        if mm < lim and mm + total - 2 * ov < best:
            best, bshift = mm + total - 2 * ov, s
    cb = max(-bshift, 0)
    ce = min(Lc, La - bshift)
    ovl = ce - cb
    return best, ovl, bshift, best - total + 2 * ovl, int(bshift != -Lc)


def mutate(rng, s, k):
    s = list(s)
    for _ in range(k):
        i = rng.randrange(len(s))
        s[i] = rng.choice([b for b in "ACGT" if b != s[i]])
    return "".join(s)


@pytest.mark.parametrize("seed", range(40))
def test_shifted_hamming_matches_argmin(seed):
    rng = random.Random(seed)
    La = rng.choice([50, 64, 100, 101, 150, 200, 250])
    Lc = rng.choice([50, 63, 100, 150, 249])
    g = rand_seq(rng, 600)
    a0 = rng.randrange(0, 300)
    a = g[a0:a0 + La]
    c0 = a0 + rng.randrange(-Lc + 20, La - 20)
    c0 = max(0, c0)
    c = mutate(rng, g[c0:c0 + Lc], rng.randrange(0, 8))
    if len(c) < Lc:
        c = c + rand_seq(rng, Lc - len(c))
    if seed % 3 == 0:
        c = rc(c)
    res = _oracle.CoAlign()
    L.co_shd(enc(a), La, enc(c), Lc, 30, ctypes.c_float(0.2), ctypes.c_float(0.3), ctypes.byref(res))
    got = (res.score, res.overlap, res.shift, res.nops, res.valid)
    assert got == py_shd(a, c, 30, 0.2, 0.3)


def test_pair_flags_equal_mate_membership():
    rng = random.Random(7)
    for _ in range(500):
        pool = rng.sample(range(60), rng.randrange(0, 30))
        l1 = sorted(rng.sample(pool, rng.randrange(0, len(pool) + 1)))
        l2 = sorted(rng.sample(pool, rng.randrange(0, len(pool) + 1)))
        a1 = (ctypes.c_uint32 * max(1, len(l1)))(*l1)
        a2 = (ctypes.c_uint32 * max(1, len(l2)))(*l2)
        f1 = (ctypes.c_uint8 * max(1, len(l1)))()
        f2 = (ctypes.c_uint8 * max(1, len(l2)))()
        L.co_pair_flags(a1, len(l1), a2, len(l2), f1, f2)
        s1, s2 = set(l1), set(l2)
        assert [bool(f1[i]) for i in range(len(l1))] == [(x ^ 1) in s2 for x in l1]
        assert [bool(f2[i]) for i in range(len(l2))] == [(x ^ 1) in s1 for x in l2]


@pytest.mark.parametrize("bits", [1, 2, 8])
def test_quality_codec(bits):
    rng = random.Random(bits)
    q = "".join(chr(33 + rng.randrange(0, 42)) for _ in range(150))
    n = (bits * 150 + 31) // 32
    e = (ctypes.c_uint32 * n)()
    L.co_encode_quality(q.encode(), 150, bits, e)
    out = ctypes.create_string_buffer(151)
    L.co_decode_quality(e, 150, bits, out)
    dec = out.raw[:150].decode("latin1")
    if bits == 8:
        assert dec == q
    else:
        bounds = {1: [13, 256], 2: [4, 13, 20, 256]}[bits]
        chars = {1: "(5", 2: "$(19"}[bits]
        exp = "".join(chars[next(i for i, b in enumerate(bounds) if ord(ch) - 33 <= b)] for ch in q)
        assert dec == exp


def test_quality_weights():
    w = (ctypes.c_float * 256)()
    L.co_quality_weights(w)
    for i in range(256):
        p = 1.0 if i < 33 else 10.0 ** (-(i - 33) / 10.0)
        assert abs(w[i] - max(0.001, 1.0 - p)) < 1e-6


def test_threshold():
    for cov, exp in [(1.0, 10), (4.0, 10), (30.0, 75), (40.0, 100), (50.0, 125), (30.9, 75)]:
        assert L.co_threshold(ctypes.c_float(cov)) == exp
