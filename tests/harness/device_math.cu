// Host build of the per-thread device helpers of care_b200/csrc/device.cuh,
// so that their results can be compared with the CPU oracle without a GPU.
// Test infrastructure only.
#include "../../care_b200/csrc/device.cuh"

#include <cstring>

using namespace careb200;

template <int NW>
static void shd_nw(const uint32_t* a, int la, const uint32_t* c, int lc, int min_overlap, float mer,
                   float ratio, int* out) {
    uint32_t Ah[NW + 2], Al[NW + 2], Ch[NW + 2], Cl[NW + 2], Rh[NW + 2], Rl[NW + 2];
    load_planes<NW>(a, la, Ah, Al);
    load_planes<NW>(c, lc, Ch, Cl);
    int mextab[kMaxLen + 1];
    for (int i = 0; i <= kMaxLen; i++) mextab[i] = f2i_rz(fmul_rn((float)i, mer));
    const int lo = f2i_rz(fmul_rn((float)la, ratio));
    const int minov = min_overlap > lo ? min_overlap : lo;
    const ShdResult f = shifted_hamming<NW>(Ah, Al, la, Ch, Cl, lc, minov, mextab);
    revcomp_planes<NW>(Ch, Cl, lc, Rh, Rl);
    const ShdResult r = shifted_hamming<NW>(Ah, Al, la, Rh, Rl, lc, minov, mextab);
    const ShdResult* rs[2] = {&f, &r};
    for (int k = 0; k < 2; k++) {
        out[5 * k + 0] = rs[k]->score; out[5 * k + 1] = rs[k]->overlap; out[5 * k + 2] = rs[k]->shift;
        out[5 * k + 3] = rs[k]->nops; out[5 * k + 4] = rs[k]->valid;
    }
    out[10] = choose_orientation(f, r, la, ratio, min_overlap, fmul_rn(0.06f, 4.0f));
}

extern "C" {

// forward and reverse-complement alignments + orientation, NW = plane words
int hd_shd(const uint32_t* a, int la, const uint32_t* c, int lc, int min_overlap, float mer, float ratio,
           int nw, int* out) {
    switch (nw) {
        case 4: shd_nw<4>(a, la, c, lc, min_overlap, mer, ratio, out); return 0;
        case 5: shd_nw<5>(a, la, c, lc, min_overlap, mer, ratio, out); return 0;
        case 6: shd_nw<6>(a, la, c, lc, min_overlap, mer, ratio, out); return 0;
        case 8: shd_nw<8>(a, la, c, lc, min_overlap, mer, ratio, out); return 0;
    }
    return -1;
}

// canonical k-mer at each position, as the candidate kernel computes it
void hd_canonical_kmers(const uint32_t* seq, int len, int k, unsigned long long* out) {
    uint32_t padded[kMaxLen / 16 + 4];
    const int n = (len + 15) / 16;
    for (int i = 0; i < n + 2; i++) padded[i] = i < n ? seq[i] : 0u;
    for (int p = 0; p + k <= len; p++) {
        const unsigned long long fw = kmer_at(padded, k, p);
        const unsigned long long rv = revcomp64(fw) >> (64 - 2 * k);
        out[p] = fw < rv ? fw : rv;
    }
}

unsigned long long hd_murmur64(unsigned long long x) { return murmur64(x); }

int hd_unpruned_words(int la, int lc, int minov) { return unpruned_words(la, lc, minov); }

// forward alignments of (a, c) and (c, a) from one scan (equal lengths);
// out: score, overlap, shift, nops, valid of (a, c) then of (c, a)
int hd_shd_pair(const uint32_t* a, const uint32_t* c, int len, int min_overlap, float mer, float ratio, int* out) {
    constexpr int NW = 8;
    if (len > 32 * NW) return -1;
    uint32_t Ah[NW + 2], Al[NW + 2], Ch[NW + 2], Cl[NW + 2];
    load_planes<NW>(a, len, Ah, Al);
    load_planes<NW>(c, len, Ch, Cl);
    int mextab[kMaxLen + 1];
    for (int i = 0; i <= kMaxLen; i++) mextab[i] = f2i_rz(fmul_rn((float)i, mer));
    const int lo = f2i_rz(fmul_rn((float)len, ratio));
    const int minov = min_overlap > lo ? min_overlap : lo;
    ShdResult ac, ca;
    shifted_hamming_pair<NW>(Ah, Al, Ch, Cl, len, minov, mextab, ac, ca);
    const ShdResult* rs[2] = {&ac, &ca};
    for (int k = 0; k < 2; k++) {
        out[5 * k + 0] = rs[k]->score; out[5 * k + 1] = rs[k]->overlap; out[5 * k + 2] = rs[k]->shift;
        out[5 * k + 3] = rs[k]->nops; out[5 * k + 4] = rs[k]->valid;
    }
    return 0;
}
}
