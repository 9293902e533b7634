// Miller-Rabin to base 2 on eight candidates at once with AVX-512 IFMA
// (52-bit multiply-add), one candidate per 64-bit lane: the strong
// probable-prime test of crypto-primes' MillerRabin::test_base_two, which
// primality/src/lib.rs:12-19 calls for the transcript's prime.
//
// Each candidate n (odd, > 1, at most 64L bits) is held as K = ceil(64L / 52)
// limbs of 52 bits.  The exponentiation 2^d mod n runs in Montgomery form with
// radix 2^(52K) (the test's verdict does not depend on the radix): every bit of
// d is a Montgomery squaring, and a set bit a modular doubling.  The lanes run
// the same 64L iterations, so each candidate's leading zero bits square 1 into
// 1.  The verdict is the scalar test's for every input: this path is a speed-up
// and is checked against the scalar test (tests/test_host_abi.py).
#include <immintrin.h>

#include <cstdint>
#include <cstring>

namespace zg {

namespace {

constexpr uint64_t kMask52 = (1ull << 52) - 1;

// 64L-bit little-endian words -> K limbs of 52 bits
inline void to52(const uint64_t *w, int L, int K, uint64_t *l) {
    for (int k = 0; k < K; k++) {
        const int bit = 52 * k, wi = bit / 64, sh = bit % 64;
        uint64_t v = wi < L ? w[wi] >> sh : 0;
        if (sh > 12 && wi + 1 < L) v |= w[wi + 1] << (64 - sh);
        l[k] = v & kMask52;
    }
}

template <int K>
struct V {
    __m512i l[K];
};

#define ZG_IFMA __attribute__((target("avx512f,avx512ifma,avx512vl,avx512dq,avx512bw")))

// Carry-propagate limbs held in 64-bit lanes (each below 2^63) to 52 bits;
// the carry out of the top limb is returned (zero for values below 2^(52K)).
template <int K>
ZG_IFMA inline __m512i normalize(V<K> &x) {
    const __m512i m = _mm512_set1_epi64((long long)kMask52);
    __m512i c = _mm512_setzero_si512();
    for (int k = 0; k < K; k++) {
        const __m512i t = _mm512_add_epi64(x.l[k], c);
        c = _mm512_srli_epi64(t, 52);
        x.l[k] = _mm512_and_si512(t, m);
    }
    return c;
}

// x >= n per lane, for normalized x (with an extra top word xt) and n
template <int K>
ZG_IFMA inline __mmask8 geq(const V<K> &x, __m512i xt, const V<K> &n) {
    __mmask8 gt = _mm512_cmpneq_epi64_mask(xt, _mm512_setzero_si512());
    __mmask8 eq = (__mmask8)~gt;
    for (int k = K - 1; k >= 0; k--) {
        gt |= eq & _mm512_cmpgt_epu64_mask(x.l[k], n.l[k]);
        eq &= _mm512_cmpeq_epi64_mask(x.l[k], n.l[k]);
    }
    return gt | eq;
}

// x -= n on the lanes of mask (x >= n there), limbs normalized
template <int K>
ZG_IFMA inline void sub_masked(V<K> &x, const V<K> &n, __mmask8 mask) {
    const __m512i m = _mm512_set1_epi64((long long)kMask52);
    __m512i br = _mm512_setzero_si512();
    for (int k = 0; k < K; k++) {
        __m512i t = _mm512_sub_epi64(_mm512_sub_epi64(x.l[k], n.l[k]), br);
        br = _mm512_srli_epi64(t, 63);  // borrow: the difference went negative
        t = _mm512_and_si512(t, m);
        x.l[k] = _mm512_mask_mov_epi64(x.l[k], mask, t);
    }
}

// Montgomery product a b 2^(-52K) mod n (a, b < n; result < n), per lane
template <int K>
ZG_IFMA inline void mont_mul(const V<K> &a, const V<K> &b, const V<K> &n, __m512i n0, V<K> &out) {
    __m512i t[K + 1];
    const __m512i z = _mm512_setzero_si512();
    for (int k = 0; k <= K; k++) t[k] = z;
    for (int i = 0; i < K; i++) {
        const __m512i bi = b.l[i];
        for (int j = 0; j < K; j++) {
            t[j] = _mm512_madd52lo_epu64(t[j], a.l[j], bi);
            t[j + 1] = _mm512_madd52hi_epu64(t[j + 1], a.l[j], bi);
        }
        const __m512i m = _mm512_madd52lo_epu64(z, t[0], n0);  // t0 * n0 mod 2^52
        for (int j = 0; j < K; j++) {
            t[j] = _mm512_madd52lo_epu64(t[j], m, n.l[j]);
            t[j + 1] = _mm512_madd52hi_epu64(t[j + 1], m, n.l[j]);
        }
        // t[0] is now 0 mod 2^52: shift down one limb, carrying its high part
        const __m512i c = _mm512_srli_epi64(t[0], 52);
        for (int j = 0; j < K; j++) t[j] = t[j + 1];
        t[0] = _mm512_add_epi64(t[0], c);
        t[K] = z;
    }
    V<K> r;
    for (int k = 0; k < K; k++) r.l[k] = t[k];
    const __m512i top = normalize<K>(r);  // r < 2n
    sub_masked<K>(r, n, geq<K>(r, top, n));
    out = r;
}

// x = 2x mod n on the lanes of mask (x < n, normalized)
template <int K>
ZG_IFMA inline void dbl_mod(V<K> &x, const V<K> &n, __mmask8 mask) {
    V<K> y;
    for (int k = 0; k < K; k++) y.l[k] = _mm512_slli_epi64(x.l[k], 1);
    const __m512i top = normalize<K>(y);
    sub_masked<K>(y, n, geq<K>(y, top, n));
    for (int k = 0; k < K; k++) x.l[k] = _mm512_mask_mov_epi64(x.l[k], mask, y.l[k]);
}

template <int K>
ZG_IFMA inline __mmask8 veq(const V<K> &x, const V<K> &y) {
    __mmask8 e = 0xFF;
    for (int k = 0; k < K; k++) e &= _mm512_cmpeq_epi64_mask(x.l[k], y.l[k]);
    return e;
}

template <int K>
ZG_IFMA void mr8(const uint64_t *cand, int L, int count, uint8_t *ok) {
    alignas(64) uint64_t nl[K][8], one[K][8], mone[K][8], n0s[8];
    int s_of[8], topbit = 0;
    uint64_t d[8][4];
    bool valid[8];
    for (int c = 0; c < 8; c++) {
        uint64_t w[4] = {1, 0, 0, 0};  // padding lanes test n = 3 (any odd n > 1)
        w[0] = 3;
        valid[c] = c < count;
        if (valid[c])
            for (int i = 0; i < L; i++) w[i] = cand[(size_t)c * L + i];
        uint64_t l[K];
        to52(w, L, K, l);
        for (int k = 0; k < K; k++) nl[k][c] = l[k];
        // n0 = -n^-1 mod 2^52
        uint64_t inv = w[0];
        for (int i = 0; i < 6; i++) inv *= 2 - w[0] * inv;
        n0s[c] = (0 - inv) & kMask52;
        // R' = 2^(52K) mod n: from 2^(b-1) < n (b the bit length), doubled
        int b = 64 * L;
        while (b > 0 && !((w[(b - 1) / 64] >> ((b - 1) % 64)) & 1)) b--;
        uint64_t y[5] = {0, 0, 0, 0, 0};
        y[(b - 1) / 64] = 1ull << ((b - 1) % 64);
        for (int k = 0; k < 52 * K - b + 1; k++) {
            uint64_t cr = 0;
            for (int i = 0; i < L; i++) {
                const uint64_t nc = y[i] >> 63;
                y[i] = (y[i] << 1) | cr;
                cr = nc;
            }
            bool ge = cr != 0;
            if (!ge) {
                ge = true;
                for (int i = L - 1; i >= 0; i--)
                    if (y[i] != w[i]) {
                        ge = y[i] > w[i];
                        break;
                    }
            }
            if (ge) {
                unsigned __int128 br = 0;
                for (int i = 0; i < L; i++) {
                    const unsigned __int128 t = (unsigned __int128)y[i] - w[i] - (uint64_t)br;
                    y[i] = (uint64_t)t;
                    br = (t >> 64) & 1;
                }
            }
        }
        uint64_t ol[K], ml[K], mw[4] = {0, 0, 0, 0};
        to52(y, L, K, ol);
        for (int k = 0; k < K; k++) one[k][c] = ol[k];
        // -1 in Montgomery form: n - R' mod n
        unsigned __int128 br = 0;
        for (int i = 0; i < L; i++) {
            const unsigned __int128 t = (unsigned __int128)w[i] - y[i] - (uint64_t)br;
            mw[i] = (uint64_t)t;
            br = (t >> 64) & 1;
        }
        to52(mw, L, K, ml);
        for (int k = 0; k < K; k++) mone[k][c] = ml[k];
        // n - 1 = 2^s d
        uint64_t nm1[4] = {0, 0, 0, 0};
        for (int i = 0; i < L; i++) nm1[i] = w[i];
        nm1[0] -= 1;
        int s = 0;
        while (!((nm1[s / 64] >> (s % 64)) & 1)) s++;
        s_of[c] = s;
        for (int i = 0; i < 4; i++) d[c][i] = 0;
        for (int i = 0; i + s < 64 * L; i++)
            if ((nm1[(i + s) / 64] >> ((i + s) % 64)) & 1) d[c][i / 64] |= 1ull << (i % 64);
        for (int i = 64 * L - 1; i >= 0; i--)
            if ((d[c][i / 64] >> (i % 64)) & 1) {
                if (i > topbit) topbit = i;
                break;
            }
    }
    V<K> n, x, vone, vmone;
    for (int k = 0; k < K; k++) {
        n.l[k] = _mm512_load_si512(nl[k]);
        vone.l[k] = _mm512_load_si512(one[k]);
        vmone.l[k] = _mm512_load_si512(mone[k]);
    }
    const __m512i n0 = _mm512_load_si512(n0s);
    x = vone;
    for (int bit = topbit; bit >= 0; bit--) {
        mont_mul<K>(x, x, n, n0, x);
        __mmask8 m = 0;
        for (int c = 0; c < 8; c++)
            if ((d[c][bit / 64] >> (bit % 64)) & 1) m |= (__mmask8)(1u << c);
        if (m) dbl_mod<K>(x, n, m);
    }
    // strong probable prime: 2^d = +-1, or 2^(d 2^r) = -1 for some 0 < r < s
    __mmask8 pass = veq<K>(x, vone) | veq<K>(x, vmone), done = pass;
    int smax = 0;
    for (int c = 0; c < 8; c++) smax = s_of[c] > smax ? s_of[c] : smax;
    for (int r = 1; r < smax; r++) {
        mont_mul<K>(x, x, n, n0, x);
        __mmask8 live = 0;
        for (int c = 0; c < 8; c++)
            if (r < s_of[c]) live |= (__mmask8)(1u << c);
        live &= (__mmask8)~done;
        const __mmask8 is_one = veq<K>(x, vone) & live, is_mone = veq<K>(x, vmone) & live;
        pass |= is_mone;
        done |= is_one | is_mone;
    }
    for (int c = 0; c < count; c++) ok[c] = (pass >> c) & 1;
}

}  // namespace

bool mr_ifma_available() {
    static const int have = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512ifma") &&
                            __builtin_cpu_supports("avx512vl") && __builtin_cpu_supports("avx512dq") &&
                            __builtin_cpu_supports("avx512bw");
    return have != 0;
}

// count (1..8) odd candidates n > 1 of L limbs; ok[c] = the base-2 verdict
void mr_base2_x8(const uint64_t *cand, int L, int count, uint8_t *ok) {
    switch (L) {
        case 1: mr8<2>(cand, L, count, ok); break;
        case 2: mr8<3>(cand, L, count, ok); break;
        case 3: mr8<4>(cand, L, count, ok); break;
        default: mr8<5>(cand, L, count, ok); break;
    }
}

}  // namespace zg
