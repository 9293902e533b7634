// Wide two's-complement integers (crypto-bigint Int<N>, wrapping) and the
// Montgomery prime field MontyField<L> (R = 2^(64L)) for host and device.
// The reference uses crypto-bigint 0.7 / crypto-primitives for both
// (utils/src/mul_by_scalar.rs:31-125, utils/src/field/monty.rs).
#pragma once
#include <cstdint>
#include <cstring>

#ifndef ZG_HD
#ifdef __CUDACC__
#define ZG_HD __host__ __device__ __forceinline__
#else
#define ZG_HD inline
#endif
#endif

namespace zg {

typedef unsigned __int128 u128;
typedef __int128 i128;

constexpr int MAX_FIELD_LIMBS = 4;
constexpr int MAX_COMB_LIMBS = 8;

// ---------------------------------------------------------------- wide ints
ZG_HD void wide_add(uint64_t *acc, const uint64_t *x, int n) {
    uint64_t c = 0;
    for (int i = 0; i < n; i++) {
        u128 s = (u128)acc[i] + x[i] + c;
        acc[i] = (uint64_t)s;
        c = (uint64_t)(s >> 64);
    }
}

// acc += x * s (mod 2^(64n)), s a signed 128-bit scalar.
ZG_HD void wide_mul_i128_add(uint64_t *acc, const uint64_t *x, i128 s, int n) {
    uint64_t s0 = (uint64_t)(u128)s, s1 = (uint64_t)((u128)s >> 64);
    uint64_t sg = s < 0 ? ~0ull : 0ull;
    uint64_t prod[MAX_COMB_LIMBS];
    for (int i = 0; i < n; i++) prod[i] = 0;
    for (int i = 0; i < n; i++) {
        uint64_t c = 0;
        for (int j = 0; i + j < n; j++) {
            uint64_t sj = j == 0 ? s0 : (j == 1 ? s1 : sg);
            u128 t = (u128)x[i] * sj + prod[i + j] + c;
            prod[i + j] = (uint64_t)t;
            c = (uint64_t)(t >> 64);
        }
    }
    wide_add(acc, prod, n);
}

// Sign-extend a signed value of `from` limbs to `to` limbs.
ZG_HD void wide_sext(const uint64_t *x, int from, uint64_t *out, int to) {
    uint64_t sg = (x[from - 1] >> 63) ? ~0ull : 0ull;
    for (int i = 0; i < to; i++) out[i] = i < from ? x[i] : sg;
}

// --------------------------------------------------------------- the field
struct FieldCfg {
    int L;
    uint64_t p[MAX_FIELD_LIMBS];
    uint64_t n0;                           // -p^-1 mod 2^64
    uint64_t one[MAX_FIELD_LIMBS];         // R mod p
    uint64_t r2[MAX_FIELD_LIMBS];          // R^2 mod p
    uint64_t rpow[4][MAX_FIELD_LIMBS];     // R^(k+2) mod p, k = 0..3
};

template <int L>
ZG_HD int ucmp(const uint64_t *a, const uint64_t *b) {
    for (int i = L - 1; i >= 0; i--)
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
}
template <int L>
ZG_HD uint64_t usub(uint64_t *a, const uint64_t *b) {
    uint64_t br = 0;
    for (int i = 0; i < L; i++) {
        u128 s = (u128)a[i] - b[i] - br;
        a[i] = (uint64_t)s;
        br = (uint64_t)(s >> 64) & 1;
    }
    return br;
}
template <int L>
ZG_HD uint64_t uadd(uint64_t *a, const uint64_t *b) {
    uint64_t c = 0;
    for (int i = 0; i < L; i++) {
        u128 s = (u128)a[i] + b[i] + c;
        a[i] = (uint64_t)s;
        c = (uint64_t)(s >> 64);
    }
    return c;
}
template <int L>
ZG_HD bool uzero(const uint64_t *a) {
    uint64_t o = 0;
    for (int i = 0; i < L; i++) o |= a[i];
    return o == 0;
}

template <int L>
ZG_HD void fadd(uint64_t *a, const uint64_t *b, const uint64_t *p) {
    uint64_t c = uadd<L>(a, b);
    if (c || ucmp<L>(a, p) >= 0) usub<L>(a, p);
}
template <int L>
ZG_HD void fsub(uint64_t *a, const uint64_t *b, const uint64_t *p) {
    if (usub<L>(a, b)) uadd<L>(a, p);
}
template <int L>
ZG_HD void fneg(uint64_t *a, const uint64_t *p) {
    if (uzero<L>(a)) return;
    uint64_t t[L];
    for (int i = 0; i < L; i++) t[i] = p[i];
    usub<L>(t, a);
    for (int i = 0; i < L; i++) a[i] = t[i];
}

// Montgomery product a*b*R^-1 mod p for a < R, b < p (CIOS).
template <int L>
ZG_HD void fmul(const uint64_t *a, const uint64_t *b, const uint64_t *p, uint64_t n0,
                uint64_t *out) {
    uint64_t t[L + 2];
    for (int i = 0; i < L + 2; i++) t[i] = 0;
    for (int i = 0; i < L; i++) {
        uint64_t c = 0;
        for (int j = 0; j < L; j++) {
            u128 s = (u128)a[j] * b[i] + t[j] + c;
            t[j] = (uint64_t)s;
            c = (uint64_t)(s >> 64);
        }
        u128 s = (u128)t[L] + c;
        t[L] = (uint64_t)s;
        t[L + 1] = (uint64_t)(s >> 64);
        uint64_t m = t[0] * n0;
        s = (u128)m * p[0] + t[0];
        c = (uint64_t)(s >> 64);
        for (int j = 1; j < L; j++) {
            s = (u128)m * p[j] + t[j] + c;
            t[j - 1] = (uint64_t)s;
            c = (uint64_t)(s >> 64);
        }
        s = (u128)t[L] + c;
        t[L - 1] = (uint64_t)s;
        t[L] = t[L + 1] + (uint64_t)(s >> 64);
    }
    if (t[L] || ucmp<L>(t, p) >= 0) usub<L>(t, p);
    for (int i = 0; i < L; i++) out[i] = t[i];
}

// F::from_with_cfg(&Int<limbs>) in Montgomery form: sign and magnitude, the
// magnitude reduced digit by digit (digit k of L limbs weighs R^k).
template <int L>
ZG_HD void from_signed(const uint64_t *x, int limbs, const FieldCfg &f, uint64_t *out) {
    bool neg = (x[limbs - 1] >> 63) != 0;
    uint64_t mag[MAX_COMB_LIMBS + MAX_FIELD_LIMBS];
    int nd = (limbs + L - 1) / L;
    for (int i = 0; i < nd * L; i++) mag[i] = i < limbs ? x[i] : 0;
    if (neg) {
        uint64_t c = 1;
        for (int i = 0; i < limbs; i++) {
            u128 s = (u128)(~mag[i]) + c;
            mag[i] = (uint64_t)s;
            c = (uint64_t)(s >> 64);
        }
    }
    uint64_t acc[L];
    for (int i = 0; i < L; i++) acc[i] = 0;
    for (int k = 0; k < nd; k++) {
        if (uzero<L>(mag + k * L)) continue;
        uint64_t t[L];
        fmul<L>(mag + k * L, f.rpow[k], f.p, f.n0, t);
        fadd<L>(acc, t, f.p);
    }
    if (neg) fneg<L>(acc, f.p);
    for (int i = 0; i < L; i++) out[i] = acc[i];
}

template <int L>
ZG_HD void from_i128(i128 v, const FieldCfg &f, uint64_t *out) {
    uint64_t x[2] = {(uint64_t)(u128)v, (uint64_t)((u128)v >> 64)};
    from_signed<L>(x, 2, f, out);
}

// Host-side configuration of MontyField for an odd modulus p of L limbs.
inline void field_cfg_init(FieldCfg &f, const uint64_t *p, int L) {
    std::memset(&f, 0, sizeof f);
    f.L = L;
    for (int i = 0; i < L; i++) f.p[i] = p[i];
    uint64_t inv = p[0];
    for (int i = 0; i < 6; i++) inv *= 2 - p[0] * inv;
    f.n0 = (uint64_t)0 - inv;
    // R mod p and R^2 mod p by modular doubling.
    uint64_t x[MAX_FIELD_LIMBS] = {1, 0, 0, 0};
    auto dbl = [&](uint64_t *v) {
        uint64_t c = 0;
        for (int i = 0; i < L; i++) {
            uint64_t nc = v[i] >> 63;
            v[i] = (v[i] << 1) | c;
            c = nc;
        }
        bool ge = c != 0;
        if (!ge) {
            ge = true;
            for (int i = L - 1; i >= 0; i--)
                if (v[i] != f.p[i]) {
                    ge = v[i] > f.p[i];
                    break;
                }
        }
        if (ge) {
            uint64_t br = 0;
            for (int i = 0; i < L; i++) {
                u128 s = (u128)v[i] - f.p[i] - br;
                v[i] = (uint64_t)s;
                br = (uint64_t)(s >> 64) & 1;
            }
        }
    };
    // 1 mod p (p > 1)
    for (int i = 0; i < 64 * L; i++) dbl(x);
    for (int i = 0; i < L; i++) f.one[i] = x[i];
    for (int i = 0; i < 64 * L; i++) dbl(x);
    for (int i = 0; i < L; i++) f.r2[i] = x[i];
    for (int i = 0; i < L; i++) f.rpow[0][i] = f.r2[i];
    for (int k = 1; k < 4; k++) {
        if (L == 3) fmul<3>(f.rpow[k - 1], f.r2, f.p, f.n0, f.rpow[k]);
        else if (L == 4) fmul<4>(f.rpow[k - 1], f.r2, f.p, f.n0, f.rpow[k]);
        else if (L == 2) fmul<2>(f.rpow[k - 1], f.r2, f.p, f.n0, f.rpow[k]);
        else fmul<1>(f.rpow[k - 1], f.r2, f.p, f.n0, f.rpow[k]);
    }
}

}  // namespace zg
