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

// acc += x * s (mod 2^(64n)) for a signed 64-bit scalar: x * (s mod 2^64),
// minus x * 2^64 when s < 0.
ZG_HD void wide_mul_s64_add(uint64_t *acc, const uint64_t *x, int64_t s, int n) {
    const uint64_t s0 = (uint64_t)s;
    uint64_t c = 0, borrow = 0;
    for (int i = 0; i < n; i++) {
        u128 t = (u128)x[i] * s0 + acc[i] + c;
        uint64_t v = (uint64_t)t;
        c = (uint64_t)(t >> 64);
        if (s < 0 && i > 0) {  // subtract x[i-1] at limb i
            const uint64_t sub = x[i - 1], before = v;
            v = before - sub - borrow;
            borrow = (before < sub || (before == sub && borrow)) ? 1u : 0u;
        }
        acc[i] = v;
    }
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

#ifdef __CUDA_ARCH__
// One word step of the CIOS loop (accumulate a*b_i, reduce by m*p), each in
// one asm block so that its carry chains stay together while independent
// products interleave.  Generated for N = 2, 4, 6, 8 words.
template <int N>
__device__ __forceinline__ void mont_step(uint32_t (&t)[N + 2], const uint32_t (&a)[N],
                                          const uint32_t (&p)[N], uint32_t bi, uint32_t n0);
template <int N>
__device__ __forceinline__ void mont_sub(const uint32_t (&t)[N + 2], const uint32_t (&p)[N],
                                         uint32_t (&d)[N], uint32_t &top);
template <>
__device__ __forceinline__ void mont_step<2>(uint32_t (&t)[4], const uint32_t (&a)[2],
                                             const uint32_t (&p)[2], uint32_t bi, uint32_t n0) {
    asm("{\n\t.reg .u32 m;\n\tmad.lo.cc.u32 %0, %4, %8, %0;\n\tmadc.lo.cc.u32 %1, %5, %8, %1;\n\taddc.cc.u32 %2, %2, 0;\n\taddc.u32 %3, %3, 0;\n\tmad.hi.cc.u32 %1, %4, %8, %1;\n\tmadc.hi.cc.u32 %2, %5, %8, %2;\n\taddc.u32 %3, %3, 0;\n\tmul.lo.u32 m, %0, %9;\n\tmad.lo.cc.u32 %0, m, %6, %0;\n\tmadc.lo.cc.u32 %1, m, %7, %1;\n\taddc.cc.u32 %2, %2, 0;\n\taddc.u32 %3, %3, 0;\n\tmad.hi.cc.u32 %1, m, %6, %1;\n\tmadc.hi.cc.u32 %2, m, %7, %2;\n\taddc.u32 %3, %3, 0;\n\t}"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3])
        : "r"(a[0]), "r"(a[1]), "r"(p[0]), "r"(p[1]), "r"(bi), "r"(n0));
}
template <>
__device__ __forceinline__ void mont_sub<2>(const uint32_t (&t)[4], const uint32_t (&p)[2],
                                            uint32_t (&d)[2], uint32_t &top) {
    asm("sub.cc.u32 %0, %3, %6;\n\tsubc.cc.u32 %1, %4, %7;\n\tsubc.u32 %2, %5, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(top)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(p[0]), "r"(p[1]));
}
template <>
__device__ __forceinline__ void mont_step<4>(uint32_t (&t)[6], const uint32_t (&a)[4],
                                             const uint32_t (&p)[4], uint32_t bi, uint32_t n0) {
    asm("{\n\t.reg .u32 m;\n\tmad.lo.cc.u32 %0, %6, %14, %0;\n\tmadc.lo.cc.u32 %1, %7, %14, %1;\n\tmadc.lo.cc.u32 %2, %8, %14, %2;\n\tmadc.lo.cc.u32 %3, %9, %14, %3;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.u32 %5, %5, 0;\n\tmad.hi.cc.u32 %1, %6, %14, %1;\n\tmadc.hi.cc.u32 %2, %7, %14, %2;\n\tmadc.hi.cc.u32 %3, %8, %14, %3;\n\tmadc.hi.cc.u32 %4, %9, %14, %4;\n\taddc.u32 %5, %5, 0;\n\tmul.lo.u32 m, %0, %15;\n\tmad.lo.cc.u32 %0, m, %10, %0;\n\tmadc.lo.cc.u32 %1, m, %11, %1;\n\tmadc.lo.cc.u32 %2, m, %12, %2;\n\tmadc.lo.cc.u32 %3, m, %13, %3;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.u32 %5, %5, 0;\n\tmad.hi.cc.u32 %1, m, %10, %1;\n\tmadc.hi.cc.u32 %2, m, %11, %2;\n\tmadc.hi.cc.u32 %3, m, %12, %3;\n\tmadc.hi.cc.u32 %4, m, %13, %4;\n\taddc.u32 %5, %5, 0;\n\t}"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(bi), "r"(n0));
}
template <>
__device__ __forceinline__ void mont_sub<4>(const uint32_t (&t)[6], const uint32_t (&p)[4],
                                            uint32_t (&d)[4], uint32_t &top) {
    asm("sub.cc.u32 %0, %5, %10;\n\tsubc.cc.u32 %1, %6, %11;\n\tsubc.cc.u32 %2, %7, %12;\n\tsubc.cc.u32 %3, %8, %13;\n\tsubc.u32 %4, %9, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(top)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]));
}
template <>
__device__ __forceinline__ void mont_step<6>(uint32_t (&t)[8], const uint32_t (&a)[6],
                                             const uint32_t (&p)[6], uint32_t bi, uint32_t n0) {
    asm("{\n\t.reg .u32 m;\n\tmad.lo.cc.u32 %0, %8, %20, %0;\n\tmadc.lo.cc.u32 %1, %9, %20, %1;\n\tmadc.lo.cc.u32 %2, %10, %20, %2;\n\tmadc.lo.cc.u32 %3, %11, %20, %3;\n\tmadc.lo.cc.u32 %4, %12, %20, %4;\n\tmadc.lo.cc.u32 %5, %13, %20, %5;\n\taddc.cc.u32 %6, %6, 0;\n\taddc.u32 %7, %7, 0;\n\tmad.hi.cc.u32 %1, %8, %20, %1;\n\tmadc.hi.cc.u32 %2, %9, %20, %2;\n\tmadc.hi.cc.u32 %3, %10, %20, %3;\n\tmadc.hi.cc.u32 %4, %11, %20, %4;\n\tmadc.hi.cc.u32 %5, %12, %20, %5;\n\tmadc.hi.cc.u32 %6, %13, %20, %6;\n\taddc.u32 %7, %7, 0;\n\tmul.lo.u32 m, %0, %21;\n\tmad.lo.cc.u32 %0, m, %14, %0;\n\tmadc.lo.cc.u32 %1, m, %15, %1;\n\tmadc.lo.cc.u32 %2, m, %16, %2;\n\tmadc.lo.cc.u32 %3, m, %17, %3;\n\tmadc.lo.cc.u32 %4, m, %18, %4;\n\tmadc.lo.cc.u32 %5, m, %19, %5;\n\taddc.cc.u32 %6, %6, 0;\n\taddc.u32 %7, %7, 0;\n\tmad.hi.cc.u32 %1, m, %14, %1;\n\tmadc.hi.cc.u32 %2, m, %15, %2;\n\tmadc.hi.cc.u32 %3, m, %16, %3;\n\tmadc.hi.cc.u32 %4, m, %17, %4;\n\tmadc.hi.cc.u32 %5, m, %18, %5;\n\tmadc.hi.cc.u32 %6, m, %19, %6;\n\taddc.u32 %7, %7, 0;\n\t}"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(bi), "r"(n0));
}
template <>
__device__ __forceinline__ void mont_sub<6>(const uint32_t (&t)[8], const uint32_t (&p)[6],
                                            uint32_t (&d)[6], uint32_t &top) {
    asm("sub.cc.u32 %0, %7, %14;\n\tsubc.cc.u32 %1, %8, %15;\n\tsubc.cc.u32 %2, %9, %16;\n\tsubc.cc.u32 %3, %10, %17;\n\tsubc.cc.u32 %4, %11, %18;\n\tsubc.cc.u32 %5, %12, %19;\n\tsubc.u32 %6, %13, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(top)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]));
}
template <>
__device__ __forceinline__ void mont_step<8>(uint32_t (&t)[10], const uint32_t (&a)[8],
                                             const uint32_t (&p)[8], uint32_t bi, uint32_t n0) {
    asm("{\n\t.reg .u32 m;\n\tmad.lo.cc.u32 %0, %10, %26, %0;\n\tmadc.lo.cc.u32 %1, %11, %26, %1;\n\tmadc.lo.cc.u32 %2, %12, %26, %2;\n\tmadc.lo.cc.u32 %3, %13, %26, %3;\n\tmadc.lo.cc.u32 %4, %14, %26, %4;\n\tmadc.lo.cc.u32 %5, %15, %26, %5;\n\tmadc.lo.cc.u32 %6, %16, %26, %6;\n\tmadc.lo.cc.u32 %7, %17, %26, %7;\n\taddc.cc.u32 %8, %8, 0;\n\taddc.u32 %9, %9, 0;\n\tmad.hi.cc.u32 %1, %10, %26, %1;\n\tmadc.hi.cc.u32 %2, %11, %26, %2;\n\tmadc.hi.cc.u32 %3, %12, %26, %3;\n\tmadc.hi.cc.u32 %4, %13, %26, %4;\n\tmadc.hi.cc.u32 %5, %14, %26, %5;\n\tmadc.hi.cc.u32 %6, %15, %26, %6;\n\tmadc.hi.cc.u32 %7, %16, %26, %7;\n\tmadc.hi.cc.u32 %8, %17, %26, %8;\n\taddc.u32 %9, %9, 0;\n\tmul.lo.u32 m, %0, %27;\n\tmad.lo.cc.u32 %0, m, %18, %0;\n\tmadc.lo.cc.u32 %1, m, %19, %1;\n\tmadc.lo.cc.u32 %2, m, %20, %2;\n\tmadc.lo.cc.u32 %3, m, %21, %3;\n\tmadc.lo.cc.u32 %4, m, %22, %4;\n\tmadc.lo.cc.u32 %5, m, %23, %5;\n\tmadc.lo.cc.u32 %6, m, %24, %6;\n\tmadc.lo.cc.u32 %7, m, %25, %7;\n\taddc.cc.u32 %8, %8, 0;\n\taddc.u32 %9, %9, 0;\n\tmad.hi.cc.u32 %1, m, %18, %1;\n\tmadc.hi.cc.u32 %2, m, %19, %2;\n\tmadc.hi.cc.u32 %3, m, %20, %3;\n\tmadc.hi.cc.u32 %4, m, %21, %4;\n\tmadc.hi.cc.u32 %5, m, %22, %5;\n\tmadc.hi.cc.u32 %6, m, %23, %6;\n\tmadc.hi.cc.u32 %7, m, %24, %7;\n\tmadc.hi.cc.u32 %8, m, %25, %8;\n\taddc.u32 %9, %9, 0;\n\t}"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8]), "+r"(t[9])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]), "r"(bi), "r"(n0));
}
template <>
__device__ __forceinline__ void mont_sub<8>(const uint32_t (&t)[10], const uint32_t (&p)[8],
                                            uint32_t (&d)[8], uint32_t &top) {
    asm("sub.cc.u32 %0, %9, %18;\n\tsubc.cc.u32 %1, %10, %19;\n\tsubc.cc.u32 %2, %11, %20;\n\tsubc.cc.u32 %3, %12, %21;\n\tsubc.cc.u32 %4, %13, %22;\n\tsubc.cc.u32 %5, %14, %23;\n\tsubc.cc.u32 %6, %15, %24;\n\tsubc.cc.u32 %7, %16, %25;\n\tsubc.u32 %8, %17, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(top)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]), "r"(t[8]), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]));
}

// Montgomery product over N 32-bit words, R = 2^(32 N) (CIOS, Koc, Acar and
// Kaliski 1996), with PTX carry chains: per word b_i, the low halves of a*b_i
// are added with one carry chain and the high halves, one word up, with a
// second; the reduction by m*p (m = t_0 * n0 mod 2^32) likewise, then the
// accumulator shifts down one word.  t < 2p throughout for a < R, b < p, so
// one conditional subtraction ends it.
template <int N>
__device__ __forceinline__ void mont_mul32(const uint32_t (&a)[N], const uint32_t (&b)[N],
                                           const uint32_t (&p)[N], uint32_t n0, uint32_t (&out)[N]) {
    uint32_t t[N + 2];
#pragma unroll
    for (int i = 0; i < N + 2; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        mont_step<N>(t, a, p, b[i], n0);
        // t_0 is now zero: shift down one word
#pragma unroll
        for (int j = 0; j <= N; j++) t[j] = t[j + 1];
        t[N + 1] = 0;
    }
    // d = t - p over N + 1 words; keep t if that borrows
    uint32_t d[N], top;
    mont_sub<N>(t, p, d, top);
    const bool keep = (top >> 31) != 0;
#pragma unroll
    for (int j = 0; j < N; j++) out[j] = keep ? t[j] : d[j];
}
#endif

// Montgomery product a*b*R^-1 mod p for a < R, b < p (CIOS).  On the device
// the 32-bit carry-chain form above; on the host 64-bit limbs.
template <int L>
ZG_HD void fmul(const uint64_t *a, const uint64_t *b, const uint64_t *p, uint64_t n0,
                uint64_t *out) {
#ifdef __CUDA_ARCH__
    uint32_t aw[2 * L], bw[2 * L], pw[2 * L], ow[2 * L];
#pragma unroll
    for (int i = 0; i < L; i++) {
        aw[2 * i] = (uint32_t)a[i];
        aw[2 * i + 1] = (uint32_t)(a[i] >> 32);
        bw[2 * i] = (uint32_t)b[i];
        bw[2 * i + 1] = (uint32_t)(b[i] >> 32);
        pw[2 * i] = (uint32_t)p[i];
        pw[2 * i + 1] = (uint32_t)(p[i] >> 32);
    }
    mont_mul32<2 * L>(aw, bw, pw, (uint32_t)n0, ow);
#pragma unroll
    for (int i = 0; i < L; i++) out[i] = (uint64_t)ow[2 * i] | ((uint64_t)ow[2 * i + 1] << 32);
    return;
#else
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
#endif
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
