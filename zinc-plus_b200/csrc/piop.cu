// Zinc+ prover steps 3 and 6 on the trace columns (protocol/src/prover.rs:
// 385-415 and 497-532), the data-parallel parts around the PCS and sumcheck.
//
//  k_eval_proj     step 3, evaluation projection: project_trace_coeffs (a binary
//                  coefficient becomes one or zero, an integer F::from_with_cfg;
//                  piop/src/projections.rs:140-220) then
//                  evaluate_trace_to_column_mles (each polynomial's inner product
//                  with the powers of the projecting element a, :227-301).  A
//                  binary cell is the sum of a^l over its set bits.
//  k_lifted_bin    step 6, lifted evaluations (compute_lifted_evals,
//  k_lifted_int    protocol/src/lib.rs:327-395): coefficient l of binary column c
//                  is sum_b eq(b, r0) [bit l of c[b]]; an integer column's single
//                  coefficient is sum_b eq(b, r0) F(c[b]).  Per-block partial sums,
//                  then k_lifted_reduce.
// Field elements are Montgomery inners (F::Inner of MontyField) of 3 or 4 limbs.
#include <cstring>
#include <vector>

#include "zg_internal.h"

namespace zg {
namespace {

constexpr uint32_t kLiftChunkLog = 12;  // inputs b per block of the lifted sums

// Lazy sums of field elements (each < p < 2^(64L)): 2L 32-bit words plus a
// 32-bit top word, added with one PTX carry chain and no reduction; up to 2^32
// addends cannot overflow.  lazy_reduce brings V = lo + top 2^(64L) to the
// canonical residue with two Montgomery products: lo * (R mod p) R^-1 = lo mod p
// and top * (R^2 mod p) R^-1 = top R mod p (R = 2^(64L); both factors < R).
template <int L>
struct Lazy {
    uint32_t w[2 * L + 1];
};

template <int L>
__device__ __forceinline__ void lazy_zero(Lazy<L> &a) {
#pragma unroll
    for (int i = 0; i < 2 * L + 1; i++) a.w[i] = 0;
}

template <int L>
__device__ __forceinline__ void lazy_add(Lazy<L> &a, const uint64_t *b) {
    uint32_t v[2 * L];
#pragma unroll
    for (int i = 0; i < L; i++) {
        v[2 * i] = (uint32_t)b[i];
        v[2 * i + 1] = (uint32_t)(b[i] >> 32);
    }
    if constexpr (L == 3) {
        asm("add.cc.u32 %0, %0, %7;\n\taddc.cc.u32 %1, %1, %8;\n\taddc.cc.u32 %2, %2, %9;\n\t"
            "addc.cc.u32 %3, %3, %10;\n\taddc.cc.u32 %4, %4, %11;\n\taddc.cc.u32 %5, %5, %12;\n\t"
            "addc.u32 %6, %6, 0;"
            : "+r"(a.w[0]), "+r"(a.w[1]), "+r"(a.w[2]), "+r"(a.w[3]), "+r"(a.w[4]), "+r"(a.w[5]), "+r"(a.w[6])
            : "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]));
    } else {
        static_assert(L == 4, "lazy sums are for 3- or 4-limb fields");
        asm("add.cc.u32 %0, %0, %9;\n\taddc.cc.u32 %1, %1, %10;\n\taddc.cc.u32 %2, %2, %11;\n\t"
            "addc.cc.u32 %3, %3, %12;\n\taddc.cc.u32 %4, %4, %13;\n\taddc.cc.u32 %5, %5, %14;\n\t"
            "addc.cc.u32 %6, %6, %15;\n\taddc.cc.u32 %7, %7, %16;\n\taddc.u32 %8, %8, 0;"
            : "+r"(a.w[0]), "+r"(a.w[1]), "+r"(a.w[2]), "+r"(a.w[3]), "+r"(a.w[4]), "+r"(a.w[5]), "+r"(a.w[6]),
              "+r"(a.w[7]), "+r"(a.w[8])
            : "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]));
    }
}

// a += b for two lazy sums (reductions; the top words stay far below 2^32).
template <int L>
__device__ __forceinline__ void lazy_merge(Lazy<L> &a, const Lazy<L> &b) {
    uint64_t c = 0;
#pragma unroll
    for (int i = 0; i < 2 * L + 1; i++) {
        const uint64_t t = (uint64_t)a.w[i] + b.w[i] + c;
        a.w[i] = (uint32_t)t;
        c = t >> 32;
    }
}

// Canonical residue of a lazy sum below 8p: subtract 4p, 2p, p where they fit
// (pm[k] = p << k as 2L + 1 words, k = 0..2).
template <int L>
__device__ __forceinline__ void lazy_reduce_small(const Lazy<L> &a, const uint32_t (*pm)[2 * L + 1],
                                                  uint64_t *out) {
    uint32_t v[2 * L + 1];
#pragma unroll
    for (int i = 0; i < 2 * L + 1; i++) v[i] = a.w[i];
#pragma unroll
    for (int k = 2; k >= 0; k--) {
        uint32_t t[2 * L + 1];
        uint64_t br = 0;
#pragma unroll
        for (int i = 0; i < 2 * L + 1; i++) {
            const uint64_t d = (uint64_t)v[i] - pm[k][i] - br;
            t[i] = (uint32_t)d;
            br = (d >> 32) & 1u;
        }
#pragma unroll
        for (int i = 0; i < 2 * L + 1; i++) v[i] = br ? v[i] : t[i];
    }
#pragma unroll
    for (int i = 0; i < L; i++) out[i] = (uint64_t)v[2 * i] | ((uint64_t)v[2 * i + 1] << 32);
}

template <int L>
__device__ __forceinline__ void lazy_reduce(const Lazy<L> &a, const FieldCfg &f, uint64_t *out) {
    uint64_t lo[L], hi[L], t[L];
#pragma unroll
    for (int i = 0; i < L; i++) {
        lo[i] = (uint64_t)a.w[2 * i] | ((uint64_t)a.w[2 * i + 1] << 32);
        hi[i] = i == 0 ? a.w[2 * L] : 0;
    }
    fmul<L>(lo, f.one, f.p, f.n0, out);
    fmul<L>(hi, f.r2, f.p, f.n0, t);
    fadd<L>(out, t, f.p);
}

// Byte tables of the powers of a: tab[j][v] = sum of a^(8j + i) over the set
// bits i of v (8j + i < D), canonical.  One thread per (j, v).
template <int L>
__global__ void k_pow_tables(const uint64_t *__restrict__ pw, uint32_t D, FieldCfg f, uint64_t *__restrict__ tab) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x, nbytes = (D + 7) / 8;
    if (e >= nbytes * 256) return;
    const uint32_t j = e >> 8, v = e & 255u;
    uint64_t acc[L];
#pragma unroll
    for (int k = 0; k < L; k++) acc[k] = 0;
    for (uint32_t i = 0; i < 8; i++)
        if (((v >> i) & 1u) && 8 * j + i < D) fadd<L>(acc, pw + (size_t)(8 * j + i) * L, f.p);
#pragma unroll
    for (int k = 0; k < L; k++) tab[(size_t)e * L + k] = acc[k];
}

// One cell per thread (grid-stride): a binary cell is the sum of ceil(D/8)
// table entries (a lazy sum below 8p, then three conditional subtractions); an
// integer cell is F::from_with_cfg of the value.
template <int L>
__global__ void __launch_bounds__(256) k_eval_proj(const uint64_t *__restrict__ bin, uint32_t n_bin,
                                                   uint64_t dmask, const int64_t *__restrict__ ints,
                                                   uint32_t n_int, uint32_t nv,
                                                   const uint64_t *__restrict__ tab, uint32_t D, FieldCfg f,
                                                   uint64_t *__restrict__ out) {
    // dynamic shared memory only (the kernel may take the device's whole
    // opt-in limit): [ceil(D/8)][256][L] table words, then p, 2p, 4p
    extern __shared__ uint64_t stab[];
    const uint32_t nbytes = (D + 7) / 8;
    uint32_t(*pm)[2 * L + 1] = reinterpret_cast<uint32_t(*)[2 * L + 1]>(stab + (size_t)nbytes * 256 * L);
    for (uint32_t i = threadIdx.x; i < nbytes * 256 * L; i += blockDim.x) stab[i] = tab[i];
    if (threadIdx.x < 3) {
        uint32_t c = 0;
        for (int i = 0; i < 2 * L; i++) {
            const uint32_t w = (uint32_t)(f.p[i / 2] >> (32 * (i & 1)));
            pm[threadIdx.x][i] = (w << threadIdx.x) | c;
            c = threadIdx.x ? w >> (32 - threadIdx.x) : 0u;
        }
        pm[threadIdx.x][2 * L] = c;
    }
    __syncthreads();
    const size_t total = (size_t)(n_bin + n_int) << nv, nbin_cells = (size_t)n_bin << nv;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        uint64_t acc[L];
        if (e < nbin_cells) {
            const uint64_t x = bin[e] & dmask;
            Lazy<L> z;
            lazy_zero(z);
            for (uint32_t j = 0; j < nbytes; j++) lazy_add<L>(z, stab + ((size_t)j * 256 + ((x >> (8 * j)) & 255u)) * L);
            lazy_reduce_small<L>(z, pm, acc);
        } else {
            const int64_t v = ints[e - nbin_cells];
            const uint64_t w2[2] = {(uint64_t)v, v < 0 ? ~0ull : 0ull};
            from_signed<L>(w2, 2, f, acc);
        }
#pragma unroll
        for (int w = 0; w < L; w++) out[e * L + w] = acc[w];
    }
}

// Block (LB lanes, 256 / LB rows): column blockIdx.y, inputs b of chunk
// blockIdx.x; thread (l, w) adds eq[b] for b = chunk start + w, + rows, ...
// when bit l of the cell is set.  partials: [column][chunk][LB][L].
template <int L, int LB>
__global__ void __launch_bounds__(256) k_lifted_bin(const uint64_t *__restrict__ bin, uint32_t nv,
                                                    uint64_t dmask, const uint64_t *__restrict__ eq, FieldCfg f,
                                                    uint64_t *__restrict__ partials) {
    __shared__ Lazy<L> red[256];
    // a tile of 256 inputs: their cells and eq entries, loaded coalesced, then
    // read by every lane as shared-memory broadcasts (one load per warp and
    // input from L2 left the kernel waiting: 15 long-scoreboard stalls per issue)
    constexpr uint32_t kTile = 256;
    __shared__ uint64_t sx[kTile];
    __shared__ uint64_t se[kTile * L];
    const uint32_t l = threadIdx.x, w = threadIdx.y, rows = blockDim.y;
    const uint32_t tid = w * LB + l, nthr = LB * rows;
    const size_t n = (size_t)1 << nv, b0 = (size_t)blockIdx.x << kLiftChunkLog;
    const size_t b1 = b0 + ((size_t)1 << kLiftChunkLog) < n ? b0 + ((size_t)1 << kLiftChunkLog) : n;
    const uint64_t *col = bin + ((size_t)blockIdx.y << nv);
    Lazy<L> acc;
    lazy_zero(acc);
    for (size_t tb = b0; tb < b1; tb += kTile) {
        const uint32_t cnt = b1 - tb < kTile ? (uint32_t)(b1 - tb) : kTile;
        for (uint32_t i = tid; i < cnt; i += nthr) sx[i] = col[tb + i] & dmask;
        for (uint32_t i = tid; i < cnt * L; i += nthr) se[i] = eq[tb * L + i];
        __syncthreads();
        uint32_t j = w;
        for (; j + 7 * rows < cnt; j += 8 * rows)
#pragma unroll
            for (int u = 0; u < 8; u++)
                if ((sx[j + u * rows] >> l) & 1u) lazy_add<L>(acc, se + (size_t)(j + u * rows) * L);
        for (; j < cnt; j += rows)
            if ((sx[j] >> l) & 1u) lazy_add<L>(acc, se + (size_t)j * L);
        __syncthreads();
    }
    const uint32_t t = w * LB + l;
    red[t] = acc;
    __syncthreads();
    for (uint32_t h = rows / 2; h > 0; h >>= 1) {
        if (w < h) lazy_merge<L>(red[t], red[t + h * LB]);
        __syncthreads();
    }
    if (w == 0) {
        uint32_t *po = reinterpret_cast<uint32_t *>(partials) +
                       (((size_t)blockIdx.y * gridDim.x + blockIdx.x) * LB + l) * (2 * L + 2);
#pragma unroll
        for (int k = 0; k < 2 * L + 1; k++) po[k] = red[l].w[k];
        po[2 * L + 1] = 0;
    }
}

// Integer columns: 256 threads per chunk, partials [column][chunk][L].
template <int L>
__global__ void __launch_bounds__(256) k_lifted_int(const int64_t *__restrict__ ints, uint32_t nv,
                                                    const uint64_t *__restrict__ eq, FieldCfg f,
                                                    uint64_t *__restrict__ partials) {
    __shared__ uint64_t red[256 * L];
    const size_t n = (size_t)1 << nv, b0 = (size_t)blockIdx.x << kLiftChunkLog;
    const size_t b1 = b0 + ((size_t)1 << kLiftChunkLog) < n ? b0 + ((size_t)1 << kLiftChunkLog) : n;
    const int64_t *col = ints + ((size_t)blockIdx.y << nv);
    uint64_t acc[L];
#pragma unroll
    for (int k = 0; k < L; k++) acc[k] = 0;
    for (size_t b = b0 + threadIdx.x; b < b1; b += blockDim.x) {
        const int64_t v = col[b];
        const uint64_t w2[2] = {(uint64_t)v, v < 0 ? ~0ull : 0ull};
        uint64_t fv[L], t[L];
        from_signed<L>(w2, 2, f, fv);
        fmul<L>(fv, eq + b * L, f.p, f.n0, t);
        fadd<L>(acc, t, f.p);
    }
#pragma unroll
    for (int k = 0; k < L; k++) red[threadIdx.x * L + k] = acc[k];
    __syncthreads();
    for (uint32_t h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) fadd<L>(red + threadIdx.x * L, red + (threadIdx.x + h) * L, f.p);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        uint64_t *po = partials + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * L;
#pragma unroll
        for (int k = 0; k < L; k++) po[k] = red[k];
    }
}

// eq(b, r) over nv variables as lo[b mod 2^a] * hi[b >> a] (a = nv / 2): the
// half tables over the first a and the last nv - a variables first (one thread
// per entry, a chain of at most 14 products), then one product per entry.
// Field products are exact, so the grouping does not change any value.
template <int L>
__global__ void k_eq_halves(const uint64_t *__restrict__ r, const uint64_t *__restrict__ omr, uint32_t nv,
                            FieldCfg f, uint64_t *__restrict__ halves) {
    const uint32_t a = nv / 2, na = 1u << a, nb = 1u << (nv - a);
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= na + nb) return;
    const bool hi = e >= na;
    const uint32_t idx = hi ? e - na : e, k0 = hi ? a : 0, kn = hi ? nv - a : a;
    uint64_t acc[L];
#pragma unroll
    for (int w = 0; w < L; w++) acc[w] = f.one[w];
    for (uint32_t k = 0; k < kn; k++) {
        const uint64_t *sel = ((idx >> k) & 1u) ? r + (size_t)(k0 + k) * L : omr + (size_t)(k0 + k) * L;
        uint64_t t[L];
        fmul<L>(acc, sel, f.p, f.n0, t);
#pragma unroll
        for (int w = 0; w < L; w++) acc[w] = t[w];
    }
#pragma unroll
    for (int w = 0; w < L; w++) halves[(size_t)e * L + w] = acc[w];
}

template <int L>
__global__ void __launch_bounds__(256) k_eq_outer(const uint64_t *__restrict__ halves, uint32_t nv, FieldCfg f,
                                                  uint64_t *__restrict__ eq) {
    const uint32_t a = nv / 2, na = 1u << a;
    const size_t n = (size_t)1 << nv;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint64_t t[L];
        fmul<L>(halves + (i & (na - 1)) * L, halves + (na + (i >> a)) * L, f.p, f.n0, t);
#pragma unroll
        for (int w = 0; w < L; w++) eq[i * L + w] = t[w];
    }
}

// out[o] = sum over `chunks` partials of slot o (slots: stride `width`).
// lazy: the partials are lazy sums (2L + 2 words each, the last zero), else
// canonical field elements (L words).
template <int L>
__global__ void k_lifted_reduce(const uint64_t *__restrict__ partials, uint32_t nslots, uint32_t chunks,
                                uint32_t width, bool lazy, FieldCfg f, uint64_t *__restrict__ out) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nslots) return;
    const uint32_t col = o / width, lane = o % width;
    uint64_t acc[L];
    if (lazy) {
        Lazy<L> z, q;
        lazy_zero(z);
        for (uint32_t c = 0; c < chunks; c++) {
            const uint32_t *pq = reinterpret_cast<const uint32_t *>(partials) +
                                 (((size_t)col * chunks + c) * width + lane) * (2 * L + 2);
#pragma unroll
            for (int k = 0; k < 2 * L + 1; k++) q.w[k] = pq[k];
            lazy_merge<L>(z, q);
        }
        lazy_reduce<L>(z, f, acc);
    } else {
#pragma unroll
        for (int k = 0; k < L; k++) acc[k] = 0;
        for (uint32_t c = 0; c < chunks; c++)
            fadd<L>(acc, partials + (((size_t)col * chunks + c) * width + lane) * L, f.p);
    }
#pragma unroll
    for (int k = 0; k < L; k++) out[(size_t)o * L + k] = acc[k];
}

// precombined[b] = sum_j gamma_j v_j[b] (multipoint_eval.rs:160-182): one
// product per column, summed lazily, one reduction per entry.
template <int L>
__global__ void __launch_bounds__(256) k_precombine(const uint64_t *__restrict__ mles, uint32_t ncols, uint32_t nv,
                                                    const uint64_t *__restrict__ gammas, FieldCfg f,
                                                    uint64_t *__restrict__ out) {
    const size_t n = (size_t)1 << nv;
    for (size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x; b < n; b += (size_t)gridDim.x * blockDim.x) {
        Lazy<L> z;
        lazy_zero(z);
        for (uint32_t j = 0; j < ncols; j++) {
            uint64_t t[L];
            fmul<L>(gammas + (size_t)j * L, mles + (((size_t)j << nv) + b) * L, f.p, f.n0, t);
            lazy_add<L>(z, t);
        }
        uint64_t r[L];
        lazy_reduce<L>(z, f, r);
#pragma unroll
        for (int w = 0; w < L; w++) out[b * L + w] = r[w];
    }
}

// out[b] = sum_{e < count} weights[e] * mles[idx[e]][b]: a combination of a few
// columns, without visiting the columns whose weight is zero.
template <int L>
__global__ void __launch_bounds__(256) k_precombine_sparse(const uint64_t *__restrict__ mles, uint32_t nv,
                                                           const uint32_t *__restrict__ idx,
                                                           const uint64_t *__restrict__ weights, uint32_t count,
                                                           FieldCfg f, uint64_t *__restrict__ out) {
    const size_t n = (size_t)1 << nv;
    for (size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x; b < n; b += (size_t)gridDim.x * blockDim.x) {
        Lazy<L> z;
        lazy_zero(z);
        for (uint32_t e = 0; e < count; e++) {
            uint64_t t[L];
            fmul<L>(weights + (size_t)e * L, mles + (((size_t)idx[e] << nv) + b) * L, f.p, f.n0, t);
            lazy_add<L>(z, t);
        }
        uint64_t r[L];
        lazy_reduce<L>(z, f, r);
#pragma unroll
        for (int w = 0; w < L; w++) out[b * L + w] = r[w];
    }
}

// partials[k][blockIdx.x] = sum over this block's share of b of eq[b] * mles[k][b]
// (grid: (blocks per MLE, MLEs)); lazy sums, one reduction per block.
template <int L>
__global__ void __launch_bounds__(256) k_mle_dots(const uint64_t *__restrict__ mles, uint32_t nv,
                                                  const uint64_t *__restrict__ eq, FieldCfg f,
                                                  uint64_t *__restrict__ partials) {
    __shared__ Lazy<L> red[256];
    const size_t n = (size_t)1 << nv;
    const uint64_t *v = mles + ((size_t)blockIdx.y << nv) * L;
    Lazy<L> z;
    lazy_zero(z);
    for (size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x; b < n; b += (size_t)gridDim.x * blockDim.x) {
        uint64_t t[L];
        fmul<L>(eq + b * L, v + b * L, f.p, f.n0, t);
        lazy_add<L>(z, t);
    }
    red[threadIdx.x] = z;
    __syncthreads();
    for (unsigned h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) lazy_merge<L>(red[threadIdx.x], red[threadIdx.x + h]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        uint64_t r[L];
        lazy_reduce<L>(red[0], f, r);
#pragma unroll
        for (int w = 0; w < L; w++) partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * L + w] = r[w];
    }
}

// Step 2 on the combined path for a term that multiplies two columns
// (compute_combined_polynomials, ideal_check/combined_poly_builder.rs:30-95):
// coefficient m (blockIdx.y) of the product polynomial at row b, times eq[b],
// summed over the rows b < 2^nv - 1 (the last row is zero).  Binary x binary:
// the coefficient is the count of bit pairs i + j = m, one popcount of u and
// the bit-reversed w shifted into place, times the table small[count] = F(count);
// binary x integer: F(y) where bit m is set; integer x integer: F(x) F(y) at m = 0.
// partials[m][block]: lazy sums reduced once per block.
template <int L>
__global__ void __launch_bounds__(256) k_ic_product(IcFactor fa, IcFactor fb, uint64_t dmask, uint32_t nv,
                                                    const uint64_t *__restrict__ eq,
                                                    const uint64_t *__restrict__ small, FieldCfg f,
                                                    uint64_t *__restrict__ partials) {
    __shared__ Lazy<L> red[256];
    const size_t n = (size_t)1 << nv;
    const uint32_t m = blockIdx.y;
    Lazy<L> z;
    lazy_zero(z);
    for (size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x; b + 1 < n; b += (size_t)gridDim.x * blockDim.x) {
        const size_t ra = b + fa.shift, rb = b + fb.shift;
        uint64_t t[L];
        if (fa.bin && fb.bin) {
            const uint64_t u = ra < n ? fa.bin[ra] & dmask : 0, w = rb < n ? fb.bin[rb] & dmask : 0;
            const uint64_t rw = __brevll(w);
            const uint64_t sh = m <= 63 ? (rw >> (63 - m)) : (rw << (m - 63));
            const int cnt = __popcll(u & sh);
            if (!cnt) continue;
            fmul<L>(small + (size_t)cnt * L, eq + b * L, f.p, f.n0, t);
        } else if (fa.bin || fb.bin) {
            const IcFactor &fbin = fa.bin ? fa : fb, &fint = fa.bin ? fb : fa;
            const size_t rbin = fa.bin ? ra : rb, rint = fa.bin ? rb : ra;
            const uint64_t u = rbin < n ? fbin.bin[rbin] & dmask : 0;
            if (!((u >> m) & 1)) continue;
            const int64_t y = rint < n ? fint.ints[rint] : 0;
            if (!y) continue;
            uint64_t fy[L];
            from_i128<L>((i128)y, f, fy);
            fmul<L>(fy, eq + b * L, f.p, f.n0, t);
        } else {
            const int64_t x = ra < n ? fa.ints[ra] : 0, y = rb < n ? fb.ints[rb] : 0;
            if (!x || !y) continue;
            uint64_t fx[L], fy[L], xy[L];
            from_i128<L>((i128)x, f, fx);
            from_i128<L>((i128)y, f, fy);
            fmul<L>(fx, fy, f.p, f.n0, xy);
            fmul<L>(xy, eq + b * L, f.p, f.n0, t);
        }
        lazy_add<L>(z, t);
    }
    red[threadIdx.x] = z;
    __syncthreads();
    for (unsigned h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) lazy_merge<L>(red[threadIdx.x], red[threadIdx.x + h]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        uint64_t r[L];
        lazy_reduce<L>(red[0], f, r);
#pragma unroll
        for (int w = 0; w < L; w++) partials[((size_t)m * gridDim.x + blockIdx.x) * L + w] = r[w];
    }
}

struct PiopCols {
    const uint64_t *bin;
    uint32_t n_bin, D;
    const int64_t *ints;
    uint32_t n_int, nv;
};

// Device views of the columns: the caller's device pointers, or copies at
// the start of `arena` (host columns).  Returns the bytes used.
size_t stage_cols(const PiopCols &c, int on_device, cudaStream_t s, uint8_t *arena, const uint64_t *&bin,
                  const int64_t *&ints, zg_status &st) {
    st = ZG_OK;
    if (on_device) {
        bin = c.bin;
        ints = c.ints;
        return 0;
    }
    const size_t n = (size_t)1 << c.nv, bb = (size_t)c.n_bin * n * 8, ib = (size_t)c.n_int * n * 8;
    if ((bb && cudaMemcpyAsync(arena, c.bin, bb, cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        (ib && cudaMemcpyAsync(arena + bb, c.ints, ib, cudaMemcpyHostToDevice, s) != cudaSuccess)) {
        set_error("piop: copying the columns to the device failed");
        st = ZG_ERR_CUDA;
    }
    bin = reinterpret_cast<const uint64_t *>(arena);
    ints = reinterpret_cast<const int64_t *>(arena + bb);
    return bb + ib;
}

size_t staged_bytes(const PiopCols &c, int on_device) {
    return on_device ? 0 : ((size_t)c.n_bin + c.n_int) * ((size_t)8 << c.nv);
}

template <int L>
zg_status eval_projection_t(zg_ctx *ctx, const FieldCfg &f, const PiopCols &c, const uint64_t *a, int on_device,
                            uint64_t *out) {
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)1 << c.nv, fb = 8 * L, cells = (size_t)(c.n_bin + c.n_int) * n;
    std::vector<uint64_t> pw((size_t)64 * L, 0);
    std::memcpy(pw.data(), f.one, fb);
    for (uint32_t l = 1; l < c.D; l++) fmul<L>(&pw[(size_t)(l - 1) * L], a, f.p, f.n0, &pw[(size_t)l * L]);
    const uint32_t nbytes = (c.D + 7) / 8;
    const size_t tab_bytes = (size_t)nbytes * 256 * fb;
    const size_t sb = (staged_bytes(c, on_device) + 255) / 256 * 256;
    ZG_TRY(ctx->sc_arena.ensure(sb + 64 * fb + tab_bytes + (on_device ? 0 : cells * fb)));
    uint8_t *arena = ctx->sc_arena.as<uint8_t>();
    const uint64_t *bin_d;
    const int64_t *ints_d;
    zg_status sst;
    stage_cols(c, on_device, s, arena, bin_d, ints_d, sst);
    ZG_TRY(sst);
    uint64_t *pw_d = reinterpret_cast<uint64_t *>(arena + sb), *tab_d = pw_d + 64 * L;
    uint64_t *out_d = on_device ? out : tab_d + (size_t)nbytes * 256 * L;
    ZG_CUDA(cudaMemcpyAsync(pw_d, pw.data(), 64 * fb, cudaMemcpyHostToDevice, s));
    const uint64_t dmask = c.D >= 64 ? ~0ull : ((1ull << c.D) - 1);
    const unsigned blocks = (unsigned)std::min<size_t>((cells + 255) / 256, (size_t)ctx->num_sms * 8);
    if (cells) {
        ZG_KBEGIN(ctx, s, "k_pow_tables");
        k_pow_tables<L><<<(nbytes * 256 + 255) / 256, 256, 0, s>>>(pw_d, c.D, f, tab_d);
        ZG_KEND(ctx, s);
        if (tab_bytes + 3 * (2 * L + 1) * 4 > 48 * 1024) ZG_CUDA(allow_max_smem(k_eval_proj<L>));
        ZG_KBEGIN(ctx, s, "k_eval_proj");
        k_eval_proj<L><<<blocks, 256, tab_bytes + 3 * (2 * L + 1) * 4, s>>>(bin_d, c.n_bin, dmask, ints_d, c.n_int,
                                                                            c.nv, tab_d, c.D, f, out_d);
        ZG_KEND(ctx, s);
    }
    if (!on_device) ZG_CUDA(cudaMemcpyAsync(out, out_d, cells * fb, cudaMemcpyDeviceToHost, s));
    ZG_CUDA(ctx_sync(ctx));
    return ZG_OK;
}

template <int L>
zg_status lifted_evals_t(zg_ctx *ctx, const FieldCfg &f, const PiopCols &c, const uint64_t *point,
                         int on_device, uint64_t *out) {
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)1 << c.nv, fb = 8 * L;
    const uint32_t LB = c.D > 32 ? 64 : 32;
    const uint32_t chunks = (uint32_t)((n + (1u << kLiftChunkLog) - 1) >> kLiftChunkLog);
    std::vector<uint64_t> omr((size_t)std::max<uint32_t>(c.nv, 1) * L, 0);
    for (uint32_t k = 0; k < c.nv; k++) {
        std::memcpy(&omr[(size_t)k * L], f.one, fb);
        fsub<L>(&omr[(size_t)k * L], point + (size_t)k * L, f.p);
    }
    const size_t nv1 = std::max<uint32_t>(c.nv, 1);
    const size_t pb = (size_t)c.n_bin * chunks * LB * (fb + 8) + (size_t)c.n_int * chunks * fb;
    const size_t ob = ((size_t)c.n_bin * LB + c.n_int) * fb;
    const size_t sb = (staged_bytes(c, on_device) + 255) / 256 * 256;
    const size_t halves = ((size_t)1 << (c.nv / 2)) + ((size_t)1 << (c.nv - c.nv / 2));
    ZG_TRY(ctx->sc_arena.ensure(sb + 2 * nv1 * fb + n * fb + pb + ob + halves * fb + 64));
    uint8_t *arena = ctx->sc_arena.as<uint8_t>();
    const uint64_t *bin_d;
    const int64_t *ints_d;
    zg_status sst;
    stage_cols(c, on_device, s, arena, bin_d, ints_d, sst);
    ZG_TRY(sst);
    uint64_t *r_d = reinterpret_cast<uint64_t *>(arena + sb), *omr_d = r_d + nv1 * L, *eq_d = omr_d + nv1 * L;
    uint64_t *part_d = eq_d + n * L, *res_d = part_d + pb / 8;
    ZG_CUDA(cudaMemcpyAsync(r_d, point, (size_t)c.nv * fb, cudaMemcpyHostToDevice, s));
    ZG_CUDA(cudaMemcpyAsync(omr_d, omr.data(), (size_t)c.nv * fb, cudaMemcpyHostToDevice, s));
    uint64_t *half_d = res_d + ob / 8;
    ZG_KBEGIN(ctx, s, "k_eq_halves");
    k_eq_halves<L><<<(unsigned)((halves + 127) / 128), 128, 0, s>>>(r_d, omr_d, c.nv, f, half_d);
    ZG_KEND(ctx, s);
    ZG_KBEGIN(ctx, s, "k_eq_outer");
    k_eq_outer<L><<<(unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8), 256, 0, s>>>(
        half_d, c.nv, f, eq_d);
    ZG_KEND(ctx, s);
    const uint64_t dmask = c.D >= 64 ? ~0ull : ((1ull << c.D) - 1);
    uint64_t *part_int = part_d + (size_t)c.n_bin * chunks * LB * (L + 1);
    uint64_t *res_int = res_d + (size_t)c.n_bin * LB * L;
    if (c.n_bin) {
        ZG_KBEGIN(ctx, s, "k_lifted_bin");
        dim3 g(chunks, c.n_bin);
        if (LB == 64)
            k_lifted_bin<L, 64><<<g, dim3(64, 4), 0, s>>>(bin_d, c.nv, dmask, eq_d, f, part_d);
        else
            k_lifted_bin<L, 32><<<g, dim3(32, 8), 0, s>>>(bin_d, c.nv, dmask, eq_d, f, part_d);
        ZG_KEND(ctx, s);
        ZG_KBEGIN(ctx, s, "k_lifted_reduce");
        const uint32_t slots = c.n_bin * LB;
        k_lifted_reduce<L><<<(slots + 127) / 128, 128, 0, s>>>(part_d, slots, chunks, LB, true, f, res_d);
        ZG_KEND(ctx, s);
    }
    if (c.n_int) {
        ZG_KBEGIN(ctx, s, "k_lifted_int");
        k_lifted_int<L><<<dim3(chunks, c.n_int), 256, 0, s>>>(ints_d, c.nv, eq_d, f, part_int);
        ZG_KEND(ctx, s);
        ZG_KBEGIN(ctx, s, "k_lifted_reduce");
        k_lifted_reduce<L><<<(c.n_int + 127) / 128, 128, 0, s>>>(part_int, c.n_int, chunks, 1, false, f, res_int);
        ZG_KEND(ctx, s);
    }
    std::vector<uint64_t> res(((size_t)c.n_bin * LB + c.n_int) * L);
    if (!res.empty()) ZG_CUDA(cudaMemcpyAsync(res.data(), res_d, res.size() * 8, cudaMemcpyDeviceToHost, s));
    ZG_CUDA(ctx_sync(ctx));
    for (uint32_t col = 0; col < c.n_bin; col++)
        std::memcpy(out + (size_t)col * c.D * L, &res[(size_t)col * LB * L], (size_t)c.D * fb);
    if (c.n_int)
        std::memcpy(out + (size_t)c.n_bin * c.D * L, &res[(size_t)c.n_bin * LB * L], (size_t)c.n_int * fb);
    return ZG_OK;
}

zg_status piop_args(zg_ctx *ctx, const uint8_t *modulus, uint32_t limbs, const PiopCols &c,
                    const uint64_t *elems, const void *out, FieldCfg &f) {
    if (!ctx || !modulus || !elems || !out || (c.n_bin && !c.bin) || (c.n_int && !c.ints)) {
        set_error("piop: null argument");
        return ZG_ERR_INVALID_PARAM;
    }
    if (limbs != 3 && limbs != 4) {
        set_error("piop: field limbs must be 3 or 4 (got %u)", limbs);
        return ZG_ERR_INVALID_PARAM;
    }
    if (c.nv > 28 || (c.n_bin && (c.D < 1 || c.D > 64)) || (size_t)c.n_bin + c.n_int > 4096) {
        set_error("piop: num_vars above 28, BinaryPoly width outside 1..64 or more than 4096 columns");
        return ZG_ERR_INVALID_PARAM;
    }
    uint64_t p[4] = {0, 0, 0, 0};
    std::memcpy(p, modulus, 8 * limbs);
    if (!(p[0] & 1)) {
        set_error("piop: the modulus must be odd");
        return ZG_ERR_INVALID_PARAM;
    }
    field_cfg_init(f, p, (int)limbs);
    return ZG_OK;
}

// get_field_challenge (transcript/src/traits.rs:333-340): the inner's bytes
// from the XOF, F::new_with_cfg (to Montgomery form).
template <int L>
void field_challenge_h(zg_transcript *t, const FieldCfg &f, uint64_t *out) {
    uint8_t b[8 * L];
    tr_challenge(t, b, sizeof b);
    uint64_t x[L];
    std::memcpy(x, b, sizeof b);
    fmul<L>(x, f.r2, f.p, f.n0, out);
}

// Step 5 up to the sumcheck: challenges, then the packed MLEs
// [eq_r, next_1 .. next_S, precombined, down_1 .. down_S] in ctx->piop_arena.
template <int L>
zg_status multipoint_prepare(zg_ctx *ctx, zg_transcript *t, const FieldCfg &f, const uint64_t *trace,
                             uint32_t ncols, uint32_t nv, const uint64_t *point, const uint32_t *src,
                             const uint32_t *shift, uint32_t S, int on_device, uint32_t *n_amounts,
                             uint64_t **packed) {
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)1 << nv, fb = 8 * L, mle = n * fb;
    std::vector<uint64_t> alphas((size_t)S * L, 0), gammas((size_t)ncols * L);
    for (uint32_t k = 0; k < S; k++) field_challenge_h<L>(t, f, &alphas[(size_t)k * L]);
    for (uint32_t j = 0; j < ncols; j++) field_challenge_h<L>(t, f, &gammas[(size_t)j * L]);
    // sum_k alpha_k next_{c_k} v_{src_k} = sum_c next_c (sum_{k: c_k = c} alpha_k v_{src_k}):
    // one selector and one weighted column combination per distinct shift amount.
    // Each combination is kept sparse: its distinct source columns and their
    // summed alphas, stored amount by amount (at most S entries in all).
    std::vector<uint32_t> amounts;
    std::vector<std::vector<uint32_t>> srcs;
    std::vector<std::vector<uint64_t>> wts;
    for (uint32_t k = 0; k < S; k++) {
        uint32_t m = 0;
        while (m < amounts.size() && amounts[m] != shift[k]) m++;
        if (m == amounts.size()) {
            amounts.push_back(shift[k]);
            srcs.emplace_back();
            wts.emplace_back();
        }
        uint32_t e = 0;
        while (e < srcs[m].size() && srcs[m][e] != src[k]) e++;
        if (e == srcs[m].size()) {
            srcs[m].push_back(src[k]);
            wts[m].resize(wts[m].size() + L, 0);
        }
        fadd<L>(&wts[m][(size_t)e * L], &alphas[(size_t)k * L], f.p);
    }
    const uint32_t M = (uint32_t)amounts.size();
    std::vector<uint32_t> sp_idx, sp_off(M + 1, 0);
    std::vector<uint64_t> sp_w;
    for (uint32_t m = 0; m < M; m++) {
        sp_idx.insert(sp_idx.end(), srcs[m].begin(), srcs[m].end());
        sp_w.insert(sp_w.end(), wts[m].begin(), wts[m].end());
        sp_off[m + 1] = (uint32_t)sp_idx.size();
    }
    const size_t nsp = sp_idx.size();
    *n_amounts = M;
    std::vector<uint64_t> omr((size_t)nv * L);
    for (uint32_t k = 0; k < nv; k++) {
        std::memcpy(&omr[(size_t)k * L], f.one, fb);
        fsub<L>(&omr[(size_t)k * L], point + (size_t)k * L, f.p);
    }
    const size_t halves = ((size_t)1 << (nv / 2)) + ((size_t)1 << (nv - nv / 2));
    const size_t npk = 2 + 2 * (size_t)M;
    const size_t staged = on_device ? 0 : (size_t)ncols * mle;
    const size_t small = (2 * (size_t)nv + halves + ncols + nsp) * fb + nsp * 4;
    ZG_TRY(ctx->piop_arena.ensure(npk * mle + staged + small + 256));
    uint8_t *ar = ctx->piop_arena.as<uint8_t>();
    uint64_t *pk = reinterpret_cast<uint64_t *>(ar);
    const uint64_t *tr = on_device ? trace : reinterpret_cast<const uint64_t *>(ar + npk * mle);
    uint64_t *r_d = reinterpret_cast<uint64_t *>(ar + npk * mle + staged), *omr_d = r_d + (size_t)nv * L;
    uint64_t *half_d = omr_d + (size_t)nv * L, *gam_d = half_d + halves * L, *wgt_d = gam_d + (size_t)ncols * L;
    if (!on_device) ZG_CUDA(cudaMemcpyAsync(const_cast<uint64_t *>(tr), trace, staged, cudaMemcpyHostToDevice, s));
    ZG_CUDA(cudaMemcpyAsync(r_d, point, (size_t)nv * fb, cudaMemcpyHostToDevice, s));
    ZG_CUDA(cudaMemcpyAsync(omr_d, omr.data(), (size_t)nv * fb, cudaMemcpyHostToDevice, s));
    ZG_CUDA(cudaMemcpyAsync(gam_d, gammas.data(), (size_t)ncols * fb, cudaMemcpyHostToDevice, s));
    uint32_t *idx_d = reinterpret_cast<uint32_t *>(wgt_d + nsp * L);
    if (nsp) {
        ZG_CUDA(cudaMemcpyAsync(wgt_d, sp_w.data(), nsp * fb, cudaMemcpyHostToDevice, s));
        ZG_CUDA(cudaMemcpyAsync(idx_d, sp_idx.data(), nsp * 4, cudaMemcpyHostToDevice, s));
    }
    uint64_t *eq = pk;  // MLE 0
    ZG_KBEGIN(ctx, s, "k_eq_halves");
    k_eq_halves<L><<<(unsigned)((halves + 127) / 128), 128, 0, s>>>(r_d, omr_d, nv, f, half_d);
    ZG_KEND(ctx, s);
    const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8);
    ZG_KBEGIN(ctx, s, "k_eq_outer");
    k_eq_outer<L><<<grid, 256, 0, s>>>(half_d, nv, f, eq);
    ZG_KEND(ctx, s);
    // next_c(r', b) = 0 for b < c, eq(r', b - c) for b >= c (build_next_c_r_mle,
    // poly/src/utils.rs:207-236), one per distinct shift amount, each paired with
    // its weighted combination of the source columns
    for (uint32_t m = 0; m < M; m++) {
        uint64_t *nx = pk + (size_t)(1 + m) * n * L;
        const size_t c = amounts[m];
        if (c) ZG_CUDA(cudaMemsetAsync(nx, 0, c * fb, s));
        ZG_CUDA(cudaMemcpyAsync(nx + c * L, eq, (n - c) * fb, cudaMemcpyDeviceToDevice, s));
    }
    ZG_KBEGIN(ctx, s, "k_precombine");
    k_precombine<L><<<grid, 256, 0, s>>>(tr, ncols, nv, gam_d, f, pk + (size_t)(1 + M) * n * L);
    for (uint32_t m = 0; m < M; m++)
        k_precombine_sparse<L><<<grid, 256, 0, s>>>(tr, nv, idx_d + sp_off[m], wgt_d + (size_t)sp_off[m] * L,
                                                    sp_off[m + 1] - sp_off[m], f, pk + (size_t)(2 + M + m) * n * L);
    ZG_KEND(ctx, s);
    ZG_CUDA(ctx_sync(ctx));
    *packed = pk;
    return ZG_OK;
}

// Blocks per column of the CPR's closing dot products (and their partials).
constexpr size_t kCprDotBlocks = 64;

// Step 4 for a linear UAIR up to the sumcheck: the folding challenge and the
// packed MLEs [last-row selector, eq_r, f, up_1 .. up_J, down_1 .. down_S] in
// ctx->piop_arena (combined_poly_resolver.rs:71-178).  coeffs: n_cons x (J + S)
// Montgomery inners (constraint k's coefficients over up then down columns);
// folded_out: J + S inners A_j = sum_k alpha^k coeffs[k][j].
template <int L>
zg_status cpr_prepare(zg_ctx *ctx, zg_transcript *t, const FieldCfg &f, const uint64_t *trace, uint32_t J,
                      uint32_t nv, const uint64_t *point, const uint32_t *src, const uint32_t *shift, uint32_t S,
                      uint32_t n_cons, const uint64_t *coeffs, int on_device, std::vector<uint64_t> &folded,
                      std::vector<uint64_t> &alpha_pows, uint64_t **packed) {
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)1 << nv, fb = 8 * L, mle = n * fb;
    uint64_t alpha[L], pw[L];
    field_challenge_h<L>(t, f, alpha);  // the folding challenge
    folded.assign((size_t)(J + S) * L, 0);
    alpha_pows.assign((size_t)n_cons * L, 0);
    std::memcpy(pw, f.one, fb);
    for (uint32_t k = 0; k < n_cons; k++) {
        std::memcpy(&alpha_pows[(size_t)k * L], pw, fb);
        for (uint32_t j = 0; j < J + S; j++) {
            uint64_t tm[L];
            fmul<L>(pw, coeffs + ((size_t)k * (J + S) + j) * L, f.p, f.n0, tm);
            fadd<L>(&folded[(size_t)j * L], tm, f.p);
        }
        uint64_t nx[L];
        fmul<L>(pw, alpha, f.p, f.n0, nx);
        std::memcpy(pw, nx, fb);
    }
    std::vector<uint64_t> omr((size_t)nv * L);
    for (uint32_t k = 0; k < nv; k++) {
        std::memcpy(&omr[(size_t)k * L], f.one, fb);
        fsub<L>(&omr[(size_t)k * L], point + (size_t)k * L, f.p);
    }
    const size_t halves = ((size_t)1 << (nv / 2)) + ((size_t)1 << (nv - nv / 2));
    const size_t npk = 3 + (size_t)J + S;
    const size_t small = (2 * (size_t)nv + halves + (size_t)(J + S) * (1 + kCprDotBlocks)) * fb;
    ZG_TRY(ctx->piop_arena.ensure(npk * mle + small + 256));
    uint8_t *ar = ctx->piop_arena.as<uint8_t>();
    uint64_t *pk = reinterpret_cast<uint64_t *>(ar);
    uint64_t *r_d = reinterpret_cast<uint64_t *>(ar + npk * mle), *omr_d = r_d + (size_t)nv * L;
    uint64_t *half_d = omr_d + (size_t)nv * L, *fold_d = half_d + halves * L;
    uint64_t *up = pk + 3 * n * L, *down = up + (size_t)J * n * L;
    ZG_CUDA(cudaMemcpyAsync(up, trace, (size_t)J * mle, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            s));
    ZG_CUDA(cudaMemcpyAsync(r_d, point, (size_t)nv * fb, cudaMemcpyHostToDevice, s));
    ZG_CUDA(cudaMemcpyAsync(omr_d, omr.data(), (size_t)nv * fb, cudaMemcpyHostToDevice, s));
    // last-row selector: one at index 2^nv - 1
    ZG_CUDA(cudaMemsetAsync(pk, 0, mle, s));
    ZG_CUDA(cudaMemcpyAsync(pk + (n - 1) * L, f.one, fb, cudaMemcpyHostToDevice, s));
    ZG_KBEGIN(ctx, s, "k_eq_halves");
    k_eq_halves<L><<<(unsigned)((halves + 127) / 128), 128, 0, s>>>(r_d, omr_d, nv, f, half_d);
    ZG_KEND(ctx, s);
    ZG_KBEGIN(ctx, s, "k_eq_outer");
    k_eq_outer<L><<<(unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8), 256, 0, s>>>(
        half_d, nv, f, pk + n * L);
    ZG_KEND(ctx, s);
    // down column k: up column src[k] from row shift[k] on, zero padded
    for (uint32_t k = 0; k < S; k++) {
        uint64_t *dk = down + (size_t)k * n * L;
        const size_t c = shift[k];
        ZG_CUDA(cudaMemcpyAsync(dk, up + ((size_t)src[k] * n + c) * L, (n - c) * fb, cudaMemcpyDeviceToDevice, s));
        if (c) ZG_CUDA(cudaMemsetAsync(dk + (n - c) * L, 0, c * fb, s));
    }
    // f = sum_j A_j v_j over the up and down columns: the comb's linear part as
    // one MLE, so the sumcheck carries [sel, eq_r, f] instead of every column
    ZG_CUDA(cudaMemcpyAsync(fold_d, folded.data(), (size_t)(J + S) * fb, cudaMemcpyHostToDevice, s));
    ZG_KBEGIN(ctx, s, "k_precombine");
    k_precombine<L><<<(unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8), 256, 0, s>>>(
        up, J + S, nv, fold_d, f, pk + 2 * n * L);
    ZG_KEND(ctx, s);
    ZG_CUDA(ctx_sync(ctx));
    *packed = pk;
    return ZG_OK;
}

// After the CPR sumcheck: the J + S up and down columns (packed after [sel, eq,
// f]) evaluated at its point r*: eq(r*, .) into the eq slot, then one dot
// product per column.
template <int L>
zg_status cpr_column_evals(zg_ctx *ctx, const FieldCfg &f, uint64_t *pk, uint32_t K, uint32_t nv,
                           const uint64_t *point, uint64_t *evals) {
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)1 << nv, fb = 8 * L, mle = n * fb;
    const size_t halves = ((size_t)1 << (nv / 2)) + ((size_t)1 << (nv - nv / 2));
    uint8_t *ar = reinterpret_cast<uint8_t *>(pk);
    uint64_t *r_d = reinterpret_cast<uint64_t *>(ar + (3 + (size_t)K) * mle), *omr_d = r_d + (size_t)nv * L;
    uint64_t *half_d = omr_d + (size_t)nv * L, *part_d = half_d + halves * L + (size_t)K * L;
    std::vector<uint64_t> omr((size_t)nv * L);
    for (uint32_t k = 0; k < nv; k++) {
        std::memcpy(&omr[(size_t)k * L], f.one, fb);
        fsub<L>(&omr[(size_t)k * L], point + (size_t)k * L, f.p);
    }
    ZG_CUDA(cudaMemcpyAsync(r_d, point, (size_t)nv * fb, cudaMemcpyHostToDevice, s));
    ZG_CUDA(cudaMemcpyAsync(omr_d, omr.data(), (size_t)nv * fb, cudaMemcpyHostToDevice, s));
    uint64_t *eq = pk + n * L;
    ZG_KBEGIN(ctx, s, "k_eq_halves");
    k_eq_halves<L><<<(unsigned)((halves + 127) / 128), 128, 0, s>>>(r_d, omr_d, nv, f, half_d);
    ZG_KEND(ctx, s);
    ZG_KBEGIN(ctx, s, "k_eq_outer");
    k_eq_outer<L><<<(unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8), 256, 0, s>>>(
        half_d, nv, f, eq);
    ZG_KEND(ctx, s);
    const unsigned G = (unsigned)std::max<size_t>(1, std::min<size_t>(kCprDotBlocks, n / 2048));
    ZG_KBEGIN(ctx, s, "k_mle_dots");
    k_mle_dots<L><<<dim3(G, K), 256, 0, s>>>(pk + 3 * n * L, nv, eq, f, part_d);
    ZG_KEND(ctx, s);
    std::vector<uint64_t> part((size_t)K * G * L);
    ZG_CUDA(cudaMemcpyAsync(part.data(), part_d, part.size() * 8, cudaMemcpyDeviceToHost, s));
    ZG_CUDA(ctx_sync(ctx));
    for (uint32_t k = 0; k < K; k++) {
        uint64_t acc[L] = {};
        for (unsigned g = 0; g < G; g++) fadd<L>(acc, &part[((size_t)k * G + g) * L], f.p);
        std::memcpy(evals + (size_t)k * L, acc, fb);
    }
    return ZG_OK;
}

template <int L>
zg_status ic_product_sums_t(zg_ctx *ctx, const FieldCfg &f, const uint64_t *point, uint32_t nv, const IcFactor &a,
                            const IcFactor &b, uint32_t D, std::vector<uint64_t> &out, uint32_t &len) {
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)1 << nv, fb = 8 * L;
    const uint32_t la = a.bin ? D : 1, lb = b.bin ? D : 1;
    len = la + lb - 1;
    const size_t halves = ((size_t)1 << (nv / 2)) + ((size_t)1 << (nv - nv / 2));
    const unsigned G = (unsigned)std::max<size_t>(1, std::min<size_t>(128, n / 4096));
    // [eq: n][r: nv][1 - r: nv][halves][small: 65][partials: len x G]
    const size_t need = (n + 2 * (size_t)nv + halves + 65 + (size_t)len * G) * fb + 256;
    ZG_TRY(ctx->piop_arena.ensure(need));
    uint64_t *eq = ctx->piop_arena.as<uint64_t>(), *r_d = eq + n * L, *omr_d = r_d + (size_t)nv * L;
    uint64_t *half_d = omr_d + (size_t)nv * L, *small_d = half_d + halves * L, *part_d = small_d + 65 * L;
    std::vector<uint64_t> omr((size_t)nv * L), small(65 * (size_t)L, 0);
    for (uint32_t k = 0; k < nv; k++) {
        std::memcpy(&omr[(size_t)k * L], f.one, fb);
        fsub<L>(&omr[(size_t)k * L], point + (size_t)k * L, f.p);
    }
    for (int c = 1; c <= 64; c++) {  // small[c] = F(c) = (c - 1) * one + one
        std::memcpy(&small[(size_t)c * L], &small[(size_t)(c - 1) * L], fb);
        fadd<L>(&small[(size_t)c * L], f.one, f.p);
    }
    ZG_CUDA(cudaMemcpyAsync(r_d, point, (size_t)nv * fb, cudaMemcpyHostToDevice, s));
    ZG_CUDA(cudaMemcpyAsync(omr_d, omr.data(), (size_t)nv * fb, cudaMemcpyHostToDevice, s));
    ZG_CUDA(cudaMemcpyAsync(small_d, small.data(), small.size() * 8, cudaMemcpyHostToDevice, s));
    ZG_KBEGIN(ctx, s, "k_eq_halves");
    k_eq_halves<L><<<(unsigned)((halves + 127) / 128), 128, 0, s>>>(r_d, omr_d, nv, f, half_d);
    ZG_KEND(ctx, s);
    ZG_KBEGIN(ctx, s, "k_eq_outer");
    k_eq_outer<L><<<(unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8), 256, 0, s>>>(
        half_d, nv, f, eq);
    ZG_KEND(ctx, s);
    const uint64_t dmask = D >= 64 ? ~0ull : ((1ull << D) - 1);
    ZG_KBEGIN(ctx, s, "k_ic_product");
    k_ic_product<L><<<dim3(G, len), 256, 0, s>>>(a, b, dmask, nv, eq, small_d, f, part_d);
    ZG_KEND(ctx, s);
    std::vector<uint64_t> part((size_t)len * G * L);
    ZG_CUDA(cudaMemcpyAsync(part.data(), part_d, part.size() * 8, cudaMemcpyDeviceToHost, s));
    ZG_CUDA(ctx_sync(ctx));
    out.assign((size_t)len * L, 0);
    for (uint32_t m = 0; m < len; m++)
        for (unsigned g = 0; g < G; g++) fadd<L>(&out[(size_t)m * L], &part[((size_t)m * G + g) * L], f.p);
    return ZG_OK;
}

}  // namespace

zg_status ic_product_sums(zg_ctx *ctx, const FieldCfg &f, const uint64_t *point, uint32_t nv, const IcFactor &a,
                          const IcFactor &b, uint32_t D, std::vector<uint64_t> &out, uint32_t &len) {
    if (D == 0 || D > 64 || nv == 0 || nv > 28 || (!a.bin && !a.ints) || (!b.bin && !b.ints)) {
        set_error("ideal check: product term with an empty factor or out-of-range sizes");
        return ZG_ERR_INVALID_PARAM;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    return f.L == 3 ? ic_product_sums_t<3>(ctx, f, point, nv, a, b, D, out, len)
                    : ic_product_sums_t<4>(ctx, f, point, nv, a, b, D, out, len);
}

}  // namespace zg

using namespace zg;

extern "C" zg_status zg_piop_eval_projection(zg_ctx *ctx, const uint8_t *modulus, uint32_t limbs,
                                             const uint64_t *bin_cols, uint32_t n_bin, uint32_t degree_plus_one,
                                             const int64_t *int_cols, uint32_t n_int, uint32_t nvars,
                                             const uint64_t *a, int on_device, uint64_t *mles_out) {
    try {
        const PiopCols c{bin_cols, n_bin, degree_plus_one, int_cols, n_int, nvars};
        FieldCfg f;
        ZG_TRY(piop_args(ctx, modulus, limbs, c, a, mles_out, f));
        std::lock_guard<std::mutex> lk(ctx->mu);
        ZG_CUDA(cudaSetDevice(ctx->device));
        return limbs == 3 ? eval_projection_t<3>(ctx, f, c, a, on_device, mles_out)
                          : eval_projection_t<4>(ctx, f, c, a, on_device, mles_out);
    } catch (const std::exception &e) {
        set_error("piop: %s", e.what());
        return ZG_ERR_OOM;
    }
}

extern "C" zg_status zg_piop_lifted_evals(zg_ctx *ctx, const uint8_t *modulus, uint32_t limbs,
                                          const uint64_t *bin_cols, uint32_t n_bin, uint32_t degree_plus_one,
                                          const int64_t *int_cols, uint32_t n_int, uint32_t nvars,
                                          const uint64_t *point, int cols_on_device, uint64_t *coeffs_out) {
    try {
        const PiopCols c{bin_cols, n_bin, degree_plus_one, int_cols, n_int, nvars};
        FieldCfg f;
        ZG_TRY(piop_args(ctx, modulus, limbs, c, point, coeffs_out, f));
        std::lock_guard<std::mutex> lk(ctx->mu);
        ZG_CUDA(cudaSetDevice(ctx->device));
        return limbs == 3 ? lifted_evals_t<3>(ctx, f, c, point, cols_on_device, coeffs_out)
                          : lifted_evals_t<4>(ctx, f, c, point, cols_on_device, coeffs_out);
    } catch (const std::exception &e) {
        set_error("piop: %s", e.what());
        return ZG_ERR_OOM;
    }
}

extern "C" zg_status zg_piop_multipoint_eval(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus,
                                             uint32_t limbs, const uint64_t *trace_mles, uint32_t num_cols,
                                             uint32_t nvars, const uint64_t *eval_point,
                                             const uint32_t *shift_src, const uint32_t *shift_amount,
                                             uint32_t n_shifts, int mles_on_device, uint8_t *proof,
                                             size_t *proof_len, uint64_t *r0_out) {
    try {
        if (!ctx || !t || !modulus || !trace_mles || !eval_point || !proof || !proof_len || num_cols == 0 ||
            (n_shifts && (!shift_src || !shift_amount))) {
            set_error("multipoint eval: null argument or no columns");
            return ZG_ERR_INVALID_PARAM;
        }
        if (limbs != 3 && limbs != 4) {
            set_error("multipoint eval: field limbs must be 3 or 4 (got %u)", limbs);
            return ZG_ERR_INVALID_PARAM;
        }
        if (nvars == 0 || nvars > 28 || n_shifts > 1024 || num_cols > 4096) {
            set_error("multipoint eval: num_vars must be 1..28, at most 1024 shifts and 4096 columns");
            return ZG_ERR_INVALID_PARAM;
        }
        for (uint32_t k = 0; k < n_shifts; k++)
            if (shift_src[k] >= num_cols || (uint64_t)shift_amount[k] >= (1ull << nvars)) {
                set_error("shift %u: source column %u or shift %u out of range", k, shift_src[k], shift_amount[k]);
                return ZG_ERR_INVALID_PARAM;
            }
        uint64_t p[4] = {0, 0, 0, 0};
        std::memcpy(p, modulus, 8 * limbs);
        if (!(p[0] & 1)) {
            set_error("multipoint eval: the modulus must be odd");
            return ZG_ERR_INVALID_PARAM;
        }
        uint32_t M = 0;  // distinct shift amounts
        uint64_t *packed = nullptr;
        {
            std::lock_guard<std::mutex> lk(ctx->mu);
            ZG_CUDA(cudaSetDevice(ctx->device));
            field_cfg_init(t->f, p, (int)limbs);
            t->has_field = true;
            const zg_status st =
                limbs == 3 ? multipoint_prepare<3>(ctx, t, t->f, trace_mles, num_cols, nvars, eval_point, shift_src,
                                                   shift_amount, n_shifts, mles_on_device, &M, &packed)
                           : multipoint_prepare<4>(ctx, t, t->f, trace_mles, num_cols, nvars, eval_point, shift_src,
                                                   shift_amount, n_shifts, mles_on_device, &M, &packed);
            if (st != ZG_OK) return st;
        }
        // comb = eq * precombined + sum_k alpha_k next_k v_{src_k}, degree 2
        // (multipoint_eval.rs:195-213), with the shift terms grouped by amount:
        // eq * precombined + sum_c next_c * w_c, every product with coefficient one
        std::vector<uint64_t> coeffs((size_t)(1 + M) * limbs);
        for (uint32_t k = 0; k <= M; k++) std::memcpy(&coeffs[(size_t)k * limbs], t->f.one, 8 * limbs);
        std::vector<uint32_t> offsets(2 + M), indices(2 * (1 + M));
        for (uint32_t k = 0; k <= 1 + M; k++) offsets[k] = 2 * k;
        indices[0] = 0;
        indices[1] = 1 + M;
        for (uint32_t m = 0; m < M; m++) {
            indices[2 * (1 + m)] = 1 + m;
            indices[2 * (1 + m) + 1] = 2 + M + m;
        }
        zg_sumcheck_group g{};
        g.degree = 2;
        g.n_mles = 2 + 2 * M;
        g.n_products = 1 + M;
        g.mles = packed;
        g.coeffs = coeffs.data();
        g.offsets = offsets.data();
        g.indices = indices.data();
        return zg_sumcheck_prove(ctx, t, modulus, limbs, nvars, 0, &g, 1, 1, proof, proof_len, r0_out, nullptr);
    } catch (const std::exception &e) {
        set_error("multipoint eval: %s", e.what());
        return ZG_ERR_OOM;
    }
}

zg_status zg::cpr_prove_impl(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus, uint32_t limbs,
                             const uint64_t *trace_mles, uint32_t num_cols, uint32_t nvars,
                             const uint64_t *eval_point, const uint32_t *shift_src, const uint32_t *shift_amount,
                             uint32_t n_shifts, uint32_t n_constraints, const uint64_t *coeffs,
                             const std::vector<CprProduct> &products, int mles_on_device, uint8_t *proof,
                             size_t *proof_len, uint64_t *point_out, uint64_t *evals_out) {
    try {
        if (!ctx || !t || !modulus || !trace_mles || !eval_point || !proof || !proof_len || !coeffs ||
            num_cols == 0 || n_constraints == 0 || (n_shifts && (!shift_src || !shift_amount))) {
            set_error("CPR: null argument, no columns or no constraints");
            return ZG_ERR_INVALID_PARAM;
        }
        if (limbs != 3 && limbs != 4) {
            set_error("CPR: field limbs must be 3 or 4 (got %u)", limbs);
            return ZG_ERR_INVALID_PARAM;
        }
        if (nvars < 2 || nvars > 28 || n_shifts > 1024 || num_cols > 4096 || n_constraints > 65536) {
            set_error("CPR: num_vars must be 2..28 (the protocol is not needed for 1), at most 1024 shifts, "
                      "4096 columns and 65536 constraints");
            return ZG_ERR_INVALID_PARAM;
        }
        for (uint32_t k = 0; k < n_shifts; k++)
            if (shift_src[k] >= num_cols || (uint64_t)shift_amount[k] >= (1ull << nvars)) {
                set_error("shift %u: source column %u or shift %u out of range", k, shift_src[k], shift_amount[k]);
                return ZG_ERR_INVALID_PARAM;
            }
        uint64_t p[4] = {0, 0, 0, 0};
        std::memcpy(p, modulus, 8 * limbs);
        if (!(p[0] & 1)) {
            set_error("CPR: the modulus must be odd");
            return ZG_ERR_INVALID_PARAM;
        }
        const uint32_t J = num_cols, S = n_shifts;
        uint32_t max_factors = 1;
        for (const CprProduct &q : products) {
            if (q.constraint >= n_constraints || q.cols.empty()) {
                set_error("CPR: product term of constraint %u out of range or without columns", q.constraint);
                return ZG_ERR_INVALID_PARAM;
            }
            for (uint32_t c : q.cols)
                if (c >= J + S) {
                    set_error("CPR: product column %u out of range", c);
                    return ZG_ERR_INVALID_PARAM;
                }
            max_factors = std::max<uint32_t>(max_factors, (uint32_t)q.cols.size());
        }
        if (max_factors + 2 > 8) {
            set_error("CPR: products of %u columns make the sumcheck degree exceed 8", max_factors);
            return ZG_ERR_INVALID_PARAM;
        }
        std::vector<uint64_t> folded, alpha_pows;
        uint64_t *packed = nullptr;
        {
            std::lock_guard<std::mutex> lk(ctx->mu);
            ZG_CUDA(cudaSetDevice(ctx->device));
            field_cfg_init(t->f, p, (int)limbs);
            t->has_field = true;
            const zg_status st =
                limbs == 3 ? cpr_prepare<3>(ctx, t, t->f, trace_mles, J, nvars, eval_point, shift_src, shift_amount, S,
                                            n_constraints, coeffs, mles_on_device, folded, alpha_pows, &packed)
                           : cpr_prepare<4>(ctx, t, t->f, trace_mles, J, nvars, eval_point, shift_src, shift_amount, S,
                                            n_constraints, coeffs, mles_on_device, folded, alpha_pows, &packed);
            if (st != ZG_OK) return st;
        }
        // comb = (sum_j A_j v_j) * eq_r * (1 - selector), degree max_degree + 2 = 3
        // (combined_poly_resolver.rs:147-172): the sum is the precombined MLE f,
        // times two affine factors; the round polynomials are those of the
        // reference's comb over every column
        const uint32_t fm[2] = {1, 0};
        std::vector<uint64_t> fa(2 * (size_t)limbs, 0), fbv(2 * (size_t)limbs, 0);
        std::memcpy(&fbv[0], t->f.one, 8 * limbs);      // eq_r: 0 + 1 * eq_r
        std::memcpy(&fa[limbs], t->f.one, 8 * limbs);   // 1 - sel: one + (p - one) * sel
        std::memcpy(&fbv[limbs], t->f.p, 8 * limbs);
        {
            uint64_t *b1 = &fbv[limbs];
            unsigned __int128 br = 0;
            for (uint32_t w = 0; w < limbs; w++) {
                const unsigned __int128 d = (unsigned __int128)b1[w] - t->f.one[w] - (uint64_t)br;
                b1[w] = (uint64_t)d;
                br = (d >> 64) & 1;
            }
        }
        // product terms (constraints of degree above one): alpha^k c_t times the
        // product of their columns, which the sumcheck then carries as MLEs too
        // (packed after [sel, eq, f]); the comb's degree is the longest product + 2
        std::vector<uint64_t> pcoeffs((size_t)limbs, 0);
        std::memcpy(pcoeffs.data(), t->f.one, 8 * limbs);
        std::vector<uint32_t> poff{0, 1}, pidx{2};
        for (const CprProduct &q : products) {
            uint64_t c[4], cm[4];
            if (limbs == 3) {
                from_i128<3>((i128)q.coeff, t->f, c);
                fmul<3>(c, &alpha_pows[(size_t)q.constraint * 3], t->f.p, t->f.n0, cm);
            } else {
                from_i128<4>((i128)q.coeff, t->f, c);
                fmul<4>(c, &alpha_pows[(size_t)q.constraint * 4], t->f.p, t->f.n0, cm);
            }
            pcoeffs.insert(pcoeffs.end(), cm, cm + limbs);
            for (uint32_t col : q.cols) pidx.push_back(3 + col);
            poff.push_back((uint32_t)pidx.size());
        }
        zg_sumcheck_group g{};
        g.degree = max_factors + 2;
        g.n_mles = products.empty() ? 3 : 3 + J + S;
        g.n_products = (uint32_t)poff.size() - 1;
        g.mles = packed;
        g.coeffs = pcoeffs.data();
        g.offsets = poff.data();
        g.indices = pidx.data();
        g.n_factors = 2;
        g.factor_mles = fm;
        g.factor_a = fa.data();
        g.factor_b = fbv.data();
        std::vector<uint64_t> pt((size_t)nvars * limbs), evals((size_t)(J + S) * limbs);
        ZG_TRY(zg_sumcheck_prove(ctx, t, modulus, limbs, nvars, 1, &g, 1, 1, proof, proof_len, pt.data(),
                                 nullptr));
        if (point_out) std::memcpy(point_out, pt.data(), pt.size() * 8);
        // finalize_prover (combined_poly_resolver.rs:192-247): the up and down
        // columns at the sumcheck point, absorbed as random-field elements
        std::lock_guard<std::mutex> lk(ctx->mu);
        ZG_CUDA(cudaSetDevice(ctx->device));
        ZG_TRY(limbs == 3 ? cpr_column_evals<3>(ctx, t->f, packed, J + S, nvars, pt.data(), evals.data())
                          : cpr_column_evals<4>(ctx, t->f, packed, J + S, nvars, pt.data(), evals.data()));
        for (uint32_t j = 0; j < J + S; j++) tr_absorb_field(t, &evals[(size_t)j * limbs]);
        if (evals_out) std::memcpy(evals_out, evals.data(), evals.size() * 8);
        return ZG_OK;
    } catch (const std::exception &e) {
        set_error("CPR: %s", e.what());
        return ZG_ERR_OOM;
    }
}

extern "C" zg_status zg_piop_cpr_linear_prove(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus,
                                              uint32_t limbs, const uint64_t *trace_mles, uint32_t num_cols,
                                              uint32_t nvars, const uint64_t *eval_point,
                                              const uint32_t *shift_src, const uint32_t *shift_amount,
                                              uint32_t n_shifts, uint32_t n_constraints, const uint64_t *coeffs,
                                              int mles_on_device, uint8_t *proof, size_t *proof_len,
                                              uint64_t *point_out, uint64_t *evals_out) {
    return cpr_prove_impl(ctx, t, modulus, limbs, trace_mles, num_cols, nvars, eval_point, shift_src, shift_amount,
                          n_shifts, n_constraints, coeffs, {}, mles_on_device, proof, proof_len, point_out,
                          evals_out);
}

// Step 2 for a linear UAIR (IdealCheckProtocol::prove_linear, piop/src/ideal_check.rs:
// 137-176, MLE first): the point r from the transcript, every up column and every
// shifted (down) column evaluated coefficient-wise at r (the lifted-evaluation sums
// on copies of the columns, the down ones shifted up and zero padded, the last row
// of every copy cleared as the reference's evaluate_combined_polynomials reads it), each
// constraint's coefficients applied to those polynomial values, and the trimmed
// combined values absorbed constraint after constraint.
namespace zg {
// absorb == false: the point is drawn and the combined values are computed
// (untrimmed, lengths_out left alone) but nothing is absorbed, for callers that
// add more terms before the values go into the transcript.
zg_status ideal_check_linear_impl(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus, uint32_t limbs,
                                  const uint64_t *bin_cols, uint32_t n_bin, uint32_t degree_plus_one,
                                  const int64_t *int_cols, uint32_t n_int, uint32_t nvars, const uint32_t *shift_src,
                                  const uint32_t *shift_amount, uint32_t n_shifts, uint32_t n_constraints,
                                  const uint64_t *coeffs, int cols_on_device, uint64_t *point_out,
                                  uint64_t *combined_out, uint32_t *lengths_out, bool absorb) {
    try {
        const uint32_t D = degree_plus_one, J = n_bin + n_int, S = n_shifts;
        const PiopCols c0{bin_cols, n_bin, D, int_cols, n_int, nvars};
        FieldCfg f;
        if (!t || !point_out || !combined_out || !lengths_out || !coeffs || n_constraints == 0 || J == 0 ||
            (S && (!shift_src || !shift_amount)) || S > 1024 || n_constraints > 65536) {
            set_error("ideal check: null argument, no columns or constraints, or more than 1024 shifts");
            return ZG_ERR_INVALID_PARAM;
        }
        ZG_TRY(piop_args(ctx, modulus, limbs, c0, coeffs, combined_out, f));
        if (nvars == 0) {
            set_error("ideal check: num_vars must be at least 1");
            return ZG_ERR_INVALID_PARAM;
        }
        for (uint32_t k = 0; k < S; k++)
            if (shift_src[k] >= J || (uint64_t)shift_amount[k] >= (1ull << nvars)) {
                set_error("shift %u: source column %u or shift %u out of range", k, shift_src[k], shift_amount[k]);
                return ZG_ERR_INVALID_PARAM;
            }
        const size_t n = (size_t)1 << nvars, L = limbs, fb = 8 * L;
        std::lock_guard<std::mutex> lk(ctx->mu);
        ZG_CUDA(cudaSetDevice(ctx->device));
        field_cfg_init(t->f, f.p, (int)limbs);
        t->has_field = true;
        // the evaluation point: get_field_challenges(num_vars)
        for (uint32_t k = 0; k < nvars; k++) {
            if (L == 3) field_challenge_h<3>(t, f, point_out + k * L);
            else field_challenge_h<4>(t, f, point_out + k * L);
        }
        // extended columns: binary up, binary down, then integer up, integer down
        std::vector<uint32_t> dbin, dint;  // shift indices by source kind
        for (uint32_t k = 0; k < S; k++) (shift_src[k] < n_bin ? dbin : dint).push_back(k);
        const uint32_t nb2 = n_bin + (uint32_t)dbin.size(), ni2 = n_int + (uint32_t)dint.size();
        ZG_TRY(ctx->piop_arena.ensure(((size_t)nb2 + ni2) * n * 8 + 256));
        uint64_t *eb = ctx->piop_arena.as<uint64_t>();
        int64_t *ei = reinterpret_cast<int64_t *>(eb + (size_t)nb2 * n);
        cudaStream_t s = ctx->stream;
        const cudaMemcpyKind kind = cols_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        if (n_bin) ZG_CUDA(cudaMemcpyAsync(eb, bin_cols, (size_t)n_bin * n * 8, kind, s));
        if (n_int) ZG_CUDA(cudaMemcpyAsync(ei, int_cols, (size_t)n_int * n * 8, kind, s));
        auto shifted = [&](void *dst, const void *src_col, size_t c) -> cudaError_t {
            cudaError_t e = cudaMemcpyAsync(dst, static_cast<const uint8_t *>(src_col) + c * 8, (n - c) * 8, kind, s);
            if (e == cudaSuccess && c) e = cudaMemsetAsync(static_cast<uint8_t *>(dst) + (n - c) * 8, 0, c * 8, s);
            return e;
        };
        for (size_t q = 0; q < dbin.size(); q++)
            ZG_CUDA(shifted(eb + (n_bin + q) * n, bin_cols + (size_t)shift_src[dbin[q]] * n, shift_amount[dbin[q]]));
        for (size_t q = 0; q < dint.size(); q++)
            ZG_CUDA(shifted(ei + (n_int + q) * n, int_cols + (size_t)(shift_src[dint[q]] - n_bin) * n,
                            shift_amount[dint[q]]));
        // evaluate_combined_polynomials (ideal_check/combined_poly_builder.rs:232-252)
        // reads zero on the last row of every up and down column: clear entry
        // 2^nvars - 1 of each extended column (one strided memset per kind)
        if (nb2) ZG_CUDA(cudaMemset2DAsync(eb + (n - 1), n * 8, 0, 8, nb2, s));
        if (ni2) ZG_CUDA(cudaMemset2DAsync(ei + (n - 1), n * 8, 0, 8, ni2, s));
        const PiopCols ext{eb, nb2, D, ei, ni2, nvars};
        std::vector<uint64_t> vals(((size_t)nb2 * D + ni2) * L);
        ZG_TRY(L == 3 ? lifted_evals_t<3>(ctx, f, ext, point_out, 1, vals.data())
                      : lifted_evals_t<4>(ctx, f, ext, point_out, 1, vals.data()));
        // position of shift k among the extended binary (or integer) columns
        std::vector<uint32_t> ext_pos(S);
        for (size_t q = 0; q < dbin.size(); q++) ext_pos[dbin[q]] = n_bin + (uint32_t)q;
        for (size_t q = 0; q < dint.size(); q++) ext_pos[dint[q]] = n_int + (uint32_t)q;
        // column value (D coefficients) of column index j in [up (bin, int), down (shift order)]
        static const uint64_t zero[4] = {0, 0, 0, 0};
        auto column = [&](uint32_t j, uint32_t l) -> const uint64_t * {
            if (j < n_bin) return &vals[((size_t)j * D + l) * L];
            if (j < J) return l == 0 ? &vals[((size_t)nb2 * D + (j - n_bin)) * L] : zero;
            const uint32_t k = j - J;
            if (shift_src[k] < n_bin) return &vals[((size_t)ext_pos[k] * D + l) * L];
            return l == 0 ? &vals[((size_t)nb2 * D + ext_pos[k]) * L] : zero;
        };
        for (uint32_t k = 0; k < n_constraints; k++) {
            uint64_t *out = combined_out + (size_t)k * D * L;
            std::memset(out, 0, (size_t)D * fb);
            for (uint32_t j = 0; j < J + S; j++) {
                const uint64_t *cf = coeffs + ((size_t)k * (J + S) + j) * L;
                bool nz = false;
                for (size_t w = 0; w < L; w++) nz |= cf[w] != 0;
                if (!nz) continue;
                for (uint32_t l = 0; l < D; l++) {
                    uint64_t tm[4];
                    if (L == 3) {
                        fmul<3>(cf, column(j, l), f.p, f.n0, tm);
                        fadd<3>(out + (size_t)l * L, tm, f.p);
                    } else {
                        fmul<4>(cf, column(j, l), f.p, f.n0, tm);
                        fadd<4>(out + (size_t)l * L, tm, f.p);
                    }
                }
            }
            if (!absorb) continue;
            // DynamicPolynomialF::new_trimmed, then absorb_random_field_slice
            uint32_t len = D;
            while (len > 0) {
                bool nz = false;
                for (size_t w = 0; w < L; w++) nz |= out[(size_t)(len - 1) * L + w] != 0;
                if (nz) break;
                len--;
            }
            lengths_out[k] = len;
            for (uint32_t l = 0; l < len; l++) tr_absorb_field(t, out + (size_t)l * L);
        }
        return ZG_OK;
    } catch (const std::exception &e) {
        set_error("ideal check: %s", e.what());
        return ZG_ERR_OOM;
    }
}
}  // namespace zg

extern "C" zg_status zg_piop_ideal_check_linear(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus,
                                                uint32_t limbs, const uint64_t *bin_cols, uint32_t n_bin,
                                                uint32_t degree_plus_one, const int64_t *int_cols, uint32_t n_int,
                                                uint32_t nvars, const uint32_t *shift_src,
                                                const uint32_t *shift_amount, uint32_t n_shifts,
                                                uint32_t n_constraints, const uint64_t *coeffs, int cols_on_device,
                                                uint64_t *point_out, uint64_t *combined_out, uint32_t *lengths_out) {
    return ideal_check_linear_impl(ctx, t, modulus, limbs, bin_cols, n_bin, degree_plus_one, int_cols, n_int, nvars,
                                   shift_src, shift_amount, n_shifts, n_constraints, coeffs, cols_on_device,
                                   point_out, combined_out, lengths_out, true);
}
