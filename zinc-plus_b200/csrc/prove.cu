// Prove-phase kernels (zip-plus/src/pcs/phase_prove.rs:119-304).
//
//  k_eq_table      eq(x, r) over the hypercube (poly/src/utils.rs:24-101)
//  k_project_rows  w'[j][c] = <eval, alphas> in CombR (phase_prove.rs:154-174)
//                  and per-block partial sums of F(w') * q1 (b rows, :179-193)
//  k_combined_row  combined_row[c] = sum_poly sum_j s_j * w'[j][c] (:205-244)
//  k_openings      column values and Merkle siblings of the opened columns in
//                  proof byte order (open_merkle_trees_for_column, :285-304;
//                  write_merkle_proof, pcs_transcript.rs:210-221)
#include "zg_internal.h"
#include "zg_prove.h"

namespace zg {

template <int L>
__global__ void k_eq_table(const uint64_t *__restrict__ r, const uint64_t *__restrict__ omr,
                           uint32_t n, FieldCfg f, uint64_t *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (1u << n)) return;
    uint64_t acc[L];
    for (int k = 0; k < L; k++) acc[k] = f.one[k];
    for (uint32_t k = 0; k < n; k++) {
        const uint64_t *sel = ((i >> k) & 1u) ? r + (size_t)k * L : omr + (size_t)k * L;
        uint64_t t[L];
        fmul<L>(acc, sel, f.p, f.n0, t);
        for (int w = 0; w < L; w++) acc[w] = t[w];
    }
    for (int w = 0; w < L; w++) out[(size_t)i * L + w] = acc[w];
}

// eq(x, r) over n <= 20 variables as an outer product: with n = a + b,
// eq[i] = eq_lo[i mod 2^a] * eq_hi[i >> a], the half tables (over the first a
// and the last b coordinates) being rebuilt by every block in shared memory.
// Field products are exact, so the grouping does not change any value.
template <int L>
__global__ void __launch_bounds__(256) k_eq_table_split(const uint64_t *__restrict__ r,
                                                        const uint64_t *__restrict__ omr,
                                                        uint32_t n, FieldCfg f,
                                                        uint64_t *__restrict__ out) {
    extern __shared__ uint64_t tab[];  // [2^a + 2^b][L]
    const uint32_t a = n / 2, b = n - a;
    const uint32_t na = 1u << a, nb = 1u << b;
    for (uint32_t e = threadIdx.x; e < na + nb; e += blockDim.x) {
        const bool hi = e >= na;
        const uint32_t idx = hi ? e - na : e, k0 = hi ? a : 0, kn = hi ? b : a;
        // the product of the kn factors as a balanced tree: depth ceil(log2 kn)
        // instead of a chain of kn dependent Montgomery products
        uint64_t v[10][L];
        for (uint32_t k = 0; k < kn; k++) {
            const uint64_t *sel = ((idx >> k) & 1u) ? r + (size_t)(k0 + k) * L : omr + (size_t)(k0 + k) * L;
            for (int w = 0; w < L; w++) v[k][w] = sel[w];
        }
        uint32_t width = kn;
        if (width == 0) {
            for (int w = 0; w < L; w++) v[0][w] = f.one[w];
            width = 1;
        }
        while (width > 1) {
            const uint32_t half = width / 2;
            for (uint32_t i = 0; i < half; i++) {
                uint64_t t[L];
                fmul<L>(v[2 * i], v[2 * i + 1], f.p, f.n0, t);
                for (int w = 0; w < L; w++) v[i][w] = t[w];
            }
            if (width & 1)
                for (int w = 0; w < L; w++) v[half][w] = v[width - 1][w];
            width = half + (width & 1);
        }
        for (int w = 0; w < L; w++) tab[(size_t)e * L + w] = v[0][w];
    }
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (1u << n)) return;
    uint64_t t[L];
    fmul<L>(&tab[(size_t)(i & (na - 1)) * L], &tab[(size_t)(na + (i >> a)) * L], f.p, f.n0, t);
    for (int w = 0; w < L; w++) out[(size_t)i * L + w] = t[w];
}

// One thread per (poly, row j, column c).  Binary evaluations (binary == 1)
// project to sum_{bit i set} alpha_i; i32 (binary == 0) and i64 (binary == 2)
// evaluations project to themselves (alphas = [1]).
// The projection fits in 3 limbs (|w'| < 64 * 2^127); it is sign-extended (or
// truncated) to comb_limbs.
template <int L>
__global__ void __launch_bounds__(256) k_project_rows(const void *__restrict__ evals, int binary,
                                                      const i128 *__restrict__ alphas, uint32_t D,
                                                      uint64_t dmask, const uint64_t *__restrict__ q1,
                                                      uint32_t row_len, uint32_t num_rows,
                                                      uint32_t comb_limbs, FieldCfg f,
                                                      uint64_t *__restrict__ wprime,
                                                      uint64_t *__restrict__ partial) {
    __shared__ i128 s_alpha[64];
    __shared__ uint64_t s_red[256 * L];
    const uint32_t b = blockIdx.z, j = blockIdx.y;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (binary == 1) {
        for (uint32_t i = threadIdx.x; i < D; i += blockDim.x) s_alpha[i] = alphas[(size_t)b * D + i];
    }
    __syncthreads();
    uint64_t fe[L];
    for (int w = 0; w < L; w++) fe[w] = 0;
    if (c < row_len) {
        const size_t e = ((size_t)b * num_rows + j) * row_len + c;
        uint64_t w3[3] = {0, 0, 0};
        if (binary == 1) {
            uint64_t x = static_cast<const uint64_t *>(evals)[e] & dmask;
            while (x) {
                const int bit = __ffsll((long long)x) - 1;
                const i128 a = s_alpha[bit];
                const uint64_t add[3] = {(uint64_t)(u128)a, (uint64_t)((u128)a >> 64),
                                         a < 0 ? ~0ull : 0ull};
                wide_add(w3, add, 3);
                x &= x - 1;
            }
        } else {
            const int64_t v = binary == 2 ? static_cast<const int64_t *>(evals)[e]
                                          : (int64_t) static_cast<const int32_t *>(evals)[e];
            w3[0] = (uint64_t)v;
            w3[1] = w3[2] = v < 0 ? ~0ull : 0ull;
        }
        uint64_t *wo = wprime + e * comb_limbs;
        const uint64_t sg = (w3[2] >> 63) ? ~0ull : 0ull;
        for (uint32_t k = 0; k < comb_limbs; k++) wo[k] = k < 3 ? w3[k] : sg;
        // |w3| < 2^134 (at most 64 alphas of 128 bits, or one 64-bit value) is
        // below R, which is all the Montgomery product asks of its first operand.
        // Times q1 (the Montgomery form Q R of the eq entry) it gives the plain
        // residue of |w3| Q: one product where the conversion to Montgomery form
        // took another.  The block's plain sum is put into Montgomery form once,
        // times R^2 (the sum is linear, so the same value).
        const bool neg = (w3[2] >> 63) != 0;
        uint64_t mag[L];
        uint64_t cy = neg ? 1 : 0;
        for (int w = 0; w < L; w++) {
            const uint64_t v = w < 3 ? (neg ? ~w3[w] : w3[w]) : 0;
            mag[w] = v + cy;
            cy = mag[w] < cy;
        }
        fmul<L>(mag, q1 + (size_t)c * L, f.p, f.n0, fe);
        if (neg) fneg<L>(fe, f.p);
    }
    for (int w = 0; w < L; w++) s_red[threadIdx.x * L + w] = fe[w];
    __syncthreads();
    for (uint32_t h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) fadd<L>(&s_red[threadIdx.x * L], &s_red[(threadIdx.x + h) * L], f.p);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        uint64_t *po = partial + (((size_t)b * num_rows + j) * gridDim.x + blockIdx.x) * L;
        uint64_t m[L];
        fmul<L>(&s_red[0], f.r2, f.p, f.n0, m);
        for (int w = 0; w < L; w++) po[w] = m[w];
    }
}

// blockDim (32, Y): 32 columns per block, the batch x num_rows products of a
// column split over Y threads, whose partial sums (exact, wrapping at
// 64 * comb_limbs bits, so their order is free) are added in shared memory.
// With one thread per column, a tall matrix (RAA: 256 rows of 256) ran a
// chain of 256 dependent multiply-adds on 256 threads.
__global__ void __launch_bounds__(1024) k_combined_row(const uint64_t *__restrict__ wprime,
                                                       const i128 *__restrict__ coeffs,
                                                       uint32_t batch, uint32_t num_rows,
                                                       uint32_t row_len, uint32_t comb_limbs,
                                                       uint64_t *__restrict__ out) {
    extern __shared__ uint64_t part[];  // [Y][32][comb_limbs]
    const uint32_t tx = threadIdx.x, ty = threadIdx.y, Y = blockDim.y;
    const uint32_t c = blockIdx.x * 32 + tx;
    uint64_t acc[MAX_COMB_LIMBS];
    for (uint32_t k = 0; k < comb_limbs; k++) acc[k] = 0;
    const uint32_t total = batch * num_rows;
    if (c < row_len)
        for (uint32_t q = ty; q < total; q += Y)  // q = b * num_rows + j
            wide_mul_i128_add(acc, wprime + ((size_t)q * row_len + c) * comb_limbs, coeffs[q % num_rows],
                              (int)comb_limbs);
    for (uint32_t k = 0; k < comb_limbs; k++) part[((size_t)ty * 32 + tx) * comb_limbs + k] = acc[k];
    __syncthreads();
    if (ty != 0 || c >= row_len) return;
    for (uint32_t y = 1; y < Y; y++) {
        const uint64_t *p = part + ((size_t)y * 32 + tx) * comb_limbs;
        uint64_t carry = 0;
        for (uint32_t k = 0; k < comb_limbs; k++) {
            const uint64_t t = acc[k] + carry, c1 = t < carry;
            const uint64_t u = t + p[k], c2 = u < t;
            acc[k] = u;
            carry = c1 | c2;
        }
    }
    for (uint32_t k = 0; k < comb_limbs; k++) out[(size_t)c * comb_limbs + k] = acc[k];
}

// One block per opening: column bytes, u64 leaf_index, u64 leaf_count,
// u64 path length, then the sibling path bottom-up.
__global__ void k_openings(const uint8_t *__restrict__ cw, uint32_t leaf_bytes,
                           const uint8_t *__restrict__ tree, uint32_t depth, uint32_t width,
                           const uint32_t *__restrict__ idxs, uint8_t *__restrict__ out) {
    const uint32_t o = blockIdx.x, idx = idxs[o];
    const size_t open_bytes = (size_t)leaf_bytes + 24 + 32 * (size_t)depth;
    uint8_t *dst = out + (size_t)o * open_bytes;
    const uint32_t *src = reinterpret_cast<const uint32_t *>(cw + (size_t)idx * leaf_bytes);
    uint32_t *d32 = reinterpret_cast<uint32_t *>(dst);
    for (uint32_t w = threadIdx.x; w < leaf_bytes / 4; w += blockDim.x) d32[w] = src[w];
    if (threadIdx.x < 6) {
        const uint64_t v[3] = {idx, width, depth};
        const uint32_t word = threadIdx.x & 1 ? (uint32_t)(v[threadIdx.x / 2] >> 32)
                                              : (uint32_t)v[threadIdx.x / 2];
        reinterpret_cast<uint32_t *>(dst + leaf_bytes)[threadIdx.x] = word;
    }
    const uint32_t nw = 8 * depth;
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
        const uint32_t k = w / 8, part = w % 8;
        const uint64_t node = 2ull * width - 2ull * (width >> k) + ((idx >> k) ^ 1u);
        reinterpret_cast<uint32_t *>(dst + leaf_bytes + 24)[w] =
            reinterpret_cast<const uint32_t *>(tree)[node * 8 + part];
    }
}

// ---------------------------------------------------------------------------
template <int L>
static zg_status eq_table_t(zg_ctx *ctx, const uint64_t *r_d, const uint64_t *omr_d, uint32_t n,
                            const FieldCfg &f, uint64_t *out_d, cudaStream_t s) {
    const uint32_t m = 1u << n;
    ZG_KBEGIN(ctx, s, "k_eq_table");
    if (n >= 2 && n <= 20) {
        const size_t sm = ((size_t)(1u << (n / 2)) + (1u << (n - n / 2))) * L * 8;
        if (sm > 48 * 1024)
            ZG_CUDA(allow_max_smem(k_eq_table_split<L>));
        k_eq_table_split<L><<<(m + 255) / 256, 256, sm, s>>>(r_d, omr_d, n, f, out_d);
    } else {
        k_eq_table<L><<<(m + 255) / 256, 256, 0, s>>>(r_d, omr_d, n, f, out_d);
    }
    ZG_KEND(ctx, s);
    return ZG_OK;
}

zg_status launch_eq_table(zg_ctx *ctx, const uint64_t *r_d, const uint64_t *omr_d, uint32_t n,
                          const FieldCfg &f, uint64_t *out_d, cudaStream_t s) {
    return f.L == 3 ? eq_table_t<3>(ctx, r_d, omr_d, n, f, out_d, s)
                    : eq_table_t<4>(ctx, r_d, omr_d, n, f, out_d, s);
}

template <int L>
static zg_status project_t(zg_ctx *ctx, const ProjectArgs &a, cudaStream_t s) {
    dim3 grid((a.row_len + 255) / 256, a.num_rows, a.batch);
    ZG_KBEGIN(ctx, s, "k_project_rows");
    k_project_rows<L><<<grid, 256, 0, s>>>(a.evals, a.binary, a.alphas, a.D, a.dmask, a.q1,
                                           a.row_len, a.num_rows, a.comb_limbs, *a.f, a.wprime,
                                           a.partial);
    ZG_KEND(ctx, s);
    return ZG_OK;
}

zg_status launch_project_rows(zg_ctx *ctx, const ProjectArgs &a, cudaStream_t s) {
    return a.f->L == 3 ? project_t<3>(ctx, a, s) : project_t<4>(ctx, a, s);
}

zg_status launch_combined_and_openings(zg_ctx *ctx, const CombineArgs &a, cudaStream_t s) {
    ZG_KBEGIN(ctx, s, "k_combined_row");
    // Y threads per column: about 2^17 threads in all, at most the rows, at most
    // 32, and their partials within 48 KB of shared memory
    uint32_t Y = 1;
    const uint32_t rows = a.batch * a.num_rows;
    while (Y < 32 && 2 * Y <= rows && (size_t)a.row_len * Y < (1u << 17) &&
           (size_t)2 * Y * 32 * a.comb_limbs * 8 <= 48 * 1024)
        Y *= 2;
    k_combined_row<<<(a.row_len + 31) / 32, dim3(32, Y), (size_t)Y * 32 * a.comb_limbs * 8, s>>>(
        a.wprime, a.coeffs, a.batch, a.num_rows, a.row_len, a.comb_limbs, a.comb_out);
    ZG_KEND(ctx, s);
    ZG_KBEGIN(ctx, s, "k_openings");
    k_openings<<<a.n_open, 128, 0, s>>>(a.cw, a.leaf_bytes, a.tree, a.depth, a.width, a.idxs,
                                        a.open_out);
    ZG_KEND(ctx, s);
    return ZG_OK;
}

}  // namespace zg
