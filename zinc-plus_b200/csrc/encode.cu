// Linear-code encoders on sm_100a: the IPRS radix-8 pseudo-NTT over the
// integers (zip-plus/src/code/iprs/pntt/radix8.rs:21-161) and the RAA code
// (zip-plus/src/code/raa.rs:93-127).
//
// Layouts.  Evaluations: nrows rows of row_len values, row-major.
// Intermediates: row-major [grow][position][lane].  The final codeword is
// written either leaf-major [position][grow][lane] (a Merkle leaf's preimage
// is then contiguous) or row-major like the reference's DenseRowMatrix.
//
// Arithmetic is wrapping two's complement at the codeword width (i64 lanes for
// binary polynomials, i128 for i32 evaluations).  Wrapping arithmetic is a
// ring homomorphism, so the order of additions does not change any output,
// and when the reference's checked arithmetic does not overflow the values are
// identical.
#include <type_traits>
#include <algorithm>

#include "zg_internal.h"
#include "zg_umma.cuh"

namespace zg {

__device__ __forceinline__ uint32_t octet_reverse(uint32_t x, uint32_t digits) {
    // octet_reversal.rs:6-29: reverse the base-8 digits of x.
    uint32_t r = 0;
    for (uint32_t i = 0; i < digits; i++) {
        r = (r << 3) | (x & 7u);
        x >>= 3;
    }
    return r;
}

// ---------------------------------------------------------------------------
// Leaf-major position of (codeword position p, global row grow).  The rows of a
// launch form segments of 2^seg_log rows, one polynomial each, and every
// segment is its own C x 2^seg_log block (its polynomial's codeword); seg_log
// >= 32 means a single segment of nrows rows.
__device__ __forceinline__ size_t lm_pos(size_t p, uint32_t grow, uint32_t nrows, uint32_t C,
                                         uint32_t seg_log) {
    if (seg_log >= 32) return p * nrows + grow;
    const size_t seg = grow >> seg_log;
    return ((seg * C + p) << seg_log) + (grow & ((1u << seg_log) - 1u));
}

// Base layer, binary evaluations (base_multiply_into_output, radix8.rs:117-161):
//   out[ch*bd + rb][lane] = sum_c bit_lane(in[octrev(ch) + c*8^depth]) * bm[rb][c]
// Block: 32 base rows x ceil(D/8) lane groups; the chunk's inputs are staged
// in shared memory.  Binary sums are < 2^31 for every legal code (|bm| <= 32769,
// base_len < 2^14), so they accumulate in int32.
template <bool FINAL, bool LEAF_MAJOR>
__global__ void __launch_bounds__(256) k_base_bin(const uint64_t *__restrict__ evals,
                                                  const int32_t *__restrict__ bmT, void *out,
                                                  uint32_t row_len, uint32_t bd, uint32_t bl,
                                                  uint32_t depth, uint32_t C, uint32_t D,
                                                  uint64_t dmask, uint32_t nrows,
                                                  uint32_t seg_log) {
    extern __shared__ uint64_t sx[];
    const uint32_t grow = blockIdx.z, ch = blockIdx.y;
    const uint32_t oct = octet_reverse(ch, depth);
    const uint32_t shift = 3 * depth;
    const uint64_t *row = evals + (size_t)grow * row_len;
    const uint32_t tid = threadIdx.y * 32 + threadIdx.x, nthr = 32 * blockDim.y;
    for (uint32_t c = tid; c < bl; c += nthr) sx[c] = row[oct + ((size_t)c << shift)] & dmask;
    __syncthreads();
    const uint32_t rb = blockIdx.x * 32 + threadIdx.x;
    if (rb >= bd) return;
    const uint32_t g = threadIdx.y;
    int32_t acc[8];
#pragma unroll
    for (int j = 0; j < 8; j++) acc[j] = 0;
    const int32_t *bcol = bmT + rb;
    for (uint32_t c = 0; c < bl; c++) {
        const uint32_t x = (uint32_t)(sx[c] >> (8 * g));
        const int32_t b = __ldg(bcol + (size_t)c * bd);
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] += (int32_t)((x >> j) & 1u) * b;
    }
    const size_t p = (size_t)ch * bd + rb;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const uint32_t lane = 8 * g + j;
        if (lane >= D) break;
        if (FINAL) {
            int64_t *o = static_cast<int64_t *>(out);
            size_t idx = LEAF_MAJOR ? lm_pos(p, grow, nrows, C, seg_log) * D + lane : ((size_t)grow * C + p) * D + lane;
            o[idx] = acc[j];
        } else {
            static_cast<int32_t *>(out)[((size_t)grow * C + p) * D + lane] = acc[j];
        }
    }
}

// Base layer, binary evaluations, two coefficient lanes per 64-bit multiply.
// A lane's sum is |sum_c bm[rb][c] * bit| <= base_len * 32769 < 2^29 whenever
// base_len < 16383, so lanes 2j and 2j+1 share one int64 accumulator as
// lane_2j + 2^30 * lane_2j+1: each step adds bm * (b_2j + 2^30 b_2j+1), one
// 32x32->64 multiply-add for two lanes.  The packed multipliers of a byte of
// lane bits come from a 256-entry table.  Each thread owns 8 base rows x 8
// lanes; a block owns 128 base rows and every lane group of one chunk.
constexpr uint32_t kBase2Rows = 128;

template <bool FINAL, bool LEAF_MAJOR>
__global__ void __launch_bounds__(128) k_base_bin2(const uint64_t *__restrict__ evals,
                                                   const int32_t *__restrict__ bmP, void *out,
                                                   uint32_t row_len, uint32_t bd, uint32_t bdp,
                                                   uint32_t bl, uint32_t depth, uint32_t C,
                                                   uint32_t D, uint64_t dmask, uint32_t nrows,
                                                   uint32_t seg_log) {
    extern __shared__ __align__(16) uint8_t smem2[];
    uint4 *lut = reinterpret_cast<uint4 *>(smem2);  // 256 x 4 packed multipliers
    uint8_t *sxb = smem2 + 256 * sizeof(uint4);     // [group][c] lane bits
    const uint32_t ngroups = blockDim.y;
    const uint32_t grow = blockIdx.z, ch = blockIdx.y;
    const uint32_t tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * ngroups;
    for (uint32_t v = tid; v < 256; v += nthr) {
        uint32_t m[4];
#pragma unroll
        for (int j = 0; j < 4; j++) m[j] = ((v >> (2 * j)) & 1u) | (((v >> (2 * j + 1)) & 1u) << 30);
        lut[v] = make_uint4(m[0], m[1], m[2], m[3]);
    }
    const uint32_t oct = octet_reverse(ch, depth), shift = 3 * depth;
    const uint64_t *row = evals + (size_t)grow * row_len;
    for (uint32_t c = tid; c < bl; c += nthr) {
        const uint64_t x = row[oct + ((size_t)c << shift)] & dmask;
        for (uint32_t g = 0; g < ngroups; g++) sxb[(size_t)g * bl + c] = (uint8_t)(x >> (8 * g));
    }
    __syncthreads();
    const uint32_t r0 = (blockIdx.x * blockDim.x + threadIdx.x) * 8;
    if (r0 >= bd) return;
    const uint32_t g = threadIdx.y;
    long long acc[8][4];
#pragma unroll
    for (int r = 0; r < 8; r++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[r][j] = 0;
    const int4 *bp = reinterpret_cast<const int4 *>(bmP + r0);
    const uint32_t bstride = bdp / 4;
    const uint8_t *xg = sxb + (size_t)g * bl;
#pragma unroll 2
    for (uint32_t c = 0; c < bl; c++) {
        const uint4 m = lut[xg[c]];
        const int4 b0 = __ldg(bp + (size_t)c * bstride), b1 = __ldg(bp + (size_t)c * bstride + 1);
        const int bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
        const int mv[4] = {(int)m.x, (int)m.y, (int)m.z, (int)m.w};
#pragma unroll
        for (int r = 0; r < 8; r++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[r][j] += (long long)bv[r] * mv[j];
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const uint32_t rb = r0 + r;
        if (rb >= bd) break;
        const size_t p = (size_t)ch * bd + rb;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const long long a = acc[r][j];
            const long long lo = (long long)((unsigned long long)a << 34) >> 34;
            const long long hi = (a - lo) >> 30;
            const long long v2[2] = {lo, hi};
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const uint32_t lane = 8 * g + 2 * j + h;
                if (lane >= D) continue;
                if (FINAL) {
                    int64_t *o = static_cast<int64_t *>(out);
                    o[LEAF_MAJOR ? lm_pos(p, grow, nrows, C, seg_log) * D + lane : ((size_t)grow * C + p) * D + lane] = v2[h];
                } else {
                    static_cast<int32_t *>(out)[((size_t)grow * C + p) * D + lane] = (int32_t)v2[h];
                }
            }
        }
    }
}

// Base layer, binary evaluations: the packed-lane multiply of k_base_bin2
// with the block's slice of the base matrix (TR rows x base_len) staged in
// shared memory once and reused by kBase3Chunks chunks, so the inner loop reads
// only shared memory.  Thread = (row octet, lane group, chunk); a warp holds
// all row octets of one chunk, so its base-matrix reads are broadcasts.
constexpr uint32_t kBase3Chunks = 8;

template <uint32_t TR, bool FINAL, bool LEAF_MAJOR>
__global__ void __launch_bounds__(512) k_base_bin3(const uint64_t *__restrict__ evals,
                                                   const int32_t *__restrict__ bmP, void *out,
                                                   uint32_t row_len, uint32_t bd, uint32_t bdp,
                                                   uint32_t bl, uint32_t depth, uint32_t nch,
                                                   uint32_t C, uint32_t D, uint32_t ngroups,
                                                   uint64_t dmask, uint32_t nrows,
                                                   uint32_t seg_log) {
    extern __shared__ __align__(16) uint8_t smem3[];
    constexpr uint32_t RO = TR / 8;
    int4 *bmS = reinterpret_cast<int4 *>(smem3);                  // [bl][TR/4]
    uint4 *lut = reinterpret_cast<uint4 *>(smem3 + (size_t)bl * TR * 4);
    uint8_t *xs = reinterpret_cast<uint8_t *>(lut + 256);           // [chunk][group][bl]
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t rb0 = blockIdx.x * TR, ch0 = blockIdx.y * kBase3Chunks, grow = blockIdx.z;
    // base-matrix slice (rows past bd read as zero)
    for (uint32_t e = tid; e < bl * (TR / 4); e += nthr) {
        const uint32_t c = e / (TR / 4), r4 = (e % (TR / 4)) * 4;
        int4 v = make_int4(0, 0, 0, 0);
        if (rb0 + r4 < bdp) v = __ldg(reinterpret_cast<const int4 *>(bmP + (size_t)c * bdp + rb0 + r4));
        bmS[e] = v;
    }
    for (uint32_t v = tid; v < 256; v += nthr) {
        uint32_t m[4];
#pragma unroll
        for (int j = 0; j < 4; j++) m[j] = ((v >> (2 * j)) & 1u) | (((v >> (2 * j + 1)) & 1u) << 30);
        lut[v] = make_uint4(m[0], m[1], m[2], m[3]);
    }
    const uint32_t shift = 3 * depth;
    const uint64_t *row = evals + (size_t)grow * row_len;
    for (uint32_t e = tid; e < kBase3Chunks * bl; e += nthr) {
        const uint32_t chl = e / bl, c = e % bl, ch = ch0 + chl;
        uint64_t x = 0;
        if (ch < nch) x = row[octet_reverse(ch, depth) + ((size_t)c << shift)] & dmask;
        for (uint32_t g = 0; g < ngroups; g++) xs[((size_t)chl * ngroups + g) * bl + c] = (uint8_t)(x >> (8 * g));
    }
    __syncthreads();
    const uint32_t ro = tid % RO, g = (tid / RO) % ngroups, chl = tid / (RO * ngroups);
    const uint32_t ch = ch0 + chl, r0 = rb0 + 8 * ro;
    if (chl >= kBase3Chunks || ch >= nch || r0 >= bd) return;
    long long acc[8][4];
#pragma unroll
    for (int r = 0; r < 8; r++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[r][j] = 0;
    const uint8_t *xg = xs + ((size_t)chl * ngroups + g) * bl;
    const int4 *bs = bmS + 2 * ro;
#pragma unroll 4
    for (uint32_t c = 0; c < bl; c++) {
        const uint4 m = lut[xg[c]];
        const int4 b0 = bs[(size_t)c * (TR / 4)], b1 = bs[(size_t)c * (TR / 4) + 1];
        const int bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
        const int mv[4] = {(int)m.x, (int)m.y, (int)m.z, (int)m.w};
#pragma unroll
        for (int r = 0; r < 8; r++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[r][j] += (long long)bv[r] * mv[j];
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const uint32_t rb = r0 + r;
        if (rb >= bd) break;
        const size_t p = (size_t)ch * bd + rb;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const long long a = acc[r][j];
            const long long lo = (long long)((unsigned long long)a << 34) >> 34;
            const long long hi = (a - lo) >> 30;
            const long long v2[2] = {lo, hi};
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const uint32_t lane = 8 * g + 2 * j + h;
                if (lane >= D) continue;
                if (FINAL) {
                    int64_t *o = static_cast<int64_t *>(out);
                    o[LEAF_MAJOR ? lm_pos(p, grow, nrows, C, seg_log) * D + lane : ((size_t)grow * C + p) * D + lane] = v2[h];
                } else {
                    static_cast<int32_t *>(out)[((size_t)grow * C + p) * D + lane] = (int32_t)v2[h];
                }
            }
        }
    }
}

// Base layer, binary evaluations, on the tensor cores.  For one chunk of one
// codeword row the base layer is the exact integer product
//   base[rb][lane] = sum_c bm[rb][c] * bit_lane(x_c),
// an (bd x bl) by (bl x D) matrix product with {0,1} entries on the right.
// bm in [-32769, 32767] splits exactly into unsigned bytes,
//   bm = l0 + 256 l1 - 65536 [bm < 0],   l0, l1 in [0, 255],
// so three u8 x u8 -> s32 MMAs (m16n8k32) per tile give the exact result; no
// partial sum exceeds 255 * bl < 2^31.  A (the limbs) is staged in shared
// memory and read with ldmatrix; B is built in registers from the lane masks
// with byte permutes (bit n of the input words is column n of B).
//
// Block: 4 warps over a 64-row slice of the base matrix; warp (mw, cw) owns
// rows 32 mw .. 32 mw + 31 (two m16 tiles) and every other (row, chunk) pair of
// the block's kMmaPairs pairs.  Lanes are processed 32 at a time (four n8 tiles).
constexpr uint32_t kMmaRows = 64;
constexpr uint32_t kMmaPairs = 8;  // default pairs per block (variants: 4, 8, 16)

__device__ __forceinline__ void mma_u8_16x8x32(int (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                               uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t (&r)[4], const void *smem_ptr) {
    const uint32_t addr = (uint32_t)__cvta_generic_to_shared(smem_ptr);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

// B fragments of four n8 tiles from four input words: word i holds the lanes
// of input k0 + 4t + i; the result for tile nt has byte i = bit (8 nt + g).
__device__ __forceinline__ void bits_to_bfrag(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3,
                                              uint32_t g, uint32_t (&b)[4]) {
    const uint32_t y0 = (x0 >> g) & 0x01010101u, y1 = (x1 >> g) & 0x01010101u;
    const uint32_t y2 = (x2 >> g) & 0x01010101u, y3 = (x3 >> g) & 0x01010101u;
    const uint32_t lo01 = __byte_perm(y0, y1, 0x5140), hi01 = __byte_perm(y0, y1, 0x7362);
    const uint32_t lo23 = __byte_perm(y2, y3, 0x5140), hi23 = __byte_perm(y2, y3, 0x7362);
    b[0] = __byte_perm(lo01, lo23, 0x5410);
    b[1] = __byte_perm(lo01, lo23, 0x7632);
    b[2] = __byte_perm(hi01, hi23, 0x5410);
    b[3] = __byte_perm(hi01, hi23, 0x7632);
}

template <uint32_t PAIRS>
__global__ void __launch_bounds__(128) k_base_mma(const uint64_t *__restrict__ evals,
                                                  const uint8_t *__restrict__ bmL,
                                                  int32_t *__restrict__ out, uint32_t row_len,
                                                  uint32_t bd, uint32_t bl, uint32_t blp,
                                                  uint32_t depth, uint32_t nch, uint32_t C,
                                                  uint32_t D, uint64_t dmask, uint32_t nrows) {
    extern __shared__ __align__(16) uint8_t smem_m[];
    const uint32_t astride = blp + 16;  // padded row: conflict-free ldmatrix
    uint8_t *As = smem_m;                                               // [3][64][astride]
    uint64_t *Xs = reinterpret_cast<uint64_t *>(smem_m + 3 * kMmaRows * astride);  // [pairs][blp]
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t rb0 = blockIdx.x * kMmaRows;
    const uint32_t pair0 = blockIdx.y * PAIRS, npairs = nrows * nch;
    // A slice: 16-byte pieces (limb, row, k); rows past bd and k past bl are zero
    const uint32_t pieces_per_row = blp / 16;
    for (uint32_t e = tid; e < 3 * kMmaRows * pieces_per_row; e += nthr) {
        const uint32_t limb = e / (kMmaRows * pieces_per_row);
        const uint32_t rem = e % (kMmaRows * pieces_per_row);
        const uint32_t row = rem / pieces_per_row, k = (rem % pieces_per_row) * 16;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (rb0 + row < bd && k < bl)
            v = __ldg(reinterpret_cast<const uint4 *>(bmL + ((size_t)limb * bd + rb0 + row) * blp + k));
        *reinterpret_cast<uint4 *>(As + ((size_t)limb * kMmaRows + row) * astride + k) = v;
    }
    const uint32_t shift = 3 * depth;
    for (uint32_t e = tid; e < PAIRS * blp; e += nthr) {
        const uint32_t pi = e / blp, c = e % blp, pair = pair0 + pi;
        uint64_t x = 0;
        if (pair < npairs && c < bl) {
            const uint32_t grow = pair / nch, ch = pair % nch;
            x = evals[(size_t)grow * row_len + octet_reverse(ch, depth) + ((size_t)c << shift)] & dmask;
        }
        Xs[e] = x;
    }
    __syncthreads();
    const uint32_t lane = tid & 31, warp = tid >> 5;
    const uint32_t mw = warp & 1, cw = warp >> 1;
    const uint32_t g = lane >> 2, t = lane & 3;
    const uint32_t lrow = lane & 15, lk = (lane >> 4) * 16;
    for (uint32_t pi = cw; pi < PAIRS; pi += 2) {
        const uint32_t pair = pair0 + pi;
        if (pair >= npairs) break;
        const uint32_t grow = pair / nch, ch = pair % nch;
        const uint64_t *xp = Xs + (size_t)pi * blp;
        for (uint32_t half = 0; half * 32 < D; half++) {
            int acc[2][4][3][4];
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int b = 0; b < 4; b++)
#pragma unroll
                    for (int c = 0; c < 3; c++)
#pragma unroll
                        for (int d = 0; d < 4; d++) acc[a][b][c][d] = 0;
            for (uint32_t k0 = 0; k0 < blp; k0 += 32) {
                uint32_t afr[2][3][4];
#pragma unroll
                for (int mt = 0; mt < 2; mt++)
#pragma unroll
                    for (int limb = 0; limb < 3; limb++)
                        ldmatrix_x4(afr[mt][limb], As + ((size_t)limb * kMmaRows + 32 * mw + 16 * mt + lrow) * astride + k0 + lk);
                uint32_t xw[8];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    xw[i] = (uint32_t)(xp[k0 + 4 * t + i] >> (32 * half));
                    xw[4 + i] = (uint32_t)(xp[k0 + 16 + 4 * t + i] >> (32 * half));
                }
                uint32_t b0[4], b1[4];
                bits_to_bfrag(xw[0], xw[1], xw[2], xw[3], g, b0);
                bits_to_bfrag(xw[4], xw[5], xw[6], xw[7], g, b1);
#pragma unroll
                for (int mt = 0; mt < 2; mt++)
#pragma unroll
                    for (int nt = 0; nt < 4; nt++)
#pragma unroll
                        for (int limb = 0; limb < 3; limb++) mma_u8_16x8x32(acc[mt][nt][limb], afr[mt][limb], b0[nt], b1[nt]);
            }
#pragma unroll
            for (int mt = 0; mt < 2; mt++)
#pragma unroll
                for (int nt = 0; nt < 4; nt++)
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const uint32_t r = rb0 + 32 * mw + 16 * mt + g + (e >= 2 ? 8 : 0);
                        const uint32_t ln = 32 * half + 8 * nt + 2 * t + (e & 1);
                        if (r < bd && ln < D) {
                            const long long v = (long long)acc[mt][nt][0][e] + 256ll * acc[mt][nt][1][e] -
                                                65536ll * acc[mt][nt][2][e];
                            out[((size_t)grow * C + (size_t)ch * bd + r) * D + ln] = (int32_t)v;
                        }
                    }
        }
    }
}

// Base layer on the 5th-generation tensor cores (tcgen05, accumulators in
// tensor memory).  The same sums as k_base_mma, as one GEMM per tile:
//   D[m][n] = sum_k bits[m][k] * (bm[n][k] + off[n]),
//   out = D[m][n] - off[n] * popcount(bits[m][.]),
// m = (pair, lane) of 128 input rows, n = NT base rows, k < round_up(bl, 128).
// The offset brings every base row into [-2^15, 2^15), so two 8-bit MMAs
// give it exactly: the u8 low byte and the s8 high byte (x 256).  The table
// holds -off[n].
//
// Tile pairs are taken in octet-reversed chunk order: slot q of a codeword row
// is chunk octet_reverse(q), whose inputs are evals[q + k 8^depth], so the
// tile's pairs read adjacent evaluations.  Input bits are expanded into the A
// tile (K-major, 128-byte swizzle) by the CTA's threads; the pre-swizzled
// base-matrix tile arrives by one bulk copy per (limb, 128-column atom); one
// thread issues the MMAs and commits them to an mbarrier; TMEM lane m is A row
// m, so a warp holds one pair's 32 lanes (D <= 32) and writes each base row's
// lanes as one 128-byte line.  Waits are bounded (umma::mbar_wait*): on a
// timeout the CTA sets the device status word, stores nothing, frees its
// tensor memory and returns.

// Expands the input bits of m-tile `mt` into the A tile: tasks (pair, 32-lane
// half, 8 inputs) strided over `nthr` threads starting at `t0`.
__device__ __forceinline__ void umma_fill_a(uint8_t *A, const uint64_t *__restrict__ evals, uint32_t mt,
                                            uint32_t t0, uint32_t nthr, uint32_t lp, uint32_t kp,
                                            uint32_t bl, uint32_t shift, uint32_t nch, uint32_t row_len,
                                            uint64_t dmask, uint32_t npairs) {
    const uint32_t ppt = 128 / lp, halves = lp / 32, ntask = ppt * halves * (kp / 8);
    for (uint32_t task = t0; task < ntask; task += nthr) {
        const uint32_t pi = task % ppt, rest = task / ppt;
        const uint32_t hw = rest % halves, g8 = rest / halves;
        const uint32_t gp = mt * ppt + pi;
        uint32_t x[8];
        if (gp < npairs) {
            const uint64_t *src = evals + (size_t)(gp / nch) * row_len + (gp % nch);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const uint32_t k = 8 * g8 + i;
                x[i] = k < bl ? (uint32_t)((__ldg(src + ((size_t)k << shift)) & dmask) >> (32 * hw)) : 0u;
            }
        } else {
#pragma unroll
            for (int i = 0; i < 8; i++) x[i] = 0;
        }
#pragma unroll
        for (uint32_t g = 0; g < 8; g++) {
            uint32_t b0[4], b1[4];
            bits_to_bfrag(x[0], x[1], x[2], x[3], g, b0);
            bits_to_bfrag(x[4], x[5], x[6], x[7], g, b1);
#pragma unroll
            for (uint32_t bb = 0; bb < 4; bb++) {
                const uint32_t row = pi * lp + 32 * hw + g + 8 * bb;
                *reinterpret_cast<uint2 *>(A + umma::sw128_offset(row, 8 * g8, 128)) = make_uint2(b0[bb], b1[bb]);
            }
        }
    }
}

// Set bits of A row `row`.  Chunks are read in the order j ^ (row % 8), so
// eight consecutive rows touch all 32 banks (conflict-free).
__device__ __forceinline__ uint32_t umma_row_popcount(const uint8_t *A, uint32_t row, uint32_t atoms) {
    uint32_t c = 0;
    for (uint32_t a = 0; a < atoms; a++)
#pragma unroll
        for (uint32_t j = 0; j < 8; j++) {
            const uint4 v = *reinterpret_cast<const uint4 *>(A + a * 128 * 128 + row * 128 + ((j ^ (row & 7u)) << 4));
            c = __dp4a(v.x, 0x01010101u, c);
            c = __dp4a(v.y, 0x01010101u, c);
            c = __dp4a(v.z, 0x01010101u, c);
            c = __dp4a(v.w, 0x01010101u, c);
        }
    return c;
}

// Epilogue of one 32-column chunk: TMEM columns col (low limb) and col + NT
// (high limb) of this warp's lanes, base rows r0 .. r0 + 31 (nvalid of them
// below bd) written at o[q * D].  DS = D when it is 32 or 64 (immediate store
// offsets), 0 for any other D.
template <uint32_t DS, uint32_t NT>
__device__ __forceinline__ void umma_store_chunk(uint32_t taddr, const int32_t *__restrict__ noff, uint32_t r0,
                                                 bool live, int32_t *o, uint32_t cnt, uint32_t D,
                                                 uint32_t nvalid) {
    uint32_t lo[32], hi[32];
    umma::tmem_ld32(taddr, lo);
    umma::tmem_ld32(taddr + NT, hi);
    int4 o4[8];  // -off of the chunk's rows (table padded to whole 128-row tiles)
#pragma unroll
    for (int v = 0; v < 8; v++) o4[v] = __ldg(reinterpret_cast<const int4 *>(noff + r0) + v);
    umma::tmem_wait_ld();
    if (!live) return;
    const uint32_t Dv = DS ? DS : D;
#define ZG_UMMA_VAL(q)                                                                             \
    (int32_t)(lo[q] + (hi[q] << 8) +                                                               \
              (uint32_t)((q & 3) == 0 ? o4[q >> 2].x : (q & 3) == 1 ? o4[q >> 2].y : (q & 3) == 2 ? o4[q >> 2].z : o4[q >> 2].w) * cnt)
    if (nvalid >= 32) {
#pragma unroll
        for (uint32_t q = 0; q < 32; q++) o[q * Dv] = ZG_UMMA_VAL(q);
    } else {
#pragma unroll
        for (uint32_t q = 0; q < 32; q++)
            if (q < nvalid) o[q * Dv] = ZG_UMMA_VAL(q);
    }
#undef ZG_UMMA_VAL
}

// One tile per CTA (4 warps).
template <uint32_t NT, uint32_t DS>
__global__ void __launch_bounds__(128) k_base_umma(const uint64_t *__restrict__ evals,
                                                   const uint8_t *__restrict__ bm_img,
                                                   const int32_t *__restrict__ bm_noff,
                                                   int32_t *__restrict__ out, uint32_t row_len,
                                                   uint32_t bd, uint32_t bl, uint32_t kp,
                                                   uint32_t depth, uint32_t nch, uint32_t C,
                                                   uint32_t D, uint64_t dmask, uint32_t npairs,
                                                   uint32_t lp, uint32_t *status) {
    using namespace umma;
    constexpr uint32_t kCols = 2 * NT;  // two limb accumulators of NT columns
    extern __shared__ __align__(16) uint8_t smem_u[];
    uint8_t *As = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_u) + 1023) & ~uintptr_t(1023));
    uint8_t *Bs = As + 128 * kp;  // [limb][kp / 128][NT][128]
    uint64_t *bars = reinterpret_cast<uint64_t *>(Bs + 2 * NT * kp);  // loaded, MMA done
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t atoms = kp / 128, mt = blockIdx.x, nt = blockIdx.y;

    if (warp == 0) {
        tmem_alloc(tslot, kCols);
        tmem_relinquish();
    }
    if (tid == 32) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (tid == 32) {
        // base-matrix limbs of rows nt*NT .. +NT: NT x 128 bytes per (limb, atom)
        mbar_arrive_expect_tx(&bars[0], 2 * NT * kp);
        const uint32_t t_img = (nt * NT) / kUmmaImgRows, row0 = (nt * NT) % kUmmaImgRows;
        for (uint32_t l = 0; l < 2; l++)
            for (uint32_t a = 0; a < atoms; a++)
                bulk_g2s(Bs + (size_t)(l * atoms + a) * NT * 128,
                         bm_img + ((((size_t)t_img * 2 + l) * atoms + a) * kUmmaImgRows + row0) * 128,
                         NT * 128, &bars[0]);
    }
    umma_fill_a(As, evals, mt, tid, 128, lp, kp, bl, 3 * depth, nch, row_len, dmask, npairs);
    fence_async_smem();
    __syncthreads();

    // every thread observes the copy's completion itself
    const bool loaded = mbar_wait(&bars[0], 0);
    if (tid == 0) {
        if (!loaded) {
            report_status(status, kStatusLoadTimeout);
            mbar_arrive(&bars[1]);
        } else {
            tc_fence_after();
            const uint32_t id_lo = idesc_i8(128, NT, false, false);
            const uint32_t id_hi = idesc_i8(128, NT, true, true);
            const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs), b1 = b0 + atoms * NT * 128;
            for (uint32_t ks = 0; ks < kp / 32; ks++) {
                const uint32_t a = ks >> 2, o = (ks & 3) * 32;
                const uint64_t ad = sdesc_k_sw128(a0 + a * 128 * 128 + o);
                mma_i8(tmem, ad, sdesc_k_sw128(b0 + a * NT * 128 + o), id_lo, ks > 0);
                mma_i8(tmem + NT, ad, sdesc_k_sw128(b1 + a * NT * 128 + o), id_hi, ks > 0);
            }
            mma_commit(&bars[1]);
        }
    }
    __syncwarp();

    const uint32_t cnt = umma_row_popcount(As, tid, atoms);  // while the MMAs run
    const bool done = mbar_wait(&bars[1], 0);
    tc_fence_after();
    const bool ok = done && loaded;
    if (!done && lane == 0) report_status(status, kStatusMmaTimeout);
    if (ok) {
        const uint32_t ppt = 128 / lp, gp = mt * ppt + tid / lp, ln = tid % lp;
        const bool live = gp < npairs && ln < D;
        size_t ob = 0;
        if (live) {
            const uint32_t ch = octet_reverse(gp % nch, depth);
            ob = ((size_t)(gp / nch) * C + (size_t)ch * bd) * D + ln;
        }
        const uint32_t lane_base = tmem + ((32 * warp) << 16);
#pragma unroll 1
        for (uint32_t c = 0; c < NT / 32; c++) {
            const uint32_t r0 = nt * NT + 32 * c;
            umma_store_chunk<DS, NT>(lane_base + 32 * c, bm_noff, r0, live, out + ob + (size_t)r0 * D, cnt, D,
                                     r0 < bd ? bd - r0 : 0);
        }
    }
    // on a timeout, give copies and MMAs still in flight a second bounded wait
    if (tid == 32 && !loaded) mbar_wait(&bars[0], 0);
    if (tid == 0 && !done) mbar_wait(&bars[1], 0);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kCols);
    }
}

// Persistent, warp-specialised form of k_base_umma.  One CTA per SM walks a
// contiguous range of tiles in (m-tile, n-tile) order, so most consecutive
// tiles share their input rows, which are expanded once per m-tile.  Roles:
//   warps 0-7   epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (one A row
//               per thread) and columns of half w / 4 of the tile;
//   warp 8      producer: one bulk copy per (limb, atom) of the next base tile;
//   warp 9      MMA issuer: 2 x kp/32 MMAs per tile into one of two
//               accumulator sets, committed to the operand and TMEM barriers;
//   warps 10-11 A expansion: input bits of the next m-tile and their per-row
//               popcounts.
// A and B tiles are double-buffered in shared memory and the accumulators in
// TMEM (4 NT columns), so the MMAs of tile j+1 overlap the epilogue of tile j.
// Every wait is bounded; a timeout sets the shared abort word, every role
// leaves its loop, in-flight copies and MMAs get one more bounded wait, and
// the CTA frees its tensor memory and returns.
constexpr uint32_t kUmmaEpiWarps = 8;
constexpr uint32_t kUmmaPThreads = 32 * (kUmmaEpiWarps + 4);

template <uint32_t NT, uint32_t DS>
__global__ void __launch_bounds__(kUmmaPThreads, 1) k_base_umma_p(const uint64_t *__restrict__ evals,
                                                                 const uint8_t *__restrict__ bm_img,
                                                                 const int32_t *__restrict__ bm_noff,
                                                                 int32_t *__restrict__ out, uint32_t row_len,
                                                                 uint32_t bd, uint32_t bl, uint32_t kp,
                                                                 uint32_t depth, uint32_t nch, uint32_t C,
                                                                 uint32_t D, uint64_t dmask, uint32_t npairs,
                                                                 uint32_t lp, uint32_t ntn, uint32_t ntiles,
                                                                 uint32_t *status) {
    using namespace umma;
    constexpr uint32_t kAcc = 2 * NT;    // one accumulator set: two limbs of NT columns
    constexpr uint32_t kCols = 2 * kAcc; // two sets
    constexpr uint32_t kEpiThreads = 32 * kUmmaEpiWarps;
    constexpr uint32_t kProducer = kUmmaEpiWarps, kIssuer = kUmmaEpiWarps + 1, kExpand = kUmmaEpiWarps + 2;
    extern __shared__ __align__(16) uint8_t smem_u[];
    uint8_t *As = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_u) + 1023) & ~uintptr_t(1023));
    const uint32_t a_bytes = 128 * kp, b_bytes = 2 * NT * kp;
    uint8_t *Bs = As + 2 * a_bytes;
    uint32_t *cnt_s = reinterpret_cast<uint32_t *>(Bs + 2 * b_bytes);  // [2][128]
    uint64_t *bars = reinterpret_cast<uint64_t *>(cnt_s + 256);
    uint64_t *a_full = bars, *a_empty = bars + 2, *b_full = bars + 4, *b_empty = bars + 6;
    uint64_t *t_full = bars + 8, *t_empty = bars + 10, *fin = bars + 12;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 13);
    volatile uint32_t *abort = tslot + 1;
    uint32_t *go = tslot + 2;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ppt = 128 / lp, atoms = kp / 128;
    const uint32_t t0 = (uint32_t)((uint64_t)blockIdx.x * ntiles / gridDim.x);
    const uint32_t t1 = (uint32_t)((uint64_t)(blockIdx.x + 1) * ntiles / gridDim.x);

    if (warp == 0) {
        tmem_alloc(tslot, kCols);
        tmem_relinquish();
    }
    if (tid == 32) {
        for (int i = 0; i < 2; i++) {
            mbar_init(&a_full[i], 64);               // the expansion threads
            mbar_init(&a_empty[i], 1 + kEpiThreads); // MMA commit + the epilogue's popcount reads
            mbar_init(&b_full[i], 1);
            mbar_init(&b_empty[i], 1);
            mbar_init(&t_full[i], 1);
            mbar_init(&t_empty[i], kEpiThreads);
        }
        mbar_init(fin, 1);
        *abort = 0;
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == kProducer) {
        if (lane == 0) {
            int last_par[2] = {-1, -1};
            for (uint32_t t = t0, j = 0; t < t1; t++, j++) {
                const uint32_t s = j & 1;
                if (!mbar_wait_or_abort(&b_empty[s], ((j >> 1) & 1) ^ 1, abort)) break;
                const uint32_t n = t % ntn;
                const uint32_t t_img = (n * NT) / kUmmaImgRows, row0 = (n * NT) % kUmmaImgRows;
                mbar_arrive_expect_tx(&b_full[s], b_bytes);
                for (uint32_t l = 0; l < 2; l++)
                    for (uint32_t a = 0; a < atoms; a++)
                        bulk_g2s(Bs + s * b_bytes + (l * atoms + a) * NT * 128,
                                 bm_img + ((((size_t)t_img * 2 + l) * atoms + a) * kUmmaImgRows + row0) * 128,
                                 NT * 128, &b_full[s]);
                last_par[s] = (int)((j >> 1) & 1);
            }
            // copies still in flight (none on the normal path)
            for (int s = 0; s < 2; s++)
                if (last_par[s] >= 0) mbar_wait(&b_full[s], (uint32_t)last_par[s]);
        }
        __syncwarp();
    } else if (warp == kIssuer) {
        if (lane == 0) {
            const uint32_t id_lo = idesc_i8(128, NT, false, false), id_hi = idesc_i8(128, NT, true, true);
            uint32_t u = 0;
            for (uint32_t t = t0, j = 0; t < t1; t++, j++) {
                const uint32_t m = t / ntn;
                const bool new_m = t == t0 || m != (t - 1) / ntn;
                if (new_m && t != t0) u++;
                const uint32_t sa = u & 1, s = j & 1, acc = j & 1;
                if (new_m && !mbar_wait_or_abort(&a_full[sa], (u >> 1) & 1, abort)) break;
                if (!mbar_wait_or_abort(&b_full[s], (j >> 1) & 1, abort)) break;
                if (!mbar_wait_or_abort(&t_empty[acc], ((j >> 1) & 1) ^ 1, abort)) break;
                tc_fence_after();
                const uint32_t a0 = smem_u32(As + sa * a_bytes), b0 = smem_u32(Bs + s * b_bytes);
                const uint32_t b1 = b0 + atoms * NT * 128, d = tmem + acc * kAcc;
                for (uint32_t ks = 0; ks < kp / 32; ks++) {
                    const uint32_t a = ks >> 2, o = (ks & 3) * 32;
                    const uint64_t ad = sdesc_k_sw128(a0 + a * 128 * 128 + o);
                    mma_i8(d, ad, sdesc_k_sw128(b0 + a * NT * 128 + o), id_lo, ks > 0);
                    mma_i8(d + NT, ad, sdesc_k_sw128(b1 + a * NT * 128 + o), id_hi, ks > 0);
                }
                mma_commit(&b_empty[s]);
                mma_commit(&t_full[acc]);
                if (t + 1 == t1 || (t + 1) / ntn != m) mma_commit(&a_empty[sa]);
            }
            mma_commit(fin);
            mbar_wait(fin, 0);  // every MMA retired
        }
        __syncwarp();
    } else if (warp >= kExpand) {
        // A expansion: 64 threads; one of them waits, all follow its verdict
        const uint32_t et = tid - 32 * kExpand;
        uint32_t u = 0;
        for (uint32_t t = t0; t < t1; t++) {
            const uint32_t m = t / ntn;
            if (t != t0 && m == (t - 1) / ntn) continue;
            const uint32_t sa = u & 1;
            if (et == 0) *go = mbar_wait_or_abort(&a_empty[sa], ((u >> 1) & 1) ^ 1, abort) ? 1u : 0u;
            named_bar_sync(1, 64);
            if (!*go) break;
            uint8_t *A = As + sa * a_bytes;
            umma_fill_a(A, evals, m, et, 64, lp, kp, bl, 3 * depth, nch, row_len, dmask, npairs);
            named_bar_sync(1, 64);
            for (uint32_t row = et; row < 128; row += 64) cnt_s[sa * 128 + row] = umma_row_popcount(A, row, atoms);
            fence_async_smem();
            mbar_arrive(&a_full[sa]);
            u++;
        }
    } else {
        // epilogue: TMEM lane / A row `row`, columns of half `h` of the tile
        const uint32_t qd = warp & 3, h = warp >> 2, row = 32 * qd + lane, ln = row % lp;
        constexpr uint32_t kChunks = NT / 32 / (kUmmaEpiWarps / 4);
        uint32_t u = 0, cnt = 0;
        for (uint32_t t = t0, j = 0; t < t1; t++, j++) {
            const uint32_t m = t / ntn, n = t % ntn;
            const bool new_m = t == t0 || m != (t - 1) / ntn;
            if (new_m && t != t0) u++;
            const uint32_t acc = j & 1;
            bool ok = mbar_wait_or_abort(&t_full[acc], (j >> 1) & 1, abort);
            if (ok && new_m) ok = mbar_wait_or_abort(&a_full[u & 1], (u >> 1) & 1, abort);
            if (!__all_sync(0xFFFFFFFFu, ok)) break;
            tc_fence_after();
            if (new_m) {
                cnt = cnt_s[(u & 1) * 128 + row];
                mbar_arrive(&a_empty[u & 1]);
            }
            const uint32_t gp = m * ppt + row / lp;
            const bool live = gp < npairs && ln < D;
            size_t ob = 0;
            if (live) {
                const uint32_t ch = octet_reverse(gp % nch, depth);
                ob = ((size_t)(gp / nch) * C + (size_t)ch * bd) * D + ln;
            }
            const uint32_t lane_base = tmem + ((32 * qd) << 16) + acc * kAcc;
#pragma unroll 1
            for (uint32_t c = h * kChunks; c < (h + 1) * kChunks; c++) {
                const uint32_t r0 = n * NT + 32 * c;
                umma_store_chunk<DS, NT>(lane_base + 32 * c, bm_noff, r0, live, out + ob + (size_t)r0 * D, cnt, D,
                                         r0 < bd ? bd - r0 : 0);
            }
            tc_fence_before();
            mbar_arrive(&t_empty[acc]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (tid == 0 && *abort) report_status(status, kStatusMmaTimeout);
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kCols);
    }
}

// Both radix-8 stages of a depth-2 code (combine_stages, radix8.rs:58-113) for
// one base position rb of one codeword row and one coefficient lane, entirely
// in registers: the thread holds the 64 base outputs x[8 q + c0] (chunk 8q+c0,
// position rb), and for each r0 computes the stage-0 outputs y[q] of the eight
// chunk groups, then the stage-1 outputs, written at positions
// (8 r1 + r0) * bd + rb.  Block: D lanes x RB positions; the positions'
// twiddles (576 each, in use order) are staged in shared memory.
constexpr uint32_t kStageRB = 8;

// d = a * b + c with a 64-bit accumulator (one wide multiply-add).
__device__ __forceinline__ int64_t mad_wide_s32(int32_t a, int32_t b, int64_t c) {
    int64_t d;
    asm("mad.wide.s32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint32_t mad_lo_u32(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// Output element of position p = k * bd + rb (k = 8 r1 + r0) is out[A + k * S]:
// leaf-major single block: A = (rb * nrows + grow) * D + lane, S = bd * nrows * D;
// leaf-major segments of 2^seg_log rows: A = (((seg * C + rb) << seg_log) + r) * D + lane,
// S = (bd << seg_log) * D; row-major: A = (grow * C + rb) * D + lane, S = bd * D.
__global__ void __launch_bounds__(256, 2) k_stages2_reg(const int32_t *__restrict__ base,
                                                     int64_t *__restrict__ out,
                                                     const int32_t *__restrict__ tw2r, uint32_t C,
                                                     uint32_t bd, uint32_t D, uint32_t nrows,
                                                     uint32_t seg_log, bool leaf_major) {
    __shared__ __align__(16) int32_t ts[kStageRB * 576];
    const uint32_t lane = threadIdx.x, yi = threadIdx.y, RB = blockDim.y;
    const uint32_t rb0 = blockIdx.x * RB, grow = blockIdx.y;
    const uint32_t npos = min(RB, bd - rb0);
    const uint32_t tid = yi * blockDim.x + lane, nthr = blockDim.x * RB;
    for (uint32_t e = tid; e < npos * 576; e += nthr) ts[e] = __ldg(tw2r + (size_t)rb0 * 576 + e);
    __syncthreads();
    const uint32_t rb = rb0 + yi;
    if (yi >= npos) return;
    size_t A, S;
    if (!leaf_major) {
        A = ((size_t)grow * C + rb) * D + lane;
        S = (size_t)bd * D;
    } else if (seg_log >= 32) {
        A = ((size_t)rb * nrows + grow) * D + lane;
        S = (size_t)bd * nrows * D;
    } else {
        const size_t seg = grow >> seg_log;
        A = ((((seg * C + rb) << seg_log) + (grow & ((1u << seg_log) - 1u))) * D) + lane;
        S = ((size_t)bd << seg_log) * D;
    }
    int64_t *o = out + A;
    const int32_t *src = base + ((size_t)grow * C + rb) * D + lane;
    const size_t pstride = (size_t)bd * D;  // next chunk, same position
    int32_t x[64];
#pragma unroll
    for (int c = 0; c < 64; c++) x[c] = __ldg(src + (size_t)c * pstride);
    const int32_t *T = ts + yi * 576;
#pragma unroll
    for (int r0 = 0; r0 < 8; r0++) {
        const int4 ta = *reinterpret_cast<const int4 *>(T + r0 * 8);
        const int4 tb = *reinterpret_cast<const int4 *>(T + r0 * 8 + 4);
        const int32_t t0[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
        // stage 0: int32 inputs, twiddles below 2^17: exact 32x32->64 products
        int64_t y[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            int64_t acc = x[8 * q];
#pragma unroll
            for (int j = 1; j < 8; j++) acc = mad_wide_s32(x[8 * q + j], t0[j], acc);
            y[q] = acc;
        }
        // stage 1 modulo 2^64: y = hi * 2^32 + lo, lo the signed low word
        int32_t lo[8];
        uint32_t hi[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            lo[q] = (int32_t)(uint32_t)(uint64_t)y[q];
            hi[q] = (uint32_t)((uint64_t)y[q] >> 32) + (uint32_t)(lo[q] < 0);
        }
#pragma unroll
        for (int r1 = 0; r1 < 8; r1++) {
            const int4 ua = *reinterpret_cast<const int4 *>(T + 64 + (r0 * 8 + r1) * 8);
            const int4 ub = *reinterpret_cast<const int4 *>(T + 64 + (r0 * 8 + r1) * 8 + 4);
            const int32_t t1[8] = {ua.x, ua.y, ua.z, ua.w, ub.x, ub.y, ub.z, ub.w};
            int64_t acc = y[0];
            uint32_t hacc = 0;
#pragma unroll
            for (int j = 1; j < 8; j++) {
                acc = mad_wide_s32(lo[j], t1[j], acc);
                hacc = mad_lo_u32(hi[j], (uint32_t)t1[j], hacc);
            }
            const uint64_t z = (uint64_t)acc + ((uint64_t)hacc << 32);
            o[(size_t)(8 * r1 + r0) * S] = (int64_t)z;
        }
    }
}

// One radix-8 stage (combine_stages, radix8.rs:58-113 with
// apply_radix_8_butterflies, butterfly.rs:24-43) on 64-bit lanes:
//   y_r = x_0 + sum_{j=1..7} x_j * tw[k][i][j-1][(r*j) mod 8]
// One thread per (row, block position q, lane) computes all eight outputs.
// Twiddles are stored [(j-1)*8 + t][i] for stage k.
template <typename Tin, bool FINAL, bool LEAF_MAJOR>
__global__ void __launch_bounds__(256) k_stage_bin(const Tin *__restrict__ in,
                                                   int64_t *__restrict__ out,
                                                   const int32_t *__restrict__ tw, uint32_t C,
                                                   uint32_t sub, uint32_t D, uint32_t nrows,
                                                   uint32_t seg_log) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t C8 = C / 8;
    const size_t total = (size_t)nrows * C8 * D;
    if (t >= total) return;
    const uint32_t lane = (uint32_t)(t % D);
    const size_t rq = t / D;
    const uint32_t q = (uint32_t)(rq % C8), grow = (uint32_t)(rq / C8);
    const uint32_t blk = q / sub, i = q % sub;
    const size_t base = (size_t)grow * C + (size_t)blk * 8 * sub + i;
    // Inputs as a signed low word and a high word: x * tw mod 2^64 =
    // lo * tw + ((hi * tw) mod 2^32) * 2^32 (hi = 0 for int32 inputs).
    int64_t xf[8];
    int32_t lo[8];
    uint32_t hi[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        xf[j] = (int64_t)in[(base + (size_t)j * sub) * D + lane];
        lo[j] = (int32_t)(uint32_t)(uint64_t)xf[j];
        hi[j] = sizeof(Tin) == 4 ? 0u : (uint32_t)((uint64_t)(xf[j] - (int64_t)lo[j]) >> 32);
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
        int64_t acc = xf[0];
        uint32_t hacc = 0;
#pragma unroll
        for (int j = 1; j < 8; j++) {
            const int32_t t = __ldg(tw + (size_t)((j - 1) * 8 + ((r * j) & 7)) * sub + i);
            acc += (int64_t)lo[j] * (int64_t)t;
            if (sizeof(Tin) != 4) hacc += hi[j] * (uint32_t)t;
        }
        const uint64_t y = (uint64_t)acc + ((uint64_t)hacc << 32);
        const size_t p = (size_t)blk * 8 * sub + (size_t)r * sub + i;
        const size_t idx = (FINAL && LEAF_MAJOR) ? lm_pos(p, grow, nrows, C, seg_log) * D + lane
                                                 : ((size_t)grow * C + p) * D + lane;
        out[idx] = (int64_t)y;
    }
}

// ---------------------------------------------------------------------------
// Base layer, integer evaluations -> i128 codeword.  i32 evaluations
// (MulByScalar i32 x i64 -> i128, utils/src/mul_by_scalar.rs:89-95): |sum| <
// 2^31 * 32769 * 2^14 < 2^61 fits i64, the base values are i64.  i64
// evaluations (MulByScalar i64 x i64 -> i128, mul_by_scalar.rs:110-116): the
// sum needs i128 (< 2^63 * 2^16 * 2^14), the base values are i128.
template <typename TE, bool FINAL, bool LEAF_MAJOR>
__global__ void __launch_bounds__(256) k_base_int(const TE *__restrict__ evals,
                                                  const int32_t *__restrict__ bmT, void *out,
                                                  uint32_t row_len, uint32_t bd, uint32_t bl,
                                                  uint32_t depth, uint32_t C, uint32_t nrows,
                                                  uint32_t seg_log) {
    using Acc = typename std::conditional<sizeof(TE) == 4, int64_t, i128>::type;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nrows * C) return;
    const uint32_t p = (uint32_t)(t % C), grow = (uint32_t)(t / C);
    const uint32_t ch = p / bd, rb = p % bd;
    const uint32_t oct = octet_reverse(ch, depth), shift = 3 * depth;
    const TE *row = evals + (size_t)grow * row_len;
    Acc acc = 0;
    if (sizeof(TE) == 8 && bl <= (1u << 14)) {
        // x = hi * 2^32 + lo: with |bm| < 2^16 and bl <= 2^14 both partial sums
        // stay below 2^62 in magnitude, so two int64 sums are exact
        int64_t slo = 0, shi = 0;
        for (uint32_t c = 0; c < bl; c++) {
            const int64_t x = (int64_t)__ldg(row + oct + ((size_t)c << shift));
            const int64_t m = __ldg(bmT + (size_t)c * bd + rb);
            slo += (int64_t)(uint32_t)x * m;
            shi += (x >> 32) * m;
        }
        acc = (Acc)(((i128)shi << 32) + (i128)slo);
    } else {
        for (uint32_t c = 0; c < bl; c++)
            acc += (Acc)__ldg(row + oct + ((size_t)c << shift)) * (Acc)__ldg(bmT + (size_t)c * bd + rb);
    }
    if (FINAL) {
        i128 *o = static_cast<i128 *>(out);
        o[LEAF_MAJOR ? lm_pos(p, grow, nrows, C, seg_log) : (size_t)grow * C + p] = (i128)acc;
    } else {
        static_cast<Acc *>(out)[(size_t)grow * C + p] = acc;
    }
}

// Radix-8 stage on i128 values (MulByScalar i128 x i64, mul_by_scalar.rs:97-108).
template <typename Tin, bool FINAL, bool LEAF_MAJOR>
__global__ void __launch_bounds__(256) k_stage_i128(const Tin *__restrict__ in,
                                                    i128 *__restrict__ out,
                                                    const int32_t *__restrict__ tw, uint32_t C,
                                                    uint32_t sub, uint32_t nrows,
                                                    uint32_t seg_log) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t C8 = C / 8;
    if (t >= (size_t)nrows * C8) return;
    const uint32_t q = (uint32_t)(t % C8), grow = (uint32_t)(t / C8);
    const uint32_t blk = q / sub, i = q % sub;
    const size_t base = (size_t)grow * C + (size_t)blk * 8 * sub + i;
    u128 x[8];
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = (u128)(i128)in[base + (size_t)j * sub];
#pragma unroll
    for (int r = 0; r < 8; r++) {
        u128 y = x[0];
#pragma unroll
        for (int j = 1; j < 8; j++)
            y += x[j] * (u128)(i128)__ldg(tw + (size_t)((j - 1) * 8 + ((r * j) & 7)) * sub + i);
        const size_t p = (size_t)blk * 8 * sub + (size_t)r * sub + i;
        out[(FINAL && LEAF_MAJOR) ? lm_pos(p, grow, nrows, C, seg_log) : (size_t)grow * C + p] = (i128)y;
    }
}

// ---------------------------------------------------------------------------
// RAA (raa.rs:93-127) for binary evaluations: repeat x rep, permute by perm1,
// prefix-sum, permute by perm2, prefix-sum, on i32 lanes (wrapping).  One
// block per (row, group of LG lanes); the first prefix sum stays in shared
// memory.  perm[i] is the source position of output i (clone_shuffled).  The
// sign-flipping variant (raa_sign_flip.rs:31-69) negates the odd entries of
// the repeated row and of the first prefix sum: a gathered entry is negated
// when its source position is odd.
template <int LG>
__device__ void block_exclusive_scan(uint32_t (&v)[LG], uint32_t *warp_tot) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    uint32_t inc[LG];
#pragma unroll
    for (int l = 0; l < LG; l++) {
        uint32_t s = v[l];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t u = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += u;
        }
        inc[l] = s;
        if (lane == 31) warp_tot[wid * LG + l] = s;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int l = 0; l < LG; l++) {
            uint32_t s = lane < nw ? warp_tot[lane * LG + l] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t u = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += u;
            }
            if (lane < nw) warp_tot[lane * LG + l] = s;  // inclusive over warps
        }
    }
    __syncthreads();
#pragma unroll
    for (int l = 0; l < LG; l++) {
        uint32_t before = wid > 0 ? warp_tot[(wid - 1) * LG + l] : 0;
        v[l] = before + inc[l] - v[l];
    }
    __syncthreads();
}

template <int LG>
__global__ void k_raa_bin(const uint64_t *__restrict__ evals, const uint32_t *__restrict__ perm1,
                          const uint32_t *__restrict__ perm2, int32_t *__restrict__ out,
                          uint32_t row_len, uint32_t n, uint32_t D, uint64_t dmask,
                          uint32_t nrows, bool leaf_major, uint32_t seg_log, bool flip) {
    extern __shared__ uint32_t sm[];
    uint32_t *pre = sm;                 // n x LG
    uint32_t *wt = sm + (size_t)n * LG; // 32 x LG
    const uint32_t grow = blockIdx.x, lane0 = blockIdx.y * LG;
    const uint64_t *row = evals + (size_t)grow * row_len;
    // positions [i0, i0 + per) of this thread; n is a power of two, and
    // blockDim.x is 32 or 256, so either n is a multiple or per == 1.
    const uint32_t per = n >= blockDim.x ? n / blockDim.x : 1;
    const uint32_t i0 = threadIdx.x * per;
    const uint32_t cnt = i0 < n ? min(per, n - i0) : 0;
    // pass 1
    uint32_t tot[LG];
#pragma unroll
    for (int l = 0; l < LG; l++) tot[l] = 0;
    for (uint32_t k = 0; k < cnt; k++) {
        const uint32_t i = i0 + k;
        const uint32_t s1 = perm1[i];
        const uint64_t x = (row[s1 % row_len] & dmask) >> lane0;
        // sign-flip code: the repeated row's odd entries are negated (mod 2^32)
        const uint32_t neg = (flip && (s1 & 1u)) ? ~0u : 0u;
#pragma unroll
        for (int l = 0; l < LG; l++) {
            tot[l] += ((uint32_t)((x >> l) & 1u) ^ neg) - neg;
            pre[(size_t)i * LG + l] = tot[l];
        }
    }
    uint32_t off[LG];
#pragma unroll
    for (int l = 0; l < LG; l++) off[l] = tot[l];
    block_exclusive_scan<LG>(off, wt);
    for (uint32_t k = 0; k < cnt; k++)
#pragma unroll
        for (int l = 0; l < LG; l++) pre[(size_t)(i0 + k) * LG + l] += off[l];
    __syncthreads();
    // pass 2
#pragma unroll
    for (int l = 0; l < LG; l++) tot[l] = 0;
    for (uint32_t k = 0; k < cnt; k++) {
        const uint32_t src = perm2[i0 + k];
        const uint32_t neg = (flip && (src & 1u)) ? ~0u : 0u;  // first accumulation's odd entries
#pragma unroll
        for (int l = 0; l < LG; l++) tot[l] += (pre[(size_t)src * LG + l] ^ neg) - neg;
    }
#pragma unroll
    for (int l = 0; l < LG; l++) off[l] = tot[l];
    block_exclusive_scan<LG>(off, wt);
#pragma unroll
    for (int l = 0; l < LG; l++) tot[l] = off[l];
    for (uint32_t k = 0; k < cnt; k++) {
        const uint32_t i = i0 + k;
        const uint32_t src = perm2[i];
        const uint32_t neg = (flip && (src & 1u)) ? ~0u : 0u;
#pragma unroll
        for (int l = 0; l < LG; l++) {
            tot[l] += (pre[(size_t)src * LG + l] ^ neg) - neg;
            const uint32_t lane = lane0 + l;
            if (lane < D) {
                size_t idx = leaf_major ? lm_pos(i, grow, nrows, n, seg_log) * D + lane
                                        : ((size_t)grow * n + i) * D + lane;
                out[idx] = (int32_t)tot[l];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Selected positions of LinearCode::encode_wide (iprs.rs:148-150) on a row of
// CL-limb integers (wrapping).  Position P = ch * bd + rb of the codeword only
// depends on the 8^depth base outputs at base position rb (one per chunk), and
// stage k combines the chunks that differ in base-8 digit k of the chunk index
// (twiddle position (ch mod 8^k) * bd + rb).  One block per position: its
// threads compute the chunks' base outputs, then the stages run in shared memory.
struct TwOffsets {
    uint32_t off[4];
};

__global__ void __launch_bounds__(256) k_encode_wide_at(const uint64_t *__restrict__ row,
                                                        const int32_t *__restrict__ bmT,
                                                        const int32_t *__restrict__ tw, TwOffsets to,
                                                        uint32_t bd, uint32_t bl, uint32_t depth,
                                                        uint32_t CL, const uint32_t *__restrict__ pos,
                                                        uint64_t *__restrict__ out) {
    extern __shared__ uint64_t sv[];  // two buffers of nch x CL limbs
    const uint32_t P = pos[blockIdx.x], rb = P % bd, nch = 1u << (3 * depth);
    uint64_t *cur = sv, *nxt = sv + (size_t)nch * CL;
    for (uint32_t ch = threadIdx.x; ch < nch; ch += blockDim.x) {
        uint64_t acc[MAX_COMB_LIMBS];
        for (uint32_t w = 0; w < CL; w++) acc[w] = 0;
        const uint32_t oct = octet_reverse(ch, depth);
        for (uint32_t c = 0; c < bl; c++)
            wide_mul_s64_add(acc, row + ((size_t)oct + ((size_t)c << (3 * depth))) * CL,
                             (int64_t)__ldg(bmT + (size_t)c * bd + rb), (int)CL);
        for (uint32_t w = 0; w < CL; w++) cur[(size_t)ch * CL + w] = acc[w];
    }
    __syncthreads();
    for (uint32_t k = 0; k < depth; k++) {
        const uint32_t stride = 1u << (3 * k);
        const size_t sub = (size_t)bd << (3 * k);
        for (uint32_t ch = threadIdx.x; ch < nch; ch += blockDim.x) {
            const uint32_t r = (ch / stride) % 8, g0 = ch - r * stride;
            const size_t i = (size_t)(ch % stride) * bd + rb;
            uint64_t acc[MAX_COMB_LIMBS];
            for (uint32_t w = 0; w < CL; w++) acc[w] = cur[(size_t)g0 * CL + w];
            for (uint32_t j = 1; j < 8; j++) {
                const int32_t t = __ldg(tw + to.off[k] + (size_t)((j - 1) * 8 + ((r * j) & 7)) * sub + i);
                wide_mul_s64_add(acc, cur + (size_t)(g0 + j * stride) * CL, (int64_t)t, (int)CL);
            }
            for (uint32_t w = 0; w < CL; w++) nxt[(size_t)ch * CL + w] = acc[w];
        }
        __syncthreads();
        uint64_t *tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
    const uint32_t chp = P / bd;
    for (uint32_t w = threadIdx.x; w < CL; w += blockDim.x) out[(size_t)blockIdx.x * CL + w] = cur[(size_t)chp * CL + w];
}

static inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

zg_status launch_encode_wide_at(zg_params *p, zg_ctx *ctx, const uint64_t *row_d, uint32_t CL,
                                const uint32_t *pos_d, uint32_t n, uint64_t *out_d, cudaStream_t s) {
    const zg_params_info &I = p->info;
    if (p->d.code_kind != ZG_CODE_IPRS || I.depth > 3 || CL > (uint32_t)MAX_COMB_LIMBS || n == 0) {
        set_error("selected-position encode_wide needs an IPRS code of depth <= 3");
        return ZG_ERR_INVALID_PARAM;
    }
    TwOffsets to{};
    for (uint32_t k = 0; k < I.depth; k++) to.off[k] = (uint32_t)p->tw_dev_off[k];
    const uint32_t nch = 1u << (3 * I.depth);
    const size_t smem = (size_t)2 * nch * CL * 8;
    ZG_CUDA(allow_max_smem(k_encode_wide_at));
    ZG_KBEGIN(ctx, s, "k_encode_wide_at");
    k_encode_wide_at<<<n, std::min<uint32_t>(256, std::max<uint32_t>(32, nch)), smem, s>>>(
        row_d, p->d_bmT, p->d_tw, to, I.base_dim, I.base_len, I.depth, CL, pos_d, out_d);
    ZG_KEND(ctx, s);
    return ZG_OK;
}

// IPRS encode of i32 or i64 evaluation rows into i128 codewords: the base
// layer (i64 values for i32 evaluations, i128 for i64) then the radix-8
// stages on i128.
template <typename TE>
static zg_status encode_int_rows(zg_params *p, zg_ctx *ctx, const TE *ev, uint8_t *out_d, uint32_t nrows,
                                 bool leaf_major, uint32_t seg_log, cudaStream_t s) {
    using Base = typename std::conditional<sizeof(TE) == 4, int64_t, i128>::type;
    const zg_params_info &I = p->info;
    const uint32_t C = I.codeword_len, L = I.row_len;
    const uint32_t bd = I.base_dim, bl = I.base_len, depth = I.depth;
    const char *kname = sizeof(TE) == 4 ? "k_base_i32" : "k_base_i64";
    const size_t nbase = (size_t)nrows * C;
    if (depth == 0) {
        ZG_KBEGIN(ctx, s, kname);
        if (leaf_major)
            k_base_int<TE, true, true><<<blocks_for(nbase, 256), 256, 0, s>>>(ev, p->d_bmT, out_d, L, bd, bl, depth, C, nrows, seg_log);
        else
            k_base_int<TE, true, false><<<blocks_for(nbase, 256), 256, 0, s>>>(ev, p->d_bmT, out_d, L, bd, bl, depth, C, nrows, seg_log);
        ZG_KEND(ctx, s);
        return ZG_OK;
    }
    ZG_TRY(ctx->stage_a.ensure(nbase * sizeof(Base)));
    ZG_TRY(ctx->stage_b.ensure(nbase * 16));
    ZG_TRY(ctx->stage_c.ensure(depth > 2 ? nbase * 16 : 16));
    Base *base = ctx->stage_a.as<Base>();
    ZG_KBEGIN(ctx, s, kname);
    k_base_int<TE, false, false><<<blocks_for(nbase, 256), 256, 0, s>>>(ev, p->d_bmT, base, L, bd, bl, depth, C, nrows, seg_log);
    ZG_KEND(ctx, s);
    const size_t nthr = (size_t)nrows * (C / 8);
    const unsigned nb = blocks_for(nthr, 256);
    i128 *prev = nullptr;
    for (uint32_t k = 0; k < depth; k++) {
        const uint32_t sub = bd << (3 * k);
        const int32_t *tw = p->d_tw + p->tw_dev_off[k];
        const bool last = k + 1 == depth;
        i128 *dst = last ? reinterpret_cast<i128 *>(out_d)
                         : (k % 2 == 0 ? ctx->stage_b.as<i128>() : ctx->stage_c.as<i128>());
        ZG_KBEGIN(ctx, s, k == 0 ? "k_stage_i128[0]" : "k_stage_i128[1+]");
        if (k == 0) {
            if (last && leaf_major)
                k_stage_i128<Base, true, true><<<nb, 256, 0, s>>>(base, dst, tw, C, sub, nrows, seg_log);
            else if (last)
                k_stage_i128<Base, true, false><<<nb, 256, 0, s>>>(base, dst, tw, C, sub, nrows, seg_log);
            else
                k_stage_i128<Base, false, false><<<nb, 256, 0, s>>>(base, dst, tw, C, sub, nrows, seg_log);
        } else {
            if (last && leaf_major)
                k_stage_i128<i128, true, true><<<nb, 256, 0, s>>>(prev, dst, tw, C, sub, nrows, seg_log);
            else if (last)
                k_stage_i128<i128, true, false><<<nb, 256, 0, s>>>(prev, dst, tw, C, sub, nrows, seg_log);
            else
                k_stage_i128<i128, false, false><<<nb, 256, 0, s>>>(prev, dst, tw, C, sub, nrows, seg_log);
        }
        ZG_KEND(ctx, s);
        prev = dst;
    }
    return ZG_OK;
}

zg_status launch_encode(zg_params *p, zg_ctx *lane, const void *evals_d, uint32_t nrows,
                        uint8_t *out_d, bool leaf_major, cudaStream_t s, uint32_t seg_rows,
                        int base_variant) {
    zg_ctx *ctx = lane;
    uint32_t seg_log = 32;
    if (seg_rows != 0 && seg_rows != nrows) {
        if ((seg_rows & (seg_rows - 1)) != 0 || nrows % seg_rows != 0 || !leaf_major) {
            set_error("segmented encode needs power-of-two segments that divide %u rows", nrows);
            return ZG_ERR_INVALID_PARAM;
        }
        seg_log = 0;
        while ((1u << seg_log) < seg_rows) seg_log++;
    }
    if (nrows > 65535) {
        set_error("too many codeword rows (%u) for one launch", nrows);
        return ZG_ERR_INVALID_PARAM;
    }
    const zg_params_info &I = p->info;
    const uint32_t C = I.codeword_len, L = I.row_len, D = p->D;
    const uint64_t dmask = D >= 64 ? ~0ull : ((1ull << D) - 1);
    if (p->d.code_kind != ZG_CODE_IPRS) {
        const bool flip = p->d.code_kind == ZG_CODE_RAA_SIGN_FLIP;
        if (p->d.eval_kind != ZG_EVAL_BINPOLY) {
            set_error("RAA encoding is defined for binary polynomial evaluations");
            return ZG_ERR_INVALID_PARAM;
        }
        // lanes per block so that n x LG x 4 bytes fits the shared memory budget
        int LG = 8;
        while (LG > 1 && (size_t)C * LG * 4 > 96 * 1024) LG /= 2;
        if ((size_t)C * LG * 4 > 200 * 1024) {
            set_error("RAA codeword length %u exceeds the shared-memory kernel", C);
            return ZG_ERR_INVALID_PARAM;
        }
        unsigned threads = C >= 256 ? 256 : 32;
        size_t smem = ((size_t)C * LG + 32 * LG) * 4;
        dim3 grid(nrows, (D + LG - 1) / LG);
        const uint32_t *p1 = p->d_perm, *p2 = p->d_perm + C;
        int32_t *o = reinterpret_cast<int32_t *>(out_d);
        const uint64_t *ev = static_cast<const uint64_t *>(evals_d);
#define ZG_RAA(LGV)                                                                               \
    do {                                                                                          \
        ZG_CUDA(allow_max_smem(k_raa_bin<LGV>));                                                 \
        k_raa_bin<LGV><<<grid, threads, smem, s>>>(ev, p1, p2, o, L, C, D, dmask, nrows,          \
                                                   leaf_major, seg_log, flip);                             \
    } while (0)
        ZG_KBEGIN(ctx, s, "k_raa_bin");
        switch (LG) {
            case 8: ZG_RAA(8); break;
            case 4: ZG_RAA(4); break;
            case 2: ZG_RAA(2); break;
            default: ZG_RAA(1); break;
        }
#undef ZG_RAA
        ZG_KEND(ctx, s);
        return ZG_OK;
    }

    const uint32_t bd = I.base_dim, bl = I.base_len, depth = I.depth;
    const uint32_t nch = 1u << (3 * depth);
    if (p->d.eval_kind == ZG_EVAL_BINPOLY) {
        const uint64_t *ev = static_cast<const uint64_t *>(evals_d);
        const uint32_t ngroups = (D + 7) / 8;
        // packed-lane base kernel when every lane sum fits the 30-bit field
        const bool packed = (uint64_t)bl * 32769u < (1ull << 29);
        const uint32_t bdp = (bd + 7) / 8 * 8;
        dim3 block2(16, ngroups), grid2((bd + kBase2Rows - 1) / kBase2Rows, nch, nrows);
        const size_t smem2 = 256 * sizeof(uint4) + (size_t)ngroups * bl;
        dim3 block(32, ngroups);
        dim3 grid((bd + 31) / 32, nch, nrows);
        size_t smem = (size_t)bl * 8;
        // shared-memory staged variant: 64-row slices, 8 chunks per block
        constexpr uint32_t TR3 = 64;
        const size_t smem3 = (size_t)bl * TR3 * 4 + 256 * sizeof(uint4) + (size_t)kBase3Chunks * ngroups * bl;
        const uint32_t threads3 = (TR3 / 8) * ngroups * kBase3Chunks;
        bool staged = packed && smem3 <= 200 * 1024 && threads3 <= 512;
        if (base_variant == 2 || base_variant == 3) staged = false;
        const bool use_packed = packed && base_variant != 3;
        auto base_launch = [&](void *dst, bool final_out, bool lm) -> zg_status {
            ZG_KBEGIN(ctx, s, "k_base_bin");
            if (staged) {
                dim3 g3((bd + TR3 - 1) / TR3, (nch + kBase3Chunks - 1) / kBase3Chunks, nrows);
                ZG_CUDA(allow_max_smem(k_base_bin3<TR3, true, true>));
                ZG_CUDA(allow_max_smem(k_base_bin3<TR3, true, false>));
                ZG_CUDA(allow_max_smem(k_base_bin3<TR3, false, false>));
                if (final_out && lm)
                    k_base_bin3<TR3, true, true><<<g3, threads3, smem3, s>>>(ev, p->d_bmP, dst, L, bd, bdp, bl, depth, nch, C, D, ngroups, dmask, nrows, seg_log);
                else if (final_out)
                    k_base_bin3<TR3, true, false><<<g3, threads3, smem3, s>>>(ev, p->d_bmP, dst, L, bd, bdp, bl, depth, nch, C, D, ngroups, dmask, nrows, seg_log);
                else
                    k_base_bin3<TR3, false, false><<<g3, threads3, smem3, s>>>(ev, p->d_bmP, dst, L, bd, bdp, bl, depth, nch, C, D, ngroups, dmask, nrows, seg_log);
            } else if (use_packed) {
                if (smem2 > 48 * 1024) {
                    ZG_CUDA(allow_max_smem(k_base_bin2<true, true>));
                    ZG_CUDA(allow_max_smem(k_base_bin2<true, false>));
                    ZG_CUDA(allow_max_smem(k_base_bin2<false, false>));
                }
                if (final_out && lm)
                    k_base_bin2<true, true><<<grid2, block2, smem2, s>>>(ev, p->d_bmP, dst, L, bd, bdp, bl, depth, C, D, dmask, nrows, seg_log);
                else if (final_out)
                    k_base_bin2<true, false><<<grid2, block2, smem2, s>>>(ev, p->d_bmP, dst, L, bd, bdp, bl, depth, C, D, dmask, nrows, seg_log);
                else
                    k_base_bin2<false, false><<<grid2, block2, smem2, s>>>(ev, p->d_bmP, dst, L, bd, bdp, bl, depth, C, D, dmask, nrows, seg_log);
            } else {
                if (smem > 48 * 1024) {
                    ZG_CUDA(allow_max_smem(k_base_bin<true, true>));
                    ZG_CUDA(allow_max_smem(k_base_bin<true, false>));
                    ZG_CUDA(allow_max_smem(k_base_bin<false, false>));
                }
                if (final_out && lm)
                    k_base_bin<true, true><<<grid, block, smem, s>>>(ev, p->d_bmT, dst, L, bd, bl, depth, C, D, dmask, nrows, seg_log);
                else if (final_out)
                    k_base_bin<true, false><<<grid, block, smem, s>>>(ev, p->d_bmT, dst, L, bd, bl, depth, C, D, dmask, nrows, seg_log);
                else
                    k_base_bin<false, false><<<grid, block, smem, s>>>(ev, p->d_bmT, dst, L, bd, bl, depth, C, D, dmask, nrows, seg_log);
            }
            ZG_KEND(ctx, s);
            return ZG_OK;
        };
        if (depth == 0) return base_launch(out_d, true, leaf_major);
        ZG_TRY(ctx->stage_a.ensure((size_t)nrows * C * D * 4));
        int32_t *base = ctx->stage_a.as<int32_t>();
        // tcgen05 base layer, persistent and warp-specialised (default; variants
        // 6 = 128 and 7 = 64 base rows per tile), one CTA per SM
        if (p->d_bmU && D <= 64 && (base_variant == -1 || base_variant == 6 || base_variant == 7)) {
            const uint32_t NT = base_variant == 7 ? 64 : 128;
            const uint32_t lp = D <= 32 ? 32 : 64, kp = p->umma_kp;
            const uint64_t npairs = (uint64_t)nrows * nch;
            const uint64_t ntm = (npairs + 128 / lp - 1) / (128 / lp), ntn = (bd + NT - 1) / NT;
            const uint64_t ntiles = ntm * ntn;
            const size_t smem_p = 1024 + (size_t)2 * 128 * kp + (size_t)2 * 2 * NT * kp + 1024 + 128;
            if (smem_p <= (size_t)max_smem_optin() && ntiles < (1ull << 31) && npairs < (1ull << 32)) {
                const unsigned g = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)std::max(ctx->num_sms, 1));
                ZG_KBEGIN(ctx, s, "k_base_bin");
#define ZG_UMMA_P(NTV, DSV)                                                                              \
    do {                                                                                                 \
        ZG_CUDA(allow_max_smem(k_base_umma_p<NTV, DSV>));                                                \
        k_base_umma_p<NTV, DSV><<<g, kUmmaPThreads, smem_p, s>>>(ev, p->d_bmU, p->d_bmOff, base, L, bd, bl, kp, \
                                                                 depth, nch, C, D, dmask, (uint32_t)npairs, lp, \
                                                                 (uint32_t)ntn, (uint32_t)ntiles, ctx->status); \
    } while (0)
                if (NT == 64) {
                    if (D == 32) ZG_UMMA_P(64, 32); else if (D == 64) ZG_UMMA_P(64, 64); else ZG_UMMA_P(64, 0);
                } else {
                    if (D == 32) ZG_UMMA_P(128, 32); else if (D == 64) ZG_UMMA_P(128, 64); else ZG_UMMA_P(128, 0);
                }
#undef ZG_UMMA_P
                ZG_KEND(ctx, s);
                goto stages;
            }
        }
        // tcgen05 base layer, one tile per CTA (variant 8 = 128 base rows per
        // tile, 9 = 64; also when the persistent kernel's buffers do not fit)
        if (p->d_bmU && D <= 64 && (base_variant == -1 || base_variant == 6 || base_variant == 7 ||
                                    base_variant == 8 || base_variant == 9)) {
            const uint32_t NT = (base_variant == 7 || base_variant == 9) ? 64 : 128;
            const uint32_t lp = D <= 32 ? 32 : 64, kp = p->umma_kp;
            const uint64_t npairs = (uint64_t)nrows * nch;
            // operand tiles, barriers and TMEM slot, 1024-byte alignment slack; at
            // least a 1/(512/(2 NT) + 1) share of the SM's 228 KiB so that the CTAs
            // resident on one SM never ask for more than its 512 TMEM columns
            size_t smem_u = 1024 + (size_t)128 * kp + (size_t)2 * NT * kp + 32;
            smem_u = std::max<size_t>(smem_u, 233472 / (512 / (2 * NT) + 1));
            const uint64_t gx = (npairs + 128 / lp - 1) / (128 / lp);
            if (smem_u <= (size_t)max_smem_optin() && gx < (1ull << 31)) {
                dim3 gu((unsigned)gx, (bd + NT - 1) / NT);
                ZG_KBEGIN(ctx, s, "k_base_bin");
#define ZG_UMMA_S(NTV, DSV)                                                                              \
    do {                                                                                                 \
        ZG_CUDA(allow_max_smem(k_base_umma<NTV, DSV>));                                                  \
        k_base_umma<NTV, DSV><<<gu, 128, smem_u, s>>>(ev, p->d_bmU, p->d_bmOff, base, L, bd, bl, kp, depth, nch, C, \
                                                      D, dmask, (uint32_t)npairs, lp, ctx->status);      \
    } while (0)
                if (NT == 64) {
                    if (D == 32) ZG_UMMA_S(64, 32); else if (D == 64) ZG_UMMA_S(64, 64); else ZG_UMMA_S(64, 0);
                } else {
                    if (D == 32) ZG_UMMA_S(128, 32); else if (D == 64) ZG_UMMA_S(128, 64); else ZG_UMMA_S(128, 0);
                }
#undef ZG_UMMA_S
                ZG_KEND(ctx, s);
                goto stages;
            }
        }
        {
        const uint32_t blp = (bl + 31) / 32 * 32;
        // tensor-core variants by pairs per block: 0 = 8 (default), 4 = 4, 5 = 16
        const uint32_t pairs = base_variant == 4 ? 4 : base_variant == 5 ? 16 : kMmaPairs;
        const size_t smem_m = (size_t)3 * kMmaRows * (blp + 16) + (size_t)pairs * blp * 8;
        const uint64_t mma_gy = ((uint64_t)nrows * nch + pairs - 1) / pairs;
        if (p->d_bmL && smem_m <= 200 * 1024 && mma_gy <= 65535 &&
            (base_variant == -1 || base_variant == 0 || base_variant == 4 || base_variant == 5)) {
            dim3 gm((bd + kMmaRows - 1) / kMmaRows, (unsigned)mma_gy);
            ZG_KBEGIN(ctx, s, "k_base_bin");
            if (pairs == 4) {
                ZG_CUDA(allow_max_smem(k_base_mma<4>));
                k_base_mma<4><<<gm, 128, smem_m, s>>>(ev, p->d_bmL, base, L, bd, bl, blp, depth, nch, C, D, dmask, nrows);
            } else if (pairs == 16) {
                ZG_CUDA(allow_max_smem(k_base_mma<16>));
                k_base_mma<16><<<gm, 128, smem_m, s>>>(ev, p->d_bmL, base, L, bd, bl, blp, depth, nch, C, D, dmask, nrows);
            } else {
                ZG_CUDA(allow_max_smem(k_base_mma<kMmaPairs>));
                k_base_mma<kMmaPairs><<<gm, 128, smem_m, s>>>(ev, p->d_bmL, base, L, bd, bl, blp, depth, nch, C, D, dmask, nrows);
            }
            ZG_KEND(ctx, s);
        } else {
            ZG_TRY(base_launch(base, false, false));
        }
        }
    stages:
        if (depth == 2 && p->d_tw2r && D <= 64) {
            // both stages in one kernel, register resident
            const uint32_t RB = std::max<uint32_t>(1, std::min<uint32_t>(kStageRB, 256 / D));
            dim3 b2(D, RB), g2((bd + RB - 1) / RB, nrows);
            int64_t *o = reinterpret_cast<int64_t *>(out_d);
            ZG_KBEGIN(ctx, s, "k_stages2_bin");
            k_stages2_reg<<<g2, b2, 0, s>>>(base, o, p->d_tw2r, C, bd, D, nrows, seg_log, leaf_major);
            ZG_KEND(ctx, s);
            return ZG_OK;
        }
        ZG_TRY(ctx->stage_b.ensure((size_t)nrows * C * D * 8 * (depth > 1 ? 1 : 0) + 8));
        const size_t nthr = (size_t)nrows * (C / 8) * D;
        const unsigned tb = 256, nb = blocks_for(nthr, tb);
        int64_t *prev = nullptr;
        for (uint32_t k = 0; k < depth; k++) {
            const uint32_t sub = bd << (3 * k);
            const int32_t *tw = p->d_tw + p->tw_dev_off[k];
            const bool last = k + 1 == depth;
            int64_t *dst = last ? reinterpret_cast<int64_t *>(out_d)
                                : (k % 2 == 0 ? ctx->stage_b.as<int64_t>() : nullptr);
            if (!last && k % 2 == 1) {
                // a third buffer is needed only for depth >= 3
                ZG_TRY(ctx->stage_c.ensure((size_t)nrows * C * D * 8));
                dst = ctx->stage_c.as<int64_t>();
            }
            ZG_KBEGIN(ctx, s, k == 0 ? "k_stage_bin[0]" : "k_stage_bin[1+]");
            if (k == 0) {
                if (last && leaf_major)
                    k_stage_bin<int32_t, true, true><<<nb, tb, 0, s>>>(base, dst, tw, C, sub, D, nrows, seg_log);
                else if (last)
                    k_stage_bin<int32_t, true, false><<<nb, tb, 0, s>>>(base, dst, tw, C, sub, D, nrows, seg_log);
                else
                    k_stage_bin<int32_t, false, false><<<nb, tb, 0, s>>>(base, dst, tw, C, sub, D, nrows, seg_log);
            } else {
                if (last && leaf_major)
                    k_stage_bin<int64_t, true, true><<<nb, tb, 0, s>>>(prev, dst, tw, C, sub, D, nrows, seg_log);
                else if (last)
                    k_stage_bin<int64_t, true, false><<<nb, tb, 0, s>>>(prev, dst, tw, C, sub, D, nrows, seg_log);
                else
                    k_stage_bin<int64_t, false, false><<<nb, tb, 0, s>>>(prev, dst, tw, C, sub, D, nrows, seg_log);
            }
            ZG_KEND(ctx, s);
            prev = dst;
        }
        return ZG_OK;
    }

    // i32 and i64 evaluations
    if (p->d.eval_kind == ZG_EVAL_I64)
        return encode_int_rows<int64_t>(p, ctx, static_cast<const int64_t *>(evals_d), out_d, nrows, leaf_major,
                                        seg_log, s);
    return encode_int_rows<int32_t>(p, ctx, static_cast<const int32_t *>(evals_d), out_d, nrows, leaf_major,
                                    seg_log, s);
}

}  // namespace zg
