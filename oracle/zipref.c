/*
 * zipref.c -- CPU restatement (oracle) of the Zip+ commit/prove/verify path of
 * NethermindEth/zinc-plus.  TEST INFRASTRUCTURE ONLY: the checker for the
 * product's CUDA path and the timed CPU baseline.  The product never links it.
 *
 * Every function cites the reference file:line it restates.  Paths are relative
 * to the reference workspace root.
 *
 * Parity pins (see tests/test_oracle_pins.py): octet-reversal KATs, F65537
 * twiddle KAT, pNTT == NTT mod 65537, RAA 16-element KAT (which pins the
 * rand 0.9 StdRng/ChaCha12 shuffle), Merkle round trip, proof-size formula,
 * BLAKE3 against the `blake3` wheel.  Field bytes follow crypto-bigint
 * MontyForm (R = 2^(64*LIMBS)).
 */
#include "zipref.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__AVX512F__)
#include <immintrin.h>
#endif

typedef __int128 i128;
typedef unsigned __int128 u128;

/* Bits at or above the coefficient count of a BinaryPoly are not part of it. */
static uint64_t dmask(uint32_t D) { return D >= 64 ? ~0ull : ((1ull << D) - 1); }

static int g_threads = 0;
void zr_set_threads(int n) { g_threads = n; }
int zr_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* ========================================================================
 * BLAKE3 (public spec; the reference uses the `blake3` 1.8 crate:
 * zip-plus/src/merkle.rs:148-221, transcript/src/lib.rs:12-77)
 * ====================================================================== */
static const uint32_t B3_IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                  0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
enum { B3_CHUNK_START = 1, B3_CHUNK_END = 2, B3_PARENT = 4, B3_ROOT = 8 };
static const uint8_t B3_PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
static uint8_t B3_SCHED[7][16];
static int b3_sched_ready = 0;

static void b3_init_sched(void) {
    if (b3_sched_ready) return;
    for (int i = 0; i < 16; i++) B3_SCHED[0][i] = (uint8_t)i;
    for (int r = 1; r < 7; r++)
        for (int i = 0; i < 16; i++) B3_SCHED[r][i] = B3_SCHED[r - 1][B3_PERM[i]];
    b3_sched_ready = 1;
}

static inline uint32_t rotr32(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

#define B3G(a, b, c, d, x, y)                                                                     \
    do {                                                                                          \
        v[a] = v[a] + v[b] + (x);                                                                 \
        v[d] = rotr32(v[d] ^ v[a], 16);                                                           \
        v[c] = v[c] + v[d];                                                                       \
        v[b] = rotr32(v[b] ^ v[c], 12);                                                           \
        v[a] = v[a] + v[b] + (y);                                                                 \
        v[d] = rotr32(v[d] ^ v[a], 8);                                                            \
        v[c] = v[c] + v[d];                                                                       \
        v[b] = rotr32(v[b] ^ v[c], 7);                                                            \
    } while (0)

#if defined(__AVX512F__) && defined(__AVX512VL__)
/* The same compression with the 4x4 state held as four 128-bit rows: the four
 * column G functions run lane-parallel, then the rows are rotated so the
 * diagonals line up as columns, and rotated back (the row-wise SIMD form the
 * BLAKE3 spec describes, which the `blake3` crate uses for one block at a time;
 * the reference hashes each Merkle leaf with one Hasher::update,
 * merkle.rs:148-168).  32-bit rotations are single AVX-512VL instructions. */
#define B3ROW_G(r0, r1, r2, r3, mx, my)                                                           \
    do {                                                                                          \
        r0 = _mm_add_epi32(_mm_add_epi32(r0, r1), mx);                                            \
        r3 = _mm_ror_epi32(_mm_xor_si128(r3, r0), 16);                                            \
        r2 = _mm_add_epi32(r2, r3);                                                               \
        r1 = _mm_ror_epi32(_mm_xor_si128(r1, r2), 12);                                            \
        r0 = _mm_add_epi32(_mm_add_epi32(r0, r1), my);                                            \
        r3 = _mm_ror_epi32(_mm_xor_si128(r3, r0), 8);                                             \
        r2 = _mm_add_epi32(r2, r3);                                                               \
        r1 = _mm_ror_epi32(_mm_xor_si128(r1, r2), 7);                                             \
    } while (0)

static void b3_compress(const uint32_t cv[8], const uint32_t m[16], uint64_t counter,
                        uint32_t block_len, uint32_t flags, uint32_t out[16]) {
    const __m128i c0 = _mm_loadu_si128((const __m128i *)cv), c1 = _mm_loadu_si128((const __m128i *)(cv + 4));
    __m128i r0 = c0, r1 = c1, r2 = _mm_loadu_si128((const __m128i *)B3_IV);
    __m128i r3 = _mm_set_epi32((int)flags, (int)block_len, (int)(uint32_t)(counter >> 32), (int)(uint32_t)counter);
    for (int r = 0; r < 7; r++) {
        const uint8_t *s = B3_SCHED[r];
        B3ROW_G(r0, r1, r2, r3, _mm_set_epi32((int)m[s[6]], (int)m[s[4]], (int)m[s[2]], (int)m[s[0]]),
                _mm_set_epi32((int)m[s[7]], (int)m[s[5]], (int)m[s[3]], (int)m[s[1]]));
        r1 = _mm_shuffle_epi32(r1, _MM_SHUFFLE(0, 3, 2, 1)); /* lanes v5 v6 v7 v4 */
        r2 = _mm_shuffle_epi32(r2, _MM_SHUFFLE(1, 0, 3, 2)); /* lanes v10 v11 v8 v9 */
        r3 = _mm_shuffle_epi32(r3, _MM_SHUFFLE(2, 1, 0, 3)); /* lanes v15 v12 v13 v14 */
        B3ROW_G(r0, r1, r2, r3, _mm_set_epi32((int)m[s[14]], (int)m[s[12]], (int)m[s[10]], (int)m[s[8]]),
                _mm_set_epi32((int)m[s[15]], (int)m[s[13]], (int)m[s[11]], (int)m[s[9]]));
        r1 = _mm_shuffle_epi32(r1, _MM_SHUFFLE(2, 1, 0, 3));
        r2 = _mm_shuffle_epi32(r2, _MM_SHUFFLE(1, 0, 3, 2));
        r3 = _mm_shuffle_epi32(r3, _MM_SHUFFLE(0, 3, 2, 1));
    }
    _mm_storeu_si128((__m128i *)out, _mm_xor_si128(r0, r2));
    _mm_storeu_si128((__m128i *)(out + 4), _mm_xor_si128(r1, r3));
    _mm_storeu_si128((__m128i *)(out + 8), _mm_xor_si128(r2, c0));
    _mm_storeu_si128((__m128i *)(out + 12), _mm_xor_si128(r3, c1));
}
#else
static void b3_compress(const uint32_t cv[8], const uint32_t m[16], uint64_t counter,
                        uint32_t block_len, uint32_t flags, uint32_t out[16]) {
    uint32_t v[16] = {cv[0],    cv[1],    cv[2],    cv[3],    cv[4],
                      cv[5],    cv[6],    cv[7],    B3_IV[0], B3_IV[1],
                      B3_IV[2], B3_IV[3], (uint32_t)counter, (uint32_t)(counter >> 32),
                      block_len, flags};
    for (int r = 0; r < 7; r++) {
        const uint8_t *s = B3_SCHED[r];
        B3G(0, 4, 8, 12, m[s[0]], m[s[1]]);
        B3G(1, 5, 9, 13, m[s[2]], m[s[3]]);
        B3G(2, 6, 10, 14, m[s[4]], m[s[5]]);
        B3G(3, 7, 11, 15, m[s[6]], m[s[7]]);
        B3G(0, 5, 10, 15, m[s[8]], m[s[9]]);
        B3G(1, 6, 11, 12, m[s[10]], m[s[11]]);
        B3G(2, 7, 8, 13, m[s[12]], m[s[13]]);
        B3G(3, 4, 9, 14, m[s[14]], m[s[15]]);
    }
    for (int i = 0; i < 8; i++) {
        out[i] = v[i] ^ v[i + 8];
        out[i + 8] = v[i + 8] ^ cv[i];
    }
}
#endif

static void b3_words(const uint8_t *b, size_t n, uint32_t m[16]) {
    uint8_t blk[64];
    memset(blk, 0, 64);
    memcpy(blk, b, n);
    for (int i = 0; i < 16; i++)
        m[i] = (uint32_t)blk[4 * i] | ((uint32_t)blk[4 * i + 1] << 8) |
               ((uint32_t)blk[4 * i + 2] << 16) | ((uint32_t)blk[4 * i + 3] << 24);
}

typedef struct {
    uint32_t cv[8];
    uint32_t m[16];
    uint64_t counter;
    uint32_t block_len;
    uint32_t flags;
} b3_output;

typedef struct {
    uint32_t cv[8];
    uint64_t counter;
    uint8_t block[64];
    uint32_t block_len;
    uint32_t blocks_compressed;
} b3_chunk;

typedef struct {
    b3_chunk chunk;
    uint32_t stack[54][8];
    uint32_t stack_len;
} b3_hasher;

static void b3_chunk_init(b3_chunk *c, uint64_t counter) {
    memcpy(c->cv, B3_IV, 32);
    c->counter = counter;
    memset(c->block, 0, 64);
    c->block_len = 0;
    c->blocks_compressed = 0;
}
static size_t b3_chunk_len(const b3_chunk *c) { return 64u * c->blocks_compressed + c->block_len; }
static uint32_t b3_start_flag(const b3_chunk *c) { return c->blocks_compressed == 0 ? B3_CHUNK_START : 0; }

static void b3_chunk_update(b3_chunk *c, const uint8_t *in, size_t n) {
    while (n) {
        if (c->block_len == 64) {
            uint32_t m[16], out[16];
            b3_words(c->block, 64, m);
            b3_compress(c->cv, m, c->counter, 64, b3_start_flag(c), out);
            memcpy(c->cv, out, 32);
            c->blocks_compressed++;
            c->block_len = 0;
            memset(c->block, 0, 64);
        }
        size_t take = 64 - c->block_len;
        if (take > n) take = n;
        memcpy(c->block + c->block_len, in, take);
        c->block_len += (uint32_t)take;
        in += take;
        n -= take;
    }
}

static b3_output b3_chunk_output(const b3_chunk *c) {
    b3_output o;
    memcpy(o.cv, c->cv, 32);
    b3_words(c->block, c->block_len, o.m);
    o.counter = c->counter;
    o.block_len = c->block_len;
    o.flags = b3_start_flag(c) | B3_CHUNK_END;
    return o;
}

static void b3_output_cv(const b3_output *o, uint32_t cv[8]) {
    uint32_t out[16];
    b3_compress(o->cv, o->m, o->counter, o->block_len, o->flags, out);
    memcpy(cv, out, 32);
}

static b3_output b3_parent_output(const uint32_t l[8], const uint32_t r[8]) {
    b3_output o;
    memcpy(o.cv, B3_IV, 32);
    memcpy(o.m, l, 32);
    memcpy(o.m + 8, r, 32);
    o.counter = 0;
    o.block_len = 64;
    o.flags = B3_PARENT;
    return o;
}

static void b3_output_root(const b3_output *o, uint8_t *out, size_t n) {
    uint64_t blk = 0;
    while (n) {
        uint32_t w[16];
        b3_compress(o->cv, o->m, blk++, o->block_len, o->flags | B3_ROOT, w);
        uint8_t bytes[64];
        for (int i = 0; i < 16; i++) {
            bytes[4 * i] = (uint8_t)w[i];
            bytes[4 * i + 1] = (uint8_t)(w[i] >> 8);
            bytes[4 * i + 2] = (uint8_t)(w[i] >> 16);
            bytes[4 * i + 3] = (uint8_t)(w[i] >> 24);
        }
        size_t take = n < 64 ? n : 64;
        memcpy(out, bytes, take);
        out += take;
        n -= take;
    }
}

static void b3_hasher_init(b3_hasher *h) {
    b3_init_sched();
    b3_chunk_init(&h->chunk, 0);
    h->stack_len = 0;
}

static void b3_hasher_update(b3_hasher *h, const uint8_t *in, size_t n) {
    while (n) {
        if (b3_chunk_len(&h->chunk) == 1024) {
            b3_output o = b3_chunk_output(&h->chunk);
            uint32_t cv[8];
            b3_output_cv(&o, cv);
            uint64_t total = h->chunk.counter + 1;
            while ((total & 1) == 0) {
                b3_output p = b3_parent_output(h->stack[--h->stack_len], cv);
                b3_output_cv(&p, cv);
                total >>= 1;
            }
            memcpy(h->stack[h->stack_len++], cv, 32);
            b3_chunk_init(&h->chunk, h->chunk.counter + 1);
        }
        size_t take = 1024 - b3_chunk_len(&h->chunk);
        if (take > n) take = n;
        b3_chunk_update(&h->chunk, in, take);
        in += take;
        n -= take;
    }
}

static void b3_hasher_xof(const b3_hasher *h, uint8_t *out, size_t n) {
    b3_output o = b3_chunk_output(&h->chunk);
    for (int i = (int)h->stack_len - 1; i >= 0; i--) {
        uint32_t cv[8];
        b3_output_cv(&o, cv);
        o = b3_parent_output(h->stack[i], cv);
    }
    b3_output_root(&o, out, n);
}

void zr_blake3_xof(const uint8_t *in, size_t n, uint8_t *out, size_t out_len) {
    b3_hasher h;
    b3_hasher_init(&h);
    b3_hasher_update(&h, in, n);
    b3_hasher_xof(&h, out, out_len);
}

void zr_blake3(const uint8_t *in, size_t n, uint8_t out[32]) { zr_blake3_xof(in, n, out, 32); }

static void cv_to_bytes(const uint32_t cv[8], uint8_t b[32]);

/* Non-root chaining value of one chunk (<= 1024 bytes) at a given counter. */
void zr_blake3_chunk_cv(const uint8_t *in, size_t n, uint64_t counter, uint8_t out[32]) {
    b3_init_sched();
    b3_chunk c;
    b3_chunk_init(&c, counter);
    b3_chunk_update(&c, in, n);
    b3_output o = b3_chunk_output(&c);
    uint32_t cv[8];
    b3_output_cv(&o, cv);
    cv_to_bytes(cv, out);
}

static void cv_from_bytes(const uint8_t b[32], uint32_t cv[8]) {
    for (int i = 0; i < 8; i++)
        cv[i] = (uint32_t)b[4 * i] | ((uint32_t)b[4 * i + 1] << 8) | ((uint32_t)b[4 * i + 2] << 16) |
                ((uint32_t)b[4 * i + 3] << 24);
}
static void cv_to_bytes(const uint32_t cv[8], uint8_t b[32]) {
    for (int i = 0; i < 8; i++) {
        b[4 * i] = (uint8_t)cv[i];
        b[4 * i + 1] = (uint8_t)(cv[i] >> 8);
        b[4 * i + 2] = (uint8_t)(cv[i] >> 16);
        b[4 * i + 3] = (uint8_t)(cv[i] >> 24);
    }
}

/* blake3::hazmat::merge_subtrees_{non_root,root}(l, r, Mode::Hash)
 * (zip-plus/src/merkle.rs:210-212). */
void zr_blake3_parent(const uint8_t l[32], const uint8_t r[32], int root, uint8_t out[32]) {
    b3_init_sched();
    uint32_t lc[8], rc[8], cv[8];
    cv_from_bytes(l, lc);
    cv_from_bytes(r, rc);
    b3_output o = b3_parent_output(lc, rc);
    if (root) {
        b3_output_root(&o, out, 32);
    } else {
        b3_output_cv(&o, cv);
        cv_to_bytes(cv, out);
    }
}

/* ========================================================================
 * rand 0.9: StdRng (ChaCha12) seed_from_u64 + SliceRandom::shuffle, as used
 * by shuffle_seeded (zip-plus/src/utils.rs:7-10) for the RAA permutations
 * (zip-plus/src/code/raa.rs:76-80).  Restated from rand_core 0.9
 * SeedableRng::seed_from_u64 (PCG32 fill), rand_chacha 0.9 (64-bit block
 * counter, zero stream), rand 0.9 seq::increasing_uniform and the
 * single-sample uniform u32 range method.
 * ====================================================================== */
typedef struct {
    uint32_t key[8];
    uint64_t ctr;
    uint32_t buf[16];
    int idx;
} stdrng;

static void chacha12_block(const uint32_t key[8], uint64_t ctr, uint32_t out[16]) {
    uint32_t x[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2],
                      key[3],      key[4],      key[5],      key[6],      key[7], (uint32_t)ctr,
                      (uint32_t)(ctr >> 32), 0, 0};
    uint32_t s[16];
    memcpy(s, x, sizeof s);
#define QR(a, b, c, d)                                                                            \
    do {                                                                                          \
        x[a] += x[b]; x[d] ^= x[a]; x[d] = (x[d] << 16) | (x[d] >> 16);                           \
        x[c] += x[d]; x[b] ^= x[c]; x[b] = (x[b] << 12) | (x[b] >> 20);                           \
        x[a] += x[b]; x[d] ^= x[a]; x[d] = (x[d] << 8) | (x[d] >> 24);                            \
        x[c] += x[d]; x[b] ^= x[c]; x[b] = (x[b] << 7) | (x[b] >> 25);                            \
    } while (0)
    for (int i = 0; i < 6; i++) {
        QR(0, 4, 8, 12); QR(1, 5, 9, 13); QR(2, 6, 10, 14); QR(3, 7, 11, 15);
        QR(0, 5, 10, 15); QR(1, 6, 11, 12); QR(2, 7, 8, 13); QR(3, 4, 9, 14);
    }
#undef QR
    for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

static void stdrng_seed(stdrng *r, uint64_t state) {
    const uint64_t MUL = 6364136223846793005ull, INC = 11634580027462260723ull;
    for (int i = 0; i < 8; i++) {
        state = state * MUL + INC;
        uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
        uint32_t rot = (uint32_t)(state >> 59);
        r->key[i] = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
    }
    r->ctr = 0;
    r->idx = 16;
}

static uint32_t stdrng_next(stdrng *r) {
    if (r->idx >= 16) {
        chacha12_block(r->key, r->ctr++, r->buf);
        r->idx = 0;
    }
    return r->buf[r->idx++];
}

/* UniformInt<u32>::sample_single(0, bound): one wide multiply with a second
 * sample to reduce bias. */
static uint32_t stdrng_range(stdrng *r, uint32_t bound) {
    uint64_t m = (uint64_t)stdrng_next(r) * bound;
    uint32_t result = (uint32_t)(m >> 32), lo = (uint32_t)m;
    if (lo > (uint32_t)(0u - bound)) {
        uint64_t m2 = (uint64_t)stdrng_next(r) * bound;
        uint32_t new_hi = (uint32_t)(m2 >> 32);
        if ((uint64_t)lo + new_hi > 0xFFFFFFFFull) result += 1;
    }
    return result;
}

void zr_shuffle_identity(uint64_t seed, uint32_t n, uint32_t *perm) {
    for (uint32_t i = 0; i < n; i++) perm[i] = i;
    if (n <= 1) return;
    stdrng r;
    stdrng_seed(&r, seed);
    uint32_t cn = 0, chunk = 0;
    uint32_t chunk_remaining = 1; /* n == 0 at construction */
    for (uint32_t i = 0; i < n; i++) {
        uint32_t next_n = cn + 1, next_rem, result;
        if (chunk_remaining == 0) {
            uint64_t product = next_n;
            uint64_t current = (uint64_t)next_n + 1;
            while (product * current <= 0xFFFFFFFFull) {
                product *= current;
                current++;
            }
            chunk = stdrng_range(&r, (uint32_t)product);
            next_rem = (uint32_t)(current - next_n) - 1;
        } else {
            next_rem = chunk_remaining - 1;
        }
        if (next_rem == 0) {
            result = chunk;
        } else {
            result = chunk % next_n;
            chunk /= next_n;
        }
        chunk_remaining = next_rem;
        cn = next_n;
        uint32_t t = perm[i];
        perm[i] = perm[result];
        perm[result] = t;
    }
}

uint32_t zr_stdrng_u32(uint64_t seed, uint32_t index) {
    stdrng r;
    stdrng_seed(&r, seed);
    uint32_t v = 0;
    for (uint32_t i = 0; i <= index; i++) v = stdrng_next(&r);
    return v;
}

/* ========================================================================
 * IPRS radix-8 pseudo-NTT over the integers
 * (zip-plus/src/code/iprs/pntt/radix8{.rs,/params.rs,/butterfly.rs,
 *  /octet_reversal.rs}, zip-plus/src/code/iprs.rs)
 * ====================================================================== */
#define F65537 65537u

/* octet_reversal.rs:6-29 */
size_t zr_octet_reversal(size_t x, size_t num_octets) {
    if (num_octets == 0) return 0;
    size_t result = 0;
    for (size_t i = 0; i < num_octets; i++) {
        size_t digit = (x >> (3 * i)) & 7;
        result |= digit << (3 * (num_octets - 1 - i));
    }
    return result;
}

/* params.rs:173-181 normalize_field_element */
static int64_t norm65537(uint64_t x) {
    int64_t v = (int64_t)x, p = F65537;
    return v >= (p - 1) / 2 ? v - p : v;
}

static uint64_t powmod(uint64_t b, uint64_t e, uint64_t m) {
    uint64_t r = 1 % m;
    b %= m;
    while (e) {
        if (e & 1) r = r * b % m;
        b = b * b % m;
        e >>= 1;
    }
    return r;
}

/* Radix2EvaluationDomain::<F65537>::new(n).elements() normalized
 * (params.rs:146-155): generator 3, two-adicity 16, so omega_n = 3^(65536/n). */
int zr_roots_of_unity(uint32_t n, int64_t *out) {
    if (n == 0 || (n & (n - 1)) || n > 65536) return -1;
    uint64_t w = powmod(3, 65536 / n, F65537), x = 1;
    for (uint32_t i = 0; i < n; i++) {
        out[i] = norm65537(x);
        x = x * w % F65537;
    }
    return 0;
}

static const int64_t BASE_TWIDDLES[8] = {1, 4096, -256, 16, -1, -4096, 256, -16};
static const uint8_t BUTTERFLY_TABLE[8][7] = {
    {0, 0, 0, 0, 0, 0, 0}, {1, 2, 3, 4, 5, 6, 7}, {2, 4, 6, 0, 2, 4, 6}, {3, 6, 1, 4, 7, 2, 5},
    {4, 0, 4, 0, 4, 0, 4}, {5, 2, 7, 4, 1, 6, 3}, {6, 4, 2, 0, 6, 4, 2}, {7, 6, 5, 4, 3, 2, 1}};

typedef struct {
    uint32_t row_len, codeword_len, depth, base_len, base_dim, base_dim_log2;
    int64_t *bm;  /* base_dim x base_len */
    int64_t **tw; /* per stage k: sub_k x 7 x 8 */
} iprs_params;

/* params.rs:59-108 Radix8PnttParams::new */
static int iprs_check(uint32_t row_len, uint32_t depth, uint32_t rep, uint32_t dims[4]) {
    uint64_t cw = (uint64_t)row_len * rep;
    if (cw >= F65537) return -1;
    if (3 * depth >= 32) return -1;
    uint64_t coeff = 1ull << (3 * depth);
    if (row_len % coeff) return -1;
    uint64_t base_len = row_len / coeff, base_dim = base_len * rep;
    if (base_dim == 0 || (base_dim & (base_dim - 1))) return -1;
    dims[0] = (uint32_t)cw;
    dims[1] = (uint32_t)base_len;
    dims[2] = (uint32_t)base_dim;
    dims[3] = depth;
    return 0;
}

/* iprs.rs:43-51 new_with_optimal_depth */
static uint32_t iprs_optimal_depth(uint32_t row_len) {
    uint32_t q = row_len / 256;
    if (q < 1) q = 1;
    uint32_t lg = 31 - (uint32_t)__builtin_clz(q);
    uint32_t d = (lg + 2) / 3;
    return d < 1 ? 1 : d;
}

uint32_t zr_iprs_optimal_depth(uint32_t row_len) { return iprs_optimal_depth(row_len); }

int zr_iprs_dims(uint32_t row_len, uint32_t depth, uint32_t rep, uint32_t out[4]) {
    return iprs_check(row_len, depth, rep, out);
}

static void iprs_free(iprs_params *p) {
    free(p->bm);
    if (p->tw) {
        for (uint32_t k = 0; k < p->depth; k++) free(p->tw[k]);
        free(p->tw);
    }
}

/* params.rs:110-196 precompute_base_matrix / precompute_butterfly_twiddles */
static int iprs_build(uint32_t row_len, uint32_t depth, uint32_t rep, iprs_params *p) {
    uint32_t dims[4];
    if (iprs_check(row_len, depth, rep, dims)) return -1;
    memset(p, 0, sizeof *p);
    p->row_len = row_len;
    p->codeword_len = dims[0];
    p->base_len = dims[1];
    p->base_dim = dims[2];
    p->depth = depth;
    p->base_dim_log2 = (uint32_t)__builtin_ctz(p->base_dim);
    p->bm = (int64_t *)malloc(sizeof(int64_t) * p->base_dim * p->base_len);
    uint64_t wbd = powmod(3, 65536 / p->base_dim, F65537), root = 1;
    for (uint32_t r = 0; r < p->base_dim; r++) {
        for (uint32_t c = 0; c < p->base_len; c++)
            p->bm[(size_t)r * p->base_len + c] = norm65537(powmod(root, c, F65537));
        root = root * wbd % F65537;
    }
    int64_t *roots = (int64_t *)malloc(sizeof(int64_t) * p->codeword_len);
    zr_roots_of_unity(p->codeword_len, roots);
    p->tw = (int64_t **)calloc(depth ? depth : 1, sizeof(int64_t *));
    for (uint32_t k = 0; k < depth; k++) {
        size_t sub = (size_t)p->base_dim << (3 * k);
        size_t pw = (size_t)1 << (3 * (depth - 1 - k));
        int64_t *t = (int64_t *)malloc(sizeof(int64_t) * sub * 56);
        for (size_t i = 0; i < sub; i++)
            for (int j = 0; j < 7; j++) {
                int64_t rt = roots[pw * i * (size_t)(j + 1)];
                uint64_t rm = (uint64_t)((rt % (int64_t)F65537 + F65537) % F65537);
                for (int tix = 0; tix < 8; tix++) {
                    uint64_t bm = (uint64_t)((BASE_TWIDDLES[tix] % (int64_t)F65537 + F65537) % F65537);
                    t[(i * 7 + j) * 8 + tix] = norm65537(bm * rm % F65537);
                }
            }
        p->tw[k] = t;
    }
    free(roots);
    return 0;
}

int zr_iprs_tables(uint32_t row_len, uint32_t depth, uint32_t rep, int64_t *base_matrix,
                   int64_t *twiddles) {
    iprs_params p;
    if (iprs_build(row_len, depth, rep, &p)) return -1;
    if (base_matrix) memcpy(base_matrix, p.bm, sizeof(int64_t) * p.base_dim * p.base_len);
    if (twiddles) {
        size_t off = 0;
        for (uint32_t k = 0; k < depth; k++) {
            size_t sub = (size_t)p.base_dim << (3 * k);
            memcpy(twiddles + off, p.tw[k], sizeof(int64_t) * sub * 56);
            off += sub * 56;
        }
    }
    iprs_free(&p);
    return 0;
}

/* Generic pNTT over "lanes" of wrapping 64-bit-limb integers.  A value is
 * `limbs` little-endian u64 words (two's complement, wrapping); lanes are
 * independent.  Element i of the output occupies out[(i*lanes + l)*limbs].
 * (radix8.rs:21-161, butterfly.rs:24-43) */
static inline void wl_mul_i64_add(uint64_t *acc, const uint64_t *x, int64_t t, uint32_t limbs) {
    /* acc += x * t (mod 2^(64*limbs)), t sign-extended */
    uint64_t tl = (uint64_t)t, th = t < 0 ? ~0ull : 0;
    uint64_t prod[8] = {0};
    for (uint32_t i = 0; i < limbs; i++) {
        u128 carry = 0;
        for (uint32_t j = 0; i + j < limbs; j++) {
            uint64_t tw = (j == 0) ? tl : th;
            u128 s = (u128)x[i] * tw + prod[i + j] + carry;
            prod[i + j] = (uint64_t)s;
            carry = s >> 64;
        }
    }
    u128 c = 0;
    for (uint32_t i = 0; i < limbs; i++) {
        u128 s = (u128)acc[i] + prod[i] + c;
        acc[i] = (uint64_t)s;
        c = s >> 64;
    }
}

static void pntt_stages_wide(const iprs_params *p, uint64_t *out, uint32_t lanes, uint32_t limbs) {
    size_t esz = (size_t)lanes * limbs;
    uint64_t *xs = (uint64_t *)malloc(sizeof(uint64_t) * 8 * esz);
    for (uint32_t k = 0; k < p->depth; k++) {
        size_t sub = (size_t)p->base_dim << (3 * k);
        const int64_t *tw = p->tw[k];
        for (size_t blk = 0; blk < p->codeword_len; blk += 8 * sub) {
            uint64_t *chunk = out + blk * esz;
            for (size_t i = 0; i < sub; i++) {
                for (int j = 0; j < 8; j++) memcpy(xs + j * esz, chunk + (j * sub + i) * esz, 8 * esz);
                for (int r = 0; r < 8; r++) {
                    uint64_t *y = chunk + (r * sub + i) * esz;
                    memcpy(y, xs, 8 * esz);
                    for (int j = 1; j < 8; j++) {
                        int64_t t = tw[(i * 7 + (j - 1)) * 8 + BUTTERFLY_TABLE[r][j - 1]];
                        for (uint32_t l = 0; l < lanes; l++)
                            wl_mul_i64_add(y + l * limbs, xs + j * esz + l * limbs, t, limbs);
                    }
                }
            }
        }
    }
    free(xs);
}

/* Radix-8 stages on i128 values (MulByScalar i128 x i64, mul_by_scalar.rs:97-108). */
static void pntt_stages_i128(const iprs_params *p, i128 *out);

/* The reference's pNTT (radix8.rs:21-161) is data parallel at two levels:
 * base_multiply_into_output maps every codeword position independently
 * (`cfg_into_iter!(0..codeword_len)`, radix8.rs:133) and combine_stages works
 * chunk by chunk (`cfg_chunks_mut!`, radix8.rs:88), while encode_rows runs the
 * rows in parallel (phase_commit.rs:166-172).  The functions below compute a
 * range of positions (base layer) or of butterfly columns (one stage), so
 * encode_poly can spread rows x positions over all threads the same way. */

/* Base layer, integer evaluations (Zip i32 -> i128, mul_by_scalar.rs:89-95;
 * the Zinc+ integer columns i64 -> i128, mul_by_scalar.rs:110-116; the base
 * sum of an i64 row stays below 2^63 * 2^16 * base_len in magnitude). */
static void int_base_range(const iprs_params *p, const void *in_v, int is_i64, i128 *out, size_t i0,
                           size_t i1) {
    const uint32_t sh = 3 * p->depth;
    const int32_t *in32 = (const int32_t *)in_v;
    const int64_t *in64 = (const int64_t *)in_v;
    for (size_t i = i0; i < i1; i++) {
        size_t chunk = i >> p->base_dim_log2, row = i & (p->base_dim - 1);
        size_t oct = zr_octet_reversal(chunk, p->depth);
        const int64_t *bm = p->bm + row * p->base_len;
        i128 acc = is_i64 ? (i128)in64[oct] : (i128)in32[oct];
        if (is_i64)
            for (size_t c = 1; c < p->base_len; c++) acc += (i128)in64[oct | (c << sh)] * bm[c];
        else
            for (size_t c = 1; c < p->base_len; c++) acc += (i128)in32[oct | (c << sh)] * bm[c];
        out[i] = acc;
    }
}

/* One radix-8 stage on i128 values (MulByScalar i128 x i64, wrapping,
 * mul_by_scalar.rs:97-108; butterfly.rs:24-43) for butterfly columns
 * [i0, i1) of the chunk starting at position blk. */
static void i128_stage_range(const iprs_params *p, uint32_t k, i128 *out, size_t blk, size_t i0, size_t i1) {
    const size_t sub = (size_t)p->base_dim << (3 * k);
    const int64_t *tw = p->tw[k];
    i128 *chunk = out + blk;
    i128 xs[8];
    for (size_t i = i0; i < i1; i++) {
        for (int j = 0; j < 8; j++) xs[j] = chunk[j * sub + i];
        for (int r = 0; r < 8; r++) {
            u128 y = (u128)xs[0];
            for (int j = 1; j < 8; j++)
                y += (u128)xs[j] * (u128)(i128)tw[(i * 7 + (j - 1)) * 8 + BUTTERFLY_TABLE[r][j - 1]];
            chunk[r * sub + i] = (i128)y;
        }
    }
}

static void pntt_stages_i128(const iprs_params *p, i128 *out) {
    for (uint32_t k = 0; k < p->depth; k++) {
        size_t sub = (size_t)p->base_dim << (3 * k);
        for (size_t blk = 0; blk < p->codeword_len; blk += 8 * sub) i128_stage_range(p, k, out, blk, 0, sub);
    }
}

/* Scalar Zip: Eval i32 -> Cw i128 (mul_by_scalar.rs:89-108). */
static void pntt_i32(const iprs_params *p, const int32_t *in, i128 *out) {
    int_base_range(p, in, 0, out, 0, p->codeword_len);
    pntt_stages_i128(p, out);
}

/* Int column Zip (IntZt of protocol/benches/e2e.rs:215-227): Eval i64 -> Cw i128. */
static void pntt_i64(const iprs_params *p, const int64_t *in, i128 *out) {
    int_base_range(p, in, 1, out, 0, p->codeword_len);
    pntt_stages_i128(p, out);
}

/* Zip+ base layer: Eval BinaryPoly<D> (u64 bit mask) -> Cw DensePolynomial<i64,
 * D>.  Each term is the widened polynomial (coefficient l = bm[c] if bit l is
 * set, else 0: binary_u64.rs:445-456) added coefficient-wise with wrapping i64
 * (dense.rs:551-574).  With AVX-512 the widen is the reference's own form
 * (binary_u64.rs:605-661: one masked broadcast per 8 coefficients), fused here
 * with the add as one masked add per 8 coefficients. */
#if defined(__AVX512F__)
static inline __attribute__((always_inline)) void bin_base_avx512(const iprs_params *p, const uint64_t *in,
                                                                  const uint32_t NV8, int64_t *out, size_t i0,
                                                                  size_t i1) {
    const uint32_t sh = 3 * p->depth;
    const __m512i one = _mm512_set1_epi64(1);
    for (size_t i = i0; i < i1; i++) {
        size_t chunk = i >> p->base_dim_log2, row = i & (p->base_dim - 1);
        size_t oct = zr_octet_reversal(chunk, p->depth);
        const int64_t *bm = p->bm + row * p->base_len;
        __m512i acc[8];
        const uint64_t x0 = in[oct];
        for (uint32_t v = 0; v < NV8; v++) acc[v] = _mm512_maskz_mov_epi64((__mmask8)(x0 >> (8 * v)), one);
        for (size_t c = 1; c < p->base_len; c++) {
            const uint64_t x = in[oct | (c << sh)];
            const __m512i b = _mm512_set1_epi64(bm[c]);
            for (uint32_t v = 0; v < NV8; v++)
                acc[v] = _mm512_mask_add_epi64(acc[v], (__mmask8)(x >> (8 * v)), acc[v], b);
        }
        for (uint32_t v = 0; v < NV8; v++) _mm512_storeu_si512((void *)(out + i * 8 * NV8 + 8 * v), acc[v]);
    }
}
#endif

static void bin_base_range(const iprs_params *p, const uint64_t *in, uint32_t D, int64_t *out, size_t i0,
                           size_t i1) {
#if defined(__AVX512F__)
    switch (D) {  /* D a multiple of 8: the vector form, with the lane count a constant */
    case 8: bin_base_avx512(p, in, 1, out, i0, i1); return;
    case 16: bin_base_avx512(p, in, 2, out, i0, i1); return;
    case 24: bin_base_avx512(p, in, 3, out, i0, i1); return;
    case 32: bin_base_avx512(p, in, 4, out, i0, i1); return;
    case 40: bin_base_avx512(p, in, 5, out, i0, i1); return;
    case 48: bin_base_avx512(p, in, 6, out, i0, i1); return;
    case 56: bin_base_avx512(p, in, 7, out, i0, i1); return;
    case 64: bin_base_avx512(p, in, 8, out, i0, i1); return;
    default: break;
    }
#endif
    const uint32_t sh = 3 * p->depth;
    const uint64_t msk = dmask(D);
    for (size_t i = i0; i < i1; i++) {
        size_t chunk = i >> p->base_dim_log2, row = i & (p->base_dim - 1);
        size_t oct = zr_octet_reversal(chunk, p->depth);
        const int64_t *bm = p->bm + row * p->base_len;
        uint64_t acc[64];
        uint64_t x0 = in[oct] & msk;
        for (uint32_t l = 0; l < D; l++) acc[l] = (x0 >> l) & 1;
        for (size_t c = 1; c < p->base_len; c++) {
            uint64_t x = in[oct | (c << sh)] & msk;
            uint64_t b = (uint64_t)bm[c];
            for (uint32_t l = 0; l < D; l++) acc[l] += ((x >> l) & 1) * b;
        }
        for (uint32_t l = 0; l < D; l++) out[i * D + l] = (int64_t)acc[l];
    }
}

/* One radix-8 stage on DensePolynomial<i64, D> values (coefficient-wise
 * wrapping i64 x twiddle, dense.rs:551-574), butterfly columns [i0, i1) of the
 * chunk starting at position blk. */
static void bin_stage_range(const iprs_params *p, uint32_t k, uint32_t D, int64_t *out, size_t blk, size_t i0,
                            size_t i1) {
    const size_t sub = (size_t)p->base_dim << (3 * k);
    const int64_t *tw = p->tw[k];
    int64_t *chunk = out + blk * D;
    uint64_t xs[8][64];
    for (size_t i = i0; i < i1; i++) {
        for (int j = 0; j < 8; j++) memcpy(xs[j], chunk + (j * sub + i) * D, 8 * D);
        for (int r = 0; r < 8; r++) {
            uint64_t t[8];
            for (int j = 1; j < 8; j++) t[j] = (uint64_t)tw[(i * 7 + (j - 1)) * 8 + BUTTERFLY_TABLE[r][j - 1]];
            int64_t *y = chunk + (r * sub + i) * D;
            uint32_t l = 0;
#if defined(__AVX512F__) && defined(__AVX512DQ__)
            for (; l + 8 <= D; l += 8) {
                __m512i acc = _mm512_loadu_si512((const void *)(xs[0] + l));
                for (int j = 1; j < 8; j++)
                    acc = _mm512_add_epi64(acc, _mm512_mullo_epi64(_mm512_loadu_si512((const void *)(xs[j] + l)),
                                                                    _mm512_set1_epi64((long long)t[j])));
                _mm512_storeu_si512((void *)(y + l), acc);
            }
#endif
            for (; l < D; l++) {
                uint64_t a = xs[0][l];
                for (int j = 1; j < 8; j++) a += xs[j][l] * t[j];
                y[l] = (int64_t)a;
            }
        }
    }
}

static void pntt_binary(const iprs_params *p, const uint64_t *in, uint32_t D, int64_t *out) {
    bin_base_range(p, in, D, out, 0, p->codeword_len);
    for (uint32_t k = 0; k < p->depth; k++) {
        size_t sub = (size_t)p->base_dim << (3 * k);
        for (size_t blk = 0; blk < p->codeword_len; blk += 8 * sub) bin_stage_range(p, k, D, out, blk, 0, sub);
    }
}

/* ========================================================================
 * RAA code (zip-plus/src/code/raa.rs:38-244), PERMUTE_IN_PLACE or copying:
 * both give the same codeword (raa.rs:430-455).
 * ====================================================================== */
typedef struct {
    uint32_t row_len, codeword_len;
    uint32_t *perm1, *perm2;
    int flip; /* RaaSignFlippingCode (zip-plus/src/code/raa_sign_flip.rs:31-69) */
} raa_params;

static int raa_build(uint32_t row_len, uint32_t rep, int flip, raa_params *r) {
    if (row_len == 0 || (row_len & (row_len - 1)) || rep == 0 || (rep & (rep - 1))) return -1;
    r->flip = flip;
    r->row_len = row_len;
    r->codeword_len = row_len * rep;
    r->perm1 = (uint32_t *)malloc(sizeof(uint32_t) * r->codeword_len);
    r->perm2 = (uint32_t *)malloc(sizeof(uint32_t) * r->codeword_len);
    zr_shuffle_identity(1, r->codeword_len, r->perm1);
    zr_shuffle_identity(2, r->codeword_len, r->perm2);
    return 0;
}
static void raa_free(raa_params *r) {
    free(r->perm1);
    free(r->perm2);
}

/* flip_even_signs (raa_sign_flip.rs:135-165): negate entries 1, 3, 5, ... of
 * n elements of esz wrapping limbs (each entry is lanes x limbs). */
static void flip_odd_entries(uint64_t *v, size_t n, uint32_t lanes, uint32_t limbs) {
    for (size_t i = 1; i < n; i += 2)
        for (uint32_t l = 0; l < lanes; l++) {
            uint64_t *x = v + (i * lanes + l) * limbs;
            u128 c = 1;
            for (uint32_t w = 0; w < limbs; w++) {
                u128 s = (u128)(~x[w]) + c;
                x[w] = (uint64_t)s;
                c = s >> 64;
            }
        }
}

/* encode_inner (raa.rs:93-127; with sign flips raa_sign_flip.rs:31-69) on
 * lanes of wrapping multi-limb values. */
static void raa_encode_wide(const raa_params *r, const uint64_t *in, uint64_t *out, uint32_t lanes,
                            uint32_t limbs) {
    size_t esz = (size_t)lanes * limbs, n = r->codeword_len;
    uint64_t *a = (uint64_t *)malloc(sizeof(uint64_t) * n * esz);
    for (size_t i = 0; i < n; i++) memcpy(a + i * esz, in + (i % r->row_len) * esz, 8 * esz);
    if (r->flip) flip_odd_entries(a, n, lanes, limbs);
    for (int pass = 0; pass < 2; pass++) {
        const uint32_t *perm = pass == 0 ? r->perm1 : r->perm2;
        for (size_t i = 0; i < n; i++) memcpy(out + i * esz, a + (size_t)perm[i] * esz, 8 * esz);
        for (size_t i = 1; i < n; i++) {
            uint64_t *cur = out + i * esz, *prev = out + (i - 1) * esz;
            for (uint32_t l = 0; l < lanes; l++) {
                u128 c = 0;
                for (uint32_t w = 0; w < limbs; w++) {
                    u128 s = (u128)cur[l * limbs + w] + prev[l * limbs + w] + c;
                    cur[l * limbs + w] = (uint64_t)s;
                    c = s >> 64;
                }
            }
        }
        if (pass == 0) {
            memcpy(a, out, 8 * n * esz);
            if (r->flip) flip_odd_entries(a, n, lanes, limbs);
        }
    }
    free(a);
}

/* Binary RAA: Eval BinaryPoly<D> -> Cw DensePolynomial<i32, D>, wrapping i32. */
static void raa_binary(const raa_params *r, const uint64_t *in, uint32_t D, int32_t *out) {
    size_t n = r->codeword_len;
    uint32_t *a = (uint32_t *)malloc(sizeof(uint32_t) * n * D);
    uint32_t *b = (uint32_t *)malloc(sizeof(uint32_t) * n * D);
    for (size_t i = 0; i < n; i++) {
        uint64_t x = in[i % r->row_len];
        for (uint32_t l = 0; l < D; l++) {
            const uint32_t v = (uint32_t)((x >> l) & 1);
            a[i * D + l] = (r->flip && (i & 1)) ? 0u - v : v;
        }
    }
    for (int pass = 0; pass < 2; pass++) {
        const uint32_t *perm = pass == 0 ? r->perm1 : r->perm2;
        for (size_t i = 0; i < n; i++) memcpy(b + i * D, a + (size_t)perm[i] * D, 4 * D);
        for (size_t i = 1; i < n; i++)
            for (uint32_t l = 0; l < D; l++) b[i * D + l] += b[(i - 1) * D + l];
        if (pass == 0 && r->flip)
            for (size_t i = 1; i < n; i += 2)
                for (uint32_t l = 0; l < D; l++) b[i * D + l] = 0u - b[i * D + l];
        uint32_t *t = a;
        a = b;
        b = t;
    }
    memcpy(out, a, 4 * n * D);
    free(a);
    free(b);
}

/* ========================================================================
 * Parameters (pcs/structs.rs:74-88 setup; code constructors)
 * ====================================================================== */
typedef struct {
    zr_desc d;
    uint32_t num_rows, row_len, codeword_len, D, cw_bytes, eval_bytes, depth;
    iprs_params iprs;
    raa_params raa;
} zparams;

static int zparams_build(const zr_desc *d, zparams *z) {
    memset(z, 0, sizeof *z);
    z->d = *d;
    if (d->num_vars > 30 || d->row_len == 0 || (d->row_len & (d->row_len - 1))) return -1;
    uint64_t poly = 1ull << d->num_vars;
    if (poly % d->row_len) return -1;
    z->num_rows = (uint32_t)(poly / d->row_len);
    z->row_len = d->row_len;
    if (d->eval_kind > ZR_EVAL_I64) return -1;
    z->D = d->eval_kind == ZR_EVAL_BINPOLY ? d->degree_plus_one : 1;
    if (d->eval_kind == ZR_EVAL_BINPOLY && (z->D == 0 || z->D > 64)) return -1;
    z->eval_bytes = d->eval_kind == ZR_EVAL_I32 ? 4 : 8;
    if (d->field_limbs < 1 || d->field_limbs > 4 || d->comb_limbs < 1 || d->comb_limbs > 8) return -1;
    if (d->code_kind == ZR_CODE_IPRS) {
        uint32_t depth = d->iprs_depth ? d->iprs_depth : iprs_optimal_depth(d->row_len);
        if (iprs_build(d->row_len, depth, d->rep, &z->iprs)) return -1;
        z->depth = depth;
        z->codeword_len = z->iprs.codeword_len;
        z->cw_bytes = d->eval_kind == ZR_EVAL_BINPOLY ? 8 * z->D : 16;
    } else {
        if (d->code_kind > ZR_CODE_RAA_SIGN_FLIP) return -1;
        if (raa_build(d->row_len, d->rep, d->code_kind == ZR_CODE_RAA_SIGN_FLIP, &z->raa)) return -1;
        z->codeword_len = z->raa.codeword_len;
        z->cw_bytes = 4 * z->D;
    }
    return 0;
}

static void zparams_free(zparams *z) {
    if (z->d.code_kind == ZR_CODE_IPRS) iprs_free(&z->iprs);
    else raa_free(&z->raa);
}

size_t zr_cw_bytes(const zr_desc *d) {
    zparams z;
    if (zparams_build(d, &z)) return 0;
    size_t r = z.cw_bytes;
    zparams_free(&z);
    return r;
}
size_t zr_eval_bytes(const zr_desc *d) { return d->eval_kind == ZR_EVAL_I32 ? 4 : 8; }
uint32_t zr_num_rows(const zr_desc *d) {
    zparams z;
    if (zparams_build(d, &z)) return 0;
    uint32_t r = z.num_rows;
    zparams_free(&z);
    return r;
}
uint32_t zr_codeword_len(const zr_desc *d) {
    zparams z;
    if (zparams_build(d, &z)) return 0;
    uint32_t r = z.codeword_len;
    zparams_free(&z);
    return r;
}

/* encode one row into cw (codeword_len x cw_bytes) */
static void encode_row(const zparams *z, const void *row, void *cw) {
    if (z->d.code_kind == ZR_CODE_IPRS) {
        if (z->d.eval_kind == ZR_EVAL_I32) pntt_i32(&z->iprs, (const int32_t *)row, (i128 *)cw);
        else if (z->d.eval_kind == ZR_EVAL_I64) pntt_i64(&z->iprs, (const int64_t *)row, (i128 *)cw);
        else pntt_binary(&z->iprs, (const uint64_t *)row, z->D, (int64_t *)cw);
    } else {
        raa_binary(&z->raa, (const uint64_t *)row, z->D, (int32_t *)cw);
    }
}

/* phase_commit.rs:159-176 encode_rows: row-major num_rows x codeword_len.
 * IPRS: rows x position tiles of the base layer, then per stage rows x
 * (chunk, butterfly-column tile), all threads at each level (the reference's
 * nested rayon over rows, positions and chunks).  RAA (repeat, permute, prefix
 * sums: sequential within a row, raa.rs:93-127): rows in parallel. */
#define ZR_TILE 256
static void encode_poly(const zparams *z, const uint8_t *evals, uint8_t *cw) {
    int nt = zr_get_threads();
    (void)nt;
    const long R = (long)z->num_rows;
    if (z->d.code_kind != ZR_CODE_IPRS) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
        for (long r = 0; r < R; r++)
            encode_row(z, evals + (size_t)r * z->row_len * z->eval_bytes,
                       cw + (size_t)r * z->codeword_len * z->cw_bytes);
        return;
    }
    const iprs_params *p = &z->iprs;
    const size_t C = p->codeword_len, ev_row = (size_t)z->row_len * z->eval_bytes,
                 cw_row = (size_t)C * z->cw_bytes;
    const int bin = z->d.eval_kind == ZR_EVAL_BINPOLY;
    const long tiles = (long)((C + ZR_TILE - 1) / ZR_TILE);
#pragma omp parallel num_threads(nt)
    {
#pragma omp for schedule(static) collapse(2)
        for (long r = 0; r < R; r++)
            for (long t = 0; t < tiles; t++) {
                const size_t i0 = (size_t)t * ZR_TILE, i1 = i0 + ZR_TILE < C ? i0 + ZR_TILE : C;
                const uint8_t *in = evals + (size_t)r * ev_row;
                uint8_t *o = cw + (size_t)r * cw_row;
                if (bin) bin_base_range(p, (const uint64_t *)in, z->D, (int64_t *)o, i0, i1);
                else int_base_range(p, in, z->d.eval_kind == ZR_EVAL_I64, (i128 *)o, i0, i1);
            }
        for (uint32_t k = 0; k < p->depth; k++) {
            const size_t sub = (size_t)p->base_dim << (3 * k);
            const size_t per_chunk = (sub + ZR_TILE - 1) / ZR_TILE;
            const long units = (long)((C / (8 * sub)) * per_chunk);
#pragma omp for schedule(static) collapse(2)
            for (long r = 0; r < R; r++)
                for (long u = 0; u < units; u++) {
                    const size_t blk = (size_t)(u / per_chunk) * 8 * sub, it = (size_t)(u % per_chunk);
                    const size_t i0 = it * ZR_TILE, i1 = i0 + ZR_TILE < sub ? i0 + ZR_TILE : sub;
                    uint8_t *o = cw + (size_t)r * cw_row;
                    if (bin) bin_stage_range(p, k, z->D, (int64_t *)o, blk, i0, i1);
                    else i128_stage_range(p, k, (i128 *)o, blk, i0, i1);
                }
        }
    }
}

int zr_encode_rows(const zr_desc *d, const void *evals, void *cw_out) {
    zparams z;
    if (zparams_build(d, &z)) return -1;
    if (d->code_kind != ZR_CODE_IPRS && d->eval_kind != ZR_EVAL_BINPOLY) {
        zparams_free(&z);
        return -1;
    }
    encode_poly(&z, (const uint8_t *)evals, (uint8_t *)cw_out);
    zparams_free(&z);
    return 0;
}

/* LinearCode::encode_wide on Int<limbs> (iprs.rs:148-150; raa.rs encode_wide) */
int zr_encode_wide(const zr_desc *d, const uint64_t *row, uint32_t limbs, uint64_t *out) {
    zparams z;
    if (zparams_build(d, &z)) return -1;
    if (d->code_kind == ZR_CODE_IPRS) {
        const iprs_params *p = &z.iprs;
        uint32_t sh = 3 * p->depth;
        for (size_t i = 0; i < p->codeword_len; i++) {
            size_t chunk = i >> p->base_dim_log2, rw = i & (p->base_dim - 1);
            size_t oct = zr_octet_reversal(chunk, p->depth);
            const int64_t *bm = p->bm + rw * p->base_len;
            uint64_t *o = out + i * limbs;
            memcpy(o, row + oct * limbs, 8 * limbs);
            for (size_t c = 1; c < p->base_len; c++)
                wl_mul_i64_add(o, row + (oct | (c << sh)) * limbs, bm[c], limbs);
        }
        pntt_stages_wide(p, out, 1, limbs);
    } else {
        raa_encode_wide(&z.raa, row, out, 1, limbs);
    }
    zparams_free(&z);
    return 0;
}

/* ========================================================================
 * Merkle tree (zip-plus/src/merkle.rs:74-257)
 * ====================================================================== */
typedef struct {
    uint32_t n_leaves, n_layers;
    uint8_t **layers; /* layers[k]: (n_leaves >> k) x 32 */
} mtree;

static void mtree_free(mtree *t) {
    for (uint32_t k = 0; k < t->n_layers; k++) free(t->layers[k]);
    free(t->layers);
}

/* build_merkle_tree_from_leaves (merkle.rs:172-221); leaves consumed */
static void mtree_build(mtree *t, uint8_t *leaves, uint32_t n) {
    uint32_t nl = 1;
    while ((1u << (nl - 1)) < n) nl++;
    t->n_leaves = n;
    t->n_layers = nl;
    t->layers = (uint8_t **)calloc(nl, sizeof(uint8_t *));
    t->layers[0] = leaves;
    int nt = zr_get_threads();
    (void)nt;
    for (uint32_t k = 1; k < nl; k++) {
        uint32_t m = n >> k;
        uint8_t *prev = t->layers[k - 1], *cur = (uint8_t *)malloc((size_t)m * 32);
        int root = (k == nl - 1);
#pragma omp parallel for schedule(static) num_threads(nt)
        for (long i = 0; i < (long)m; i++)
            zr_blake3_parent(prev + 64 * i, prev + 64 * i + 32, root, cur + 32 * i);
        t->layers[k] = cur;
    }
}

/* hash_leaves (merkle.rs:148-168): leaf j = BLAKE3(concat_r bytes(row_r[j])) */
static uint8_t *hash_leaves(const uint8_t *const *rows, uint32_t n_rows, uint32_t width,
                            uint32_t eb) {
    b3_init_sched();
    uint8_t *leaves = (uint8_t *)malloc((size_t)width * 32);
    int nt = zr_get_threads();
    (void)nt;
#pragma omp parallel num_threads(nt)
    {
        uint8_t *buf = (uint8_t *)malloc((size_t)n_rows * eb);
#pragma omp for schedule(static)
        for (long j = 0; j < (long)width; j++) {
            for (uint32_t r = 0; r < n_rows; r++) memcpy(buf + (size_t)r * eb, rows[r] + (size_t)j * eb, eb);
            zr_blake3(buf, (size_t)n_rows * eb, leaves + 32 * j);
        }
        free(buf);
    }
    return leaves;
}

int zr_merkle_root_rows(const uint8_t *rows, uint32_t n_rows, uint32_t width, uint32_t elem_bytes,
                        uint8_t root[32]) {
    if (n_rows == 0 || width == 0 || (width & (width - 1))) return -1;
    const uint8_t **rp = (const uint8_t **)malloc(sizeof(uint8_t *) * n_rows);
    for (uint32_t r = 0; r < n_rows; r++) rp[r] = rows + (size_t)r * width * elem_bytes;
    uint8_t *leaves = hash_leaves(rp, n_rows, width, elem_bytes);
    free(rp);
    mtree t;
    mtree_build(&t, leaves, width);
    memcpy(root, t.layers[t.n_layers - 1], 32);
    mtree_free(&t);
    return 0;
}

/* get_path_directions (merkle.rs:385-410) + MerkleProof::verify (:282-359).
 * Returns 0 if ok. */
static int merkle_verify(const uint8_t root[32], const uint8_t *column_bytes, size_t col_len,
                         uint64_t leaf_index, uint64_t leaf_count, const uint8_t *siblings,
                         uint64_t n_sib, uint64_t expected_index) {
    if (leaf_index != expected_index) return -1;
    uint8_t cur[32];
    zr_blake3(column_bytes, col_len, cur);
    if (leaf_count == 1) {
        if (leaf_index == 0 && n_sib == 0) return memcmp(cur, root, 32) ? -1 : 0;
        return -1;
    }
    uint8_t dirs[64];
    uint32_t nd = 0;
    uint64_t size = leaf_count, idx = leaf_index;
    while (size > 1) {
        uint64_t p2 = 1;
        while (p2 < size) p2 <<= 1;
        uint64_t split = p2 / 2;
        if (nd >= 64) return -1;
        if (idx < split) {
            dirs[nd++] = 0;
            size = split;
        } else {
            dirs[nd++] = 1;
            size -= split;
            idx -= split;
        }
    }
    if (nd != n_sib) return -1;
    /* reverse: leaf to root */
    for (uint32_t i = 0; i < nd / 2; i++) {
        uint8_t t = dirs[i];
        dirs[i] = dirs[nd - 1 - i];
        dirs[nd - 1 - i] = t;
    }
    for (uint32_t i = 0; i < nd; i++) {
        int root_merge = (i == nd - 1);
        const uint8_t *sib = siblings + 32 * i;
        uint8_t nxt[32];
        if (dirs[i] == 0) zr_blake3_parent(cur, sib, root_merge, nxt);
        else zr_blake3_parent(sib, cur, root_merge, nxt);
        memcpy(cur, nxt, 32);
    }
    return memcmp(cur, root, 32) ? -1 : 0;
}

/* ========================================================================
 * Wide integers and the Montgomery prime field (crypto-bigint Int/Uint,
 * crypto-primitives MontyField; utils/src/field/monty.rs)
 * ====================================================================== */
typedef struct {
    uint32_t L;
    uint64_t p[4], n0, one[4], r2[4], rpow[4][4]; /* rpow[k] = R^(k+2) mod p */
} fcfg;

static int ucmp(const uint64_t *a, const uint64_t *b, uint32_t L) {
    for (int i = (int)L - 1; i >= 0; i--) {
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    }
    return 0;
}
static uint64_t usub(uint64_t *a, const uint64_t *b, uint32_t L) {
    uint64_t br = 0;
    for (uint32_t i = 0; i < L; i++) {
        u128 s = (u128)a[i] - b[i] - br;
        a[i] = (uint64_t)s;
        br = (uint64_t)(s >> 64) & 1;
    }
    return br;
}
static uint64_t uadd(uint64_t *a, const uint64_t *b, uint32_t L) {
    u128 c = 0;
    for (uint32_t i = 0; i < L; i++) {
        u128 s = (u128)a[i] + b[i] + c;
        a[i] = (uint64_t)s;
        c = s >> 64;
    }
    return (uint64_t)c;
}
static int uiszero(const uint64_t *a, uint32_t L) {
    for (uint32_t i = 0; i < L; i++)
        if (a[i]) return 0;
    return 1;
}

static void fadd(const fcfg *f, uint64_t *a, const uint64_t *b) {
    uint64_t c = uadd(a, b, f->L);
    if (c || ucmp(a, f->p, f->L) >= 0) usub(a, f->p, f->L);
}
static void fsub(const fcfg *f, uint64_t *a, const uint64_t *b) {
    if (usub(a, b, f->L)) uadd(a, f->p, f->L);
}
static void fneg(const fcfg *f, uint64_t *a) {
    if (uiszero(a, f->L)) return;
    uint64_t t[4];
    memcpy(t, f->p, 8 * f->L);
    usub(t, a, f->L);
    memcpy(a, t, 8 * f->L);
}

/* CIOS Montgomery multiplication: out = a*b*R^-1 mod p (a, b < p or a < R). */
static void fmul(const fcfg *f, const uint64_t *a, const uint64_t *b, uint64_t *out) {
    uint32_t L = f->L;
    uint64_t t[6] = {0};
    for (uint32_t i = 0; i < L; i++) {
        u128 c = 0;
        for (uint32_t j = 0; j < L; j++) {
            u128 s = (u128)a[j] * b[i] + t[j] + c;
            t[j] = (uint64_t)s;
            c = s >> 64;
        }
        u128 s = (u128)t[L] + c;
        t[L] = (uint64_t)s;
        t[L + 1] = (uint64_t)(s >> 64);
        uint64_t m = t[0] * f->n0;
        s = (u128)m * f->p[0] + t[0];
        c = s >> 64;
        for (uint32_t j = 1; j < L; j++) {
            s = (u128)m * f->p[j] + t[j] + c;
            t[j - 1] = (uint64_t)s;
            c = s >> 64;
        }
        s = (u128)t[L] + c;
        t[L - 1] = (uint64_t)s;
        t[L] = t[L + 1] + (uint64_t)(s >> 64);
    }
    if (t[L] || ucmp(t, f->p, L) >= 0) usub(t, f->p, L);
    memcpy(out, t, 8 * L);
}

static void fcfg_init(fcfg *f, const uint64_t *p, uint32_t L) {
    memset(f, 0, sizeof *f);
    f->L = L;
    memcpy(f->p, p, 8 * L);
    uint64_t inv = p[0];
    for (int i = 0; i < 6; i++) inv *= 2 - p[0] * inv;
    f->n0 = (uint64_t)0 - inv;
    uint64_t x[4] = {1, 0, 0, 0};
    if (ucmp(x, f->p, L) >= 0) usub(x, f->p, L);
    for (uint32_t i = 0; i < 64 * L; i++) fadd(f, x, x);
    memcpy(f->one, x, 8 * L);
    for (uint32_t i = 0; i < 64 * L; i++) fadd(f, x, x);
    memcpy(f->r2, x, 8 * L);
    memcpy(f->rpow[0], f->r2, 8 * L);
    for (int k = 1; k < 4; k++) fmul(f, f->rpow[k - 1], f->r2, f->rpow[k]);
}

/* F::from_with_cfg(&Int<limbs>) -> Montgomery inner (signed, reduced mod p;
 * phase_verify.rs:192-196 and utils/src/field/monty.rs:98-157). */
static void f_from_int(const fcfg *f, const uint64_t *x, uint32_t limbs, uint64_t *out) {
    uint32_t L = f->L;
    int neg = (int)(x[limbs - 1] >> 63);
    uint64_t mag[16] = {0};
    memcpy(mag, x, 8 * limbs);
    if (neg) {
        u128 c = 1;
        for (uint32_t i = 0; i < limbs; i++) {
            u128 s = (u128)(~mag[i]) + c;
            mag[i] = (uint64_t)s;
            c = s >> 64;
        }
    }
    uint64_t acc[4] = {0};
    uint32_t ndig = (limbs + L - 1) / L;
    for (uint32_t k = 0; k < ndig; k++) {
        if (uiszero(mag + k * L, L)) continue;
        uint64_t t[4];
        fmul(f, mag + k * L, f->rpow[k], t);
        fadd(f, acc, t);
    }
    if (neg) fneg(f, acc);
    memcpy(out, acc, 8 * L);
}

static void f_from_i128(const fcfg *f, i128 v, uint64_t *out) {
    uint64_t x[2] = {(uint64_t)(u128)v, (uint64_t)((u128)v >> 64)};
    f_from_int(f, x, 2, out);
}

/* Strong probable-prime test to base 2 (primality/src/lib.rs:12-19, crypto-primes
 * hazmat MillerRabin::test_base_two). */
int zr_is_probable_prime_base2(const uint64_t *n, uint32_t L) {
    if (!(n[0] & 1)) return 0;
    uint64_t one[4] = {1, 0, 0, 0};
    if (ucmp(n, one, L) == 0) return 0;
    fcfg f;
    fcfg_init(&f, n, L);
    uint64_t nm1[4] = {0};
    memcpy(nm1, n, 8 * L);
    nm1[0] -= 1; /* n odd */
    uint32_t s = 0;
    while (!((nm1[s / 64] >> (s % 64)) & 1)) s++;
    /* d = nm1 >> s */
    uint64_t d[4] = {0};
    for (uint32_t i = 0; i < 64 * L - s; i++)
        if ((nm1[(i + s) / 64] >> ((i + s) % 64)) & 1) d[i / 64] |= 1ull << (i % 64);
    int top = 64 * (int)L - 1;
    while (top >= 0 && !((d[top / 64] >> (top % 64)) & 1)) top--;
    uint64_t x[4];
    memcpy(x, f.one, 8 * L);
    for (int b = top; b >= 0; b--) {
        uint64_t t[4];
        fmul(&f, x, x, t);
        memcpy(x, t, 8 * L);
        if ((d[b / 64] >> (b % 64)) & 1) fadd(&f, x, x);
    }
    uint64_t mone[4];
    memcpy(mone, f.one, 8 * L);
    fneg(&f, mone);
    if (ucmp(x, f.one, L) == 0 || ucmp(x, mone, L) == 0) return 1;
    for (uint32_t i = 1; i < s; i++) {
        uint64_t t[4];
        fmul(&f, x, x, t);
        memcpy(x, t, 8 * L);
        if (ucmp(x, f.one, L) == 0) return 0;
        if (ucmp(x, mone, L) == 0) return 1;
    }
    return 0;
}

/* ========================================================================
 * Blake3Transcript (transcript/src/lib.rs:12-77, traits.rs:329-426)
 * ====================================================================== */
struct zr_transcript {
    b3_hasher h;
};

zr_transcript *zr_tr_new(void) {
    zr_transcript *t = (zr_transcript *)malloc(sizeof *t);
    b3_hasher_init(&t->h);
    return t;
}
void zr_tr_free(zr_transcript *t) { free(t); }
void zr_tr_absorb(zr_transcript *t, const uint8_t *buf, size_t n) { b3_hasher_update(&t->h, buf, n); }
void zr_tr_absorb_slice(zr_transcript *t, const uint8_t *buf, size_t n) {
    uint8_t a = 0x06, b = 0x07;
    zr_tr_absorb(t, &a, 1);
    zr_tr_absorb(t, buf, n);
    zr_tr_absorb(t, &b, 1);
}
void zr_tr_challenge(zr_transcript *t, uint8_t *out, size_t n) {
    b3_hasher_xof(&t->h, out, n);
    uint8_t a = 0x12, b = 0x34;
    zr_tr_absorb(t, &a, 1);
    zr_tr_absorb(t, out, n);
    zr_tr_absorb(t, &b, 1);
}
void zr_tr_get_prime(zr_transcript *t, uint32_t L, uint64_t *prime_out) {
    for (;;) {
        uint8_t buf[32];
        b3_hasher_xof(&t->h, buf, 8 * L);
        zr_tr_absorb(t, buf, 8 * L);
        uint64_t c[4] = {0};
        memcpy(c, buf, 8 * L);
        if (uiszero(c, L)) continue;
        if (!(c[0] & 1)) { /* prime_candidate -= ONE, full width */
            for (uint32_t i = 0; i < L; i++)
                if (c[i]-- != 0) break;
        }
        if (zr_is_probable_prime_base2(c, L)) {
            memcpy(prime_out, c, 8 * L);
            return;
        }
    }
}
static i128 tr_i128(zr_transcript *t) {
    uint8_t b[16];
    zr_tr_challenge(t, b, 16);
    u128 v = 0;
    for (int i = 15; i >= 0; i--) v = (v << 8) | b[i];
    return (i128)v;
}
static uint32_t tr_u32(zr_transcript *t) {
    uint8_t b[4];
    zr_tr_challenge(t, b, 4);
    return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
}
/* absorb_random_field (traits.rs:393-413) */
static void tr_absorb_field(zr_transcript *t, const fcfg *f, const uint64_t *inner) {
    uint8_t c3 = 3, c5 = 5, c1 = 1;
    zr_tr_absorb(t, &c3, 1);
    zr_tr_absorb(t, (const uint8_t *)f->p, 8 * f->L);
    zr_tr_absorb(t, &c5, 1);
    zr_tr_absorb(t, &c1, 1);
    zr_tr_absorb(t, (const uint8_t *)inner, 8 * f->L);
    zr_tr_absorb(t, &c3, 1);
}

/* ========================================================================
 * Zip+ commit / prove / verify (pcs/phase_commit.rs, phase_prove.rs,
 * phase_verify.rs, pcs_transcript.rs)
 * ====================================================================== */
typedef struct {
    uint8_t *cw;  /* batch x num_rows x codeword_len x cw_bytes */
    mtree tree;
} zhint;

static void zhint_free(zhint *h) {
    free(h->cw);
    mtree_free(&h->tree);
}

/* validate_input bit budget (pcs/utils.rs:24-54) */
static int validate_bits(const zparams *z, uint32_t batch) {
    uint32_t d = 31 - (uint32_t)__builtin_clz(z->row_len);
    uint64_t t = (uint64_t)z->d.rep * d;
    if (t < 1) t = 1;
    uint32_t cwb = 0;
    while ((1ull << cwb) < t) cwb++;
    uint32_t dd = d < 1 ? 1 : d, ld = 0;
    while ((1u << ld) < dd) ld++;
    uint32_t chal = 128 * (z->D > 1 ? 2 : 1);
    uint32_t eval_bits = z->d.eval_kind == ZR_EVAL_BINPOLY ? 1 : z->d.eval_kind == ZR_EVAL_I64 ? 64 : 32;
    uint32_t lb = 0;
    while ((1u << lb) < batch) lb++;
    uint32_t actual = 2 * cwb + ld + chal + (eval_bits - 1) + lb;
    return actual <= 64 * z->d.comb_limbs ? 0 : -1;
}

static int do_commit(const zparams *z, const uint8_t *polys, uint32_t batch, zhint *h) {
    if (z->d.code_kind != ZR_CODE_IPRS && z->d.eval_kind != ZR_EVAL_BINPOLY) return -1;
    size_t rowbytes = (size_t)z->codeword_len * z->cw_bytes;
    size_t polycw = rowbytes * z->num_rows;
    size_t polyev = (size_t)z->num_rows * z->row_len * z->eval_bytes;
    h->cw = (uint8_t *)malloc(polycw * batch);
    for (uint32_t b = 0; b < batch; b++) encode_poly(z, polys + b * polyev, h->cw + b * polycw);
    uint32_t nr = z->num_rows * batch;
    const uint8_t **rows = (const uint8_t **)malloc(sizeof(uint8_t *) * nr);
    for (uint32_t r = 0; r < nr; r++) rows[r] = h->cw + (size_t)r * rowbytes;
    uint8_t *leaves = hash_leaves(rows, nr, z->codeword_len, z->cw_bytes);
    free(rows);
    mtree_build(&h->tree, leaves, z->codeword_len);
    return 0;
}

int zr_commit(const zr_desc *d, const void *polys, uint32_t batch, uint8_t root[32]) {
    zparams z;
    if (batch == 0 || zparams_build(d, &z)) return -1;
    if (validate_bits(&z, batch)) {
        zparams_free(&z);
        return -2;
    }
    zhint h;
    if (do_commit(&z, (const uint8_t *)polys, batch, &h)) {
        zparams_free(&z);
        return -1;
    }
    memcpy(root, h.tree.layers[h.tree.n_layers - 1], 32);
    zhint_free(&h);
    zparams_free(&z);
    return 0;
}

size_t zr_proof_size(const zr_desc *d, uint32_t batch) {
    zparams z;
    if (zparams_build(d, &z)) return 0;
    uint32_t depth = 0;
    while ((1u << depth) < z.codeword_len) depth++;
    size_t f = 16 * d->field_limbs;
    size_t s = (size_t)z.num_rows * f + (size_t)z.row_len * 8 * d->comb_limbs +
               (size_t)d->num_openings *
                   ((size_t)batch * z.num_rows * z.cw_bytes + 24 + 32 * (size_t)depth);
    zparams_free(&z);
    return s;
}

typedef struct {
    uint8_t *p;
    size_t len, cap;
    int overflow;
} wbuf;
static void wput(wbuf *w, const void *src, size_t n) {
    if (w->len + n > w->cap) {
        w->overflow = 1;
        return;
    }
    memcpy(w->p + w->len, src, n);
    w->len += n;
}

/* eq table: res[i] = prod_k (bit_k(i) ? r_k : 1 - r_k) (poly/src/utils.rs:24-101) */
static void build_eq(const fcfg *f, const uint64_t *r, uint32_t n, uint64_t *out) {
    uint32_t L = f->L;
    memcpy(out, f->one, 8 * L);
    size_t len = 1;
    for (int k = (int)n - 1; k >= 0; k--) {
        /* prepend variable k as the new lowest bit */
        for (long i = (long)len - 1; i >= 0; i--) {
            uint64_t b[4], t[4];
            memcpy(b, out + i * L, 8 * L);
            fmul(f, r + k * L, b, t);
            memcpy(out + (2 * i + 1) * L, t, 8 * L);
            fsub(f, b, t);
            memcpy(out + (2 * i) * L, b, 8 * L);
        }
        len *= 2;
    }
}

/* w'[i] = <eval_i, alphas> as Int<comb_limbs> (phase_prove.rs:154-174) */
static void alpha_project(const zparams *z, const uint8_t *evals, size_t n, const i128 *alphas,
                          uint64_t *out) {
    uint32_t C = z->d.comb_limbs;
    int nt = zr_get_threads();
    (void)nt;
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long i = 0; i < (long)n; i++) {
        uint64_t *o = out + (size_t)i * C;
        if (z->d.eval_kind != ZR_EVAL_BINPOLY) {
            int64_t v;
            if (z->d.eval_kind == ZR_EVAL_I64) memcpy(&v, evals + 8 * i, 8);
            else {
                int32_t v32;
                memcpy(&v32, evals + 4 * i, 4);
                v = v32;
            }
            /* ScalarProduct with alphas == [1] */
            uint64_t x[8];
            uint64_t sgn = v < 0 ? ~0ull : 0;
            x[0] = (uint64_t)v;
            for (uint32_t k = 1; k < C; k++) x[k] = sgn;
            memset(o, 0, 8 * C);
            wl_mul_i64_add(o, x, (int64_t)alphas[0], C);
            /* alphas[0] == 1 for scalars; the high part is zero */
        } else {
            uint64_t x;
            memcpy(&x, evals + 8 * i, 8);
            x &= dmask(z->D);
            memset(o, 0, 8 * C);
            while (x) {
                int b = __builtin_ctzll(x);
                i128 a = alphas[b];
                uint64_t add[8];
                add[0] = (uint64_t)(u128)a;
                add[1] = (uint64_t)((u128)a >> 64);
                uint64_t sgn = a < 0 ? ~0ull : 0;
                for (uint32_t k = 2; k < C; k++) add[k] = sgn;
                uadd(o, add, C);
                x &= x - 1;
            }
        }
    }
}

/* Int<C> * i128 wrapping, accumulate */
static void wmul_i128_add(uint64_t *acc, const uint64_t *x, i128 s, uint32_t C) {
    uint64_t sv[8];
    sv[0] = (uint64_t)(u128)s;
    if (C > 1) sv[1] = (uint64_t)((u128)s >> 64);
    uint64_t sg = s < 0 ? ~0ull : 0;
    for (uint32_t k = 2; k < C; k++) sv[k] = sg;
    uint64_t prod[8] = {0};
    for (uint32_t i = 0; i < C; i++) {
        u128 c = 0;
        for (uint32_t j = 0; i + j < C; j++) {
            u128 t = (u128)x[i] * sv[j] + prod[i + j] + c;
            prod[i + j] = (uint64_t)t;
            c = t >> 64;
        }
    }
    uadd(acc, prod, C);
}

/* When set, the next commit_prove takes its point as unsigned 256-bit integers
 * (4 u64 each) mapped into the field after the prime is drawn: prove_f's point
 * (phase_prove.rs:119-130) in a form that does not depend on the prime. */
static const uint64_t *g_point_u256 = NULL;

static void read_prime_and_points(zr_transcript *tr, const zparams *z, const int64_t *point,
                                  fcfg *f, uint64_t *pf) {
    uint64_t prime[4];
    zr_tr_get_prime(tr, z->d.field_limbs, prime);
    fcfg_init(f, prime, z->d.field_limbs);
    for (uint32_t i = 0; i < z->d.num_vars; i++) {
        if (g_point_u256) {
            uint64_t x[5] = {g_point_u256[4 * i], g_point_u256[4 * i + 1], g_point_u256[4 * i + 2],
                             g_point_u256[4 * i + 3], 0};
            f_from_int(f, x, 5, pf + i * f->L);
            continue;
        }
        i128 v = (i128)(((u128)(uint64_t)point[2 * i + 1] << 64) | (uint64_t)point[2 * i]);
        f_from_i128(f, v, pf + i * f->L);
    }
}

/* point_to_tensor (pcs/utils.rs:90-114) */
static void point_tensor(const fcfg *f, const zparams *z, const uint64_t *pf, uint64_t *q0,
                         uint64_t *q1) {
    uint32_t L = f->L, lr = (uint32_t)__builtin_ctz(z->num_rows), nv = z->d.num_vars;
    uint32_t nhi = nv - lr;
    if (lr) build_eq(f, pf + (size_t)nhi * L, lr, q0);
    else memcpy(q0, f->one, 8 * L);
    if (nhi) build_eq(f, pf, nhi, q1);
    else memcpy(q1, f->one, 8 * L);
}

/* The prove phase after the point is in the field (phase_prove.rs:132-304):
 * alphas, b, eval, coefficients, combined row and openings on `tr`, proof
 * bytes appended to w. */
static void prove_core(const zparams *z, const uint8_t *polys, uint32_t batch, const zhint *h, zr_transcript *tr,
                       const fcfg *f, const uint64_t *pf, wbuf *w, uint8_t *eval_out) {
    uint32_t L = z->d.field_limbs, C = z->d.comb_limbs, R = z->num_rows, RL = z->row_len;
    uint64_t *q0 = (uint64_t *)malloc(8 * L * (size_t)R), *q1 = (uint64_t *)malloc(8 * L * (size_t)RL);
    point_tensor(f, z, pf, q0, q1);

    size_t N = (size_t)R * RL, polyev = N * z->eval_bytes;
    uint64_t *wp = (uint64_t *)malloc(sizeof(uint64_t) * C * N * batch);
    i128 alphas[64];
    for (uint32_t b = 0; b < batch; b++) {
        uint32_t na = z->D > 1 ? z->D : 1;
        if (z->D > 1)
            for (uint32_t i = 0; i < na; i++) alphas[i] = tr_i128(tr);
        else alphas[0] = 1;
        alpha_project(z, polys + b * polyev, N, alphas, wp + (size_t)b * N * C);
    }
    /* b[j] = sum_poly <F(w'_j), q1> (phase_prove.rs:179-193) */
    uint64_t *bv = (uint64_t *)calloc((size_t)R, 8 * L);
    int nt = zr_get_threads();
    (void)nt;
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long j = 0; j < (long)R; j++) {
        uint64_t acc[4] = {0};
        for (uint32_t b = 0; b < batch; b++) {
            const uint64_t *row = wp + ((size_t)b * N + (size_t)j * RL) * C;
            for (uint32_t c = 0; c < RL; c++) {
                uint64_t fe[4], t[4];
                f_from_int(f, row + (size_t)c * C, C, fe);
                fmul(f, fe, q1 + (size_t)c * L, t);
                fadd(f, acc, t);
            }
        }
        memcpy(bv + j * L, acc, 8 * L);
    }
    /* write_field_elements (pcs_transcript.rs:99-142), LENGTH_NUM_BYTES = 0 */
    for (uint32_t j = 0; j < R; j++) {
        tr_absorb_field(tr, f, bv + (size_t)j * L);
        wput(w, f->p, 8 * L);
        wput(w, bv + (size_t)j * L, 8 * L);
    }
    uint64_t ev[4] = {0};
    for (uint32_t j = 0; j < R; j++) {
        uint64_t t[4];
        fmul(f, q0 + (size_t)j * L, bv + (size_t)j * L, t);
        fadd(f, ev, t);
    }
    i128 *coeffs = (i128 *)malloc(sizeof(i128) * R);
    if (R == 1) coeffs[0] = 1;
    else
        for (uint32_t j = 0; j < R; j++) coeffs[j] = tr_i128(tr);
    /* combined_row (phase_prove.rs:205-244) */
    uint64_t *comb = (uint64_t *)calloc((size_t)RL, 8 * C);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long c = 0; c < (long)RL; c++) {
        uint64_t *acc = comb + (size_t)c * C;
        for (uint32_t b = 0; b < batch; b++)
            for (uint32_t j = 0; j < R; j++)
                wmul_i128_add(acc, wp + ((size_t)b * N + (size_t)j * RL + c) * C, coeffs[j], C);
    }
    wput(w, comb, (size_t)RL * 8 * C);
    /* openings (phase_prove.rs:285-304, pcs_transcript.rs:210-221) */
    size_t rowbytes = (size_t)z->codeword_len * z->cw_bytes;
    uint64_t depth = h->tree.n_layers - 1;
    for (uint32_t o = 0; o < z->d.num_openings; o++) {
        uint32_t idx = tr_u32(tr) % z->codeword_len;
        for (uint32_t r = 0; r < R * batch; r++) wput(w, h->cw + (size_t)r * rowbytes + (size_t)idx * z->cw_bytes, z->cw_bytes);
        uint64_t li = idx, lc = z->codeword_len;
        wput(w, &li, 8);
        wput(w, &lc, 8);
        wput(w, &depth, 8);
        uint64_t cur = idx;
        for (uint32_t k = 0; k < depth; k++) {
            wput(w, h->tree.layers[k] + 32 * (cur ^ 1), 32);
            cur >>= 1;
        }
    }
    if (eval_out) memcpy(eval_out, ev, 8 * L);
    free(comb);
    free(coeffs);
    free(bv);
    free(wp);
    free(q0);
    free(q1);
}

int zr_commit_prove(const zr_desc *d, const void *polys_v, uint32_t batch, const int64_t *point,
                    uint8_t root[32], uint8_t *proof, size_t proof_cap, size_t *proof_len,
                    uint8_t *eval_out, uint8_t *modulus_out) {
    zparams z;
    if (batch == 0 || zparams_build(d, &z)) return -1;
    if (validate_bits(&z, batch)) {
        zparams_free(&z);
        return -2;
    }
    const uint8_t *polys = (const uint8_t *)polys_v;
    zhint h;
    if (do_commit(&z, polys, batch, &h)) {
        zparams_free(&z);
        return -1;
    }
    memcpy(root, h.tree.layers[h.tree.n_layers - 1], 32);

    zr_transcript *tr = zr_tr_new();
    zr_tr_absorb_slice(tr, root, 32);
    fcfg f;
    uint32_t L = d->field_limbs;
    uint64_t *pf = (uint64_t *)calloc((size_t)d->num_vars + 1, 8 * L);
    read_prime_and_points(tr, &z, point, &f, pf);
    wbuf w = {proof, 0, proof_cap, 0};
    prove_core(&z, polys, batch, &h, tr, &f, pf, &w, eval_out);
    *proof_len = w.len;
    if (modulus_out) memcpy(modulus_out, f.p, 8 * L);
    free(pf);
    zr_tr_free(tr);
    zhint_free(&h);
    zparams_free(&z);
    return w.overflow ? -3 : 0;
}

/* ZipPlus::prove_f (phase_prove.rs:119-130) on a transcript that is already in
 * use: the point (num_vars Montgomery inners of `field_limbs` u64) is in the
 * field of `modulus`, which nothing here draws.  The hint is rebuilt by
 * committing again (the commitment is deterministic). */
int zr_prove_f_on(const zr_desc *d, const void *polys_v, uint32_t batch, zr_transcript *tr,
                  const uint64_t *modulus, const uint64_t *point_f, uint8_t *proof, size_t proof_cap,
                  size_t *proof_len, uint8_t *eval_out) {
    zparams z;
    if (batch == 0 || zparams_build(d, &z)) return -1;
    if (validate_bits(&z, batch)) {
        zparams_free(&z);
        return -2;
    }
    zhint h;
    if (do_commit(&z, (const uint8_t *)polys_v, batch, &h)) {
        zparams_free(&z);
        return -1;
    }
    fcfg f;
    fcfg_init(&f, modulus, d->field_limbs);
    wbuf w = {proof, 0, proof_cap, 0};
    prove_core(&z, (const uint8_t *)polys_v, batch, &h, tr, &f, point_f, &w, eval_out);
    *proof_len = w.len;
    zhint_free(&h);
    zparams_free(&z);
    return w.overflow ? -3 : 0;
}

typedef struct {
    const uint8_t *p;
    size_t len, pos;
} rbuf;
static int rget(rbuf *r, void *dst, size_t n) {
    if (r->pos + n > r->len) return -1;
    memcpy(dst, r->p + r->pos, n);
    r->pos += n;
    return 0;
}

/* ZipPlus::verify_with_alphas (phase_verify.rs:137-304) after the point is in
 * the field: reads b, the combined row and the openings from rd (the PCS
 * stream) while absorbing into tr; alphas: batch x max(D, 1) per-poly
 * challenges (sample_alphas, phase_verify.rs:247-261).  0 = accept, 2 = a
 * check failed, 3 = malformed stream. */
static int verify_core(const zparams *z, const uint8_t root[32], uint32_t batch, zr_transcript *tr, const fcfg *fp,
                       const uint64_t *pf, const uint64_t *eval_f, const i128 *alphas, rbuf *rd) {
    const fcfg f = *fp;
    int rc = 0;
    const zr_desc *d = &z->d;
    uint32_t L = d->field_limbs, C = d->comb_limbs, R = z->num_rows, RL = z->row_len, D = z->D;
    uint64_t *q0 = (uint64_t *)malloc(8 * L * (size_t)R), *q1 = (uint64_t *)malloc(8 * L * (size_t)RL);
    point_tensor(&f, z, pf, q0, q1);
    uint64_t *bv = (uint64_t *)calloc((size_t)R, 8 * L);
    uint64_t *comb = NULL, *enc = NULL;
    i128 *coeffs = (i128 *)malloc(sizeof(i128) * R);
    uint8_t *col = NULL, *sib = NULL;
    for (uint32_t j = 0; j < R; j++) {
        uint64_t mod[4] = {0}, inner[4] = {0};
        if (rget(rd, mod, 8 * L) || rget(rd, inner, 8 * L)) { rc = 3; goto out; }
        if (ucmp(mod, f.p, L) != 0) { rc = 2; goto out; }
        tr_absorb_field(tr, &f, inner);
        memcpy(bv + (size_t)j * L, inner, 8 * L);
    }
    {
        uint64_t ev[4] = {0};
        for (uint32_t j = 0; j < R; j++) {
            uint64_t t[4];
            fmul(&f, q0 + (size_t)j * L, bv + (size_t)j * L, t);
            fadd(&f, ev, t);
        }
        if (memcmp(ev, eval_f, 8 * L)) { rc = 2; goto out; }
    }
    if (R == 1) coeffs[0] = 1;
    else
        for (uint32_t j = 0; j < R; j++) coeffs[j] = tr_i128(tr);
    comb = (uint64_t *)malloc((size_t)RL * 8 * C);
    if (rget(rd, comb, (size_t)RL * 8 * C)) { rc = 3; goto out; }
    enc = (uint64_t *)malloc((size_t)z->codeword_len * 8 * C);
    zr_encode_wide(d, comb, C, enc);
    {
        uint64_t lhs[4] = {0}, rhs[4] = {0};
        for (uint32_t c = 0; c < RL; c++) {
            uint64_t fe[4], t[4];
            f_from_int(&f, comb + (size_t)c * C, C, fe);
            fmul(&f, fe, q1 + (size_t)c * L, t);
            fadd(&f, lhs, t);
        }
        for (uint32_t j = 0; j < R; j++) {
            uint64_t fe[4], t[4];
            f_from_i128(&f, coeffs[j], fe);
            fmul(&f, fe, bv + (size_t)j * L, t);
            fadd(&f, rhs, t);
        }
        if (memcmp(lhs, rhs, 8 * L)) { rc = 2; goto out; }
    }
    {
        size_t colbytes = (size_t)batch * R * z->cw_bytes;
        col = (uint8_t *)malloc(colbytes);
        sib = (uint8_t *)malloc(32 * 64);
        for (uint32_t o = 0; o < d->num_openings; o++) {
            uint32_t idx = tr_u32(tr) % z->codeword_len;
            uint64_t li, lc, np;
            if (rget(rd, col, colbytes) || rget(rd, &li, 8) || rget(rd, &lc, 8) || rget(rd, &np, 8)) { rc = 3; goto out; }
            if (np == 0 || np > 64 || li >= lc) { rc = 3; goto out; }
            if (rget(rd, sib, 32 * np)) { rc = 3; goto out; }
            /* check 3 (phase_verify.rs:267-304) */
            uint64_t acc[8] = {0};
            for (uint32_t b = 0; b < batch; b++)
                for (uint32_t j = 0; j < R; j++) {
                    const uint8_t *e = col + ((size_t)b * R + j) * z->cw_bytes;
                    uint64_t v[8] = {0};
                    if (z->d.eval_kind != ZR_EVAL_BINPOLY) {
                        uint64_t x[8];
                        memcpy(x, e, 16);
                        uint64_t sg = (x[1] >> 63) ? ~0ull : 0;
                        for (uint32_t k = 2; k < C; k++) x[k] = sg;
                        memcpy(v, x, 8 * C);
                    } else {
                        for (uint32_t i = 0; i < D; i++) {
                            uint64_t x[8];
                            int64_t c64;
                            if (z->cw_bytes == 8 * D) memcpy(&c64, e + 8 * i, 8);
                            else {
                                int32_t c32;
                                memcpy(&c32, e + 4 * i, 4);
                                c64 = c32;
                            }
                            x[0] = (uint64_t)c64;
                            for (uint32_t k = 1; k < C; k++) x[k] = c64 < 0 ? ~0ull : 0;
                            wmul_i128_add(v, x, alphas[b * D + i], C);
                        }
                    }
                    wmul_i128_add(acc, v, coeffs[j], C);
                }
            if (memcmp(acc, enc + (size_t)idx * C, 8 * C)) { rc = 2; goto out; }
            if (merkle_verify(root, col, colbytes, li, lc, sib, np, idx)) { rc = 2; goto out; }
        }
    }
out:
    free(col);
    free(sib);
    free(enc);
    free(comb);
    free(coeffs);
    free(bv);
    free(q0);
    free(q1);
    return rc;
}

/* ZipPlus::verify (phase_verify.rs:100-304).  0 = accept. */
int zr_verify(const zr_desc *d, const uint8_t root[32], uint32_t batch, const int64_t *point,
              const uint8_t *eval_inner, const uint8_t *proof, size_t proof_len) {
    zparams z;
    if (batch == 0 || zparams_build(d, &z)) return -1;
    if (validate_bits(&z, batch)) {
        zparams_free(&z);
        return -2;
    }
    uint32_t L = d->field_limbs, D = z.D;
    zr_transcript *tr = zr_tr_new();
    zr_tr_absorb_slice(tr, root, 32);
    fcfg f;
    uint64_t *pf = (uint64_t *)calloc((size_t)d->num_vars + 1, 8 * L);
    read_prime_and_points(tr, &z, point, &f, pf);
    i128 *alphas = (i128 *)malloc(sizeof(i128) * batch * (D > 1 ? D : 1));
    for (uint32_t b = 0; b < batch; b++) {
        if (D > 1)
            for (uint32_t i = 0; i < D; i++) alphas[b * D + i] = tr_i128(tr);
        else alphas[b] = 1;
    }
    uint64_t ev[4] = {0};
    memcpy(ev, eval_inner, 8 * L);
    rbuf rd = {proof, proof_len, 0};
    int rc = verify_core(&z, root, batch, tr, &f, pf, ev, alphas, &rd);
    free(alphas);
    free(pf);
    zr_tr_free(tr);
    zparams_free(&z);
    return rc;
}

/* ========================================================================
 * Sumcheck (piop/src/sumcheck.rs:163-338, sumcheck/prover.rs:95-247,
 * sumcheck/verifier.rs, sumcheck/multi_degree.rs:259-355) with the
 * combination function comb(v) = sum_k coeff_k * prod_{i in S_k} v_i, the
 * form of the reference's test comb functions (sumcheck/tests/utils.rs:60-80).
 * Field elements are Montgomery inner values of L limbs.
 * ====================================================================== */
static void f_from_u64(const fcfg *f, uint64_t v, uint64_t *out) {
    uint64_t x[2] = {v, 0};
    f_from_int(f, x, 2, out);
}

/* comb(vals) for one group: the sum of products, times every affine factor */
static void sc_comb(const fcfg *f, const zr_sc_group *g, const uint64_t *vals, uint64_t *out) {
    uint32_t L = f->L;
    uint64_t acc[4] = {0};
    for (uint32_t k = 0; k < g->n_products; k++) {
        uint64_t t[4];
        memcpy(t, g->coeffs + (size_t)k * L, 8 * L);
        for (uint32_t q = g->offsets[k]; q < g->offsets[k + 1]; q++) {
            uint64_t u[4];
            fmul(f, t, vals + (size_t)g->indices[q] * L, u);
            memcpy(t, u, 8 * L);
        }
        fadd(f, acc, t);
    }
    for (uint32_t q = 0; q < g->n_factors; q++) {
        uint64_t fv[4], u[4];
        fmul(f, g->factor_b + (size_t)q * L, vals + (size_t)g->factor_mles[q] * L, fv);
        fadd(f, fv, g->factor_a + (size_t)q * L);
        fmul(f, acc, fv, u);
        memcpy(acc, u, 8 * L);
    }
    memcpy(out, acc, 8 * L);
}

/* ProverState::prove_round evaluations (before removing P(0)): evals[deg+1] */
static void sc_round_evals(const fcfg *f, const zr_sc_group *g, uint64_t *const *m, size_t half,
                           uint64_t *evals) {
    uint32_t L = f->L, K = g->n_mles, D = g->degree;
    memset(evals, 0, 8 * L * (size_t)(D + 1));
    int nt = zr_get_threads();
    (void)nt;
#pragma omp parallel num_threads(nt)
    {
        uint64_t *loc = (uint64_t *)calloc((size_t)(D + 1) * L, 8);
        uint64_t *v0 = (uint64_t *)malloc(8 * L * (size_t)K), *v1 = (uint64_t *)malloc(8 * L * (size_t)K);
        uint64_t *st = (uint64_t *)malloc(8 * L * (size_t)K), *cur = (uint64_t *)malloc(8 * L * (size_t)K);
#pragma omp for schedule(static)
        for (long b = 0; b < (long)half; b++) {
            for (uint32_t j = 0; j < K; j++) {
                memcpy(v0 + j * L, m[j] + (size_t)(2 * b) * L, 8 * L);
                memcpy(v1 + j * L, m[j] + (size_t)(2 * b + 1) * L, 8 * L);
            }
            uint64_t e[4];
            sc_comb(f, g, v0, e);
            fadd(f, loc, e);
            if (D > 0) {
                sc_comb(f, g, v1, e);
                fadd(f, loc + L, e);
                for (uint32_t j = 0; j < K; j++) {
                    memcpy(st + j * L, v1 + j * L, 8 * L);
                    fsub(f, st + j * L, v0 + j * L);
                    memcpy(cur + j * L, v1 + j * L, 8 * L);
                }
                for (uint32_t t = 2; t <= D; t++) {
                    for (uint32_t j = 0; j < K; j++) fadd(f, cur + j * L, st + j * L);
                    sc_comb(f, g, cur, e);
                    fadd(f, loc + (size_t)t * L, e);
                }
            }
        }
#pragma omp critical
        for (uint32_t t = 0; t <= D; t++) fadd(f, evals + (size_t)t * L, loc + (size_t)t * L);
        free(loc);
        free(v0);
        free(v1);
        free(st);
        free(cur);
    }
}

/* fix_variables_with_config (poly/src/mle/dense.rs:243-279) with one point */
static void sc_fold(const fcfg *f, uint64_t *m, size_t half, const uint64_t *r) {
    uint32_t L = f->L;
    for (size_t b = 0; b < half; b++) {
        uint64_t a[4], t[4];
        memcpy(a, m + (2 * b + 1) * L, 8 * L);
        fsub(f, a, m + (2 * b) * L);
        fmul(f, r, a, t);
        uint64_t s[4];
        memcpy(s, m + (2 * b) * L, 8 * L);
        fadd(f, s, t);
        memcpy(m + b * L, s, 8 * L);
    }
}

static void tr_field_challenge(zr_transcript *t, const fcfg *f, uint64_t *out) {
    /* get_field_challenge: XOF of 8L bytes as Uint<L>, F::new_with_cfg (a
     * value converted to Montgomery form), then absorbed as a field element */
    uint8_t b[32];
    zr_tr_challenge(t, b, 8 * f->L);
    uint64_t x[4] = {0};
    memcpy(x, b, 8 * f->L);
    /* value mod p in Montgomery form: montmul(x, R^2) */
    fmul(f, x, f->r2, out);
}

int zr_sumcheck_prove(zr_transcript *t, const uint64_t *modulus, uint32_t L, uint32_t nvars,
                      int multi, const zr_sc_group *groups, uint32_t ngroups, uint8_t *proof,
                      size_t cap, size_t *plen, uint64_t *point_out, uint64_t *finals_out) {
    if (nvars == 0 || ngroups == 0 || (!multi && ngroups != 1) || L < 1 || L > 4) return -1;
    fcfg f;
    fcfg_init(&f, modulus, L);
    uint64_t fe[4];
    f_from_u64(&f, nvars, fe);
    tr_absorb_field(t, &f, fe);
    f_from_u64(&f, multi ? ngroups : groups[0].degree, fe);
    tr_absorb_field(t, &f, fe);
    if (multi)
        for (uint32_t g = 0; g < ngroups; g++) {
            f_from_u64(&f, groups[g].degree, fe);
            tr_absorb_field(t, &f, fe);
        }
    size_t n = (size_t)1 << nvars;
    /* working copies */
    uint64_t ***m = (uint64_t ***)calloc(ngroups, sizeof(uint64_t **));
    for (uint32_t g = 0; g < ngroups; g++) {
        m[g] = (uint64_t **)calloc(groups[g].n_mles, sizeof(uint64_t *));
        for (uint32_t j = 0; j < groups[g].n_mles; j++) {
            m[g][j] = (uint64_t *)malloc(8 * L * n);
            memcpy(m[g][j], groups[g].mles + (size_t)j * n * L, 8 * L * n);
        }
    }
    uint32_t maxd = 0;
    for (uint32_t g = 0; g < ngroups; g++) maxd = groups[g].degree > maxd ? groups[g].degree : maxd;
    uint64_t *msgs = (uint64_t *)calloc((size_t)ngroups * nvars * (maxd + 1), 8 * L);
    uint64_t *claimed = (uint64_t *)calloc(ngroups, 8 * L);
    uint64_t *ev = (uint64_t *)calloc(maxd + 1, 8 * L);
    uint64_t r[4] = {0};
    size_t len = n;
    for (uint32_t rd = 0; rd < nvars; rd++) {
        if (rd > 0) {
            for (uint32_t g = 0; g < ngroups; g++)
                for (uint32_t j = 0; j < groups[g].n_mles; j++) sc_fold(&f, m[g][j], len / 2, r);
            len /= 2;
        }
        for (uint32_t g = 0; g < ngroups; g++) {
            sc_round_evals(&f, &groups[g], m[g], len / 2, ev);
            uint32_t D = groups[g].degree;
            if (rd == 0) {
                memcpy(claimed + (size_t)g * L, ev, 8 * L);
                if (D > 0) fadd(&f, claimed + (size_t)g * L, ev + L);
            }
            memcpy(msgs + ((size_t)g * nvars + rd) * (maxd + 1) * L, ev + L, 8 * L * (size_t)D);
            if (!multi)
                for (uint32_t e = 1; e <= D; e++) tr_absorb_field(t, &f, ev + (size_t)e * L);
        }
        if (multi)
            for (uint32_t g = 0; g < ngroups; g++)
                for (uint32_t e = 0; e < groups[g].degree; e++)
                    tr_absorb_field(t, &f, msgs + (((size_t)g * nvars + rd) * (maxd + 1) + e) * L);
        tr_field_challenge(t, &f, r);
        tr_absorb_field(t, &f, r);
        memcpy(point_out + (size_t)rd * L, r, 8 * L);
    }
    /* final evaluations of every MLE at the point (one more fold) */
    size_t fo = 0;
    for (uint32_t g = 0; g < ngroups; g++)
        for (uint32_t j = 0; j < groups[g].n_mles; j++) {
            sc_fold(&f, m[g][j], 1, r);
            memcpy(finals_out + fo * L, m[g][j], 8 * L);
            fo++;
        }
    /* transcription */
    wbuf w = {proof, 0, cap, 0};
    wput(&w, f.p, 8 * L);
    if (!multi) {
        uint32_t nm = nvars;
        wput(&w, &nm, 4);
        for (uint32_t rd = 0; rd < nvars; rd++) {
            uint32_t D = groups[0].degree;
            wput(&w, &D, 4);
            wput(&w, msgs + (size_t)rd * (maxd + 1) * L, 8 * L * (size_t)D);
        }
        wput(&w, claimed, 8 * L);
    } else {
        uint32_t ng = ngroups, nv = nvars;
        wput(&w, &ng, 4);
        wput(&w, &nv, 4);
        for (uint32_t g = 0; g < ngroups; g++) wput(&w, &groups[g].degree, 4);
        for (uint32_t g = 0; g < ngroups; g++)
            for (uint32_t rd = 0; rd < nvars; rd++)
                wput(&w, msgs + ((size_t)g * nvars + rd) * (maxd + 1) * L, 8 * L * (size_t)groups[g].degree);
        wput(&w, claimed, 8 * L * (size_t)ngroups);
    }
    *plen = w.len;
    for (uint32_t g = 0; g < ngroups; g++) {
        for (uint32_t j = 0; j < groups[g].n_mles; j++) free(m[g][j]);
        free(m[g]);
    }
    free(m);
    free(msgs);
    free(claimed);
    free(ev);
    return w.overflow ? -3 : 0;
}

/* Lagrange evaluation at x of the polynomial with values y[0..n) at 0..n-1
 * (NatEvaluatedPoly::evaluate_at_point, poly/src/univariate/nat_evaluation.rs) */
static void nat_eval(const fcfg *f, const uint64_t *y, uint32_t n, const uint64_t *x, uint64_t *out) {
    uint32_t L = f->L;
    uint64_t acc[4] = {0};
    for (uint32_t i = 0; i < n; i++) {
        uint64_t num[4], den[4];
        memcpy(num, f->one, 8 * L);
        memcpy(den, f->one, 8 * L);
        for (uint32_t j = 0; j < n; j++) {
            if (j == i) continue;
            uint64_t xj[4], t[4], dj[4];
            f_from_u64(f, j, xj);
            memcpy(t, x, 8 * L);
            fsub(f, t, xj);
            uint64_t u[4];
            fmul(f, num, t, u);
            memcpy(num, u, 8 * L);
            uint64_t xi[4];
            f_from_u64(f, i, xi);
            memcpy(dj, xi, 8 * L);
            fsub(f, dj, xj);
            fmul(f, den, dj, u);
            memcpy(den, u, 8 * L);
        }
        /* den^-1 by Fermat: den^(p-2) */
        uint64_t e[4], inv[4];
        memcpy(e, f->p, 8 * L);
        uint64_t two[4] = {2, 0, 0, 0};
        usub(e, two, L);
        memcpy(inv, f->one, 8 * L);
        for (int b = 64 * (int)L - 1; b >= 0; b--) {
            uint64_t u[4];
            fmul(f, inv, inv, u);
            memcpy(inv, u, 8 * L);
            if ((e[b / 64] >> (b % 64)) & 1) {
                fmul(f, inv, den, u);
                memcpy(inv, u, 8 * L);
            }
        }
        uint64_t t1[4], t2[4];
        fmul(f, y + (size_t)i * L, num, t1);
        fmul(f, t1, inv, t2);
        fadd(f, acc, t2);
    }
    memcpy(out, acc, 8 * L);
}

/* verify_as_subprotocol + check_and_generate_subclaim: returns 0 and the
 * subclaim (point, expected evaluation per group) if the transcription is
 * well formed; the caller compares expected with comb(finals). */
int zr_sumcheck_verify(zr_transcript *t, const uint64_t *modulus, uint32_t L, uint32_t nvars,
                       int multi, const uint32_t *degrees, uint32_t ngroups, const uint8_t *proof,
                       size_t len, uint64_t *point_out, uint64_t *expected_out) {
    fcfg f;
    fcfg_init(&f, modulus, L);
    rbuf rd = {proof, len, 0};
    uint64_t mod[4] = {0};
    if (rget(&rd, mod, 8 * L) || memcmp(mod, f.p, 8 * L)) return 3;
    uint64_t fe[4];
    f_from_u64(&f, nvars, fe);
    tr_absorb_field(t, &f, fe);
    f_from_u64(&f, multi ? ngroups : degrees[0], fe);
    tr_absorb_field(t, &f, fe);
    if (multi)
        for (uint32_t g = 0; g < ngroups; g++) {
            f_from_u64(&f, degrees[g], fe);
            tr_absorb_field(t, &f, fe);
        }
    uint32_t maxd = 0;
    for (uint32_t g = 0; g < ngroups; g++) maxd = degrees[g] > maxd ? degrees[g] : maxd;
    uint64_t *msgs = (uint64_t *)calloc((size_t)ngroups * nvars * (maxd + 1), 8 * L);
    uint64_t *claimed = (uint64_t *)calloc(ngroups, 8 * L);
    int rc = 0;
    if (!multi) {
        uint32_t nm;
        if (rget(&rd, &nm, 4) || nm != nvars) { rc = 3; goto done; }
        for (uint32_t r = 0; r < nvars; r++) {
            uint32_t D;
            if (rget(&rd, &D, 4) || D != degrees[0]) { rc = 3; goto done; }
            if (rget(&rd, msgs + (size_t)r * (maxd + 1) * L, 8 * L * (size_t)D)) { rc = 3; goto done; }
        }
        if (rget(&rd, claimed, 8 * L)) { rc = 3; goto done; }
    } else {
        uint32_t ng, nv;
        if (rget(&rd, &ng, 4) || rget(&rd, &nv, 4) || ng != ngroups || nv != nvars) { rc = 3; goto done; }
        for (uint32_t g = 0; g < ngroups; g++) {
            uint32_t D;
            if (rget(&rd, &D, 4) || D != degrees[g]) { rc = 3; goto done; }
        }
        for (uint32_t g = 0; g < ngroups; g++)
            for (uint32_t r = 0; r < nvars; r++)
                if (rget(&rd, msgs + ((size_t)g * nvars + r) * (maxd + 1) * L, 8 * L * (size_t)degrees[g])) { rc = 3; goto done; }
        if (rget(&rd, claimed, 8 * L * (size_t)ngroups)) { rc = 3; goto done; }
    }
    {
        uint64_t r[4];
        for (uint32_t k = 0; k < nvars; k++) {
            for (uint32_t g = 0; g < ngroups; g++)
                for (uint32_t e = 0; e < degrees[g]; e++)
                    tr_absorb_field(t, &f, msgs + (((size_t)g * nvars + k) * (maxd + 1) + e) * L);
            tr_field_challenge(t, &f, r);
            tr_absorb_field(t, &f, r);
            memcpy(point_out + (size_t)k * L, r, 8 * L);
        }
        for (uint32_t g = 0; g < ngroups; g++) {
            uint64_t expected[4];
            memcpy(expected, claimed + (size_t)g * L, 8 * L);
            uint32_t D = degrees[g];
            uint64_t *y = (uint64_t *)calloc((size_t)D + 1, 8 * L);
            for (uint32_t k = 0; k < nvars; k++) {
                const uint64_t *tail = msgs + ((size_t)g * nvars + k) * (maxd + 1) * L;
                if (D == 0) continue; /* constant polynomial: expected unchanged */
                memcpy(y, expected, 8 * L);
                fsub(&f, y, tail);
                memcpy(y + L, tail, 8 * L * (size_t)D);
                nat_eval(&f, y, D + 1, point_out + (size_t)k * L, expected);
            }
            free(y);
            memcpy(expected_out + (size_t)g * L, expected, 8 * L);
        }
    }
done:
    free(msgs);
    free(claimed);
    return rc;
}

void zr_sumcheck_comb(const uint64_t *modulus, uint32_t L, const zr_sc_group *g,
                      const uint64_t *vals, uint64_t *out) {
    fcfg f;
    fcfg_init(&f, modulus, L);
    sc_comb(&f, g, vals, out);
}

/* MLE evaluation sum_x mle[x] * eq(x, point) (mle_eval_with_eq_table,
 * poly/src/utils.rs:267-284); point in Montgomery form, bit 0 = point[0]. */
void zr_mle_evaluate(const uint64_t *modulus, uint32_t L, const uint64_t *mle, uint32_t nvars,
                     const uint64_t *point, uint64_t *out) {
    fcfg f;
    fcfg_init(&f, modulus, L);
    size_t n = (size_t)1 << nvars;
    uint64_t *eq = (uint64_t *)malloc(8 * L * n);
    build_eq(&f, point, nvars, eq);
    uint64_t acc[4] = {0};
    for (size_t x = 0; x < n; x++) {
        uint64_t t[4];
        fmul(&f, mle + x * L, eq + x * L, t);
        fadd(&f, acc, t);
    }
    memcpy(out, acc, 8 * L);
    free(eq);
}

/* ========================================================================
 * Zinc+ prover steps 3 and 6 on the trace columns
 * (protocol/src/prover.rs:385-415 and 497-532).
 * ====================================================================== */

/* F::from_with_cfg of a signed 64-bit trace integer (Montgomery inner). */
static void f_from_i64(const fcfg *f, int64_t v, uint64_t *out) {
    uint64_t x[2] = {(uint64_t)v, v < 0 ? ~0ull : 0ull};
    f_from_int(f, x, 2, out);
}

/* Step 3, evaluation projection: project_trace_coeffs (piop/src/projections.rs:
 * 140-220: a binary coefficient becomes one or zero, an integer F::from_with_cfg)
 * followed by evaluate_trace_to_column_mles (projections.rs:227-301: each
 * polynomial's inner product with the powers of a).  bin: n_bin columns of 2^nvars
 * BinaryPoly<D> (bit l = coefficient l); ints: n_int columns of 2^nvars i64.
 * out: (n_bin + n_int) MLEs of 2^nvars Montgomery inners, column after column. */
void zr_piop_eval_projection(const uint64_t *modulus, uint32_t L, const uint64_t *bin, uint32_t n_bin,
                             uint32_t D, const int64_t *ints, uint32_t n_int, uint32_t nvars,
                             const uint64_t *a, uint64_t *out) {
    fcfg f;
    fcfg_init(&f, modulus, L);
    const size_t n = (size_t)1 << nvars;
    uint64_t pw[64][4];
    memcpy(pw[0], f.one, 8 * L);
    for (uint32_t l = 1; l < D; l++) fmul(&f, pw[l - 1], a, pw[l]);
    for (uint32_t c = 0; c < n_bin; c++)
        for (size_t b = 0; b < n; b++) {
            const uint64_t x = bin[c * n + b];
            uint64_t acc[4] = {0};
            for (uint32_t l = 0; l < D; l++)
                if ((x >> l) & 1) fadd(&f, acc, pw[l]);
            memcpy(out + (c * n + b) * L, acc, 8 * L);
        }
    for (uint32_t c = 0; c < n_int; c++)
        for (size_t b = 0; b < n; b++) f_from_i64(&f, ints[c * n + b], out + ((n_bin + c) * n + b) * L);
}

/* Step 6, lifted evaluations: compute_lifted_evals (protocol/src/lib.rs:327-395).
 * For a binary column, coefficient l is sum_b eq(b, point) [bit l of col[b]];
 * for an integer column the single coefficient is sum_b eq(b, point) F(col[b]).
 * out: n_bin x D then n_int x 1 Montgomery inners (untrimmed: the reference's
 * DynamicPolynomialF::new_trimmed drops trailing zero coefficients). */
void zr_piop_lifted_evals(const uint64_t *modulus, uint32_t L, const uint64_t *bin, uint32_t n_bin,
                          uint32_t D, const int64_t *ints, uint32_t n_int, uint32_t nvars,
                          const uint64_t *point, uint64_t *out) {
    fcfg f;
    fcfg_init(&f, modulus, L);
    const size_t n = (size_t)1 << nvars;
    uint64_t *eq = (uint64_t *)malloc(8 * L * n);
    build_eq(&f, point, nvars, eq);
    for (uint32_t c = 0; c < n_bin; c++)
        for (uint32_t l = 0; l < D; l++) {
            uint64_t acc[4] = {0};
            for (size_t b = 0; b < n; b++)
                if ((bin[c * n + b] >> l) & 1) fadd(&f, acc, eq + b * L);
            memcpy(out + ((size_t)c * D + l) * L, acc, 8 * L);
        }
    for (uint32_t c = 0; c < n_int; c++) {
        uint64_t acc[4] = {0};
        for (size_t b = 0; b < n; b++) {
            uint64_t v[4], t[4];
            f_from_i64(&f, ints[c * n + b], v);
            fmul(&f, v, eq + b * L, t);
            fadd(&f, acc, t);
        }
        memcpy(out + ((size_t)n_bin * D + c) * L, acc, 8 * L);
    }
    free(eq);
}

/* get_field_challenge (transcript/src/traits.rs:333-340) for modulus `modulus`. */
void zr_tr_field_challenge(zr_transcript *t, const uint64_t *modulus, uint32_t L, uint64_t *out) {
    fcfg f;
    fcfg_init(&f, modulus, L);
    tr_field_challenge(t, &f, out);
}

/* absorb_random_field (transcript/src/traits.rs:393-413) for modulus `modulus`. */
void zr_tr_absorb_field(zr_transcript *t, const uint64_t *modulus, uint32_t L, const uint64_t *inner) {
    fcfg f;
    fcfg_init(&f, modulus, L);
    tr_absorb_field(t, &f, inner);
}

/* commit + prove_f: as zr_commit_prove with the point given as unsigned 256-bit
 * integers, F::from of each once the field is drawn. */
int zr_commit_prove_f(const zr_desc *d, const void *polys, uint32_t batch, const uint64_t *point_u256,
                      uint8_t root[32], uint8_t *proof, size_t proof_cap, size_t *proof_len, uint8_t *eval_out,
                      uint8_t *modulus_out) {
    int64_t dummy[2 * 32] = {0};
    g_point_u256 = point_u256;
    int rc = zr_commit_prove(d, polys, batch, dummy, root, proof, proof_cap, proof_len, eval_out, modulus_out);
    g_point_u256 = NULL;
    return rc;
}

/* LinearCode::encode_f (zip-plus/src/code.rs:69-71): a row of field elements
 * (Montgomery inners of the prime `modulus`, L limbs) encoded over the field.
 * IPRS (iprs.rs:88-106 encode_inner_f): the radix-8 pNTT with every base-matrix
 * entry and twiddle taken as F::from_with_cfg of its i64 value.  RAA and
 * sign-flipping RAA (raa.rs:93-127, raa_sign_flip.rs:31-69, encode_f calling
 * encode_inner): repeat, (negate odd entries,) permute, prefix sums, (negate,)
 * permute, prefix sums, all in the field. */
int zr_encode_f(const zr_desc *d, const uint64_t *modulus, uint32_t L, const uint64_t *row, uint64_t *out) {
    zparams z;
    if (L < 1 || L > 4 || zparams_build(d, &z)) return -1;
    fcfg f;
    fcfg_init(&f, modulus, L);
    if (d->code_kind == ZR_CODE_IPRS) {
        const iprs_params *p = &z.iprs;
        const uint32_t sh = 3 * p->depth;
        for (size_t i = 0; i < p->codeword_len; i++) {
            size_t chunk = i >> p->base_dim_log2, rw = i & (p->base_dim - 1);
            size_t oct = zr_octet_reversal(chunk, p->depth);
            const int64_t *bm = p->bm + rw * p->base_len;
            uint64_t acc[4];
            memcpy(acc, row + oct * L, 8 * L);
            for (size_t c = 1; c < p->base_len; c++) {
                uint64_t tw[4], t[4];
                f_from_i64(&f, bm[c], tw);
                fmul(&f, row + (oct | (c << sh)) * L, tw, t);
                fadd(&f, acc, t);
            }
            memcpy(out + i * L, acc, 8 * L);
        }
        uint64_t xs[8][4];
        for (uint32_t k = 0; k < p->depth; k++) {
            size_t sub = (size_t)p->base_dim << (3 * k);
            const int64_t *tw = p->tw[k];
            for (size_t blk = 0; blk < p->codeword_len; blk += 8 * sub)
                for (size_t i = 0; i < sub; i++) {
                    for (int j = 0; j < 8; j++) memcpy(xs[j], out + (blk + j * sub + i) * L, 8 * L);
                    for (int r = 0; r < 8; r++) {
                        uint64_t y[4];
                        memcpy(y, xs[0], 8 * L);
                        for (int j = 1; j < 8; j++) {
                            uint64_t fw[4], t[4];
                            f_from_i64(&f, tw[(i * 7 + (j - 1)) * 8 + BUTTERFLY_TABLE[r][j - 1]], fw);
                            fmul(&f, xs[j], fw, t);
                            fadd(&f, y, t);
                        }
                        memcpy(out + (blk + r * sub + i) * L, y, 8 * L);
                    }
                }
        }
    } else {
        const raa_params *r = &z.raa;
        const size_t n = r->codeword_len;
        uint64_t *a = (uint64_t *)malloc(8 * L * n);
        for (size_t i = 0; i < n; i++) memcpy(a + i * L, row + (i % r->row_len) * L, 8 * L);
        for (int pass = 0; pass < 2; pass++) {
            if (r->flip)
                for (size_t i = 1; i < n; i += 2) fneg(&f, a + i * L);
            const uint32_t *perm = pass == 0 ? r->perm1 : r->perm2;
            for (size_t i = 0; i < n; i++) memcpy(out + i * L, a + (size_t)perm[i] * L, 8 * L);
            for (size_t i = 1; i < n; i++) fadd(&f, out + i * L, out + (i - 1) * L);
            if (pass == 0) memcpy(a, out, 8 * L * n);
        }
        free(a);
    }
    zparams_free(&z);
    return 0;
}

/* The Zinc+ PIOP prover chain and verifier (oracle). */
#include "zinc_piop.c"
