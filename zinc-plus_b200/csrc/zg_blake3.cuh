// BLAKE3 for host and device (public BLAKE3 specification).  The reference
// hashes Merkle leaves with blake3::Hasher and merges nodes with
// blake3::hazmat::merge_subtrees_{non_root,root} (zip-plus/src/merkle.rs:148-221);
// its Fiat-Shamir transcript is a blake3::Hasher with XOF output
// (transcript/src/lib.rs:12-77).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>

#ifndef ZG_HD
#ifdef __CUDACC__
#define ZG_HD __host__ __device__ __forceinline__
#else
#define ZG_HD inline
#endif
#endif

// Host and device, not forced inline (the incremental hasher's update and XOF).
#ifndef ZG_HDN
#ifdef __CUDACC__
#define ZG_HDN __host__ __device__
#else
#define ZG_HDN inline
#endif
#endif

namespace zg {
namespace b3 {

enum : uint32_t { CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8 };
constexpr uint32_t CHUNK_LEN = 1024;

ZG_HD uint32_t iv(int i) {
    // The BLAKE3 IV (the SHA-256 initial hash values).
    const uint32_t v[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                           0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
    return v[i];
}

ZG_HD uint32_t rotr(uint32_t x, int n) {
#ifdef __CUDA_ARCH__
    return __funnelshift_r(x, x, n);
#else
    return (x >> n) | (x << (32 - n));
#endif
}

#define ZG_B3_G(a, b, c, d, x, y)                                                                 \
    do {                                                                                          \
        v##a = v##a + v##b + (x);                                                                 \
        v##d = rotr(v##d ^ v##a, 16);                                                             \
        v##c = v##c + v##d;                                                                       \
        v##b = rotr(v##b ^ v##c, 12);                                                             \
        v##a = v##a + v##b + (y);                                                                 \
        v##d = rotr(v##d ^ v##a, 8);                                                              \
        v##c = v##c + v##d;                                                                       \
        v##b = rotr(v##b ^ v##c, 7);                                                              \
    } while (0)

// One round on message words m0..m15; the message permutation between rounds
// is applied by renaming the arguments of the next call.
#define ZG_B3_ROUND(m0, m1, m2, m3, m4, m5, m6, m7, m8, m9, m10, m11, m12, m13, m14, m15)         \
    ZG_B3_G(0, 4, 8, 12, m0, m1);                                                                  \
    ZG_B3_G(1, 5, 9, 13, m2, m3);                                                                  \
    ZG_B3_G(2, 6, 10, 14, m4, m5);                                                                 \
    ZG_B3_G(3, 7, 11, 15, m6, m7);                                                                 \
    ZG_B3_G(0, 5, 10, 15, m8, m9);                                                                 \
    ZG_B3_G(1, 6, 11, 12, m10, m11);                                                               \
    ZG_B3_G(2, 7, 8, 13, m12, m13);                                                                \
    ZG_B3_G(3, 4, 9, 14, m14, m15)

// Full compression: out[0..16] (out[0..8] is the chaining value).
ZG_HD void compress(const uint32_t cv[8], const uint32_t m[16], uint64_t counter,
                    uint32_t block_len, uint32_t flags, uint32_t out[16]) {
    uint32_t v0 = cv[0], v1 = cv[1], v2 = cv[2], v3 = cv[3], v4 = cv[4], v5 = cv[5], v6 = cv[6],
             v7 = cv[7];
    uint32_t v8 = iv(0), v9 = iv(1), v10 = iv(2), v11 = iv(3);
    uint32_t v12 = (uint32_t)counter, v13 = (uint32_t)(counter >> 32), v14 = block_len, v15 = flags;
    const uint32_t m0 = m[0], m1 = m[1], m2 = m[2], m3 = m[3], m4 = m[4], m5 = m[5], m6 = m[6],
                   m7 = m[7], m8 = m[8], m9 = m[9], m10 = m[10], m11 = m[11], m12 = m[12],
                   m13 = m[13], m14 = m[14], m15 = m[15];
    // Message schedule: round r uses sigma^r applied to the words, where
    // sigma = [2,6,3,10,7,0,4,13,1,11,12,5,9,14,15,8].
    ZG_B3_ROUND(m0, m1, m2, m3, m4, m5, m6, m7, m8, m9, m10, m11, m12, m13, m14, m15);
    ZG_B3_ROUND(m2, m6, m3, m10, m7, m0, m4, m13, m1, m11, m12, m5, m9, m14, m15, m8);
    ZG_B3_ROUND(m3, m4, m10, m12, m13, m2, m7, m14, m6, m5, m9, m0, m11, m15, m8, m1);
    ZG_B3_ROUND(m10, m7, m12, m9, m14, m3, m13, m15, m4, m0, m11, m2, m5, m8, m1, m6);
    ZG_B3_ROUND(m12, m13, m9, m11, m15, m10, m14, m8, m7, m2, m5, m3, m0, m1, m6, m4);
    ZG_B3_ROUND(m9, m14, m11, m5, m8, m12, m15, m1, m13, m3, m0, m10, m2, m6, m4, m7);
    ZG_B3_ROUND(m11, m15, m5, m0, m1, m9, m8, m6, m14, m10, m2, m12, m3, m4, m7, m13);
    out[0] = v0 ^ v8;
    out[1] = v1 ^ v9;
    out[2] = v2 ^ v10;
    out[3] = v3 ^ v11;
    out[4] = v4 ^ v12;
    out[5] = v5 ^ v13;
    out[6] = v6 ^ v14;
    out[7] = v7 ^ v15;
    out[8] = v8 ^ cv[0];
    out[9] = v9 ^ cv[1];
    out[10] = v10 ^ cv[2];
    out[11] = v11 ^ cv[3];
    out[12] = v12 ^ cv[4];
    out[13] = v13 ^ cv[5];
    out[14] = v14 ^ cv[6];
    out[15] = v15 ^ cv[7];
}

// Chaining-value-only compression, in place on cv.
ZG_HD void compress_cv(uint32_t cv[8], const uint32_t m[16], uint64_t counter, uint32_t block_len,
                       uint32_t flags) {
    uint32_t out[16];
    compress(cv, m, counter, block_len, flags, out);
    for (int i = 0; i < 8; i++) cv[i] = out[i];
}

#ifdef __CUDA_ARCH__
// The compression out of line: one copy of its unrolled code for every call
// of the incremental hasher (the transcript, one thread), instead of one per
// call site.  The leaf and tree kernels inline it.
static __device__ __noinline__ void compress_ool(const uint32_t cv[8], const uint32_t m[16],
                                                 uint64_t counter, uint32_t block_len,
                                                 uint32_t flags, uint32_t out[16]) {
    compress(cv, m, counter, block_len, flags, out);
}
#endif

// The compression used by the incremental hasher: out of line on the device.
ZG_HD void compress_h(const uint32_t cv[8], const uint32_t m[16], uint64_t counter,
                      uint32_t block_len, uint32_t flags, uint32_t out[16]) {
#ifdef __CUDA_ARCH__
    compress_ool(cv, m, counter, block_len, flags, out);
#else
    compress(cv, m, counter, block_len, flags, out);
#endif
}

ZG_HD void compress_cv_h(uint32_t cv[8], const uint32_t m[16], uint64_t counter,
                         uint32_t block_len, uint32_t flags) {
    uint32_t out[16];
    compress_h(cv, m, counter, block_len, flags, out);
    for (int i = 0; i < 8; i++) cv[i] = out[i];
}

ZG_HD uint32_t load_le32(const uint8_t *p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
ZG_HD void store_le32(uint8_t *p, uint32_t v) {
    p[0] = (uint8_t)v;
    p[1] = (uint8_t)(v >> 8);
    p[2] = (uint8_t)(v >> 16);
    p[3] = (uint8_t)(v >> 24);
}

// Parent node (blake3::hazmat::merge_subtrees_*(l, r, Mode::Hash)): with
// root=true the first 32 root-output bytes, else the chaining value.
ZG_HD void parent_cv(const uint32_t l[8], const uint32_t r[8], bool root, uint32_t out[8]) {
    uint32_t m[16], cv[8];
    for (int i = 0; i < 8; i++) {
        m[i] = l[i];
        m[8 + i] = r[i];
        cv[i] = iv(i);
    }
    compress_cv(cv, m, 0, 64, PARENT | (root ? ROOT : 0));
    for (int i = 0; i < 8; i++) out[i] = cv[i];
}

// Chaining value (or, with root=true, the 32-byte hash) of one chunk of
// n <= 1024 bytes at position `counter`, read through a word loader
// `load(block, word)` returning little-endian words (zero past n).
template <class Loader>
ZG_HD void chunk_hash(const Loader &load, uint32_t n, uint64_t counter, bool root, uint32_t out[8]) {
    uint32_t cv[8];
    for (int i = 0; i < 8; i++) cv[i] = iv(i);
    uint32_t nblocks = n == 0 ? 1 : (n + 63) / 64;
    for (uint32_t b = 0; b < nblocks; b++) {
        uint32_t m[16];
        for (int w = 0; w < 16; w++) m[w] = load(b, w);
        uint32_t blen = (b + 1 < nblocks) ? 64u : n - 64u * b;
        uint32_t flags = (b == 0 ? CHUNK_START : 0) | (b + 1 == nblocks ? CHUNK_END : 0);
        if (root && b + 1 == nblocks) flags |= ROOT;
        compress_cv(cv, m, counter, blen, flags);
    }
    for (int i = 0; i < 8; i++) out[i] = cv[i];
}

// Non-root parent chaining value through the hasher's compression.
ZG_HD void parent_h(const uint32_t l[8], const uint32_t r[8], uint32_t out[8]) {
    uint32_t m[16], cv[8];
    for (int i = 0; i < 8; i++) {
        m[i] = l[i];
        m[8 + i] = r[i];
        cv[i] = iv(i);
    }
    compress_cv_h(cv, m, 0, 64, PARENT);
    for (int i = 0; i < 8; i++) out[i] = cv[i];
}

// Incremental hasher with XOF finalisation (host; used by the transcript).
struct Hasher {
    uint32_t cv[8];
    uint64_t chunk_counter = 0;
    uint8_t block[64];
    uint32_t block_len = 0;
    uint32_t blocks_compressed = 0;
    uint32_t stack[54][8];
    uint32_t stack_len = 0;

    ZG_HDN Hasher() { reset(); }
    ZG_HDN void reset() {
        for (int i = 0; i < 8; i++) cv[i] = iv(i);
        chunk_counter = 0;
        clear_block();
        block_len = 0;
        blocks_compressed = 0;
        stack_len = 0;
    }
    ZG_HDN uint32_t chunk_len() const { return 64 * blocks_compressed + block_len; }
    ZG_HDN uint32_t start_flag() const { return blocks_compressed == 0 ? CHUNK_START : 0; }
    // The block as words / cleared.  On the device, 32-bit accesses (the block
    // sits at a multiple of 8 bytes in the struct); bytes on the host.
    ZG_HDN void clear_block() {
#ifdef __CUDA_ARCH__
        uint32_t *w = reinterpret_cast<uint32_t *>(block);
        for (int i = 0; i < 16; i++) w[i] = 0;
#else
        for (int i = 0; i < 64; i++) block[i] = 0;
#endif
    }
    ZG_HDN void block_words(uint32_t m[16]) const {
#ifdef __CUDA_ARCH__
        const uint32_t *w = reinterpret_cast<const uint32_t *>(block);
        for (int i = 0; i < 16; i++) m[i] = w[i];
#else
        for (int i = 0; i < 16; i++) m[i] = load_le32(block + 4 * i);
#endif
    }
    ZG_HDN void finish_chunk_and_push() {
        uint32_t m[16];
        block_words(m);
        uint32_t c[8];
        for (int i = 0; i < 8; i++) c[i] = cv[i];
        compress_cv_h(c, m, chunk_counter, block_len, start_flag() | CHUNK_END);
        uint64_t total = chunk_counter + 1;
        while ((total & 1) == 0) {
            parent_h(stack[--stack_len], c, c);
            total >>= 1;
        }
        for (int i = 0; i < 8; i++) stack[stack_len][i] = c[i];
        stack_len++;
        chunk_counter++;
        for (int i = 0; i < 8; i++) cv[i] = iv(i);
        clear_block();
        block_len = 0;
        blocks_compressed = 0;
    }
    ZG_HDN void update(const uint8_t *in, size_t n) {
        while (n) {
            if (chunk_len() == CHUNK_LEN) finish_chunk_and_push();
            if (block_len == 64) {
                uint32_t m[16];
                block_words(m);
                compress_cv_h(cv, m, chunk_counter, 64, start_flag());
                blocks_compressed++;
                block_len = 0;
                clear_block();
            }
            // (the chunk has room for the rest of the block: at most 15 blocks
            // are compressed before its last one)
            const uint32_t bl = block_len;
            const uint32_t take = n < 64 - bl ? (uint32_t)n : 64 - bl;
            // Local restrict pointers: through `this`, every byte store could
            // alias block_len and force a reload per byte.
            uint8_t *__restrict__ dst = block + bl;
            const uint8_t *__restrict__ src = in;
#ifdef __CUDA_ARCH__
#pragma unroll 8
#endif
            for (uint32_t i = 0; i < take; i++) dst[i] = src[i];
            block_len = bl + take;
            in += take;
            n -= take;
        }
    }
    // finalize_xof().fill(out): does not change the hasher state.
    ZG_HDN void xof(uint8_t *out, size_t n) const {
        uint32_t ocv[8], m[16];
        uint32_t blen = block_len, flags = start_flag() | CHUNK_END;
        uint64_t counter = chunk_counter;
        for (int i = 0; i < 8; i++) ocv[i] = cv[i];
        block_words(m);
        for (int s = (int)stack_len - 1; s >= 0; s--) {
            uint32_t c[8];
            for (int i = 0; i < 8; i++) c[i] = ocv[i];
            compress_cv_h(c, m, counter, blen, flags);
            for (int i = 0; i < 8; i++) {
                m[i] = stack[s][i];
                m[8 + i] = c[i];
                ocv[i] = iv(i);
            }
            counter = 0;
            blen = 64;
            flags = PARENT;
        }
        uint64_t ob = 0;
        while (n) {
            uint32_t w[16];
            compress_h(ocv, m, ob++, blen, flags | ROOT, w);
            uint8_t bytes[64];
            for (int i = 0; i < 16; i++) store_le32(bytes + 4 * i, w[i]);
            size_t take = n < 64 ? n : 64;
            for (size_t i = 0; i < take; i++) out[i] = bytes[i];
            out += take;
            n -= take;
        }
    }
};

static_assert(offsetof(Hasher, block) % 4 == 0, "the block is read and cleared as words on the device");

// One-shot hash of a host buffer.
inline void hash(const uint8_t *in, size_t n, uint8_t out[32]) {
    Hasher h;
    h.update(in, n);
    h.xof(out, 32);
}

}  // namespace b3
}  // namespace zg
