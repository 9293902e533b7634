// Merkle commitment kernels (zip-plus/src/merkle.rs:74-221).
//
// Leaf j is BLAKE3 of the column's bytes over all rows (hash_leaves,
// merkle.rs:148-168).  The codeword is stored leaf-major, so each leaf's
// preimage is one contiguous range.  Interior nodes are BLAKE3 parent
// compressions (hazmat::merge_subtrees_non_root), the top one with the ROOT
// flag (merge_subtrees_root).
#include "zg_internal.h"

namespace zg {

namespace {

struct GlobalWords {
    const uint32_t *base;  // 4-byte aligned
    uint32_t n;            // bytes, multiple of 4
    __device__ __forceinline__ uint32_t operator()(uint32_t block, int w) const {
        const uint32_t off = 64u * block + 4u * (uint32_t)w;
        return off < n ? __ldg(base + off / 4) : 0u;
    }
};

// Node index of leaf g when the leaves of 2^tree_log-leaf trees are hashed in
// one launch: tree t = g >> tree_log keeps its layers in its own block of
// 2W - 1 nodes (W = 2^tree_log).  tree_log >= 32: one tree, node g.
__device__ __forceinline__ size_t leaf_node(uint32_t g, uint32_t tree_log) {
    if (tree_log >= 32) return g;
    const size_t t = g >> tree_log;
    return t * ((2ull << tree_log) - 1) + (g & ((1u << tree_log) - 1u));
}

}  // namespace

// Leaves of at most one chunk (1024 bytes): one thread per leaf, root output.
__global__ void __launch_bounds__(128) k_leaf_small(const uint8_t *__restrict__ cw, uint32_t width,
                                                    uint32_t leaf_bytes, uint32_t *__restrict__ leaves,
                                                    uint32_t tree_log) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= width) return;
    GlobalWords ld{reinterpret_cast<const uint32_t *>(cw + (size_t)j * leaf_bytes), leaf_bytes};
    uint32_t h[8];
    b3::chunk_hash(ld, leaf_bytes, 0, true, h);
    const size_t node = leaf_node(j, tree_log);
#pragma unroll
    for (int i = 0; i < 8; i++) leaves[node * 8 + i] = h[i];
}

// Leaves of at most one chunk whose size is a multiple of 16 bytes: each warp
// hashes 32 leaves, one per lane.  For every 64-byte block the warp first
// loads the 32 leaves' blocks with 16-byte loads (four lanes per leaf, so each
// instruction reads eight 64-byte runs) into shared memory, then every lane
// compresses its own leaf's block from there.
// With fuse (every block's 128 leaves in one tree of at least 128 leaves), the
// block then reduces its leaves to their subtree's root: tree levels 1..7 from
// shared memory, writing every node, so the level kernel starts at level 7.
__global__ void __launch_bounds__(128) k_leaf_small_coalesced(const uint8_t *__restrict__ cw,
                                                              uint32_t width, uint32_t leaf_bytes,
                                                              uint32_t *__restrict__ leaves,
                                                              uint32_t tree_log, int fuse) {
    __shared__ uint32_t tile[4][32 * 17];  // per warp: 32 leaves x 16 words (+1 pad)
    __shared__ uint32_t sub[128][9];       // the block's subtree level (+1 pad)
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t first = (blockIdx.x * 4 + warp) * 32;
    uint32_t *t = tile[warp];
    uint32_t cv[8];
#pragma unroll
    for (int i = 0; i < 8; i++) cv[i] = b3::iv(i);
    const uint32_t nblocks = leaf_bytes == 0 ? 1 : (leaf_bytes + 63) / 64;
    for (uint32_t blk = 0; blk < nblocks; blk++) {
#pragma unroll
        for (int it = 0; it < 4; it++) {
            const uint32_t l = it * 8 + lane / 4, piece = lane & 3;
            const uint32_t off = 64 * blk + 16 * piece;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (first + l < width && off < leaf_bytes)
                v = __ldg(reinterpret_cast<const uint4 *>(cw + (size_t)(first + l) * leaf_bytes + off));
            uint32_t *d = t + l * 17 + 4 * piece;
            d[0] = v.x;
            d[1] = v.y;
            d[2] = v.z;
            d[3] = v.w;
        }
        __syncwarp();
        uint32_t m[16];
#pragma unroll
        for (int w = 0; w < 16; w++) m[w] = t[lane * 17 + w];
        __syncwarp();
        const uint32_t blen = (blk + 1 < nblocks) ? 64u : leaf_bytes - 64u * blk;
        const uint32_t flags = (blk == 0 ? b3::CHUNK_START : 0u) |
                               (blk + 1 == nblocks ? (b3::CHUNK_END | b3::ROOT) : 0u);
        b3::compress_cv(cv, m, 0, blen, flags);
    }
    if (first + lane < width) {
        const size_t node = leaf_node(first + lane, tree_log);
#pragma unroll
        for (int i = 0; i < 8; i++) leaves[node * 8 + i] = cv[i];
    }
    if (!fuse) return;
    const uint32_t tt = threadIdx.x, g0 = blockIdx.x * 128;
    const uint32_t W = tree_log >= 32 ? width : (1u << tree_log);
    const uint32_t depth = 31 - __clz(W);
    const size_t tree_base = tree_log >= 32 ? 0 : (size_t)(g0 >> tree_log) * (2ull * W - 1);
    const uint32_t local0 = g0 & (W - 1);
#pragma unroll
    for (int i = 0; i < 8; i++) sub[tt][i] = cv[i];
    __syncthreads();
    for (uint32_t k = 1; k <= 7; k++) {
        const uint32_t n = 128u >> k;
        uint32_t l[8], r[8], o[8];
        if (tt < n)
#pragma unroll
            for (int i = 0; i < 8; i++) {
                l[i] = sub[2 * tt][i];
                r[i] = sub[2 * tt + 1][i];
            }
        __syncthreads();
        if (tt < n) {
            b3::parent_cv(l, r, k == depth, o);
            const size_t node = tree_base + (2ull * W - 2ull * (W >> k)) + (local0 >> k) + tt;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                leaves[node * 8 + i] = o[i];
                sub[tt][i] = o[i];
            }
        }
        __syncthreads();
    }
}

// Chunk chaining values of long leaves: one thread per (leaf, chunk).
__global__ void __launch_bounds__(128) k_leaf_chunks(const uint8_t *__restrict__ cw, uint32_t width,
                                                     uint32_t leaf_bytes, uint32_t nchunks,
                                                     uint32_t *__restrict__ cvs) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)width * nchunks) return;
    const uint32_t j = (uint32_t)(t / nchunks), c = (uint32_t)(t % nchunks);
    const uint32_t start = c * b3::CHUNK_LEN;
    const uint32_t len = min(b3::CHUNK_LEN, leaf_bytes - start);
    GlobalWords ld{reinterpret_cast<const uint32_t *>(cw + (size_t)j * leaf_bytes + start), len};
    uint32_t h[8];
    b3::chunk_hash(ld, len, c, false, h);
#pragma unroll
    for (int i = 0; i < 8; i++) cvs[t * 8 + i] = h[i];
}

// Chunk chaining values of long leaves whose size is a multiple of 16 bytes:
// each warp hashes 32 consecutive (leaf, chunk) items, one per lane.  For every
// 64-byte block the warp loads the 32 items' blocks with 16-byte loads (four
// lanes per block, eight 64-byte runs per instruction) into shared memory, then
// each lane compresses its own block from there.
__global__ void __launch_bounds__(128) k_leaf_chunks_coalesced(const uint8_t *__restrict__ cw,
                                                               uint32_t width, uint32_t leaf_bytes,
                                                               uint32_t nchunks,
                                                               uint32_t *__restrict__ cvs) {
    __shared__ uint32_t tile[4][32 * 17];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t total = (size_t)width * nchunks;
    const size_t first = ((size_t)blockIdx.x * 4 + warp) * 32;
    uint32_t *t = tile[warp];
    // this lane's item
    const size_t item = first + lane;
    const uint32_t my_c = (uint32_t)(item % nchunks);
    const uint32_t my_len = item < total ? min(b3::CHUNK_LEN, leaf_bytes - my_c * b3::CHUNK_LEN) : 0u;
    const uint32_t my_blocks = (my_len + 63) / 64;
    uint32_t cv[8];
#pragma unroll
    for (int i = 0; i < 8; i++) cv[i] = b3::iv(i);
    for (uint32_t blk = 0; blk < b3::CHUNK_LEN / 64; blk++) {
#pragma unroll
        for (int it = 0; it < 4; it++) {
            const uint32_t l = it * 8 + lane / 4, piece = lane & 3;
            const size_t li = first + l;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (li < total) {
                const size_t j = li / nchunks;
                const uint32_t c = (uint32_t)(li % nchunks);
                const uint32_t start = c * b3::CHUNK_LEN, off = 64 * blk + 16 * piece;
                if (start + off < leaf_bytes && off < b3::CHUNK_LEN)
                    v = __ldg(reinterpret_cast<const uint4 *>(cw + j * leaf_bytes + start + off));
            }
            uint32_t *d = t + l * 17 + 4 * piece;
            d[0] = v.x;
            d[1] = v.y;
            d[2] = v.z;
            d[3] = v.w;
        }
        __syncwarp();
        uint32_t m[16];
#pragma unroll
        for (int w = 0; w < 16; w++) m[w] = t[lane * 17 + w];
        __syncwarp();
        if (blk < my_blocks) {
            const uint32_t blen = (blk + 1 < my_blocks) ? 64u : my_len - 64u * blk;
            const uint32_t flags = (blk == 0 ? b3::CHUNK_START : 0u) |
                                   (blk + 1 == my_blocks ? b3::CHUNK_END : 0u);
            b3::compress_cv(cv, m, my_c, blen, flags);
        }
    }
    if (item < total) {
#pragma unroll
        for (int i = 0; i < 8; i++) cvs[item * 8 + i] = cv[i];
    }
}

// The same merge for a power-of-two chunk count n <= 32, in parallel: a leaf's
// n chaining values sit in n consecutive lanes (32 / n leaves per warp) and are
// reduced pairwise, log2(n) levels of parents (for such n the hasher's stack
// discipline builds exactly this perfect tree), the last with the root flag.
// One thread per leaf runs n - 1 dependent compressions; here the chain is
// log2(n) deep, at the cost of n / 2 + n / 4 + ... idle lanes per level, which
// pays only while the leaves are too few to fill the GPU.
__global__ void __launch_bounds__(128) k_leaf_merge_pow2(const uint32_t *__restrict__ cvs,
                                                         uint32_t width, uint32_t nchunks,
                                                         uint32_t *__restrict__ leaves,
                                                         uint32_t tree_log) {
    const uint32_t lane = threadIdx.x & 31;
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // (leaf, chunk) item
    const size_t total = (size_t)width * nchunks;
    uint32_t cur[8];
#pragma unroll
    for (int i = 0; i < 8; i++) cur[i] = g < total ? cvs[g * 8 + i] : 0u;
    const uint32_t c = lane & (nchunks - 1);  // chunk index within the leaf
    const uint32_t levels = 31 - __clz(nchunks);
    for (uint32_t lev = 1; lev <= levels; lev++) {
        const uint32_t half = 1u << (lev - 1);
        uint32_t r[8];
#pragma unroll
        for (int i = 0; i < 8; i++) r[i] = __shfl_down_sync(0xffffffffu, cur[i], half);
        if ((c & ((half << 1) - 1)) == 0) b3::parent_cv(cur, r, lev == levels, cur);
    }
    if (c == 0 && g < total) {
        const size_t node = leaf_node((uint32_t)(g / nchunks), tree_log);
#pragma unroll
        for (int i = 0; i < 8; i++) leaves[node * 8 + i] = cur[i];
    }
}

// Merge the chunk chaining values of each leaf in BLAKE3 tree order (the
// incremental hasher's stack discipline), root flag on the final parent.
__global__ void __launch_bounds__(128) k_leaf_merge(const uint32_t *__restrict__ cvs, uint32_t width,
                                                    uint32_t nchunks, uint32_t *__restrict__ leaves,
                                                    uint32_t tree_log) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= width) return;
    const uint32_t *cv = cvs + (size_t)j * nchunks * 8;
    uint32_t stack[33][8];
    int len = 0;
    uint32_t cur[8];
    for (uint32_t c = 0; c + 1 < nchunks; c++) {
        for (int i = 0; i < 8; i++) cur[i] = cv[(size_t)c * 8 + i];
        uint64_t total = (uint64_t)c + 1;
        while ((total & 1) == 0) {
            b3::parent_cv(stack[--len], cur, false, cur);
            total >>= 1;
        }
        for (int i = 0; i < 8; i++) stack[len][i] = cur[i];
        len++;
    }
    for (int i = 0; i < 8; i++) cur[i] = cv[(size_t)(nchunks - 1) * 8 + i];
    for (int s = len - 1; s >= 0; s--) b3::parent_cv(stack[s], cur, s == 0, cur);
    const size_t node = leaf_node(j, tree_log);
    for (int i = 0; i < 8; i++) leaves[node * 8 + i] = cur[i];
}

// One tree level: node i of the next layer from nodes 2i, 2i+1.
__global__ void __launch_bounds__(256) k_merkle_level(const uint32_t *__restrict__ prev,
                                                      uint32_t *__restrict__ next, uint32_t n_out,
                                                      bool root) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_out) return;
    uint32_t l[8], r[8], o[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        l[k] = prev[(size_t)(2 * i) * 8 + k];
        r[k] = prev[(size_t)(2 * i + 1) * 8 + k];
    }
    b3::parent_cv(l, r, root, o);
#pragma unroll
    for (int k = 0; k < 8; k++) next[(size_t)i * 8 + k] = o[k];
}

// Tree levels k0+1 .. k0+nlev of Merkle trees of `width` leaves, each stored
// layer after layer (layer k at node 2W - 2(W >> k)) in consecutive blocks of
// 2W - 1 nodes.  Block b of a tree reduces the 2^nlev nodes
// [b * 2^nlev, (b+1) * 2^nlev) of layer k0 to one node, writing every
// intermediate node; each tree's top node gets the ROOT flag.
__global__ void __launch_bounds__(256) k_tree_levels(uint32_t *__restrict__ forest, uint32_t width,
                                                     uint32_t k0, uint32_t nlev, uint32_t depth) {
    __shared__ uint32_t cvs[256][8];
    const uint32_t t = threadIdx.x;
    const uint32_t half = 1u << (nlev - 1);
    const uint32_t per_tree = width >> (k0 + nlev);
    uint32_t *tree = forest + (size_t)(blockIdx.x / per_tree) * (2ull * width - 1) * 8;
    const uint32_t bx = blockIdx.x % per_tree;
    const size_t in_off = 2ull * width - 2ull * (width >> k0);
    uint32_t cur[8];
    if (t < half) {
        const size_t node = in_off + ((size_t)bx << nlev) + 2 * t;
        uint32_t l[8], r[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            l[i] = tree[node * 8 + i];
            r[i] = tree[(node + 1) * 8 + i];
        }
        b3::parent_cv(l, r, k0 + 1 == depth, cur);
        const size_t out = 2ull * width - 2ull * (width >> (k0 + 1)) + ((size_t)bx << (nlev - 1)) + t;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            tree[out * 8 + i] = cur[i];
            cvs[t][i] = cur[i];
        }
    }
    __syncthreads();
    for (uint32_t lev = 2; lev <= nlev; lev++) {
        const uint32_t n = 1u << (nlev - lev);
        uint32_t l[8], r[8];
        if (t < n) {
#pragma unroll
            for (int i = 0; i < 8; i++) {
                l[i] = cvs[2 * t][i];
                r[i] = cvs[2 * t + 1][i];
            }
        }
        __syncthreads();
        if (t < n) {
            const uint32_t k = k0 + lev;
            b3::parent_cv(l, r, k == depth, cur);
            const size_t out = 2ull * width - 2ull * (width >> k) + ((size_t)bx << (nlev - lev)) + t;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                tree[out * 8 + i] = cur[i];
                cvs[t][i] = cur[i];
            }
        }
        __syncthreads();
    }
}

zg_status launch_leaf_hash(zg_ctx *ctx, const uint8_t *cw_d, uint32_t width, uint32_t leaf_bytes,
                           uint8_t *leaves_d, cudaStream_t s, uint32_t tree_width,
                           int leaf_variant, uint32_t *levels_done) {
    if (levels_done) *levels_done = 0;
    if (leaf_bytes % 4 != 0) {
        set_error("leaf size %u is not a multiple of 4 bytes", leaf_bytes);
        return ZG_ERR_INVALID_PARAM;
    }
    uint32_t tree_log = 32;
    if (tree_width != 0 && tree_width != width) {
        if ((tree_width & (tree_width - 1)) != 0 || width % tree_width != 0) {
            set_error("leaf hashing of several trees needs a power-of-two tree width dividing %u", width);
            return ZG_ERR_INVALID_PARAM;
        }
        tree_log = 31 - __builtin_clz(tree_width);
    }
    uint32_t *leaves = reinterpret_cast<uint32_t *>(leaves_d);
    if (leaf_bytes <= b3::CHUNK_LEN) {
        ZG_KBEGIN(ctx, s, "k_leaf_small");
        if (leaf_bytes % 16 == 0 && leaf_bytes > 0 && leaf_variant != 1) {
            const uint32_t W = tree_log >= 32 ? width : (1u << tree_log);
            const int fuse = levels_done && W >= 128 && width % 128 == 0 ? 1 : 0;
            k_leaf_small_coalesced<<<(width + 127) / 128, 128, 0, s>>>(cw_d, width, leaf_bytes, leaves,
                                                                      tree_log, fuse);
            if (fuse) *levels_done = 7;
        } else
            k_leaf_small<<<(width + 127) / 128, 128, 0, s>>>(cw_d, width, leaf_bytes, leaves, tree_log);
        ZG_KEND(ctx, s);
        return ZG_OK;
    }
    const uint32_t nchunks = (leaf_bytes + b3::CHUNK_LEN - 1) / b3::CHUNK_LEN;
    const size_t n = (size_t)width * nchunks;
    ZG_TRY(ctx->chunk_cv.ensure(n * 32));
    uint32_t *cvs = ctx->chunk_cv.as<uint32_t>();
    ZG_KBEGIN(ctx, s, "k_leaf_chunks");
    if (leaf_bytes % 16 == 0 && leaf_variant != 1)
        k_leaf_chunks_coalesced<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(cw_d, width, leaf_bytes,
                                                                             nchunks, cvs);
    else
        k_leaf_chunks<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(cw_d, width, leaf_bytes, nchunks, cvs);
    ZG_KEND(ctx, s);
    ZG_KBEGIN(ctx, s, "k_leaf_merge");
    // few leaves: one warp per leaf's chunks (the serial merge would leave most
    // SMs idle); many leaves: one thread per leaf, 32x fewer warp instructions
    if (nchunks <= 32 && (nchunks & (nchunks - 1)) == 0 && width < 16384)
        k_leaf_merge_pow2<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(cvs, width, nchunks, leaves,
                                                                      tree_log);
    else
        k_leaf_merge<<<(width + 127) / 128, 128, 0, s>>>(cvs, width, nchunks, leaves, tree_log);
    ZG_KEND(ctx, s);
    return ZG_OK;
}

zg_status launch_merkle_levels(zg_ctx *ctx, uint8_t *tree_d, uint32_t width, cudaStream_t s,
                               uint32_t ntrees, uint32_t k_start) {
    uint32_t *tree = reinterpret_cast<uint32_t *>(tree_d);
    const uint32_t depth = 31 - __builtin_clz(width);
    for (uint32_t k0 = k_start; k0 < depth;) {
        const uint32_t nlev = depth - k0 < 9 ? depth - k0 : 9;
        const uint32_t blocks = (width >> (k0 + nlev)) * ntrees;
        ZG_KBEGIN(ctx, s, "k_tree_levels");
        k_tree_levels<<<blocks, 1u << (nlev - 1), 0, s>>>(tree, width, k0, nlev, depth);
        ZG_KEND(ctx, s);
        k0 += nlev;
    }
    return ZG_OK;
}

}  // namespace zg

// ---------------------------------------------------------------------------
// Allocation-free Merkle root (no counterpart in the reference).
//
// Some callers of this library cannot allocate device memory on their request
// path: a serving loop that reserves its whole device-memory budget up front,
// or a host whose device buffers all come from its own pool.  For them
// cudaMalloc/cudaFree are off limits: they synchronize the device, stall other
// streams and can fail under memory pressure in the middle of a request.
// zg_merkle_root_noalloc_d allocates nothing.  Its scratch (the node layers,
// plus the chunk chaining values of leaves longer than one BLAKE3 chunk) is the
// file-scope 4 MiB array below, which every GPU that loads this library holds
// until the process exits.
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)4 << 20;
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_addr[kNoAllocMaxDevices] = {};  // device address of the array, per device

}  // namespace

extern "C" zg_status zg_merkle_root_noalloc_d(const void *leaves_d, uint32_t width,
                                              uint32_t leaf_bytes, uint8_t *root_d,
                                              void *stream) {
    using namespace zg;
    if (!leaves_d || !root_d) {
        set_error("zg_merkle_root_noalloc_d: null leaf or root pointer");
        return ZG_ERR_INVALID_PARAM;
    }
    if (width == 0 || (width & (width - 1)) != 0) {
        set_error("zg_merkle_root_noalloc_d: width %u is not a power of two", width);
        return ZG_ERR_INVALID_PARAM;
    }
    if (leaf_bytes == 0 || leaf_bytes % 4 != 0) {
        set_error("zg_merkle_root_noalloc_d: leaf size %u is not a positive multiple of 4",
                  leaf_bytes);
        return ZG_ERR_INVALID_PARAM;
    }
    // The leaf kernels read the preimages as 32-bit words: a pointer at an odd
    // offset into the caller's pool would fault on a misaligned load.
    if (reinterpret_cast<uintptr_t>(leaves_d) % 4 != 0) {
        set_error("zg_merkle_root_noalloc_d: leaves_d %p is not 4-byte aligned", leaves_d);
        return ZG_ERR_INVALID_PARAM;
    }
    const uint64_t nchunks =
        leaf_bytes <= b3::CHUNK_LEN ? 0 : (leaf_bytes + b3::CHUNK_LEN - 1) / b3::CHUNK_LEN;
    const uint64_t nodes = 2 * (uint64_t)width - 1;
    const uint64_t need = (nodes + (uint64_t)width * nchunks) * 32;
    if (need > kNoAllocScratchBytes) {
        set_error("zg_merkle_root_noalloc_d: %u leaves of %u bytes need %llu bytes of scratch; "
                  "the limit is %zu bytes (for example 65536 leaves of at most 1024 bytes)",
                  width, leaf_bytes, (unsigned long long)need, kNoAllocScratchBytes);
        return ZG_ERR_INVALID_PARAM;
    }
    int dev = 0;
    ZG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        set_error("zg_merkle_root_noalloc_d: device ordinal %d out of range", dev);
        return ZG_ERR_INVALID_PARAM;
    }
    void *base = nullptr;
    {
        // One-time set-up per device, with that device current: the array's
        // name is only a host-side stand-in, so its device address is looked up.
        // The address belongs to the device's primary context (the one the CUDA
        // runtime uses); it stays valid until the process exits or resets the
        // device, after which this entry point must not be called again.
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void *addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (e != cudaSuccess || !addr) {
                set_error("cudaGetSymbolAddress of the scratch array failed: %s",
                          cudaGetErrorString(e));
                return ZG_ERR_CUDA;
            }
            g_noalloc_addr[dev] = addr;
        }
        base = g_noalloc_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t *tree = static_cast<uint32_t *>(base);
    const uint8_t *cw = static_cast<const uint8_t *>(leaves_d);
    // Every node is written before it is read, so nothing needs clearing.
    if (nchunks == 0) {
        k_leaf_small<<<(width + 127) / 128, 128, 0, s>>>(cw, width, leaf_bytes, tree, 32u);
    } else {
        uint32_t *cvs = tree + nodes * 8;
        const uint64_t n = (uint64_t)width * nchunks;
        k_leaf_chunks<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(cw, width, leaf_bytes,
                                                                   (uint32_t)nchunks, cvs);
        k_leaf_merge<<<(width + 127) / 128, 128, 0, s>>>(cvs, width, (uint32_t)nchunks, tree, 32u);
    }
    ZG_CUDA(cudaGetLastError());
    uint64_t off = 0;
    for (uint32_t n = width; n > 1; n /= 2) {
        const uint32_t half = n / 2;
        k_merkle_level<<<(half + 255) / 256, 256, 0, s>>>(tree + off * 8, tree + (off + n) * 8,
                                                          half, half == 1);
        ZG_CUDA(cudaGetLastError());
        off += n;
    }
    ZG_CUDA(cudaMemcpyAsync(root_d, tree + off * 8, 32, cudaMemcpyDeviceToDevice, s));
    return ZG_OK;
}


