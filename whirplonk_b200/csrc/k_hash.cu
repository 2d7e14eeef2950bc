// k_hash.cu -- matrix commitment: BLAKE3 leaf hashing of codeword rows, Merkle
// levels, and the out-of-domain evaluation that closes irs_commit::commit.
//
// Leaves (cpp/include/whir/protocols/matrix_commit.hpp:169-195): leaf i is the
// BLAKE3 hash of row i's canonical little-endian bytes -- `depth` elements of
// 8 B (base) or 24 B (Ext3, c0 c1 c2).  Rows are gathered from the codeword
// planes written by the encoder, so each warp reads 8-byte words of 32
// consecutive rows per plane: fully coalesced.
//
// Merkle tree (merkle_tree.hpp:104-147): parent = BLAKE3(left || right),
// node array [leaves | level 1 | ... | root].  A CTA hashes a 512-leaf subtree
// (9 levels) in shared memory; a proof's tree ends with one launch for its
// top 10-18 levels (k_merkle_tail).
#include <algorithm>

#include "launch.h"
#include "blake3.cuh"
#include "sha256.cuh"
#include "state.cuh"
#include "wtx.cuh"

namespace wg {

__device__ __forceinline__ void store_node(u32* nodes, u64 idx, const unsigned cv[8]) {
    uint4* p = reinterpret_cast<uint4*>(nodes + idx * 8);
    p[0] = make_uint4(cv[0], cv[1], cv[2], cv[3]);
    p[1] = make_uint4(cv[4], cv[5], cv[6], cv[7]);
}
__device__ __forceinline__ void load_node(const u32* nodes, u64 idx, unsigned* m) {
    const uint4* p = reinterpret_cast<const uint4*>(nodes + idx * 8);
    uint4 a = p[0], b = p[1];
    m[0] = a.x; m[1] = a.y; m[2] = a.z; m[3] = a.w;
    m[4] = b.x; m[5] = b.y; m[6] = b.z; m[7] = b.w;
}

// The engine a configuration's hash_id selects (irs_commit.hpp:62-74).
constexpr int HASH_BLAKE3 = 0, HASH_SHA256 = 1;
template <int H>
__device__ __forceinline__ void hash64(const unsigned m[16], unsigned out[8]) {
    if (H == HASH_SHA256) sha256_hash64(m, out);
    else b3_hash64(m, out);
}

// Row i = words w = 0 .. depth*ncomp-1 with w -> (element w / ncomp, component w % ncomp),
// read from plane (component * depth + element).
template <int NCOMP>
__device__ __forceinline__ u64 row_word(const u64* __restrict__ planes, u64 N, u32 depth, u64 i, u32 w) {
    const u32 el = w / NCOMP, c = w - el * NCOMP;
    return planes[((u64)c * depth + el) * N + i];
}

// SHA-256 of row i's LE bytes: the 8-byte words become big-endian message
// words; the 0x80 marker follows the data (always on a word boundary) and the
// bit length closes the last block.
template <int NCOMP>
__device__ __forceinline__ void leaf_sha256(const u64* __restrict__ planes, u64 N, u32 depth, u64 i, unsigned out[8]) {
    const u32 nwords = depth * NCOMP;
    const u32 bytes = nwords * 8;
    const u32 nblk = (bytes + 9 + 63) / 64;
    unsigned h[8];
    sha256_init(h);
    for (u32 t = 0; t < nblk; ++t) {
        unsigned m[16];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const u32 w = t * 8 + q;
            if (w < nwords) {
                const u64 v = row_word<NCOMP>(planes, N, depth, i, w);
                m[2 * q] = bswap32((unsigned)v);
                m[2 * q + 1] = bswap32((unsigned)(v >> 32));
            } else {
                m[2 * q] = w == nwords ? 0x80000000u : 0u;
                m[2 * q + 1] = 0;
            }
        }
        if (t + 1 == nblk) {
            m[14] = 0;
            m[15] = bytes * 8;
        }
        sha256_compress(h, m);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) out[k] = bswap32(h[k]);
}

// blockIdx.y selects one of several independent matrices (planes and node
// arrays `plane_stride` / `node_stride` words apart).
template <int NCOMP, int H>
__global__ void __launch_bounds__(256, NCOMP == 3 ? 3 : 1) k_leaves(const u64* __restrict__ planes, u64 N, u32 depth, u32* nodes,
                                                u64 plane_stride, u64 node_stride, u32 logN, u32 perm_log_e) {
    const u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    const u64 i = codeword_row(k, logN, perm_log_e);  // the row leaf k hashes
    planes += blockIdx.y * plane_stride;
    nodes += blockIdx.y * node_stride;
    if (H == HASH_SHA256) {
        unsigned out[8];
        leaf_sha256<NCOMP>(planes, N, depth, i, out);
        store_node(nodes, k, out);
        return;
    }
    const u32 nwords = depth * NCOMP;           // 64-bit words per row
    const u32 bytes = nwords * 8;
    const u32 nblocks = (bytes + 63) / 64;
    unsigned cv[8];
    b3_init(cv);
    // Loads run ahead of the compressions: the next block's 8 words (base and
    // Ext2 rows) or the next two blocks' (Ext3 rows, 6 blocks of 8 planes each),
    // so their plane reads overlap the compressions.
    constexpr int AHEAD = NCOMP == 3 ? 2 : 1;
    u64 nxt[8], nxt2[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        nxt[q] = (u32)q < nwords ? row_word<NCOMP>(planes, N, depth, i, q) : 0;
        nxt2[q] = AHEAD == 2 && (u32)(8 + q) < nwords ? row_word<NCOMP>(planes, N, depth, i, 8 + q) : 0;
    }
    for (u32 t = 0; t < nblocks; ++t) {
        unsigned m[16];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            m[2 * q] = (unsigned)nxt[q];
            m[2 * q + 1] = (unsigned)(nxt[q] >> 32);
        }
        if (AHEAD == 2) {
#pragma unroll
            for (int q = 0; q < 8; ++q) nxt[q] = nxt2[q];
            if (t + 2 < nblocks) {
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const u32 w = (t + 2) * 8 + q;
                    nxt2[q] = w < nwords ? row_word<NCOMP>(planes, N, depth, i, w) : 0;
                }
            }
        } else if (t + 1 < nblocks) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const u32 w = (t + 1) * 8 + q;
                nxt[q] = w < nwords ? row_word<NCOMP>(planes, N, depth, i, w) : 0;
            }
        }
        const u32 len = (t + 1 == nblocks) ? bytes - 64 * t : 64;
        const unsigned flags = (t == 0 ? B3_CHUNK_START : 0u) | (t + 1 == nblocks ? (B3_CHUNK_END | B3_ROOT) : 0u);
        b3_compress(cv, m, flags, len);
    }
    store_node(nodes, k, cv);
}

// Rows wider than one chunk (1024 bytes: several committed vectors side by
// side) take BLAKE3's tree mode (blake3_engine.hpp:186-196, the hasher
// fallback): chunk c is compressed with counter c; a finished chunk's value is
// merged with the stack while the count of finished chunks has a trailing
// zero bit; the last chunk's value is merged with the stack from the top, the
// final merge carrying ROOT.  At most B3_MAX_CHUNKS chunks (16 KiB rows).
constexpr u32 B3_MAX_CHUNKS = 16;
__device__ __forceinline__ void b3_parent_cv(const unsigned l[8], const unsigned r[8], unsigned flags, unsigned out[8]) {
    unsigned m[16];
#pragma unroll
    for (int k = 0; k < 8; ++k) { m[k] = l[k]; m[8 + k] = r[k]; }
    b3_init(out);
    b3_compress(out, m, B3_PARENT | flags);
}

template <int NCOMP>
__global__ void __launch_bounds__(128) k_leaves_wide(const u64* __restrict__ planes, u64 N, u32 depth, u32* nodes,
                                                     u32 logN, u32 perm_log_e) {
    const u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    const u64 i = codeword_row(k, logN, perm_log_e);  // the row leaf k hashes
    const u32 nwords = depth * NCOMP;
    const u32 nch = (nwords + 127) / 128;
    unsigned stack[5][8];  // a tree of < 32 chunks holds at most 5 pending subtrees
    u32 sp = 0;
    unsigned cv[8];
    for (u32 c = 0; c < nch; ++c) {
        const u32 w0 = c * 128;
        const u32 cw = min(128u, nwords - w0);
        const u32 bytes = cw * 8;
        const u32 nblocks = (bytes + 63) / 64;
        b3_init(cv);
        for (u32 t = 0; t < nblocks; ++t) {
            unsigned m[16];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const u32 w = t * 8 + q;
                u64 v = 0;
                if (w < cw) v = row_word<NCOMP>(planes, N, depth, i, w0 + w);
                m[2 * q] = (unsigned)v;
                m[2 * q + 1] = (unsigned)(v >> 32);
            }
            const u32 len = (t + 1 == nblocks) ? bytes - 64 * t : 64;
            const unsigned flags = (t == 0 ? B3_CHUNK_START : 0u) |
                                   (t + 1 == nblocks ? (B3_CHUNK_END | (nch == 1 ? B3_ROOT : 0u)) : 0u);
            b3_compress(cv, m, flags, len, c);
        }
        if (c + 1 < nch) {
            for (u32 total = c + 1; (total & 1) == 0 && sp > 0; total >>= 1) {
                unsigned p[8];
                b3_parent_cv(stack[--sp], cv, 0u, p);
#pragma unroll
                for (int k = 0; k < 8; ++k) cv[k] = p[k];
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) stack[sp][k] = cv[k];
            ++sp;
        }
    }
    while (sp > 0) {
        --sp;
        unsigned p[8];
        b3_parent_cv(stack[sp], cv, sp == 0 ? B3_ROOT : 0u, p);
#pragma unroll
        for (int q = 0; q < 8; ++q) cv[q] = p[q];
    }
    store_node(nodes, k, cv);
}

__host__ __device__ __forceinline__ u64 level_offset(u32 logN, u32 l) {
    // [leaves (2^logN) | 2^(logN-1) | ... ]: offset of level l = 2^(logN+1) - 2^(logN+1-l)
    return (2ull << logN) - (2ull << (logN - l));
}

// parent = H(left || right)
template <int H>
__device__ __forceinline__ void parent_cv(const unsigned l[8], const unsigned r[8], unsigned out[8]) {
    unsigned m[16];
#pragma unroll
    for (int k = 0; k < 8; ++k) { m[k] = l[k]; m[8 + k] = r[k]; }
    hash64<H>(m, out);
}

int launch_leaves_batch(const u64* planes, u64 N, u32 depth, u32 ncomp, u32* nodes, u32 count, u64 plane_stride,
                       u64 node_stride, int hash, cudaStream_t st, u32 perm_log_e) {
    if (count == 0 || count > 65535) return -1;
    if (ncomp < 1 || ncomp > 3) return -1;  // base field, Ext2 (c0 c1 per element), Ext3
    if (N == 0 || (N & (N - 1))) return -1;
    u32 logN = 0;
    while ((1ull << logN) < N) ++logN;
    if (perm_log_e > logN) return -1;
    if (hash != HASH_SHA256 && depth * ncomp * 8 > 1024) {  // BLAKE3 tree mode, one matrix at a time
        if (count != 1 || depth * ncomp > 128 * B3_MAX_CHUNKS) return -1;
        const unsigned grid = (unsigned)((N + 127) / 128);
        if (ncomp == 1) k_leaves_wide<1><<<grid, 128, 0, st>>>(planes, N, depth, nodes, logN, perm_log_e);
        else if (ncomp == 2) k_leaves_wide<2><<<grid, 128, 0, st>>>(planes, N, depth, nodes, logN, perm_log_e);
        else k_leaves_wide<3><<<grid, 128, 0, st>>>(planes, N, depth, nodes, logN, perm_log_e);
        count_launches(1);
        return 0;
    }
    const dim3 grid((unsigned)((N + 255) / 256), count);
    if (hash == HASH_SHA256) {
        if (ncomp == 1) k_leaves<1, HASH_SHA256><<<grid, 256, 0, st>>>(planes, N, depth, nodes, plane_stride, node_stride, logN, perm_log_e);
        else if (ncomp == 2) k_leaves<2, HASH_SHA256><<<grid, 256, 0, st>>>(planes, N, depth, nodes, plane_stride, node_stride, logN, perm_log_e);
        else k_leaves<3, HASH_SHA256><<<grid, 256, 0, st>>>(planes, N, depth, nodes, plane_stride, node_stride, logN, perm_log_e);
    } else {
        if (ncomp == 1) k_leaves<1, HASH_BLAKE3><<<grid, 256, 0, st>>>(planes, N, depth, nodes, plane_stride, node_stride, logN, perm_log_e);
        else if (ncomp == 2) k_leaves<2, HASH_BLAKE3><<<grid, 256, 0, st>>>(planes, N, depth, nodes, plane_stride, node_stride, logN, perm_log_e);
        else k_leaves<3, HASH_BLAKE3><<<grid, 256, 0, st>>>(planes, N, depth, nodes, plane_stride, node_stride, logN, perm_log_e);
    }
    count_launches(1);
    return 0;
}

int launch_leaves(const u64* planes, u64 N, u32 depth, u32 ncomp, u32* nodes, int hash, cudaStream_t st,
                  u32 perm_log_e) {
    return launch_leaves_batch(planes, N, depth, ncomp, nodes, 1, 0, 0, hash, st, perm_log_e);
}

// Levels level_in + 1 .. level_in + levels (1 <= levels <= 9) of subtree
// `blk`, whose 2^levels children sit at level level_in from node blk 2^levels
// on; every produced level is written to global memory and the working level
// kept in shared memory.  CG: the children were written by other CTAs of the
// same launch, so they are read through L2.  Ends with a CTA barrier.
__device__ __forceinline__ void load_node_cg(const u32* nodes, u64 idx, unsigned* m) {
    const uint4* p = reinterpret_cast<const uint4*>(nodes + idx * 8);
    const uint4 a = __ldcg(p), b = __ldcg(p + 1);
    m[0] = a.x; m[1] = a.y; m[2] = a.z; m[3] = a.w;
    m[4] = b.x; m[5] = b.y; m[6] = b.z; m[7] = b.w;
}
template <int H, bool CG>
__device__ __forceinline__ void merkle_subtree(u32* nodes, u32 logN, u32 level_in, u32 levels, u64 blk,
                                               unsigned (*buf)[256 * 8]) {
    const u32 nparents = 1u << (levels - 1);
    const u64 in_off = level_offset(logN, level_in);
    const u64 out_off = level_offset(logN, level_in + 1);
    for (u32 t = threadIdx.x; t < nparents; t += blockDim.x) {
        unsigned m[16];
        const u64 child = (blk << levels) + 2 * t;
        if (CG) {
            load_node_cg(nodes, in_off + child, m);
            load_node_cg(nodes, in_off + child + 1, m + 8);
        } else {
            load_node(nodes, in_off + child, m);
            load_node(nodes, in_off + child + 1, m + 8);
        }
        unsigned cv[8];
        hash64<H>(m, cv);
        store_node(nodes, out_off + (blk << (levels - 1)) + t, cv);
#pragma unroll
        for (int k = 0; k < 8; ++k) buf[0][t * 8 + k] = cv[k];
    }
    __syncthreads();
    int cur = 0;
    for (u32 lv = 1; lv < levels; ++lv) {
        const u32 np = nparents >> lv;
        const u64 off = level_offset(logN, level_in + 1 + lv);
        for (u32 t = threadIdx.x; t < np; t += blockDim.x) {
            unsigned m[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) m[k] = buf[cur][t * 16 + k];
            unsigned cv[8];
            hash64<H>(m, cv);
            store_node(nodes, off + (blk << (levels - 1 - lv)) + t, cv);
#pragma unroll
            for (int k = 0; k < 8; ++k) buf[cur ^ 1][t * 8 + k] = cv[k];
        }
        __syncthreads();
        cur ^= 1;
    }
}

// Warp 0, after the root is written: root message, then the commitment's OOD
// points (irs_commit.hpp:472-554).
__device__ __forceinline__ void merkle_send_root(const u32* nodes, u32 logN, TxState* tx, ProofScalars* sc,
                                                 int commit_idx, int n_ood) {
    __threadfence();
    const u64 root = level_offset(logN, logN);
    u64 w[4];
    for (int k = 0; k < 4; ++k) w[k] = (u64)nodes[root * 8 + 2 * k] | ((u64)nodes[root * 8 + 2 * k + 1] << 32);
    WarpTx t;
    wtx_load(t, tx);
    wtx_message_words(t, w, 4);
    for (int j = 0; j < n_ood; ++j) {
        const E3 z = wtx_challenge_t(t);
        if (threadIdx.x == 0) sc->ood_pts[commit_idx][j] = z;
    }
    wtx_store(t, tx);
}

// One CTA hashes a subtree of height `levels` whose children sit at level
// `level_in`; every produced level is written to global memory.
template <int H>
__global__ void __launch_bounds__(256) k_merkle(u32* nodes, u32 logN, u32 level_in, u32 levels, TxState* tx,
                                                ProofScalars* sc, int commit_idx, int n_ood, int finish,
                                                u64 node_stride) {
    __shared__ unsigned buf[2][256 * 8];
    nodes += blockIdx.y * node_stride;
    if (levels > 0) merkle_subtree<H, false>(nodes, logN, level_in, levels, blockIdx.x, buf);
    if (finish && tx && threadIdx.x < 32) merkle_send_root(nodes, logN, tx, sc, commit_idx, n_ood);
}

// The top 10 .. 18 levels of a proof's tree in one launch: CTA b hashes the
// 512-node subtree b of level level_in (9 levels); the last CTA to finish (a
// ticket in ProofScalars) hashes the 2^(logN - level_in - 9) subtree roots up
// to the root and sends the root message -- what a subtree launch and a
// one-CTA top launch did, less one launch and its wait.
template <int H>
__global__ void __launch_bounds__(256) k_merkle_tail(u32* nodes, u32 logN, u32 level_in, TxState* tx,
                                                     ProofScalars* sc, int commit_idx, int n_ood) {
    __shared__ unsigned buf[2][256 * 8];
    __shared__ bool last;
    merkle_subtree<H, false>(nodes, logN, level_in, 9, blockIdx.x, buf);
    if (threadIdx.x == 0) {
        __threadfence();  // this CTA's subtree root (written by thread 0) before its ticket
        last = atomicAdd(&sc->counters[CTR_MERKLE_TAIL], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    merkle_subtree<H, true>(nodes, logN, level_in + 9, logN - level_in - 9, 0, buf);
    if (threadIdx.x < 32) merkle_send_root(nodes, logN, tx, sc, commit_idx, n_ood);
    if (threadIdx.x == 0) sc->counters[CTR_MERKLE_TAIL] = 0;
}

// Three tree levels at once: a thread reads 8 consecutive nodes of level
// `level_in` and writes their 4 parents, 2 grandparents and 1 great-grandparent.
template <int H>
__global__ void __launch_bounds__(256) k_merkle8(u32* nodes, u32 logN, u32 level_in, u64 node_stride) {
    const u64 g = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (1ull << (logN - level_in - 3))) return;
    nodes += blockIdx.y * node_stride;
    const u64 in = level_offset(logN, level_in) + 8 * g;
    const u64 o1 = level_offset(logN, level_in + 1) + 4 * g;
    const u64 o2 = level_offset(logN, level_in + 2) + 2 * g;
    const u64 o3 = level_offset(logN, level_in + 3) + g;
    // Each pair of children is loaded one hash ahead (ma / mb alternate), so the
    // node reads overlap the compressions.
    unsigned ma[16], mb[16], p0[8], p1[8], q0[8], q1[8];
    load_node(nodes, in + 0, ma); load_node(nodes, in + 1, ma + 8);
    load_node(nodes, in + 2, mb); load_node(nodes, in + 3, mb + 8);
    hash64<H>(ma, p0); store_node(nodes, o1 + 0, p0);
    load_node(nodes, in + 4, ma); load_node(nodes, in + 5, ma + 8);
    hash64<H>(mb, p1); store_node(nodes, o1 + 1, p1);
    load_node(nodes, in + 6, mb); load_node(nodes, in + 7, mb + 8);
    parent_cv<H>(p0, p1, q0);
    store_node(nodes, o2 + 0, q0);
    hash64<H>(ma, p0); store_node(nodes, o1 + 2, p0);
    hash64<H>(mb, p1); store_node(nodes, o1 + 3, p1);
    parent_cv<H>(p0, p1, q1);
    store_node(nodes, o2 + 1, q1);
    parent_cv<H>(q0, q1, p0);
    store_node(nodes, o3, p0);
}

// `count` trees `node_stride` words apart; the transcript step (tx non-null)
// is for a single tree only.
template <int H>
static int merkle_levels_h(u32* nodes, u32 logN, TxState* tx, ProofScalars* sc, int commit_idx, int n_ood, u32 count,
                           u64 node_stride, cudaStream_t st) {
    if (count == 0 || count > 65535 || (tx && count != 1)) return -1;
    u32 level = 0;
    // wide levels: 3 at a time while a launch still has >= 2^12 threads (and,
    // for a proof's tree, until at most 18 levels are left for k_merkle_tail)
    while (logN - level >= 3 + 12 && (!tx || logN - level > 18)) {
        const u64 threads = 1ull << (logN - level - 3);
        k_merkle8<H><<<dim3((unsigned)((threads + 255) / 256), count), 256, 0, st>>>(nodes, logN, level, node_stride);
        count_launches(1);
        level += 3;
    }
    if (logN == 0) {
        if (tx) {
            k_merkle<H><<<dim3(1, count), 32, 0, st>>>(nodes, logN, 0, 0, tx, sc, commit_idx, n_ood, 1, node_stride);
            count_launches(1);
        }
        return 0;
    }
    if (tx && logN - level > 9 && logN - level <= 18) {
        k_merkle_tail<H><<<1u << (logN - level - 9), 256, 0, st>>>(nodes, logN, level, tx, sc, commit_idx, n_ood);
        count_launches(1);
        return 0;
    }
    while (level < logN) {
        const u32 levels = (logN - level) < 9 ? (logN - level) : 9;
        const u32 ctas = 1u << (logN - level - levels);
        const int finish = (level + levels == logN) ? 1 : 0;
        k_merkle<H><<<dim3(ctas, count), 256, 0, st>>>(nodes, logN, level, levels, tx, sc, commit_idx, n_ood, finish,
                                                    node_stride);
        count_launches(1);
        level += levels;
    }
    return 0;
}

static int merkle_levels(u32* nodes, u32 logN, TxState* tx, ProofScalars* sc, int commit_idx, int n_ood, u32 count,
                         u64 node_stride, int hash, cudaStream_t st) {
    if (hash == HASH_SHA256)
        return merkle_levels_h<HASH_SHA256>(nodes, logN, tx, sc, commit_idx, n_ood, count, node_stride, st);
    return merkle_levels_h<HASH_BLAKE3>(nodes, logN, tx, sc, commit_idx, n_ood, count, node_stride, st);
}

int launch_merkle(u32* nodes, u32 logN, TxState* tx, ProofScalars* sc, int commit_idx, int n_ood, int hash,
                  cudaStream_t st) {
    return merkle_levels(nodes, logN, tx, sc, commit_idx, n_ood, 1, 0, hash, st);
}

int launch_merkle_batch(u32* nodes, u32 logN, u32 count, u64 node_stride, cudaStream_t st) {
    return merkle_levels(nodes, logN, nullptr, nullptr, 0, 0, count, node_stride, HASH_BLAKE3, st);
}

// ---------------------------------------------------------------------------
// Out-of-domain evaluation: value_(j,v) = sum_i v_i z_j^i for every point z_j
// and committed vector v (irs_commit.hpp:472-554 -> utilities.hpp:196-246),
// and the cross-witness completion of Config::prove (whir_prover.hpp:92-120),
// which evaluates the other witnesses' vectors at a witness's points.  With
// i = h 2^LO + l,
//   value = sum_h z_j^(h 2^LO) * sum_l v_(h,l) z_j^l :
// a warp owns whole blocks of 2^LO consecutive coefficients and accumulates
// the inner sum as unreduced 192-bit products against the table z_j^l, reduces
// once per block and scales by the table entry z_j^(h 2^LO).  Exact field
// sums, so the association order is free.  The last CTA (ticket) finishes the
// sums and sends the values as prover messages, point-major, every evaluated
// vector at each point.
// ---------------------------------------------------------------------------
// OOD_GRID: capacity of the per-CTA partials (the grid is 4 CTAs per SM, at most this).
constexpr int OOD_GRID = 1024, OOD_THREADS = 256;
constexpr u32 OOD_LO = 10;
constexpr int OOD_MAX_VALUES = MAX_OOD * MAX_VECTORS;

__device__ __forceinline__ E3 block_sum_e3(E3 v, E3* red) {
    v = e3_warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    E3 r = e3_zero();
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = e3_add(r, red[k]);
    __syncthreads();
    return r;  // valid in thread 0
}

static u32 ood_hi_count(u64 size) { return (u32)((size + (1ull << OOD_LO) - 1) >> OOD_LO); }

// tab[j]: z_j^l for l < 2^LO, then z_j^(h 2^LO) for h < hi_count.
__global__ void k_ood_tables(const E3* pts, int n_ood, u32 hi_count, E3* tab, bool ext2) {
    const u32 per = (1u << OOD_LO) + hi_count;
    const u64 total = (u64)per * n_ood;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const u32 j = (u32)(e / per), k = (u32)(e % per);
        const E3 z = pts[j];
        tab[e] = k < (1u << OOD_LO) ? ef_pow(z, k, ext2) : ef_pow(z, (u64)(k - (1u << OOD_LO)) << OOD_LO, ext2);
    }
}

// Sum over coefficients off .. off + len - 1 of chunk h (2^LO coefficients)
// of vector v against point table j, one value per lane (unreduced products,
// reduced once, scaled by z_j^(h 2^LO)).  Every load of a batch -- the
// coefficients and their table powers, 4 Ext3 or 8 base elements per lane --
// is issued before its products, so a warp waits for memory once per batch.
__device__ __forceinline__ E3 ood_part(const OodArgs& a, const E3* zlo, const E3* zhi, u32 v, u64 h, u32 off,
                                       u32 len, u32 lane) {
    const u64* b0 = a.v[0] + (u64)v * a.vec_stride;
    const u64 base = (h << OOD_LO) + off;
    const u64 rest = a.size > base ? a.size - base : 0;
    const u32 cnt = (u32)(rest < len ? rest : len);
    const E3* zl = zlo + off;
    E3Acc s = e3acc_zero();
    u32 l = lane;
    if (a.ext3) {  // one vector (nvec == 1): components in v[0..2]
        const u64* b1 = a.v[1];
        const u64* b2 = a.v[2];
        for (; l + 96 < cnt; l += 128) {
            E3 x[4], z[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const u64 i = base + l + 32 * k;
                x[k] = E3{b0[i], b1[i], b2[i]};
                z[k] = zl[l + 32 * k];
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) e3acc_mac(s, z[k], x[k]);
        }
        for (; l < cnt; l += 32) e3acc_mac(s, zl[l], E3{b0[base + l], b1[base + l], b2[base + l]});
    } else {
        for (; l + 224 < cnt; l += 256) {
            u64 x[8];
            E3 z[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                x[k] = b0[base + l + 32 * k];
                z[k] = zl[l + 32 * k];
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) e3acc_mac_base(s, z[k], x[k]);
        }
        for (; l < cnt; l += 32) e3acc_mac_base(s, zl[l], b0[base + l]);
    }
    return ef_mul(ef_fix(e3acc_reduce(s), a.ext2), zhi[h], a.ext2);
}

// ITEMS: one warp per (value, chunk) item, partials[k * hi_count + h] (few
// chunks per value: small vectors, many vectors); otherwise each warp strides
// over the parts of every value -- chunks cut into 2^sub_log parts, so that a
// vector of few chunks still spreads over many warps -- and a CTA sum goes to
// partials[cta * nvals + k].
template <bool ITEMS>
__global__ void __launch_bounds__(OOD_THREADS) k_ood(OodArgs a, const E3* tab, u32 hi_count, E3* partials,
                                                     unsigned* counter, u32 sub_log) {
    __shared__ E3 red[32];
    __shared__ bool is_last;
    __shared__ E3 totals[OOD_MAX_VALUES];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const u64 gw = (u64)blockIdx.x * nwarps + warp;
    const u64 nw = (u64)gridDim.x * nwarps;
    const u32 per = (1u << OOD_LO) + hi_count;
    const u32 nvals = (u32)a.n_ood * a.nvec;
    if (ITEMS) {
        const u64 items = (u64)nvals * hi_count;
        for (u64 it = gw; it < items; it += nw) {
            const u32 k = (u32)(it / hi_count), v = k % a.nvec, j = k / a.nvec;
            if (v >= a.skip_lo && v < a.skip_hi) continue;
            const E3* zlo = tab + (u64)j * per;
            const E3 val = e3_warp_sum(ood_part(a, zlo, zlo + (1u << OOD_LO), v, it % hi_count, 0, 1u << OOD_LO, lane));
            if (lane == 0) partials[it] = val;
        }
        // every warp's partials visible device-wide before this CTA takes its ticket
        __threadfence();
        __syncthreads();
    } else {
        for (int j = 0; j < a.n_ood; ++j) {
            const E3* zlo = tab + (u64)j * per;
            for (u32 v = 0; v < a.nvec; ++v) {
                if (v >= a.skip_lo && v < a.skip_hi) continue;
                E3 acc = e3_zero();
                const u32 len = 1u << (OOD_LO - sub_log), pmask = (1u << sub_log) - 1;
                for (u64 it = gw; it < ((u64)hi_count << sub_log); it += nw)
                    acc = e3_add(acc, ood_part(a, zlo, zlo + (1u << OOD_LO), v, it >> sub_log, ((u32)it & pmask) * len, len, lane));
                E3 bs = block_sum_e3(acc, red);
                if (threadIdx.x == 0) partials[(u64)blockIdx.x * nvals + (u32)j * a.nvec + v] = bs;
            }
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned ticket = atomicAdd(counter, 1u);
        is_last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    // one warp per value: the sum of its partials
    const u32 nparts = ITEMS ? hi_count : gridDim.x;
    for (u32 k = warp; k < nvals; k += nwarps) {
        const u32 v = k % a.nvec;
        if (v >= a.skip_lo && v < a.skip_hi) continue;
        E3 acc = e3_zero();
        for (u32 b = lane; b < nparts; b += 32) {
            const E3* pp = ITEMS ? &partials[(u64)k * hi_count + b] : &partials[(u64)b * nvals + k];
            acc = e3_add(acc, E3{__ldcg(&pp->c0), __ldcg(&pp->c1), __ldcg(&pp->c2)});
        }
        const E3 total = e3_warp_sum(acc);
        if (lane == 0) {
            a.out[(k / a.nvec) * a.out_stride + v] = total;
            totals[k] = total;
        }
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // warp 0 sends the values
        WarpTx t;
        wtx_load(t, a.tx);
        for (u32 k = 0; k < nvals; ++k) {
            const u32 v = k % a.nvec;
            if (v < a.skip_lo || v >= a.skip_hi) wtx_message_t(t, totals[k]);
        }
        wtx_store(t, a.tx);
    }
    if (threadIdx.x == 0) *counter = 0;
}

size_t ood_scratch_bytes(u64 max_size, u32 max_values) {
    return 256 + (size_t)OOD_GRID * max_values * sizeof(E3) +
           (size_t)MAX_OOD * ((1u << OOD_LO) + ood_hi_count(max_size)) * sizeof(E3);
}

int launch_ood(const OodArgs& a, cudaStream_t st) {
    if (a.n_ood <= 0) return 0;
    if (a.n_ood > MAX_OOD || a.size == 0 || a.nvec == 0 || a.nvec > (u32)MAX_VECTORS) return -1;
    if (a.ext3 && a.nvec != 1) return -1;
    if ((u32)a.n_ood * a.nvec > a.scratch_values) return -1;
    const u32 hc = ood_hi_count(a.size);
    char* base = reinterpret_cast<char*>(a.scratch);
    unsigned* counter = reinterpret_cast<unsigned*>(base);
    E3* partials = reinterpret_cast<E3*>(base + 256);
    E3* tab = partials + (size_t)OOD_GRID * a.scratch_values;
    const u64 entries = (u64)((1u << OOD_LO) + hc) * a.n_ood;
    k_ood_tables<<<(unsigned)std::min<u64>(2ull * device_sms(), (entries + 255) / 256), 256, 0, st>>>(a.pts, a.n_ood, hc, tab, a.ext2 != 0);
    count_launches(1);
    const u64 warps_per_cta = OOD_THREADS / 32;
    const u64 items = (u64)a.n_ood * a.nvec * hc;
    // Few chunks per value: spread (value, chunk) items over the warps (the
    // partials fit: items <= OOD_GRID * scratch_values when hc <= OOD_GRID).
    const bool by_items = hc <= OOD_GRID && items > hc;
    const u64 cap = std::min<u64>(4ull * device_sms(), (u64)OOD_GRID);
    // Chunks of one value cut into up to 8 parts while the parts still fit
    // the grid's warps once (a part is one product by the chunk's power more).
    u32 sub_log = 0;
    while (!by_items && sub_log < 3 && ((u64)hc << (sub_log + 1)) <= cap * warps_per_cta) ++sub_log;
    u64 want = ((by_items ? items : ((u64)hc << sub_log)) + warps_per_cta - 1) / warps_per_cta;
    unsigned grid = (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
    if (by_items) k_ood<true><<<grid, OOD_THREADS, 0, st>>>(a, tab, hc, partials, counter, 0);
    else k_ood<false><<<grid, OOD_THREADS, 0, st>>>(a, tab, hc, partials, counter, sub_log);
    count_launches(1);
    return 0;
}

}  // namespace wg
