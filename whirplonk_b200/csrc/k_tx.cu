// k_tx.cu -- the sequential Fiat-Shamir steps of the prover, executed on the
// device: transcript start, constraint/STIR combination challenges, proof of
// work grinding, in-domain openings (indices, row hints, Merkle paths) and
// the final-vector message.  Protocol order and byte layout follow
// cpp/include/whir/protocols/whir/whir_prover.hpp:56-407.
#include "launch.h"
#include "blake3.cuh"
#include "sha256.cuh"
#include "state.cuh"
#include "wtx.cuh"

namespace wg {

// ---------------------------------------------------------------------------
// Transcript start: ProverState::from_ds (transcript.hpp:605-610) absorbs
// protocol_id || session_id || instance bytes.
// ---------------------------------------------------------------------------
// One warp.
__global__ void k_tx_init(TxState* tx, const unsigned char* ds, u32 ds_len, unsigned char* narg, u64 narg_cap,
                          unsigned char* hints, u64 hints_cap, ProofScalars* sc, unsigned deg) {
    if (threadIdx.x >= 32) return;
    WarpTx t;
    t.h = t.r = 0;
    t.hpos = t.rpos = t.has_reader = t.err = 0;
    t.deg = deg;
    t.narg_len = t.hints_len = 0;
    t.narg_cap = narg_cap;
    t.hints_cap = hints_cap;
    t.narg = narg;
    t.hints = hints;
    wtx_absorb_bytes(t, ds, ds_len);
    wtx_store(t, tx);
    for (int i = threadIdx.x; i < 64; i += 32) sc->counters[i] = 0;
}

int launch_tx_init(TxState* tx, const unsigned char* ds, u32 ds_len, unsigned char* narg, u64 narg_cap,
                   unsigned char* hints, u64 hints_cap, ProofScalars* sc, unsigned deg, cudaStream_t st) {
    if (deg < 1 || deg > 3) return -1;
    k_tx_init<<<1, 32, 0, st>>>(tx, ds, ds_len, narg, narg_cap, hints, hints_cap, sc, deg);
    count_launches(1);
    return 0;
}

// Vector RLC, constraint RLC and "the sum" (whir_prover.hpp:122-197):
//   vrlc = geometric_challenge(V), crlc = geometric_challenge(F + O),
//   sum  = sum_f crlc_f sum_v vrlc_v eval_(f,v) + sum_i crlc_(F+i) sum_v vrlc_v ood_(i,v)
// over the O = nwit * ood initial OOD points, whose coordinates are also laid
// out contiguously for the covector.  One warp.
__global__ void k_constraint_rlc(TxState* tx, ProofScalars* sc, int n_forms, int nwit, int ood, int nvec) {
    if (threadIdx.x >= 32) return;
    const int l = threadIdx.x;
    const int n_ood = nwit * ood;
    for (int i = l; i < n_ood; i += 32) sc->init_ood_pts[i] = sc->ood_pts[i / ood][i % ood];
    const int count = n_forms + n_ood;
    WarpTx t;
    wtx_load(t, tx);
    wtx_geometric(t, sc->vrlc, nvec);
    wtx_geometric(t, sc->crlc, count);
    wtx_store(t, tx);
    E3 v = e3_zero();
    for (int r = l; r < count; r += 32) {
        const E3* vals = r < n_forms ? &sc->forms_eval[r * nvec] : &sc->init_ood_mat[(r - n_forms) * nvec];
        E3 row = e3_zero();
        for (int k = 0; k < nvec; ++k) row = e3_add(row, ef_mul(sc->vrlc[k], vals[k], t.deg == 2));
        v = e3_add(v, ef_mul(sc->crlc[r], row, t.deg == 2));
    }
    v = wtx_sum(v);
    if (l == 0) sc->sum = v;
}

int launch_constraint_rlc(TxState* tx, ProofScalars* sc, int n_forms, int nwit, int ood, int nvec, cudaStream_t st) {
    if (n_forms > MAX_FORMS || ood > MAX_OOD || nwit < 1 || nwit > MAX_WITNESSES || nvec < 1 || nvec > MAX_VECTORS)
        return -1;
    k_constraint_rlc<<<1, 32, 0, st>>>(tx, sc, n_forms, nwit, ood, nvec);
    count_launches(1);
    return 0;
}

// ---------------------------------------------------------------------------
// Proof of work (proof_of_work.hpp:95-193, 236-257): the smallest nonce n >= 0
// with LE_u64(BLAKE3(challenge || n_le || 0^24)[0..8]) <= threshold.
//
// One launch: CTAs claim chunks of POW_CHUNK consecutive nonces in increasing
// order from a counter (atomicAdd), scan a claimed chunk completely and claim
// the next one while the previous hit published in pow_best (atomicMin) is not
// below the chunk.  Every chunk that starts at or below the final minimum is
// therefore claimed and fully scanned, so the minimum is exact -- the
// reference's answer, whatever the scheduling -- and the work past it is at
// most one chunk per CTA.  The search stops at 64x the expected length
// 2^64 / threshold (miss probability e^-64), capped at POW_NONCE_LIMIT; running
// out sets TX_ERR_POW_EXHAUSTED.
// ---------------------------------------------------------------------------
constexpr u64 POW_NONCE_LIMIT = 1ull << 36;
constexpr unsigned POW_THREADS = 256, POW_CTAS_PER_SM = 2, POW_CHUNK = 2 * POW_THREADS;

// One warp.  Also resets the search state.
__global__ void k_pow_challenge(TxState* tx, ProofScalars* sc) {
    if (threadIdx.x >= 32) return;
    WarpTx t;
    wtx_load(t, tx);
    wtx_squeeze_bytes(t, sc->pow_ch, 32);
    wtx_store(t, tx);
    if (threadIdx.x == 0) {
        sc->pow_best = ~0ull;
        sc->pow_next = 0;
    }
}

// H: 0 = BLAKE3, 1 = SHA-256 (the PoW engine follows the hash_id, whir.hpp:134-140).
template <int H>
__global__ void __launch_bounds__(POW_THREADS) k_pow_search(ProofScalars* sc, u64 threshold, u64 limit) {
    __shared__ unsigned ch[8];
    __shared__ u64 claim[2];
    __shared__ int stop;
    unsigned long long* next = reinterpret_cast<unsigned long long*>(&sc->pow_next);
    if (threadIdx.x < 8) {
        const unsigned char* c = sc->pow_ch + 4 * threadIdx.x;
        ch[threadIdx.x] = (unsigned)c[0] | ((unsigned)c[1] << 8) | ((unsigned)c[2] << 16) | ((unsigned)c[3] << 24);
    }
    if (threadIdx.x == 0) claim[0] = atomicAdd(next, (unsigned long long)POW_CHUNK);
    __syncthreads();
    unsigned m[16];
#pragma unroll
    for (int k = 0; k < 8; ++k) m[k] = ch[k];
#pragma unroll
    for (int k = 10; k < 16; ++k) m[k] = 0;
    for (unsigned it = 0;; ++it) {
        const u64 base = claim[it & 1];
        if (threadIdx.x == 0) {
            stop = base >= limit || base > __ldcg(&sc->pow_best);
            // claim the next chunk now, so the counter's latency overlaps the hashing
            if (!stop) claim[(it + 1) & 1] = atomicAdd(next, (unsigned long long)POW_CHUNK);
        }
        __syncthreads();
        if (stop) break;
#pragma unroll
        for (unsigned k = 0; k < POW_CHUNK / POW_THREADS; ++k) {
            const u64 n = base + k * POW_THREADS + threadIdx.x;
            if (n >= limit) break;
            m[8] = (unsigned)n;
            m[9] = (unsigned)(n >> 32);
            unsigned h[8];
            if (H == 1) sha256_hash64(m, h);
            else b3_hash64(m, h);
            const u64 v = (u64)h[0] | ((u64)h[1] << 32);  // first 8 digest bytes, LE
            if (v <= threshold) atomicMin(reinterpret_cast<unsigned long long*>(&sc->pow_best), (unsigned long long)n);
        }
        __syncthreads();
    }
}

// The search for one PoW (challenge already squeezed, pow_best / pow_next reset).
int launch_pow_grind_only(ProofScalars* sc, u64 threshold, int hash, cudaStream_t st) {
    const double expect = threshold == 0 ? 1.8446744073709552e19 : 18446744073709551616.0 / (double)threshold;
    const u64 limit = expect * 64.0 >= (double)POW_NONCE_LIMIT ? POW_NONCE_LIMIT : (u64)(expect * 64.0) + 1;
    // Every CTA finishes the chunk it holds when the minimum turns up, so the
    // work past the answer is about one chunk per CTA: a search expected to be
    // short gets one CTA per SM (the latency of a proof alone stays that of a
    // full grid), a long one up to POW_CTAS_PER_SM per SM.  The answer does not
    // depend on the grid.
    const double want = expect / (4.0 * POW_CHUNK);
    const unsigned sms = device_sms(), cap = POW_CTAS_PER_SM * sms;
    const unsigned grid = want >= (double)cap ? cap : (want <= (double)sms ? sms : (unsigned)want);
    if (hash == 1) k_pow_search<1><<<grid, POW_THREADS, 0, st>>>(sc, threshold, limit);
    else k_pow_search<0><<<grid, POW_THREADS, 0, st>>>(sc, threshold, limit);
    count_launches(1);
    return 0;
}

__global__ void k_pow_finish(TxState* tx, ProofScalars* sc, int slot) {
    if (threadIdx.x >= 32) return;
    const u64 n = sc->pow_best;
    WarpTx t;
    wtx_load(t, tx);
    if (n == ~0ull) t.err |= TX_ERR_POW_EXHAUSTED;
    if (threadIdx.x == 0 && slot >= 0 && slot < MAX_COMMITS + 4) sc->pow_nonces[slot] = n;
    wtx_message_u64(t, n);
    wtx_store(t, tx);
}

int launch_pow(TxState* tx, ProofScalars* sc, u64 threshold, int slot, int hash, cudaStream_t st) {
    if (threshold == ~0ull) return 0;  // zero difficulty: nothing sent (proof_of_work.hpp:241)
    k_pow_challenge<<<1, 32, 0, st>>>(tx, sc);
    count_launches(1);
    launch_pow_grind_only(sc, threshold, hash, st);
    k_pow_finish<<<1, 32, 0, st>>>(tx, sc, slot);
    count_launches(1);
    return 0;
}

// Final vector: prover_message of every coefficient (whir_prover.hpp:360-362).
// One warp.
__global__ void k_send_vector(TxState* tx, const u64* c0, const u64* c1, const u64* c2, u64 size) {
    if (threadIdx.x >= 32) return;
    WarpTx t;
    wtx_load(t, tx);
    for (u64 i = 0; i < size; ++i) wtx_message_t(t, E3{c0[i], c1[i], c2[i]});
    wtx_store(t, tx);
}

int launch_send_vector(TxState* tx, const u64* c0, const u64* c1, const u64* c2, u64 size, cudaStream_t st) {
    k_send_vector<<<1, 32, 0, st>>>(tx, c0, c1, c2, size);
    count_launches(1);
    return 0;
}

// `count` Ext3 challenges in a row into sc->sc_r[slot ..] -- the folding
// randomness of a proof without constraints (whir_prover.hpp:211-218,
// verifier_message_vec).  One warp.
__global__ void k_squeeze_e3(TxState* tx, ProofScalars* sc, int slot, int count) {
    if (threadIdx.x >= 32) return;
    WarpTx t;
    wtx_load(t, tx);
    for (int k = 0; k < count; ++k) {
        const E3 r = wtx_challenge_t(t);
        if (threadIdx.x == 0) sc->sc_r[slot + k] = r;
    }
    wtx_store(t, tx);
}

int launch_squeeze_challenges(TxState* tx, ProofScalars* sc, int slot, int count, cudaStream_t st) {
    if (count <= 0) return 0;
    if (slot < 0 || slot + count > MAX_SC_ROUNDS) return -1;
    k_squeeze_e3<<<1, 32, 0, st>>>(tx, sc, slot, count);
    count_launches(1);
    return 0;
}

// ---------------------------------------------------------------------------
// Opening (irs_commit.hpp:600-713, challenge_indices.hpp:56-119,
// merkle_tree.hpp:165-211) of nwit commitments at the same rows, one CTA of
// 1024 threads:
//   1. squeeze q * ceil(log2(N)/8) bytes, index = big-endian bytes mod N;
//   2. per commitment: hint u64 (q * depth), the q rows in index order
//      (duplicates kept), then its Merkle hints -- sorted, deduplicated
//      indices climbed level by level, a node's sibling is emitted unless the
//      sibling is itself in the set.  Every commitment has the same tree shape
//      and indices, so its hint block has the same length;
//   3. (STIR) point gen^idx and value <rows, vector_rlc (x) eq_weights(last
//      folding randomness)> over the rows of all commitments side by side
//      (whir_prover.hpp:283-310).
// ---------------------------------------------------------------------------
constexpr int OPEN_THREADS = 1024;

// Exclusive prefix count of `flag` over the CTA; *total receives the sum.
__device__ u32 block_scan(bool flag, u32* warp_tot, u32* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, flag);
    const u32 pre = __popc(bal & ((1u << lane) - 1));
    if (lane == 0) warp_tot[warp] = __popc(bal);
    __syncthreads();
    if (warp == 0) {
        u32 v = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
        u32 incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            u32 t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += t;
        }
        warp_tot[lane] = incl - v;  // exclusive
        if (lane == 31) *total = incl;
    }
    __syncthreads();
    const u32 r = warp_tot[warp] + pre;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(OPEN_THREADS) k_open(OpenArgs a) {
    __shared__ u64 idx_s[MAX_QUERIES];
    __shared__ u64 cur[MAX_QUERIES];
    __shared__ u32 warp_tot[32];
    __shared__ u32 total;
    __shared__ E3 eqw[MAX_DEPTH];
    __shared__ u64 hint_base;
    __shared__ unsigned char idx_bytes[MAX_QUERIES * 8];
    __shared__ unsigned char occ[MAX_QUERIES];
    __shared__ u32 lvl_cnt[32];
    const TxState* tx = a.tx;  // hint pointers and capacity only; warp 0 carries the sponge
    ProofScalars* sc = a.sc;
    const u32 t = threadIdx.x;
    const u32 q = a.q;
    const u32 nbytes = (a.logN + 7) / 8;
    const u32 nwit = a.nwit;
    const bool x2 = tx->deg == 2;  // GoldilocksExt2 target field

    // 1. indices: warp 0 squeezes q * nbytes bytes (big-endian per index)
    WarpTx wt;
    if (t < 32) {
        wtx_load(wt, a.tx);
        if (a.N != 1) wtx_squeeze_bytes(wt, idx_bytes, q * nbytes);
    }
    __syncthreads();
    for (u32 i = t; i < q; i += blockDim.x) {
        u64 acc = 0;
        for (u32 k = 0; k < nbytes; ++k) acc = (acc << 8) | idx_bytes[i * nbytes + k];
        idx_s[i] = a.N == 1 ? 0 : (acc & (a.N - 1));  // N is a power of two
    }
    if (t == 0) hint_base = wt.hints_len;
    // eq weights of the last `fold` folding challenges (multilinear_point.hpp:40-62),
    // one entry per thread of warps 1.. (they do not wait for warp 0's squeeze)
    if (a.stir && t >= 32 && t - 32 < (1u << a.fold)) {
        const u32 i = t - 32;
        E3 acc = e3_one();
        for (u32 k = 0; k < a.fold; ++k) {
            const E3 r = sc->sc_r[a.r_offset + k];
            const bool bit = (i >> (a.fold - 1 - k)) & 1;
            acc = ef_mul(acc, bit ? r : e3_sub(e3_one(), r), x2);
        }
        eqw[i] = acc;
    }
    for (u32 s2 = t; s2 < (u32)MAX_QUERIES; s2 += blockDim.x) occ[s2] = 0;
    __syncthreads();
    for (u32 i = t; i < q; i += blockDim.x) sc->indices[i] = idx_s[i];

    // Sort + dedup: a first occurrence v goes to slot #{j : idx_j < v}; distinct
    // values get distinct, order-preserving slots, compacted with a CTA scan.
    if (t < q) {
        const u64 v = idx_s[t];
        u32 lt = 0;
        bool dup = false;
        for (u32 j = 0; j < q; ++j) {
            const u64 o = idx_s[j];
            lt += (o < v) ? 1u : 0u;
            dup |= (o == v && j < t);
        }
        if (!dup) { cur[lt] = v; occ[lt] = 1; }
    }
    __syncthreads();
    const bool present = t < q && occ[t];
    const u64 pv = present ? cur[t] : 0;
    const u32 pos = block_scan(present, warp_tot, &total);
    const u32 u = total;
    if (present) cur[pos] = pv;
    __syncthreads();

    // Merkle levels.  Per level L the nodes are the distinct values of
    // cur[j] >> L (cur is sorted, so equal values are adjacent); a node x emits
    // its sibling x ^ 1 unless the sibling is itself a node.  Warp L handles
    // level L: it walks cur in chunks of 32 lanes and ranks its emitters with a
    // ballot.  The per-level counts are prefix-summed, so every warp writes its
    // siblings at the reference's position (level by level, increasing x within
    // a level).
    const u32 warp = t >> 5, lane = t & 31;
    auto present_at = [&](u64 y, u32 L) -> bool {  // is y a node of level L?
        u32 lo = 0, hi = u;
        while (lo < hi) {
            const u32 mid = (lo + hi) >> 1;
            if ((cur[mid] >> L) < y) lo = mid + 1;
            else hi = mid;
        }
        return lo < u && (cur[lo] >> L) == y;
    };
    auto emits = [&](u32 j, u32 L) -> bool {
        if (j >= u) return false;
        const u64 x = cur[j] >> L;
        const bool first = j == 0 || (cur[j - 1] >> L) != x;
        return first && !present_at(x ^ 1, L);
    };
    if (warp < a.logN) {
        u32 cnt = 0;
        for (u32 j0 = 0; j0 < u; j0 += 32) cnt += __popc(__ballot_sync(0xFFFFFFFFu, emits(j0 + lane, warp)));
        if (lane == 0) lvl_cnt[warp] = cnt;
    }
    __syncthreads();
    u64 merkle_bytes = 0;
    for (u32 k = 0; k < a.logN; ++k) merkle_bytes += 32ull * lvl_cnt[k];
    const u64 esz = 8ull * a.ncomp;
    const u64 row_bytes = esz * a.depth;
    const u64 row_hint = 8 + row_bytes * q;
    const u64 blk = row_hint + merkle_bytes;  // hint bytes of one commitment
    const bool fits = hint_base + blk * nwit <= tx->hints_cap;

    // 2a. row hints.  Every hint word sits at a multiple of 8 bytes from the
    // commitment's hint block, so when the block starts 8-byte aligned (the
    // hints stream holds whole words) a word is one 8-byte store.
    const bool hints_al8 = (reinterpret_cast<uintptr_t>(tx->hints + hint_base) & 7) == 0;
    if (fits) {
        const u32 rw = a.depth * a.ncomp;  // words per row (<= MAX_DEPTH * 3)
        const u32 nwords = q * rw;
        for (u32 w = 0; w < nwit; ++w) {
            unsigned char* hb = tx->hints + hint_base + w * blk;
            const u64* planes = a.planes + w * a.planes_stride;
            if (t == 0) {
                const u64 len = (u64)q * a.depth;
                for (int k = 0; k < 8; ++k) hb[k] = (unsigned char)(len >> (8 * k));
            }
            for (u32 x = t; x < nwords; x += blockDim.x) {
                const u32 qi = x / rw, rem = x - qi * rw;
                const u32 el = rem / a.ncomp, c = rem - el * a.ncomp;
                const u64 v = planes[((u64)c * a.depth + el) * a.N + codeword_row(idx_s[qi], a.logN, a.perm_log_e)];
                unsigned char* dst = hb + 8 + qi * row_bytes + (u64)el * esz + 8ull * c;
                if (hints_al8) {
                    *reinterpret_cast<u64*>(dst) = v;
                } else {
#pragma unroll 1
                    for (int k = 0; k < 8; ++k) dst[k] = (unsigned char)(v >> (8 * k));
                }
            }
        }
    }

    // 3. STIR point and value of each opened row: a warp per row, its lanes over
    //    the row's elements (all commitments side by side), a warp sum at the end.
    if (a.stir) {
        const u32 dmask = (1u << a.fold) - 1;
        const u32 total = nwit * a.depth;
        const u32 nwarps = blockDim.x >> 5;
        for (u32 i = warp; i < q; i += nwarps) {
            const u64 id = codeword_row(idx_s[i], a.logN, a.perm_log_e);  // natural row = exponent of its point
            E3 val = e3_zero();
            for (u32 k = lane; k < total; k += 32) {
                const u32 w = k / a.depth, el = k - w * a.depth;
                const u64* planes = a.planes + w * a.planes_stride;
                E3 term;
                if (a.ncomp == 1) {
                    term = e3_mul_base(eqw[el & dmask], planes[(u64)el * a.N + id]);
                } else if (a.ncomp == 2) {  // Ext2 rows: planes c0, c1
                    term = ef_mul(E3{planes[(u64)el * a.N + id], planes[((u64)a.depth + el) * a.N + id], 0},
                                  eqw[el & dmask], true);
                } else {
                    term = e3_mul(E3{planes[(u64)el * a.N + id], planes[((u64)a.depth + el) * a.N + id],
                                     planes[((u64)2 * a.depth + el) * a.N + id]},
                                  eqw[el & dmask]);
                }
                if (a.use_vrlc) term = ef_mul(term, sc->vrlc[w * (a.depth >> a.fold) + (el >> a.fold)], x2);
                val = e3_add(val, term);
            }
            val = e3_warp_sum(val);
            if (lane == 0) {
                sc->stir_pts[a.ood_offset + i] = e3_base(gl_pow(a.gen, id));
                sc->stir_vals[a.ood_offset + i] = val;
            }
        }
    }

    // 2b. Merkle hints of every commitment
    if (warp < a.logN) {
        const u32 L = warp;
        u64 lvl_base = row_hint;
        for (u32 k = 0; k < L; ++k) lvl_base += 32ull * lvl_cnt[k];
        const u64 level_off = (2ull << a.logN) - (2ull << (a.logN - L));
        u32 rank = 0;
        for (u32 j0 = 0; j0 < u; j0 += 32) {
            const u32 j = j0 + lane;
            const bool e = emits(j, L);
            const unsigned m = __ballot_sync(0xFFFFFFFFu, e);
            if (e && fits) {
                const u64 x = cur[j] >> L;
                const u64 rel = lvl_base + 32ull * (rank + __popc(m & ((1u << lane) - 1)));
                for (u32 w = 0; w < nwit; ++w) {
                    const u32* nodes = a.nodes + w * a.nodes_stride;
                    const uint4* src = reinterpret_cast<const uint4*>(nodes + (level_off + (x ^ 1)) * 8);
                    const uint4 h0 = src[0], h1 = src[1];
                    unsigned char* dst = tx->hints + hint_base + w * blk + rel;
                    if (hints_al8) {
                        u64* d8 = reinterpret_cast<u64*>(dst);
                        d8[0] = (u64)h0.x | ((u64)h0.y << 32);
                        d8[1] = (u64)h0.z | ((u64)h0.w << 32);
                        d8[2] = (u64)h1.x | ((u64)h1.y << 32);
                        d8[3] = (u64)h1.z | ((u64)h1.w << 32);
                    } else {
                        const unsigned w8[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
#pragma unroll 1
                        for (int k = 0; k < 32; ++k) dst[k] = (unsigned char)(w8[k >> 2] >> (8 * (k & 3)));
                    }
                }
            }
            rank += __popc(m);
        }
    }
    if (t < 32) {
        if (!fits) wt.err |= TX_ERR_HINT_OVERFLOW;
        else wt.hints_len = hint_base + blk * nwit;
        wtx_store(wt, a.tx);
    }
}

int launch_open(const OpenArgs& a, cudaStream_t st) {
    if (a.q > (u32)MAX_QUERIES || (1u << a.fold) > (u32)MAX_DEPTH || a.nwit < 1 || a.nwit > (u32)MAX_WITNESSES) return -1;
    if (a.stir && (a.depth & ((1u << a.fold) - 1)) != 0) return -1;
    k_open<<<1, OPEN_THREADS, 0, st>>>(a);
    count_launches(1);
    return 0;
}

// STIR combination: the new commitment's OOD points/values first, then the
// in-domain ones written by k_open; RLC = geometric_challenge(O + q);
// sum += <rlc, values>.
// One warp.
__global__ void k_stir_rlc(TxState* tx, ProofScalars* sc, int commit_idx, int n_ood, int q) {
    if (threadIdx.x >= 32) return;
    const int l = threadIdx.x;
    if (l < n_ood) {
        sc->stir_pts[l] = sc->ood_pts[commit_idx][l];
        sc->stir_vals[l] = sc->ood_vals[commit_idx][l];
    }
    __syncwarp();
    const int count = n_ood + q;
    WarpTx t;
    wtx_load(t, tx);
    wtx_geometric(t, sc->stir_rlc, count);
    wtx_store(t, tx);
    E3 acc = e3_zero();
    for (int j = l; j < count; j += 32) acc = e3_add(acc, ef_mul(sc->stir_rlc[j], sc->stir_vals[j], t.deg == 2));
    acc = wtx_sum(acc);
    if (l == 0) sc->sum = e3_add(sc->sum, acc);
}

int launch_stir_rlc(TxState* tx, ProofScalars* sc, int commit_idx, int n_ood, int q, cudaStream_t st) {
    if (n_ood > MAX_OOD || q > MAX_QUERIES) return -1;
    k_stir_rlc<<<1, 32, 0, st>>>(tx, sc, commit_idx, n_ood, q);
    count_launches(1);
    return 0;
}

}  // namespace wg
