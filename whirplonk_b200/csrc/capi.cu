// capi.cu -- implementation of the C ABI declared in include/whirgpu.h.
//
// Owns the CUDA context state (device, stream, twiddle tables, workspace
// cache bounded by an HBM budget, pinned staging for proof read-back) and maps
// every failure to a status code plus a message (no exceptions cross the ABI).
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/whirgpu.h"
#include "ctx.h"
#include "host_keccak.h"
#include "launch.h"
#include "prover.h"
#include "state.cuh"

using namespace wg;

namespace {

// ---------------------------------------------------------------------------
// Host SHA3 (FIPS 202) for the domain-separator helpers, on the table-driven
// host permutation of host_keccak.cpp.
// ---------------------------------------------------------------------------
void sha3_host(const uint8_t* d, size_t n, size_t rate, uint8_t* out, size_t outlen) {
    uint64_t s[25] = {};
    size_t pos = 0;
    auto xb = [&](size_t p, uint8_t v) { s[p / 8] ^= (uint64_t)v << (8 * (p % 8)); };
    for (size_t i = 0; i < n; ++i) {
        xb(pos++, d[i]);
        if (pos == rate) { keccak_f1600_cpu(s); pos = 0; }
    }
    xb(pos, 0x06);
    xb(rate - 1, 0x80);
    keccak_f1600_cpu(s);
    for (size_t i = 0; i < outlen; ++i) out[i] = (uint8_t)(s[i / 8] >> (8 * (i % 8)));
}

void cbor_head(std::vector<uint8_t>& o, uint8_t major, uint64_t v) {
    const uint8_t m = (uint8_t)(major << 5);
    if (v < 24) o.push_back(m | (uint8_t)v);
    else if (v <= 0xFF) { o.push_back(m | 24); o.push_back((uint8_t)v); }
    else if (v <= 0xFFFF) { o.push_back(m | 25); for (int s = 8; s >= 0; s -= 8) o.push_back((uint8_t)(v >> s)); }
    else if (v <= 0xFFFFFFFFull) { o.push_back(m | 26); for (int s = 24; s >= 0; s -= 8) o.push_back((uint8_t)(v >> s)); }
    else { o.push_back(m | 27); for (int s = 56; s >= 0; s -= 8) o.push_back((uint8_t)(v >> s)); }
}
void cbor_text(std::vector<uint8_t>& o, const char* s) {
    const size_t n = std::strlen(s);
    cbor_head(o, 3, n);
    o.insert(o.end(), s, s + n);
}

// ---------------------------------------------------------------------------
// ChaCha20 block function (RFC 8439 section 2.3).
// ---------------------------------------------------------------------------
inline uint32_t rotl32(uint32_t v, int s) { return (v << s) | (v >> (32 - s)); }
#define WG_QR(a, b, c, d)                   \
    a += b; d ^= a; d = rotl32(d, 16);      \
    c += d; b ^= c; b = rotl32(b, 12);      \
    a += b; d ^= a; d = rotl32(d, 8);       \
    c += d; b ^= c; b = rotl32(b, 7);
void chacha20_words(const uint32_t key[8], uint32_t counter, const uint32_t nonce[3], uint32_t out[16]) {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                      key[4], key[5], key[6], key[7], counter, nonce[0], nonce[1], nonce[2]};
    uint32_t x[16];
    for (int i = 0; i < 16; ++i) x[i] = s[i];
    for (int i = 0; i < 10; ++i) {
        WG_QR(x[0], x[4], x[8], x[12]);
        WG_QR(x[1], x[5], x[9], x[13]);
        WG_QR(x[2], x[6], x[10], x[14]);
        WG_QR(x[3], x[7], x[11], x[15]);
        WG_QR(x[0], x[5], x[10], x[15]);
        WG_QR(x[1], x[6], x[11], x[12]);
        WG_QR(x[2], x[7], x[8], x[13]);
        WG_QR(x[3], x[4], x[9], x[14]);
    }
    for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

}  // namespace

namespace wg {

whirgpu_status fail(whirgpu_ctx* c, whirgpu_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}
whirgpu_status cuda_fail(whirgpu_ctx* c, cudaError_t e, const char* what) {
    return fail(c, e == cudaErrorMemoryAllocation ? WHIRGPU_E_OOM : WHIRGPU_E_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}
#define WG_CUDA(c, x, what)                               \
    do {                                                  \
        cudaError_t _e = (x);                             \
        if (_e != cudaSuccess) return cuda_fail(c, _e, what); \
    } while (0)

whirgpu_status ensure_pinned(whirgpu_ctx* c, size_t bytes) {
    if (c->pinned_bytes >= bytes) return WHIRGPU_OK;
    if (c->pinned) cudaFreeHost(c->pinned);
    c->pinned = nullptr;
    c->pinned_bytes = 0;
    WG_CUDA(c, cudaMallocHost(&c->pinned, bytes), "cudaMallocHost");
    c->pinned_bytes = bytes;
    return WHIRGPU_OK;
}

namespace {

void free_workspace(whirgpu_ctx* c, Workspace* w) {
    for (auto& kv : w->on_free) kv.second();
    for (auto& kv : w->plain_graphs) cudaGraphExecDestroy(kv.second.exec);
    cudaFree(w->dev);
    c->allocated -= w->plan.total_bytes;
    delete w;
}

// Runs `enqueue(stream, timer)` on the context stream.  Without the family
// timer the kernels are captured into a graph on the first call with `key`
// for this workspace (and NTT plan epoch) and replayed from then on: one graph
// launch instead of ~100 kernel launches per proof.  Returns 0 on success.
template <class F>
int run_captured(whirgpu_ctx* c, Workspace* ws, uint64_t key, F enqueue) {
    if (c->timer) return enqueue(c->stream, c->timer.get());
    const uint32_t epoch = lde_plan_epoch();
    key = key << 32 | epoch;
    auto it = ws->plain_graphs.find(key);
    if (it == ws->plain_graphs.end()) {
        for (auto jt = ws->plain_graphs.begin(); jt != ws->plain_graphs.end();) {  // captured under older plans
            if ((uint32_t)jt->first != epoch) {
                cudaGraphExecDestroy(jt->second.exec);
                jt = ws->plain_graphs.erase(jt);
            } else {
                ++jt;
            }
        }
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -1;
        set_capturing(true);
        const int rc = enqueue(c->stream, nullptr);
        set_capturing(false);
        const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
        Workspace::Captured cap;
        if (rc == 0 && ce == cudaSuccess) {
            cap.kernels = graph_kernel_nodes(g);
            if (cudaGraphInstantiate(&cap.exec, g, 0) != cudaSuccess) cap.exec = nullptr;
        }
        if (g) cudaGraphDestroy(g);
        if (!cap.exec) {  // not capturable: launch directly
            cudaGetLastError();
            return rc ? rc : enqueue(c->stream, nullptr);
        }
        it = ws->plain_graphs.emplace(key, cap).first;
    }
    count_launches(it->second.kernels);
    return cudaGraphLaunch(it->second.exec, c->stream) == cudaSuccess ? 0 : -1;
}

// Frees idle workspaces, least recently used first, until `need` more bytes
// fit under `limit` (all idle ones when limit is 0).  Returns whether they fit.
bool evict_idle(whirgpu_ctx* c, uint64_t need, uint64_t limit) {
    for (;;) {
        if (limit && c->allocated + need <= limit) return true;
        Workspace* victim = nullptr;
        std::vector<Workspace*>* owner = nullptr;
        for (auto& kv : c->cache)
            for (Workspace* w : kv.second)
                if (!w->busy && (!victim || w->last_used < victim->last_used)) { victim = w; owner = &kv.second; }
        if (!victim) return limit == 0;
        owner->erase(std::find(owner->begin(), owner->end(), victim));
        free_workspace(c, victim);
        ++c->ws_evictions;
    }
}

}  // namespace

namespace {
// Serialised plan shape: equal keys give equal plans.
std::string plan_key(const WhirSchedule& s, const ProtocolParams& pp, size_t ds_len, uint32_t nwit) {
    std::vector<uint64_t> w{s.initial.vector_size, s.initial.codeword_length, s.initial.depth, s.initial.in_domain,
                            s.initial.out_domain, s.initial_sumcheck.num_rounds, s.initial_sumcheck.pow_threshold,
                            s.initial_skip_pow, s.rounds.size()};
    for (const RoundSchedule& r : s.rounds)
        w.insert(w.end(), {r.irs.vector_size, r.irs.codeword_length, r.irs.depth, r.irs.in_domain, r.irs.out_domain,
                           r.pow_threshold, r.sumcheck.num_rounds, r.sumcheck.pow_threshold});
    w.insert(w.end(), {s.final_sumcheck.num_rounds, s.final_sumcheck.pow_threshold, s.final_pow, pp.batch_size,
                       (uint64_t)pp.hash, (uint64_t)pp.field_degree, (uint64_t)std::max<size_t>(ds_len, 96), nwit,
                       (uint64_t)pp.coset_major});
    return std::string(reinterpret_cast<const char*>(w.data()), w.size() * sizeof(uint64_t));
}
}  // namespace

whirgpu_status acquire_workspace(whirgpu_ctx* c, uint64_t n, const whirgpu_params* params, size_t ds_len, Workspace** out,
                                 uint64_t cap, uint32_t nwit) {
    WhirSchedule sched;
    try {
        sched = make_schedule(n, to_params(params));
    } catch (const std::exception& e) {
        return fail(c, WHIRGPU_E_INVALID, e.what());
    }
    return acquire_workspace_sched(c, sched, to_params(params), ds_len, out, cap, nwit);
}

// The inter-pass twiddle tables of every LDE split `plan` launches (built once
// per context and split, before any proof of the plan is enqueued or captured).
// Like the other twiddle tables they sit outside the workspace budget; under a
// budget a table is only built while it fits beside the workspaces, else the
// passes generate their factors.
void prepare_lde_tables(whirgpu_ctx* c, const ProofPlan& plan) {
    for (const CommitBuffers& cb : plan.commits) {
        const uint64_t room = c->budget ? (c->budget > c->allocated ? c->budget - c->allocated : 0) : ~0ull;
        lde_tables_prepare(c->lde_tables, cb.logN, cb.logX, c->tw.tw_hi, c->tw.tw_lo, c->stream, room);
    }
}

whirgpu_status acquire_workspace_sched(whirgpu_ctx* c, const WhirSchedule& sched, const ProtocolParams& pp_in,
                                       size_t ds_len, Workspace** out, uint64_t cap, uint32_t nwit) {
    ProtocolParams pp = pp_in;
    pp.coset_major = c->codeword_order == WHIRGPU_ORDER_COSET_MAJOR ? 1 : 0;
    ProofPlan plan;
    try {
        plan = make_plan(sched, pp, MAX_FORMS, std::max<size_t>(ds_len, 96), nwit);
    } catch (const std::exception& e) {
        return fail(c, WHIRGPU_E_INVALID, e.what());
    }
    const std::string key = plan_key(sched, pp, ds_len, nwit);
    std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
    prepare_lde_tables(c, plan);
    for (Workspace* w : c->cache[key])
        if (!w->busy) {
            w->busy = true;
            w->last_used = ++c->use_clock;
            *out = w;
            return WHIRGPU_OK;
        }
    uint64_t limit = c->budget;
    if (cap && (!limit || cap < limit)) limit = cap;
    if (limit && !evict_idle(c, plan.total_bytes, limit)) return fail(c, WHIRGPU_E_OOM, "workspace above the HBM budget");
    Workspace* w = new Workspace();
    w->plan = plan;
    cudaError_t e = cudaMalloc(&w->dev, plan.total_bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        evict_idle(c, plan.total_bytes, 0);
        e = cudaMalloc(&w->dev, plan.total_bytes);
    }
    if (e != cudaSuccess) { delete w; return cuda_fail(c, e, "cudaMalloc workspace"); }
    // Counters and tickets start at zero and reset themselves after use.
    e = cudaMemsetAsync(w->dev + plan.off_sc_scratch, 0, plan.off_tx - plan.off_sc_scratch, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { cudaFree(w->dev); delete w; return cuda_fail(c, e, "cudaMemset"); }
    c->allocated += plan.total_bytes;
    ++c->ws_allocations;
    w->busy = true;
    w->last_used = ++c->use_clock;
    c->cache[key].push_back(w);
    *out = w;
    return WHIRGPU_OK;
}

bool is_blake3(const whirgpu_params* p) { return std::memcmp(p->hash_id, BLAKE3_ENGINE_ID, 32) == 0; }
bool is_sha2(const whirgpu_params* p) { return std::memcmp(p->hash_id, SHA2_ENGINE_ID, 32) == 0; }
bool engine_supported(const whirgpu_params* p) { return is_blake3(p) || is_sha2(p); }

void release_workspace(whirgpu_ctx* c, Workspace* w) {
    if (!w) return;
    std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
    w->busy = false;
}

size_t workspace_bytes(uint64_t n, const whirgpu_params* params, uint32_t nwit) {
    try {
        return make_plan((uint32_t)n, to_params(params), MAX_FORMS, 96, nwit).total_bytes;
    } catch (const std::exception&) {
        return 0;
    }
}

ProtocolParams to_params(const whirgpu_params* p) {
    ProtocolParams q;
    q.unique_decoding = p->unique_decoding != 0;
    q.starting_log_inv_rate = p->starting_log_inv_rate;
    q.initial_folding_factor = p->initial_folding_factor;
    q.folding_factor = p->folding_factor;
    q.security_level = p->security_level;
    q.pow_bits = p->pow_bits;
    q.batch_size = p->batch_size;
    q.hash = is_sha2(p) ? 1 : 0;
    return q;
}

}  // namespace wg

extern "C" {

whirgpu_status whirgpu_ctx_create(int device, uint64_t hbm_budget, whirgpu_ctx** out) {
    if (!out) return WHIRGPU_E_INVALID;
    *out = nullptr;
    auto c = std::make_unique<whirgpu_ctx>();
    c->device = device;
    c->budget = hbm_budget;
    WG_CUDA(nullptr, cudaSetDevice(device), "cudaSetDevice");
    WG_CUDA(nullptr, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (lde_prepare() != 0 || sumcheck_prepare() != 0) return WHIRGPU_E_CUDA;
    whirgpu_ntt_load_default_plans();
    std::vector<uint64_t> st(1u << (TW_STAGE_LOG - 1)), hi(1u << TW_HALF), lo(1u << TW_HALF);
    host_twiddles(st.data(), hi.data(), lo.data());
    WG_CUDA(nullptr, cudaMalloc(&c->tw.tw_stage, st.size() * 8), "cudaMalloc twiddles");
    WG_CUDA(nullptr, cudaMalloc(&c->tw.tw_hi, hi.size() * 8), "cudaMalloc twiddles");
    WG_CUDA(nullptr, cudaMalloc(&c->tw.tw_lo, lo.size() * 8), "cudaMalloc twiddles");
    WG_CUDA(nullptr, cudaMemcpy(c->tw.tw_stage, st.data(), st.size() * 8, cudaMemcpyHostToDevice), "upload");
    WG_CUDA(nullptr, cudaMemcpy(c->tw.tw_hi, hi.data(), hi.size() * 8, cudaMemcpyHostToDevice), "upload");
    WG_CUDA(nullptr, cudaMemcpy(c->tw.tw_lo, lo.data(), lo.size() * 8, cudaMemcpyHostToDevice), "upload");
    c->tw.lde = &c->lde_tables;
    *out = c.release();
    return WHIRGPU_OK;
}

void whirgpu_ctx_destroy(whirgpu_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    {
        std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
        for (whirgpu_witness* w : c->live_witnesses) {  // their workspaces are freed below
            w->ws = nullptr;
            w->ctx = nullptr;
        }
        c->live_witnesses.clear();
    }
    zk_detach_all(c);
    for (auto& kv : c->cache)
        for (Workspace* w : kv.second) free_workspace(c, w);
    cudaFree(c->tw.tw_stage);
    cudaFree(c->tw.tw_hi);
    cudaFree(c->tw.tw_lo);
    lde_tables_free(c->lde_tables);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->mle_scratch) cudaFree(c->mle_scratch);
    if (c->kscratch) cudaFree(c->kscratch);
    c->timer.reset();
    cudaStreamDestroy(c->stream);
    delete c;
}

const char* whirgpu_last_error(const whirgpu_ctx* c) { return c ? c->err.c_str() : "no context"; }
void* whirgpu_stream(whirgpu_ctx* c) { return c ? (void*)c->stream : nullptr; }

whirgpu_status whirgpu_set_codeword_order(whirgpu_ctx* c, int order) {
    if (!c) return WHIRGPU_E_INVALID;
    if (order != WHIRGPU_ORDER_NATURAL && order != WHIRGPU_ORDER_COSET_MAJOR)
        return fail(c, WHIRGPU_E_INVALID, "unknown codeword order");
    c->codeword_order = order;
    return WHIRGPU_OK;
}

size_t whirgpu_schedule(const whirgpu_params* params, uint64_t n, uint64_t* out, size_t cap) {
    if (!params) return 0;
    try {
        WhirSchedule s = make_schedule(n, to_params(params));
        std::vector<uint64_t> v{s.rounds.size(), s.initial.codeword_length, s.initial.in_domain, s.initial.out_domain,
                                s.initial_sumcheck.pow_threshold, s.initial_skip_pow};
        for (const auto& r : s.rounds)
            v.insert(v.end(), {r.irs.vector_size, r.irs.codeword_length, r.irs.in_domain, r.irs.out_domain,
                               r.pow_threshold, r.sumcheck.pow_threshold});
        v.insert(v.end(), {s.final_sumcheck.initial_size, s.final_sumcheck.num_rounds, s.final_pow,
                           s.final_sumcheck.pow_threshold});
        for (size_t i = 0; i < v.size() && i < cap; ++i) out[i] = v[i];
        return v.size();
    } catch (const std::exception&) {
        return 0;
    }
}

uint64_t whirgpu_workspace_bytes(const whirgpu_params* params, uint64_t n) {
    return params ? workspace_bytes(n, params) : 0;
}

whirgpu_status whirgpu_cli_domain_separator(const whirgpu_params* p, uint8_t out[96]) {
    if (!p || !out) return WHIRGPU_E_INVALID;
    std::vector<uint8_t> c;
    cbor_head(c, 5, 8);
    cbor_text(c, "unique_decoding");
    c.push_back(p->unique_decoding ? 0xF5 : 0xF4);
    cbor_text(c, "starting_log_inv_rate"); cbor_head(c, 0, p->starting_log_inv_rate);
    cbor_text(c, "initial_folding_factor"); cbor_head(c, 0, p->initial_folding_factor);
    cbor_text(c, "folding_factor"); cbor_head(c, 0, p->folding_factor);
    cbor_text(c, "security_level"); cbor_head(c, 0, p->security_level);
    cbor_text(c, "pow_bits"); cbor_head(c, 0, p->pow_bits);
    cbor_text(c, "batch_size"); cbor_head(c, 0, p->batch_size);
    cbor_text(c, "hash_id"); cbor_head(c, 4, 32);
    for (int i = 0; i < 32; ++i) cbor_head(c, 0, p->hash_id[i]);
    sha3_host(c.data(), c.size(), 72, out, 64);
    std::vector<uint8_t> s;
    cbor_text(s, "Example at src/bin/main.rs:133");
    sha3_host(s.data(), s.size(), 136, out + 64, 32);
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_zk_domain_separator(const whirgpu_params* p, uint64_t vector_size, uint64_t num_polynomials,
                                          const whirgpu_zk_policy* policy, const char* session, size_t session_len,
                                          uint8_t* config_bytes, uint8_t out[96]) {
    if (!p || !out || (session_len && !session)) return WHIRGPU_E_INVALID;
    const whirgpu_zk_policy pol = policy ? *policy : zk_default_policy(p);
    std::vector<uint8_t> c;
    auto u64le = [&c](uint64_t v) {
        for (int i = 0; i < 8; ++i) c.push_back((uint8_t)(v >> (8 * i)));
    };
    static const char kMagic[] = "WHIR_ZK_CONFIG_V1";
    c.insert(c.end(), kMagic, kMagic + sizeof(kMagic) - 1);
    u64le(vector_size);
    u64le(num_polynomials);
    c.push_back(p->unique_decoding ? 1 : 0);
    for (uint64_t v : {p->starting_log_inv_rate, p->initial_folding_factor, p->folding_factor, p->security_level,
                       p->pow_bits, p->batch_size})
        u64le(v);
    c.insert(c.end(), p->hash_id, p->hash_id + 32);
    for (uint64_t v : {pol.q_delta_1, pol.q_delta_2, pol.t1, pol.t2, pol.sumcheck_round_degree}) u64le(v);
    if (config_bytes) std::memcpy(config_bytes, c.data(), c.size());
    sha3_host(c.data(), c.size(), 72, out, 64);
    std::vector<uint8_t> s;
    cbor_head(s, 3, session_len);
    s.insert(s.end(), session, session + session_len);
    sha3_host(s.data(), s.size(), 136, out + 64, 32);
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_transcript_create(whirgpu_ctx* ctx, const uint8_t protocol_id[64], const uint8_t session_id[32],
                                         const uint8_t* instance, size_t instance_len, whirgpu_transcript** out) {
    if (!ctx || !protocol_id || !session_id || !out || (instance_len && !instance)) return WHIRGPU_E_INVALID;
    auto t = new whirgpu_transcript();
    t->ctx = ctx;
    t->ds.insert(t->ds.end(), protocol_id, protocol_id + 64);
    t->ds.insert(t->ds.end(), session_id, session_id + 32);
    if (instance_len) t->ds.insert(t->ds.end(), instance, instance + instance_len);
    *out = t;
    return WHIRGPU_OK;
}

void whirgpu_transcript_destroy(whirgpu_transcript* t) { delete t; }

whirgpu_status whirgpu_proof_get(const whirgpu_transcript* t, const uint8_t** narg, size_t* narg_len,
                                 const uint8_t** hints, size_t* hints_len) {
    if (!t || !t->complete) return WHIRGPU_E_INVALID;
    if (narg) *narg = t->narg.data();
    if (narg_len) *narg_len = t->narg.size();
    if (hints) *hints = t->hints.data();
    if (hints_len) *hints_len = t->hints.size();
    return WHIRGPU_OK;
}

namespace {
// Commit of num_witnesses witnesses for a schedule (from params or given).
whirgpu_status commit_schedule(whirgpu_ctx* c, const WhirSchedule& sched, const ProtocolParams& pp,
                               const uint64_t* coeffs, uint64_t num_witnesses, int where, whirgpu_transcript* tx,
                               whirgpu_witness** out) {
    if (pp.batch_size == 0 || num_witnesses == 0) return fail(c, WHIRGPU_E_INVALID, "no vectors to commit");
    if (num_witnesses > (uint64_t)MAX_WITNESSES || pp.batch_size * num_witnesses > (uint64_t)MAX_VECTORS)
        return fail(c, WHIRGPU_E_UNSUPPORTED, "more committed vectors than this path holds");
    Workspace* ws = nullptr;
    whirgpu_status s = acquire_workspace_sched(c, sched, pp, tx->ds.size(), &ws, 0, (uint32_t)num_witnesses);
    if (s != WHIRGPU_OK) return s;
    const ProofPlan& p = ws->plan;
    const size_t coeff_bytes = (size_t)p.nvec * (8ull << p.n);
    cudaError_t e = cudaMemcpyAsync(ws->dev + p.off_coeffs, coeffs, coeff_bytes,
                                    where == WHIRGPU_INPUT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                    c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ws->dev + p.off_ds, tx->ds.data(), tx->ds.size(), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) { release_workspace(c, ws); return cuda_fail(c, e, "input copy"); }
    c->io_h2d = (where == WHIRGPU_INPUT_DEVICE ? 0 : coeff_bytes) + tx->ds.size();
    c->io_d2h = 0;
    const uint32_t ds_len = (uint32_t)tx->ds.size();
    if (run_captured(c, ws, (uint64_t)ds_len << 8 | 0x1,
                     [&](cudaStream_t st, Timer* tm) { return enqueue_commit(p, ws->dev, ds_len, c->tw, st, tm); }) != 0) {
        release_workspace(c, ws);
        return fail(c, WHIRGPU_E_INVALID, "commit launch failed");
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) { release_workspace(c, ws); return cuda_fail(c, e, "commit kernels"); }
    auto w = new whirgpu_witness();
    w->ctx = c;
    w->ws = ws;
    w->tx = tx;
    tx->complete = false;
    {
        std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
        c->live_witnesses.insert(w);
    }
    *out = w;
    return WHIRGPU_OK;
}

void to_irs(const IrsSchedule& a, whirgpu_irs_config& b) {
    b = {a.vector_size, a.codeword_length, a.depth, a.in_domain, a.out_domain};
}
IrsSchedule from_irs(const whirgpu_irs_config& b) {
    IrsSchedule a;
    a.vector_size = b.vector_size;
    a.codeword_length = b.codeword_length;
    a.depth = b.interleaving_depth;
    a.in_domain = b.in_domain_samples;
    a.out_domain = b.out_domain_samples;
    return a;
}
}  // namespace

whirgpu_status whirgpu_config_from_params(const whirgpu_params* params, uint64_t n, uint32_t field, whirgpu_config* out) {
    if (!params || !out || (field != WHIRGPU_FIELD_GOLDILOCKS1 && field != WHIRGPU_FIELD_GOLDILOCKS2 &&
                            field != WHIRGPU_FIELD_GOLDILOCKS3))
        return WHIRGPU_E_INVALID;
    ProtocolParams pp = to_params(params);
    pp.field_degree = (int)field;
    WhirSchedule s;
    try {
        s = make_schedule(n, pp);
    } catch (const std::exception&) {
        return WHIRGPU_E_INVALID;
    }
    if (s.rounds.size() > WHIRGPU_MAX_ROUNDS) return WHIRGPU_E_UNSUPPORTED;
    std::memset(out, 0, sizeof(*out));
    out->field = field;
    out->batch_size = params->batch_size;
    std::memcpy(out->hash_id, params->hash_id, 32);
    to_irs(s.initial, out->initial_committer);
    out->initial_sumcheck = {s.initial_sumcheck.num_rounds, s.initial_sumcheck.pow_threshold};
    out->initial_skip_pow = s.initial_skip_pow;
    out->num_rounds = s.rounds.size();
    for (size_t r = 0; r < s.rounds.size(); ++r) {
        to_irs(s.rounds[r].irs, out->round_configs[r].irs_committer);
        out->round_configs[r].pow_threshold = s.rounds[r].pow_threshold;
        out->round_configs[r].sumcheck = {s.rounds[r].sumcheck.num_rounds, s.rounds[r].sumcheck.pow_threshold};
    }
    out->final_sumcheck = {s.final_sumcheck.num_rounds, s.final_sumcheck.pow_threshold};
    out->final_pow = s.final_pow;
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_commit_config(whirgpu_ctx* c, const whirgpu_config* cfg, const uint64_t* coeffs,
                                     uint64_t num_witnesses, int where, whirgpu_transcript* tx, whirgpu_witness** out) {
    if (!c || !cfg || !coeffs || !tx || !out || tx->ctx != c) return fail(c, WHIRGPU_E_INVALID, "null argument");
    *out = nullptr;
    if (cfg->field != WHIRGPU_FIELD_GOLDILOCKS1 && cfg->field != WHIRGPU_FIELD_GOLDILOCKS2 &&
        cfg->field != WHIRGPU_FIELD_GOLDILOCKS3)
        return fail(c, WHIRGPU_E_INVALID, "unknown field");
    if (cfg->num_rounds > WHIRGPU_MAX_ROUNDS) return fail(c, WHIRGPU_E_INVALID, "too many rounds");
    whirgpu_params hp{};
    hp.batch_size = cfg->batch_size;
    std::memcpy(hp.hash_id, cfg->hash_id, 32);
    if (!engine_supported(&hp)) return fail(c, WHIRGPU_E_UNSUPPORTED, "only the BLAKE3 and SHA-2 engines are on this path");
    ProtocolParams pp;
    pp.batch_size = cfg->batch_size;
    pp.hash = is_sha2(&hp) ? 1 : 0;
    pp.field_degree = (int)cfg->field;
    const WhirSchedule s = schedule_from_config(cfg);
    return commit_schedule(c, s, pp, coeffs, num_witnesses, where, tx, out);
}

}  // extern "C"

namespace wg {
WhirSchedule schedule_from_config(const whirgpu_config* cfg) {
    WhirSchedule s;
    s.initial = from_irs(cfg->initial_committer);
    s.initial_sumcheck = {s.initial.vector_size, cfg->initial_sumcheck.num_rounds, cfg->initial_sumcheck.pow_threshold};
    s.initial_skip_pow = cfg->initial_skip_pow;
    uint64_t size = cfg->initial_sumcheck.num_rounds < 64 ? s.initial.vector_size >> cfg->initial_sumcheck.num_rounds : 0;
    for (uint64_t r = 0; r < cfg->num_rounds; ++r) {
        const whirgpu_round_config& rc = cfg->round_configs[r];
        RoundSchedule q;
        q.irs = from_irs(rc.irs_committer);
        q.pow_threshold = rc.pow_threshold;
        q.sumcheck = {size, rc.sumcheck.num_rounds, rc.sumcheck.pow_threshold};
        size = rc.sumcheck.num_rounds < 64 ? size >> rc.sumcheck.num_rounds : 0;
        s.rounds.push_back(q);
    }
    s.final_sumcheck = {size, cfg->final_sumcheck.num_rounds, cfg->final_sumcheck.pow_threshold};
    s.final_pow = cfg->final_pow;
    int n = 0;
    while (n < 40 && (1ull << n) < s.initial.vector_size) ++n;
    s.num_variables = (uint64_t)n;
    return s;
}
}  // namespace wg

extern "C" {

whirgpu_status whirgpu_commit_witnesses(whirgpu_ctx* c, const whirgpu_params* params, const uint64_t* coeffs,
                                        uint64_t num_witnesses, uint64_t n, int where, whirgpu_transcript* tx,
                                        whirgpu_witness** out) {
    if (!c || !params || !coeffs || !tx || !out || tx->ctx != c) return fail(c, WHIRGPU_E_INVALID, "null argument");
    *out = nullptr;
    if (!engine_supported(params)) return fail(c, WHIRGPU_E_UNSUPPORTED, "only the BLAKE3 and SHA-2 engines are on this path");
    if (n >= 40) return fail(c, WHIRGPU_E_INVALID, "num_variables too large");
    WhirSchedule s;
    try {
        s = make_schedule(n, to_params(params));
    } catch (const std::exception& e) {
        return fail(c, WHIRGPU_E_INVALID, e.what());
    }
    return commit_schedule(c, s, to_params(params), coeffs, num_witnesses, where, tx, out);
}

whirgpu_status whirgpu_commit(whirgpu_ctx* c, const whirgpu_params* params, const uint64_t* coeffs, uint64_t n,
                              int where, whirgpu_transcript* tx, whirgpu_witness** out) {
    return whirgpu_commit_witnesses(c, params, coeffs, 1, n, where, tx, out);
}

void whirgpu_witness_destroy(whirgpu_witness* w) {
    if (!w) return;
    if (w->ctx) {
        if (w->ws) {
            cudaStreamSynchronize(w->ctx->stream);
            release_workspace(w->ctx, w->ws);
        }
        std::lock_guard<std::recursive_mutex> lk(w->ctx->cache_mu);
        w->ctx->live_witnesses.erase(w);
    }
    delete w;
}

namespace {
// Device buffer for the host covectors of one prove call, freed on every return path.
struct TempDevice {
    void* p = nullptr;
    ~TempDevice() {
        if (p) cudaFree(p);
    }
};
}  // namespace

whirgpu_status whirgpu_prove_forms(whirgpu_ctx* c, whirgpu_witness* w, const whirgpu_linear_form* forms,
                                   size_t num_points, const uint64_t* evaluations, whirgpu_transcript* tx,
                                   uint64_t* evaluation_point, uint64_t* rlc) {
    if (!c || !w || !tx || w->ctx != c || w->tx != tx || !w->ws) return fail(c, WHIRGPU_E_INVALID, "bad handles");
    if (num_points > (size_t)MAX_FORMS || (num_points && (!forms || !evaluations)))
        return fail(c, WHIRGPU_E_INVALID, "bad statement");
    ProofPlan p = w->ws->plan;
    plan_set_forms(p, (int)num_points);
    const size_t cov_bytes = (size_t)24 << p.n;
    size_t host_dense = 0;
    for (size_t f = 0; f < num_points; ++f) {
        if (!forms[f].data || forms[f].kind > WHIRGPU_FORM_COVECTOR) return fail(c, WHIRGPU_E_INVALID, "bad linear form");
        if (forms[f].kind == WHIRGPU_FORM_COVECTOR && forms[f].location != WHIRGPU_INPUT_DEVICE) ++host_dense;
    }
    char* ws = w->ws->dev;
    ProofScalars* sc = plan_scalars(p, ws);
    TempDevice tmp;
    if (host_dense) WG_CUDA(c, cudaMalloc(&tmp.p, host_dense * cov_bytes), "cudaMalloc covectors");
    cudaError_t e = cudaSuccess;
    size_t slot = 0;
    for (size_t f = 0; f < num_points && e == cudaSuccess; ++f) {
        if (forms[f].kind == WHIRGPU_FORM_MLE) {
            e = cudaMemcpyAsync(ws + p.off_points + f * p.n * 24, forms[f].data, p.n * 24, cudaMemcpyHostToDevice,
                                c->stream);
            c->io_h2d += p.n * 24;
            continue;
        }
        p.dense_mask |= 1u << f;
        if (forms[f].location == WHIRGPU_INPUT_DEVICE) {
            p.dense[f] = forms[f].data;
        } else {
            uint64_t* dst = reinterpret_cast<uint64_t*>(static_cast<char*>(tmp.p) + slot++ * cov_bytes);
            e = cudaMemcpyAsync(dst, forms[f].data, cov_bytes, cudaMemcpyHostToDevice, c->stream);
            p.dense[f] = dst;
            c->io_h2d += cov_bytes;
        }
    }
    if (e == cudaSuccess && num_points) {
        e = cudaMemcpyAsync(&sc->forms_eval[0], evaluations, num_points * p.nvec * 24, cudaMemcpyHostToDevice,
                            c->stream);
        c->io_h2d += num_points * p.nvec * 24;
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "statement upload");
    // Statements with dense covectors name caller memory: launched directly.
    const int rc = p.dense_mask ? enqueue_prove(p, ws, c->tw, c->stream, c->timer.get())
                                : run_captured(c, w->ws, (uint64_t)num_points << 8 | 0x2, [&](cudaStream_t st, Timer* tm) {
                                      return enqueue_prove(p, ws, c->tw, st, tm);
                                  });
    if (rc != 0) return fail(c, WHIRGPU_E_INVALID, "prove launch failed");
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "prove kernels");
    // Read-back: transcript state, narg (exact size), hints (bounded), challenges.
    const size_t need = sizeof(TxState) + p.narg_len + p.hints_cap + 64 * 24 + MAX_FORMS * 24 + 64;
    whirgpu_status s = ensure_pinned(c, need);
    if (s != WHIRGPU_OK) return s;
    uint8_t* h = c->pinned;
    TxState* htx = reinterpret_cast<TxState*>(h);
    uint8_t* hnarg = h + sizeof(TxState);
    uint8_t* hhints = hnarg + p.narg_len;
    uint8_t* hr = hhints + p.hints_cap;
    uint8_t* hrlc = hr + 64 * 24;
    WG_CUDA(c, cudaMemcpyAsync(htx, plan_tx(p, ws), sizeof(TxState), cudaMemcpyDeviceToHost, c->stream), "read-back");
    WG_CUDA(c, cudaMemcpyAsync(hnarg, ws + p.off_narg, p.narg_len, cudaMemcpyDeviceToHost, c->stream), "read-back");
    WG_CUDA(c, cudaMemcpyAsync(hhints, ws + p.off_hints, p.hints_cap, cudaMemcpyDeviceToHost, c->stream), "read-back");
    WG_CUDA(c, cudaMemcpyAsync(hr, &sc->sc_r[0], p.total_sumcheck_rounds * 24, cudaMemcpyDeviceToHost, c->stream),
            "read-back");
    WG_CUDA(c, cudaMemcpyAsync(hrlc, &sc->crlc[0], std::max<size_t>(num_points, 1) * 24, cudaMemcpyDeviceToHost, c->stream),
            "read-back");
    WG_CUDA(c, cudaStreamSynchronize(c->stream), "prove");
    c->io_d2h += sizeof(TxState) + p.narg_len + p.hints_cap + p.total_sumcheck_rounds * 24 +
                 std::max<size_t>(num_points, 1) * 24;
    if (c->timer) {
        c->timer->harvest();
    }
    if (htx->err) {
        char buf[96];
        std::snprintf(buf, sizeof buf, "device error word 0x%x", htx->err);
        return fail(c, WHIRGPU_E_DEVICE, buf);
    }
    if (htx->narg_len != p.narg_len || htx->hints_len > p.hints_cap)
        return fail(c, WHIRGPU_E_DEVICE, "proof stream length mismatch");
    tx->narg.assign(hnarg, hnarg + p.narg_len);
    tx->hints.assign(hhints, hhints + htx->hints_len);
    tx->complete = true;
    if (evaluation_point) std::memcpy(evaluation_point, hr, p.total_sumcheck_rounds * 24);
    if (rlc && num_points) std::memcpy(rlc, hrlc, num_points * 24);
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_prove(whirgpu_ctx* c, whirgpu_witness* w, const uint64_t* points, size_t num_points,
                             const uint64_t* evaluations, whirgpu_transcript* tx, uint64_t* evaluation_point,
                             uint64_t* rlc) {
    if (!c || !w || !w->ws) return fail(c, WHIRGPU_E_INVALID, "bad handles");
    if (num_points > (size_t)MAX_FORMS || (num_points && !points)) return fail(c, WHIRGPU_E_INVALID, "bad statement");
    const uint64_t n = w->ws->plan.n;
    whirgpu_linear_form forms[MAX_FORMS];
    for (size_t f = 0; f < num_points; ++f) forms[f] = {WHIRGPU_FORM_MLE, WHIRGPU_INPUT_HOST, points + f * n * 3};
    return whirgpu_prove_forms(c, w, forms, num_points, evaluations, tx, evaluation_point, rlc);
}

whirgpu_status whirgpu_mle_evaluate(whirgpu_ctx* c, const uint64_t* coeffs, uint64_t n, int where,
                                    const uint64_t* point, uint64_t out[3]) {
    if (!c || !coeffs || !point || !out || n >= 40) return fail(c, WHIRGPU_E_INVALID, "bad argument");
    const size_t scratch = mle_eval_scratch_bytes((uint32_t)n);
    const size_t point_region = (n * 24 + 24 + 255) / 256 * 256;  // point (n Ext3) + result (1 Ext3)
    const size_t need = scratch + point_region + (where == WHIRGPU_INPUT_DEVICE ? 0 : (8ull << n));
    if (c->mle_scratch_bytes < need) {
        if (c->mle_scratch) cudaFree(c->mle_scratch);
        c->mle_scratch = nullptr;
        c->mle_scratch_bytes = 0;
        WG_CUDA(c, cudaMalloc(&c->mle_scratch, need), "cudaMalloc");
        c->mle_scratch_bytes = need;
        WG_CUDA(c, cudaMemsetAsync(c->mle_scratch, 0, need, c->stream), "cudaMemset");
    }
    char* base = c->mle_scratch;
    uint64_t* dpoint = reinterpret_cast<uint64_t*>(base + scratch);
    uint64_t* dout = dpoint + n * 3;
    const uint64_t* dcoeffs = coeffs;
    if (where != WHIRGPU_INPUT_DEVICE) {
        uint64_t* dc = reinterpret_cast<uint64_t*>(base + scratch + point_region);
        WG_CUDA(c, cudaMemcpyAsync(dc, coeffs, 8ull << n, cudaMemcpyHostToDevice, c->stream), "upload");
        dcoeffs = dc;
    }
    WG_CUDA(c, cudaMemcpyAsync(dpoint, point, n * 24, cudaMemcpyHostToDevice, c->stream), "upload");
    launch_mle_eval(dcoeffs, (uint32_t)n, dpoint, base, dout, c->stream);
    WG_CUDA(c, cudaMemcpyAsync(out, dout, 24, cudaMemcpyDeviceToHost, c->stream), "read-back");
    WG_CUDA(c, cudaStreamSynchronize(c->stream), "mle");
    return WHIRGPU_OK;
}

void whirgpu_chacha20_block(const uint8_t key[32], uint32_t counter, const uint8_t nonce[12], uint8_t out[64]) {
    uint32_t k[8], nn[3], o[16];
    for (int i = 0; i < 8; ++i) std::memcpy(&k[i], key + 4 * i, 4);
    for (int i = 0; i < 3; ++i) std::memcpy(&nn[i], nonce + 4 * i, 4);
    chacha20_words(k, counter, nn, o);
    std::memcpy(out, o, 64);
}

void whirgpu_sample_goldilocks(uint64_t seed, uint64_t* out, size_t count) {
    uint32_t key[8] = {(uint32_t)seed, (uint32_t)(seed >> 32), 0, 0, 0, 0, 0, 0};
    const uint32_t nonce[3] = {0, 0, 0};
    uint32_t counter = 0;
    size_t got = 0;
    uint32_t blk[16];
    while (got < count) {
        chacha20_words(key, counter++, nonce, blk);
        for (int w = 0; w < 8 && got < count; ++w) {
            const uint64_t v = (uint64_t)blk[2 * w] | ((uint64_t)blk[2 * w + 1] << 32);
            if (v < GL_P) out[got++] = v;
        }
        if (counter == 0) key[2] += 1;  // past 2^38 bytes: continue in the next key slot
    }
}

void* whirgpu_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    return p;
}
void whirgpu_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

whirgpu_status whirgpu_set_timing(whirgpu_ctx* c, int enabled) {
    if (!c) return WHIRGPU_E_INVALID;
    if (enabled && !c->timer) c->timer.reset(new EventTimer());
    if (!enabled && c->timer) {
        cudaStreamSynchronize(c->stream);
        c->timer->harvest();
        for (int f = 0; f < FAM_COUNT; ++f) { c->stat_launches[f] += c->timer->launches[f]; c->stat_ms[f] += c->timer->ms[f]; }
        c->timer.reset();
    }
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_kernel_stats(whirgpu_ctx* c, uint64_t launches[WHIRGPU_NUM_FAMILIES],
                                    double ms[WHIRGPU_NUM_FAMILIES], int reset) {
    if (!c) return WHIRGPU_E_INVALID;
    if (c->timer) {
        cudaStreamSynchronize(c->stream);
        c->timer->harvest();
    }
    for (int f = 0; f < FAM_COUNT; ++f) {
        uint64_t l = c->stat_launches[f] + (c->timer ? c->timer->launches[f] : 0);
        double m = c->stat_ms[f] + (c->timer ? c->timer->ms[f] : 0.0);
        if (launches) launches[f] = l;
        if (ms) ms[f] = m;
    }
    if (reset) {
        for (int f = 0; f < FAM_COUNT; ++f) { c->stat_launches[f] = 0; c->stat_ms[f] = 0; }
        if (c->timer) for (int f = 0; f < FAM_COUNT; ++f) { c->timer->launches[f] = 0; c->timer->ms[f] = 0; }
    }
    return WHIRGPU_OK;
}

uint64_t whirgpu_launch_count(void) { return launch_count(); }

whirgpu_status whirgpu_workspace_stats(whirgpu_ctx* ctx, uint64_t* cached_bytes, uint64_t* allocations,
                                       uint64_t* evictions) {
    if (!ctx) return WHIRGPU_E_INVALID;
    std::lock_guard<std::recursive_mutex> lk(ctx->cache_mu);
    if (cached_bytes) *cached_bytes = ctx->allocated;
    if (allocations) *allocations = ctx->ws_allocations;
    if (evictions) *evictions = ctx->ws_evictions;
    return WHIRGPU_OK;
}

void whirgpu_last_io_bytes(const whirgpu_ctx* c, uint64_t* h2d, uint64_t* d2h) {
    if (h2d) *h2d = c ? c->io_h2d : 0;
    if (d2h) *d2h = c ? c->io_d2h : 0;
}

}  // extern "C"

namespace wg {
static std::atomic<u64> g_launches{0};
static thread_local bool g_capturing = false;
void count_launches(u64 k) {
    if (!g_capturing) g_launches.fetch_add(k, std::memory_order_relaxed);
}
void set_capturing(bool on) { g_capturing = on; }
uint64_t graph_kernel_nodes(cudaGraph_t g) {
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return 0;
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
    uint64_t k = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
    }
    return k;
}
u64 launch_count() { return g_launches.load(std::memory_order_relaxed); }

void host_twiddles(u64* stage, u64* hi, u64* lo) {
    const u64 w11 = gl_pow_host(7, (GL_P - 1) >> TW_STAGE_LOG);
    u64 acc = 1;
    for (u32 u = 0; u < (1u << (TW_STAGE_LOG - 1)); ++u) { stage[u] = acc; acc = gl_mul_host(acc, w11); }
    const u64 w = gl_pow_host(7, (GL_P - 1) >> TW_LOG);
    acc = 1;
    for (u32 u = 0; u < (1u << TW_HALF); ++u) { lo[u] = acc; acc = gl_mul_host(acc, w); }
    const u64 wh = acc;  // w^(2^TW_HALF)
    acc = 1;
    for (u32 u = 0; u < (1u << TW_HALF); ++u) { hi[u] = acc; acc = gl_mul_host(acc, wh); }
}
}  // namespace wg
