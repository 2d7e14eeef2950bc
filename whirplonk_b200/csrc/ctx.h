// ctx.h -- internal state behind the C ABI handles, shared by capi.cu
// (single proofs) and batch.cu (batches and the serving loop).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <mutex>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/whirgpu.h"
#include "launch.h"
#include "prover.h"

namespace wg {

// Engine ids (identifiers of the reference's hash engines, blake3_engine.hpp,
// sha2_engine.hpp:38-43; carried in ProtocolParameters::hash_id).
constexpr uint8_t SHA2_ENGINE_ID[32] = {0x01, 0x8e, 0xaa, 0x24, 0x7c, 0xb8, 0x95, 0x7a, 0xb1, 0xe9, 0xfd,
                                        0xac, 0x88, 0x54, 0x50, 0x40, 0x3c, 0x5e, 0x7b, 0xda, 0x1a, 0xca,
                                        0xaa, 0x50, 0x4e, 0x4c, 0xc8, 0xf2, 0xf7, 0x6b, 0xb0, 0x76};
constexpr uint8_t BLAKE3_ENGINE_ID[32] = {0x03, 0xe0, 0x17, 0x49, 0xeb, 0xcc, 0x04, 0x77, 0x92, 0x42, 0x54,
                                          0xeb, 0x48, 0x20, 0x66, 0xb8, 0x64, 0xa8, 0xdd, 0x4d, 0x77, 0x25,
                                          0x24, 0x64, 0xca, 0x6f, 0x5b, 0x6f, 0x5c, 0xc0, 0x5b, 0x4c};

struct EventTimer : Timer {
    struct Pair { int fam; cudaEvent_t a, b; };
    std::vector<Pair> pending;
    std::vector<cudaEvent_t> pool;
    uint64_t launches[FAM_COUNT] = {};
    double ms[FAM_COUNT] = {};
    cudaEvent_t get() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void begin(int fam, cudaStream_t st) override {
        Pair p{fam, get(), nullptr};
        cudaEventRecord(p.a, st);
        pending.push_back(p);
    }
    void end(int fam, cudaStream_t st) override {
        for (auto it = pending.rbegin(); it != pending.rend(); ++it)
            if (it->fam == fam && it->b == nullptr) {
                it->b = get();
                cudaEventRecord(it->b, st);
                return;
            }
    }
    void harvest() {  // after a stream synchronisation
        for (auto& p : pending) {
            if (!p.b) continue;
            float t = 0;
            cudaEventElapsedTime(&t, p.a, p.b);
            ms[p.fam] += t;
            launches[p.fam] += 1;
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    ~EventTimer() override {
        for (auto& p : pending) { cudaEventDestroy(p.a); if (p.b) cudaEventDestroy(p.b); }
        for (auto e : pool) cudaEventDestroy(e);
    }
};


struct Workspace {
    ProofPlan plan;
    char* dev = nullptr;
    bool busy = false;
    uint64_t last_used = 0;                    // LRU stamp for eviction of idle workspaces
    std::map<const void*, std::function<void()>> on_free;  // per owner: drops state tied to `dev` (captured graphs)
    // The single-proof calls' kernels as captured graphs (commit; prove per
    // statement count), keyed with the NTT plan epoch they were captured under.
    struct Captured {
        cudaGraphExec_t exec = nullptr;
        uint64_t kernels = 0;
    };
    std::map<uint64_t, Captured> plain_graphs;
};

}  // namespace wg

struct whirgpu_ctx {
    int device = 0;
    int codeword_order = 0;  // WHIRGPU_ORDER_* of the commitments made from now on
    cudaStream_t stream = nullptr;
    uint64_t budget = 0;
    uint64_t allocated = 0;
    uint64_t ws_allocations = 0, ws_evictions = 0;  // workspaces allocated / freed to make room
    wg::DeviceTables tw;
    wg::LdeTables lde_tables;  // inter-pass twiddle factors of the LDE splits in use (tw.lde)
    std::string err;
    // Workspaces by plan shape: the schedule, hash engine, vector layout, field
    // degree and domain-separator length, serialised (plan_key).
    std::map<std::string, std::vector<wg::Workspace*>> cache;
    uint8_t* pinned = nullptr;
    size_t pinned_bytes = 0;
    char* mle_scratch = nullptr;
    size_t mle_scratch_bytes = 0;
    char* kscratch = nullptr;  // kernel-level calls (RS encode/commit, autotuner)
    size_t kscratch_bytes = 0;
    std::unique_ptr<wg::EventTimer> timer;
    uint64_t stat_launches[wg::FAM_COUNT] = {};
    double stat_ms[wg::FAM_COUNT] = {};
    uint64_t io_h2d = 0, io_d2h = 0;
    std::recursive_mutex cache_mu;  // workspace cache (the serving thread shares the context)
    uint64_t use_clock = 0;
    // Witnesses not yet destroyed: destroying the context detaches them, so a
    // witness destroyed afterwards only frees its handle.
    std::set<whirgpu_witness*> live_witnesses;
    std::set<whirgpu_zk_witness*> live_zk;  // the same for zero-knowledge witnesses
    // Device allocations of destroyed zero-knowledge witnesses, by size, for reuse.
    std::map<size_t, std::vector<char*>> zk_pool;
};

struct whirgpu_transcript {
    whirgpu_ctx* ctx = nullptr;
    std::vector<uint8_t> ds;  // protocol_id || session_id || instance
    std::vector<uint8_t> narg, hints;
    bool complete = false;
};

struct whirgpu_witness {
    whirgpu_ctx* ctx = nullptr;
    wg::Workspace* ws = nullptr;
    whirgpu_transcript* tx = nullptr;
};

namespace wg {
ProtocolParams to_params(const whirgpu_params* p);
whirgpu_status fail(whirgpu_ctx* c, whirgpu_status s, const std::string& msg);
whirgpu_status cuda_fail(whirgpu_ctx* c, cudaError_t e, const char* what);
whirgpu_status ensure_pinned(whirgpu_ctx* c, size_t bytes);
// A free workspace for (n, params, ds_len, nwit initial commitments),
// allocated on first use and kept in the context cache; marked busy until
// release_workspace.  Allocation keeps the context's bytes within min(ctx
// budget, cap) (0 = no limit) by freeing idle workspaces, least recently used
// first; a failed cudaMalloc frees every idle workspace and tries once more.
whirgpu_status acquire_workspace(whirgpu_ctx* c, uint64_t n, const whirgpu_params* params, size_t ds_len, Workspace** out,
                                 uint64_t cap = 0, uint32_t nwit = 1);
// The same for a schedule given field by field.
whirgpu_status acquire_workspace_sched(whirgpu_ctx* c, const WhirSchedule& sched, const ProtocolParams& pp, size_t ds_len,
                                       Workspace** out, uint64_t cap = 0, uint32_t nwit = 1);
void release_workspace(whirgpu_ctx* c, Workspace* w);
// Builds the context's inter-pass twiddle tables for the LDEs of `plan` (once
// per split; within the HBM budget).  Call outside any graph capture.
void prepare_lde_tables(whirgpu_ctx* c, const ProofPlan& plan);
// While set, kernel launches of this thread are stream-captured, not run: the
// launch counter skips them and graph launches add their kernel-node counts.
void set_capturing(bool on);
uint64_t graph_kernel_nodes(cudaGraph_t g);
bool is_blake3(const whirgpu_params* p);
bool is_sha2(const whirgpu_params* p);
bool engine_supported(const whirgpu_params* p);  // BLAKE3 or SHA-2
// Plan size of one proof (bytes of device workspace), or 0 when invalid.
size_t workspace_bytes(uint64_t n, const whirgpu_params* params, uint32_t nwit = 1);
// The schedule of a Config given field by field (shape checks: validate_schedule).
WhirSchedule schedule_from_config(const whirgpu_config* cfg);
// Frees the device memory of every live zero-knowledge witness of the context
// and detaches them (their later destroy only frees the handle).
void zk_detach_all(whirgpu_ctx* c);
// BlindingSizePolicy::from_whir_params (whir_zk.hpp:48-62).
whirgpu_zk_policy zk_default_policy(const whirgpu_params* p);
}  // namespace wg
