// batch.cu -- many independent proofs at once: batches captured into one CUDA
// graph, and a continuous-batching server with HBM-budget admission.
//
// Every proof owns its workspace (prover.h: all state, scratch and tickets live
// there), so proofs of different sizes run side by side on separate streams
// without interacting; the bytes of each proof are the same alone or in a mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/whirgpu.h"
#include "ctx.h"
#include "launch.h"
#include "prover.h"
#include "state.cuh"

using namespace wg;

namespace {

// One proof slot: a workspace plus pinned staging for its small inputs and its
// outputs.  The coefficients are copied straight from the caller's buffer when
// it is device or pinned host memory, else through `stage`.
struct Slot {
    Workspace* ws = nullptr;
    ProofPlan plan;           // copy with n_forms set for the request
    uint8_t* hin = nullptr;   // pinned: [ds 96 | points | evals]
    size_t hin_bytes = 0;
    uint8_t* hout = nullptr;  // pinned: [TxState | narg | hints]
    size_t hout_bytes = 0;
    uint8_t* stage = nullptr;          // pinned coefficient staging (pageable callers only)
    const void* coeff_src = nullptr;   // what the coefficient copy reads
    cudaGraphExec_t graph = nullptr;   // captured single-proof program (serving)
    uint64_t graph_kernels = 0;        // kernel nodes in `graph`
};

size_t coeff_bytes(const ProofPlan& p) { return (size_t)p.nvec * (8ull << p.n); }  // batch_size vectors
size_t points_off() { return 96; }
size_t evals_off(const ProofPlan& p) { return 96 + (size_t)MAX_FORMS * p.n * 24; }

bool is_pinned_host(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

whirgpu_status check_request(whirgpu_ctx* c, const whirgpu_request& r) {
    if (!engine_supported(&r.params)) return fail(c, WHIRGPU_E_UNSUPPORTED, "only the BLAKE3 and SHA-2 engines are on this path");
    if (r.num_variables >= 40 || r.num_points > (uint64_t)MAX_FORMS) return fail(c, WHIRGPU_E_INVALID, "bad request");
    if (r.num_points && (!r.points || !r.evaluations)) return fail(c, WHIRGPU_E_INVALID, "bad statement");
    if (!r.coeffs) return fail(c, WHIRGPU_E_INVALID, "null coefficients");
    return WHIRGPU_OK;
}

// Binds a slot to workspace `ws` (already acquired) and allocates its staging.
whirgpu_status slot_bind(whirgpu_ctx* c, const whirgpu_request& r, Workspace* ws, Slot& s) {
    s.ws = ws;
    s.plan = ws->plan;
    plan_set_forms(s.plan, (int)r.num_points);
    s.hin_bytes = evals_off(s.plan) + (size_t)MAX_FORMS * MAX_VECTORS * 24;
    s.hout_bytes = sizeof(TxState) + s.plan.narg_len + s.plan.hints_cap;
    if (cudaMallocHost(&s.hin, s.hin_bytes) != cudaSuccess || cudaMallocHost(&s.hout, s.hout_bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, WHIRGPU_E_OOM, "pinned staging");
    }
    return WHIRGPU_OK;
}

// Frees the slot's host staging and graph (not its workspace).
void slot_free_host(Slot& s) {
    if (s.graph) cudaGraphExecDestroy(s.graph);
    if (s.hin) cudaFreeHost(s.hin);
    if (s.hout) cudaFreeHost(s.hout);
    if (s.stage) cudaFreeHost(s.stage);
    s.graph = nullptr;
    s.hin = s.hout = s.stage = nullptr;
}

// Copies the request's small inputs into the pinned staging and picks the
// source of the coefficient copy (host side).
whirgpu_status slot_stage(whirgpu_ctx* c, Slot& s, const whirgpu_request& r) {
    const size_t n = s.plan.n;
    if (r.coeffs_location == WHIRGPU_INPUT_DEVICE || is_pinned_host(r.coeffs)) {
        s.coeff_src = r.coeffs;
    } else {
        if (!s.stage && cudaMallocHost(&s.stage, coeff_bytes(s.plan)) != cudaSuccess) {
            cudaGetLastError();
            s.stage = nullptr;
            return fail(c, WHIRGPU_E_OOM, "pinned coefficient staging");
        }
        std::memcpy(s.stage, r.coeffs, coeff_bytes(s.plan));
        s.coeff_src = s.stage;
    }
    std::memcpy(s.hin, r.protocol_id, 64);
    std::memcpy(s.hin + 64, r.session_id, 32);
    if (r.num_points) {
        std::memcpy(s.hin + points_off(), r.points, r.num_points * n * 24);
        std::memcpy(s.hin + evals_off(s.plan), r.evaluations, r.num_points * s.plan.nvec * 24);
    }
    return WHIRGPU_OK;
}

int copy_coeffs(const Slot& s, cudaStream_t st) {
    return cudaMemcpyAsync(s.ws->dev + s.plan.off_coeffs, s.coeff_src, coeff_bytes(s.plan), cudaMemcpyDefault, st) ==
                   cudaSuccess
               ? 0
               : -1;
}

// Enqueues (optionally) the coefficient copy, the small input copies, commit,
// prove and the proof read-back of one slot.
int slot_enqueue(whirgpu_ctx* c, Slot& s, cudaStream_t st, bool with_coeffs) {
    const ProofPlan& p = s.plan;
    char* ws = s.ws->dev;
    const size_t n = p.n;
    if (with_coeffs && copy_coeffs(s, st) != 0) return -1;
    if (cudaMemcpyAsync(ws + p.off_ds, s.hin, 96, cudaMemcpyHostToDevice, st) != cudaSuccess) return -1;
    ProofScalars* sc = plan_scalars(p, ws);
    if (p.n_forms) {
        if (cudaMemcpyAsync(ws + p.off_points, s.hin + points_off(), p.n_forms * n * 24, cudaMemcpyHostToDevice, st) !=
            cudaSuccess)
            return -1;
        if (cudaMemcpyAsync(&sc->forms_eval[0], s.hin + evals_off(p), (size_t)p.n_forms * p.nvec * 24,
                            cudaMemcpyHostToDevice, st) !=
            cudaSuccess)
            return -1;
    }
    if (enqueue_commit(p, ws, 96, c->tw, st, nullptr) != 0) return -2;
    if (enqueue_prove(p, ws, c->tw, st, nullptr) != 0) return -2;
    uint8_t* h = s.hout;
    if (cudaMemcpyAsync(h, plan_tx(p, ws), sizeof(TxState), cudaMemcpyDeviceToHost, st) != cudaSuccess) return -1;
    if (cudaMemcpyAsync(h + sizeof(TxState), ws + p.off_narg, p.narg_len, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return -1;
    if (cudaMemcpyAsync(h + sizeof(TxState) + p.narg_len, ws + p.off_hints, p.hints_cap, cudaMemcpyDeviceToHost, st) !=
        cudaSuccess)
        return -1;
    return 0;
}

// Checks the device status words and copies the proof out of the staging.
whirgpu_status slot_collect(whirgpu_ctx* c, Slot& s, std::vector<uint8_t>& narg, std::vector<uint8_t>& hints) {
    const TxState* t = reinterpret_cast<const TxState*>(s.hout);
    if (t->err) return fail(c, WHIRGPU_E_DEVICE, "device error word");
    if (t->narg_len != s.plan.narg_len || t->hints_len > s.plan.hints_cap)
        return fail(c, WHIRGPU_E_DEVICE, "proof stream length mismatch");
    const uint8_t* h = s.hout + sizeof(TxState);
    narg.assign(h, h + s.plan.narg_len);
    hints.assign(h + s.plan.narg_len, h + s.plan.narg_len + t->hints_len);
    return WHIRGPU_OK;
}

}  // namespace

// ===========================================================================
// Batches
// ===========================================================================
struct whirgpu_batch {
    whirgpu_ctx* ctx = nullptr;
    int mode = 0;
    std::vector<whirgpu_request> reqs;
    std::vector<Slot> slots;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork = nullptr;
    cudaStream_t main = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t graph_kernels = 0;
    std::vector<std::vector<uint8_t>> narg, hints;
    std::vector<whirgpu_status> status;
};

namespace {

whirgpu_status batch_enqueue_all(whirgpu_batch* b) {
    whirgpu_ctx* c = b->ctx;
    if (cudaEventRecord(b->fork, b->main) != cudaSuccess) return cuda_fail(c, cudaGetLastError(), "fork");
    for (size_t i = 0; i < b->slots.size(); ++i) {
        cudaStream_t st = b->streams[i % b->streams.size()];
        cudaStreamWaitEvent(st, b->fork, 0);
        if (slot_enqueue(c, b->slots[i], st, true) != 0) return fail(c, WHIRGPU_E_CUDA, "batch enqueue");
    }
    for (size_t k = 0; k < b->streams.size(); ++k) {
        cudaEventRecord(b->joins[k], b->streams[k]);
        cudaStreamWaitEvent(b->main, b->joins[k], 0);
    }
    return WHIRGPU_OK;
}

}  // namespace

extern "C" {

whirgpu_status whirgpu_batch_create(whirgpu_ctx* c, const whirgpu_request* reqs, size_t count, int mode,
                                    whirgpu_batch** out) {
    if (!c || !reqs || !out || count == 0 || mode < 0 || mode > 2) return fail(c, WHIRGPU_E_INVALID, "bad batch");
    *out = nullptr;
    auto b = std::make_unique<whirgpu_batch>();
    b->ctx = c;
    b->mode = mode;
    b->reqs.assign(reqs, reqs + count);
    b->slots.resize(count);
    auto unwind = [&](whirgpu_status st) {
        for (auto& sl : b->slots) {
            slot_free_host(sl);
            release_workspace(c, sl.ws);
        }
        return st;
    };
    for (size_t i = 0; i < count; ++i) {
        whirgpu_status st = check_request(c, reqs[i]);
        Workspace* ws = nullptr;
        if (st == WHIRGPU_OK) st = acquire_workspace(c, reqs[i].num_variables, &reqs[i].params, 96, &ws);
        if (st == WHIRGPU_OK) st = slot_bind(c, reqs[i], ws, b->slots[i]);
        else b->slots[i].ws = nullptr;
        if (st == WHIRGPU_OK) st = slot_stage(c, b->slots[i], reqs[i]);
        if (st != WHIRGPU_OK) return unwind(st);
    }
    const size_t nstreams = mode == 2 ? 1 : std::min<size_t>(count, 64);
    b->streams.resize(nstreams);
    b->joins.resize(nstreams);
    for (size_t k = 0; k < nstreams; ++k) {
        cudaStreamCreateWithFlags(&b->streams[k], cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&b->joins[k], cudaEventDisableTiming);
    }
    cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking);
    b->narg.resize(count);
    b->hints.resize(count);
    b->status.assign(count, WHIRGPU_E_INVALID);
    if (mode == 0) {
        // One graph: a fork event, one branch per proof, a join.
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return cuda_fail(c, cudaGetLastError(), "begin capture");
        set_capturing(true);
        whirgpu_status st = batch_enqueue_all(b.get());
        set_capturing(false);
        cudaError_t ce = cudaStreamEndCapture(b->main, &g);
        if (st == WHIRGPU_OK && ce != cudaSuccess) st = cuda_fail(c, ce, "end capture");
        if (st == WHIRGPU_OK) {
            b->graph_kernels = graph_kernel_nodes(g);
            ce = cudaGraphInstantiate(&b->exec, g, 0);
            if (ce != cudaSuccess) st = cuda_fail(c, ce, "graph instantiate");
        }
        if (g) cudaGraphDestroy(g);
        if (st != WHIRGPU_OK) {
            whirgpu_batch_destroy(b.release());
            return st;
        }
    }
    *out = b.release();
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_batch_run(whirgpu_batch* b) {
    if (!b) return WHIRGPU_E_INVALID;
    whirgpu_ctx* c = b->ctx;
    for (size_t i = 0; i < b->slots.size(); ++i) {
        const void* before = b->slots[i].coeff_src;
        whirgpu_status st = slot_stage(c, b->slots[i], b->reqs[i]);
        if (st != WHIRGPU_OK) return st;
        if (b->mode == 0 && b->slots[i].coeff_src != before)
            return fail(c, WHIRGPU_E_INVALID, "coefficient memory changed kind since the batch was captured");
    }
    if (b->mode == 0) {
        count_launches(b->graph_kernels);
        cudaError_t e = cudaGraphLaunch(b->exec, b->main);
        if (e != cudaSuccess) return cuda_fail(c, e, "graph launch");
        e = cudaStreamSynchronize(b->main);
        if (e != cudaSuccess) return cuda_fail(c, e, "batch");
    } else if (b->mode == 1) {
        whirgpu_status st = batch_enqueue_all(b);
        if (st != WHIRGPU_OK) return st;
        cudaError_t e = cudaStreamSynchronize(b->main);
        if (e != cudaSuccess) return cuda_fail(c, e, "batch");
    } else {
        // plain: one proof at a time, each waited for before the next starts
        for (size_t i = 0; i < b->slots.size(); ++i) {
            if (slot_enqueue(c, b->slots[i], b->streams[0], true) != 0) return fail(c, WHIRGPU_E_CUDA, "enqueue");
            cudaError_t e = cudaStreamSynchronize(b->streams[0]);
            if (e != cudaSuccess) return cuda_fail(c, e, "proof");
        }
    }
    whirgpu_status worst = WHIRGPU_OK;
    for (size_t i = 0; i < b->slots.size(); ++i) {
        b->status[i] = slot_collect(c, b->slots[i], b->narg[i], b->hints[i]);
        if (b->status[i] != WHIRGPU_OK) worst = b->status[i];
    }
    return worst;
}

whirgpu_status whirgpu_batch_proof(const whirgpu_batch* b, size_t i, const uint8_t** narg, size_t* narg_len,
                                   const uint8_t** hints, size_t* hints_len) {
    if (!b || i >= b->slots.size()) return WHIRGPU_E_INVALID;
    if (b->status[i] != WHIRGPU_OK) return b->status[i];
    if (narg) *narg = b->narg[i].data();
    if (narg_len) *narg_len = b->narg[i].size();
    if (hints) *hints = b->hints[i].data();
    if (hints_len) *hints_len = b->hints[i].size();
    return WHIRGPU_OK;
}

void whirgpu_batch_destroy(whirgpu_batch* b) {
    if (!b) return;
    if (b->main) cudaStreamSynchronize(b->main);
    for (auto st : b->streams) cudaStreamSynchronize(st);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (auto& s : b->slots) {
        slot_free_host(s);
        release_workspace(b->ctx, s.ws);
    }
    for (auto st : b->streams) cudaStreamDestroy(st);
    for (auto e : b->joins) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->main) cudaStreamDestroy(b->main);
    delete b;
}

}  // extern "C"

// ===========================================================================
// Serving: continuous batching with HBM-budget admission
// ===========================================================================
namespace {

using Clock = std::chrono::steady_clock;

struct Ticket {
    uint64_t id = 0;
    whirgpu_request req{};
    size_t bytes = 0;                             // workspace bytes it needs
    Clock::time_point t_submit, t_start, t_done;
    Slot* slot = nullptr;
    int stream = -1;
    cudaEvent_t done_ev = nullptr;
    bool finished = false;
    whirgpu_status status = WHIRGPU_OK;
    std::vector<uint8_t> narg, hints;
};

}  // namespace

struct whirgpu_server {
    whirgpu_ctx* ctx = nullptr;
    uint64_t budget = 0;
    uint32_t max_inflight = 0;
    std::mutex mu;
    std::condition_variable cv_done;
    std::map<uint64_t, std::unique_ptr<Ticket>> tickets;
    std::deque<uint64_t> queue;                 // waiting for admission, arrival order
    std::vector<uint64_t> inflight;
    // Streams in SERVER_LEVELS priority pools of max_inflight each: stream k
    // serves level k / max_inflight (server_level: small proofs on the
    // highest-priority streams, so their blocks are scheduled ahead of a large
    // proof's when both are pending; the large proofs are throughput-bound).
    std::vector<cudaStream_t> streams;
    std::vector<int> stream_busy;
    // Captured single-proof programs, one per (workspace, statement count):
    // the workspace addresses and staging buffers are baked into the graph.
    std::map<std::pair<Workspace*, int>, std::unique_ptr<Slot>> programs;
    uint64_t next_id = 1;
    uint64_t in_use = 0;                        // workspace bytes of admitted requests
    std::atomic<bool> stop{false};
    std::thread worker;
    uint64_t admitted_total = 0, peak_inflight = 0, peak_bytes = 0;
};

namespace {

// The cached program for a request: acquires a free workspace of the right
// shape and, on first use of that workspace, captures its commit + prove
// (everything but the coefficient copy, which reads the caller's buffer and is
// issued before each launch).  The program is dropped with its workspace when
// the context evicts it.
whirgpu_status program_for(whirgpu_server* s, const whirgpu_request& r, cudaStream_t cs, Slot** out) {
    whirgpu_ctx* c = s->ctx;
    whirgpu_status st = check_request(c, r);
    if (st != WHIRGPU_OK) return st;
    Workspace* ws = nullptr;
    st = acquire_workspace(c, r.num_variables, &r.params, 96, &ws, s->budget);
    if (st != WHIRGPU_OK) return st;
    auto key = std::make_pair(ws, (int)r.num_points);
    auto it = s->programs.find(key);
    if (it != s->programs.end()) {
        *out = it->second.get();
        return WHIRGPU_OK;
    }
    auto slot = std::make_unique<Slot>();
    st = slot_bind(c, r, ws, *slot);
    if (st == WHIRGPU_OK) st = slot_stage(c, *slot, r);
    if (st != WHIRGPU_OK) {
        slot_free_host(*slot);
        release_workspace(c, ws);
        return st;
    }
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        slot_free_host(*slot);
        release_workspace(c, ws);
        return fail(c, WHIRGPU_E_CUDA, "begin capture");
    }
    set_capturing(true);
    const int rc = slot_enqueue(c, *slot, cs, false);
    set_capturing(false);
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    if (rc == 0 && e == cudaSuccess) {
        slot->graph_kernels = graph_kernel_nodes(g);
        e = cudaGraphInstantiate(&slot->graph, g, 0);
    }
    if (g) cudaGraphDestroy(g);
    if (rc != 0 || e != cudaSuccess) {
        cudaGetLastError();
        slot_free_host(*slot);
        release_workspace(c, ws);
        return fail(c, WHIRGPU_E_CUDA, "capture of the proof program");
    }
    *out = slot.get();
    s->programs[key] = std::move(slot);
    ws->on_free[s] = [s, ws] {
        for (auto pit = s->programs.begin(); pit != s->programs.end();) {
            if (pit->first.first != ws) { ++pit; continue; }
            slot_free_host(*pit->second);
            pit = s->programs.erase(pit);
        }
    };
    return WHIRGPU_OK;
}

// Priority level of a request: 0 (high) for proofs of up to 2^18
// coefficients -- latency-bound chains of small kernels -- 1 above.
constexpr int SERVER_LEVELS = 2;
int server_level(const whirgpu_request& r) { return r.num_variables <= 18 ? 0 : 1; }

// Admits queued requests that fit the HBM budget and a free stream of their
// priority level, in arrival order; a later request may pass an earlier one
// that does not fit yet.
void admit(whirgpu_server* s) {
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        if (s->inflight.size() >= s->max_inflight) break;
        Ticket& t = *s->tickets[*it];
        if (s->budget && s->in_use + t.bytes > s->budget) { ++it; continue; }
        int k = -1;
        const size_t base = (size_t)server_level(t.req) * s->max_inflight;
        for (size_t j = base; j < base + s->max_inflight; ++j)
            if (!s->stream_busy[j]) { k = (int)j; break; }
        if (k < 0) { ++it; continue; }
        Slot* slot = nullptr;
        whirgpu_status st = program_for(s, t.req, s->streams[k], &slot);
        if (st == WHIRGPU_OK) {
            st = slot_stage(s->ctx, *slot, t.req);
            cudaError_t e = cudaSuccess;
            if (st == WHIRGPU_OK) {
                e = copy_coeffs(*slot, s->streams[k]) == 0 ? cudaSuccess : cudaErrorInvalidValue;
                if (e == cudaSuccess) {
                    count_launches(slot->graph_kernels);
                    e = cudaGraphLaunch(slot->graph, s->streams[k]);
                }
                if (e == cudaSuccess) e = cudaEventRecord(t.done_ev, s->streams[k]);
                if (e != cudaSuccess) st = cuda_fail(s->ctx, e, "proof launch");
            }
            if (st != WHIRGPU_OK) release_workspace(s->ctx, slot->ws);
        }
        if (st != WHIRGPU_OK) {
            t.status = st;
            t.finished = true;
            t.t_done = Clock::now();
            it = s->queue.erase(it);
            s->cv_done.notify_all();
            continue;
        }
        t.slot = slot;
        t.stream = k;
        t.t_start = Clock::now();
        s->stream_busy[k] = 1;
        s->in_use += t.bytes;
        s->peak_bytes = std::max<uint64_t>(s->peak_bytes, s->in_use);
        s->inflight.push_back(t.id);
        s->admitted_total++;
        s->peak_inflight = std::max<uint64_t>(s->peak_inflight, s->inflight.size());
        it = s->queue.erase(it);
    }
}

void reap(whirgpu_server* s) {
    for (size_t i = 0; i < s->inflight.size();) {
        Ticket& t = *s->tickets[s->inflight[i]];
        const cudaError_t q = cudaEventQuery(t.done_ev);
        if (q == cudaErrorNotReady) { ++i; continue; }
        t.status = q == cudaSuccess ? slot_collect(s->ctx, *t.slot, t.narg, t.hints) : WHIRGPU_E_CUDA;
        t.finished = true;
        t.t_done = Clock::now();
        s->stream_busy[t.stream] = 0;
        s->in_use -= t.bytes;
        release_workspace(s->ctx, t.slot->ws);  // back to the pool with its captured program
        t.slot = nullptr;
        s->inflight.erase(s->inflight.begin() + i);
        s->cv_done.notify_all();
    }
}

void server_loop(whirgpu_server* s) {
    cudaSetDevice(s->ctx->device);
    while (!s->stop.load()) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            reap(s);
            admit(s);
        }
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

}  // namespace

extern "C" {

whirgpu_status whirgpu_server_create(whirgpu_ctx* c, uint64_t hbm_budget, uint32_t max_inflight, whirgpu_server** out) {
    if (!c || !out || max_inflight == 0) return WHIRGPU_E_INVALID;
    auto s = std::make_unique<whirgpu_server>();
    s->ctx = c;
    s->budget = hbm_budget;
    s->max_inflight = max_inflight;
    int least = 0, greatest = 0;  // numerically: greatest <= least
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    s->streams.resize((size_t)SERVER_LEVELS * max_inflight);
    s->stream_busy.assign(s->streams.size(), 0);
    for (size_t k = 0; k < s->streams.size(); ++k) {
        const int level = (int)(k / max_inflight);  // 0: greatest priority
        const int prio = greatest + (least - greatest) * level / (SERVER_LEVELS - 1);
        cudaStreamCreateWithPriority(&s->streams[k], cudaStreamNonBlocking, prio);
    }
    whirgpu_server* raw = s.release();
    raw->worker = std::thread(server_loop, raw);
    *out = raw;
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_server_submit(whirgpu_server* s, const whirgpu_request* r, uint64_t* ticket) {
    if (!s || !r || !ticket || !r->coeffs) return WHIRGPU_E_INVALID;
    if (r->num_points > (uint64_t)MAX_FORMS || (r->num_points && (!r->points || !r->evaluations)))
        return WHIRGPU_E_INVALID;
    const size_t bytes = workspace_bytes(r->num_variables, &r->params);
    if (bytes == 0) return WHIRGPU_E_INVALID;
    if (s->budget && bytes > s->budget) return WHIRGPU_E_OOM;  // could never be admitted
    // The request's buffers are borrowed until poll returns the result: the
    // only copy is into the workspace's pinned staging at admission.
    auto t = std::make_unique<Ticket>();
    t->req = *r;
    t->bytes = bytes;
    t->t_submit = Clock::now();
    cudaEventCreateWithFlags(&t->done_ev, cudaEventDisableTiming);
    std::lock_guard<std::mutex> lk(s->mu);
    t->id = s->next_id++;
    *ticket = t->id;
    s->queue.push_back(t->id);
    s->tickets[t->id] = std::move(t);
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_server_poll(whirgpu_server* s, uint64_t ticket, uint32_t timeout_ms, whirgpu_result* out) {
    if (!s || !out) return WHIRGPU_E_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return WHIRGPU_E_INVALID;
    Ticket* t = it->second.get();
    if (!t->finished) {
        s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [t] { return t->finished; });
        if (!t->finished) return WHIRGPU_E_TIMEOUT;
    }
    out->status = t->status;
    out->narg = t->narg.data();
    out->narg_len = t->narg.size();
    out->hints = t->hints.data();
    out->hints_len = t->hints.size();
    out->queue_ms = t->stream >= 0 ? std::chrono::duration<double, std::milli>(t->t_start - t->t_submit).count() : 0.0;
    out->total_ms = std::chrono::duration<double, std::milli>(t->t_done - t->t_submit).count();
    return WHIRGPU_OK;
}

void whirgpu_server_release(whirgpu_server* s, uint64_t ticket) {
    if (!s) return;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end() || !it->second->finished) return;
    if (it->second->done_ev) cudaEventDestroy(it->second->done_ev);
    s->tickets.erase(it);
}

void whirgpu_server_stats(whirgpu_server* s, uint64_t* admitted, uint64_t* peak_inflight, uint64_t* peak_bytes,
                          uint64_t* queued) {
    if (!s) return;
    std::lock_guard<std::mutex> lk(s->mu);
    if (admitted) *admitted = s->admitted_total;
    if (peak_inflight) *peak_inflight = s->peak_inflight;
    if (peak_bytes) *peak_bytes = s->peak_bytes;
    if (queued) *queued = s->queue.size();
}

void whirgpu_server_destroy(whirgpu_server* s) {
    if (!s) return;
    // Drain: in-flight proofs finish; requests never admitted fail.
    for (;;) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->inflight.empty()) {
                for (uint64_t id : s->queue) {
                    Ticket& t = *s->tickets[id];
                    t.status = WHIRGPU_E_INVALID;
                    t.finished = true;
                }
                s->queue.clear();
                s->cv_done.notify_all();
                break;
            }
        }
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    s->stop.store(true);
    if (s->worker.joinable()) s->worker.join();
    for (auto& kv : s->tickets)
        if (kv.second->done_ev) cudaEventDestroy(kv.second->done_ev);
    {
        std::lock_guard<std::recursive_mutex> lk(s->ctx->cache_mu);
        for (auto& kv : s->programs) {
            kv.first.first->on_free.erase(s);
            slot_free_host(*kv.second);
        }
        s->programs.clear();
    }
    for (auto st : s->streams) cudaStreamDestroy(st);
    delete s;
}

}  // extern "C"
