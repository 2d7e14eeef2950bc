// k_rs.cu -- kernel-level entry points of the Reed-Solomon commitment and the
// NTT pass-plan autotuner.
//
// whirgpu_rs_encode / whirgpu_rs_commit_batch expose the encoder and the
// matrix commitment on their own: a vector of 2^log_len base-field words is
// committed as irs_commit::commit does for one vector
// (cpp/include/whir/protocols/irs_commit.hpp:402-470): interleaving depth d,
// block b = v[b m .. (b+1) m) with m = 2^log_len / d, codeword of length
// N = 2^log_expansion m per block (mod_ntt.hpp:49-130), row i = the d values
// X_b[i], leaf = BLAKE3(row bytes) (matrix_commit.hpp:169-195), Merkle root
// (merkle_tree.hpp:104-147).  The transcript and OOD steps of a proof are not
// part of these calls.
//
// The autotuner times every valid pass plan (split of log N into <= 3 radices
// of at most 2^11, columns per CTA per pass) for one LDE shape on synthetic
// data, checks that each plan produces the same codeword (a position-keyed
// 64-bit XOR digest) and installs the fastest one for that shape.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/whirgpu.h"
#include "ctx.h"
#include "gl.cuh"
#include "launch.h"

namespace wg {

__device__ __forceinline__ u64 mix64(u64 x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

// Canonical pseudo-random words (a function of seed and position only).
__global__ void k_fill_canonical(u64* p, u64 n, u64 seed) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        p[i] = mix64(seed ^ mix64(i)) % GL_P;
}

// XOR over i of mix64(i * K + v_i): order-free digest of the array.
__global__ void k_digest(const u64* p, u64 n, unsigned long long* out) {
    u64 acc = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        acc ^= mix64(i * 0x9E3779B97F4A7C15ull + p[i]);
    for (int o = 16; o; o >>= 1) acc ^= __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicXor(out, (unsigned long long)acc);
}

namespace {

// Device scratch owned by the context for the kernel-level calls (grown on demand).
whirgpu_status kernel_scratch(whirgpu_ctx* c, size_t bytes, char** out) {
    if (bytes <= c->kscratch_bytes) {
        *out = c->kscratch;
        return WHIRGPU_OK;
    }
    cudaStreamSynchronize(c->stream);
    if (c->kscratch) {
        cudaFree(c->kscratch);
        c->allocated -= c->kscratch_bytes;
        c->kscratch = nullptr;
        c->kscratch_bytes = 0;
    }
    if (c->budget && c->allocated + bytes > c->budget) return fail(c, WHIRGPU_E_OOM, "kernel scratch above the HBM budget");
    cudaError_t e = cudaMalloc(&c->kscratch, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c->kscratch = nullptr;
        return fail(c, WHIRGPU_E_OOM, "kernel scratch");
    }
    c->kscratch_bytes = bytes;
    c->allocated += bytes;
    *out = c->kscratch;
    return WHIRGPU_OK;
}

LdeArgs lde_args(whirgpu_ctx* c, const u64* src, u64 m, u32 planes, u32 logN, u64* tmp, u64* out) {
    LdeArgs L{};
    L.src[0] = L.src[1] = L.src[2] = src;
    L.m = m;
    L.depth = planes;  // consecutive blocks of all vectors: plane p reads src + p m
    L.planes = planes;
    L.logN = logN;
    L.tmp = tmp;
    L.out = out;
    L.tw_stage = c->tw.tw_stage;
    L.tw_hi = c->tw.tw_hi;
    L.tw_lo = c->tw.tw_lo;
    L.tables = &c->lde_tables;
    return L;
}

// The inter-pass tables of `pl` (kernel-level calls run outside graph capture).
void prepare_plan_tables(whirgpu_ctx* c, const LdePlan& pl) {
    std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
    const uint64_t room = c->budget ? (c->budget > c->allocated ? c->budget - c->allocated : 0) : ~0ull;
    lde_tables_prepare_plan(c->lde_tables, pl, c->tw.tw_hi, c->tw.tw_lo, c->stream, room);
}

bool shape_ok(uint32_t log_len, uint32_t log_expansion, uint32_t log_depth) {
    return log_depth <= 6 && log_len >= log_depth && log_len <= 30 && log_expansion <= 16 &&
           log_len - log_depth + log_expansion <= TW_LOG;
}

}  // namespace
}  // namespace wg

using namespace wg;

extern "C" {

whirgpu_status whirgpu_rs_encode(whirgpu_ctx* c, const uint64_t* d_vectors, size_t count, uint32_t log_len,
                                 uint32_t log_expansion, uint32_t log_depth, uint64_t* d_tmp, uint64_t* d_planes) {
    if (!c || !d_vectors || !d_tmp || !d_planes || count == 0) return WHIRGPU_E_INVALID;
    if (!shape_ok(log_len, log_expansion, log_depth)) return fail(c, WHIRGPU_E_INVALID, "rs_encode shape");
    const u64 planes = (u64)count << log_depth;
    if (planes > 65535) return fail(c, WHIRGPU_E_INVALID, "too many planes");
    const u32 logN = log_len - log_depth + log_expansion;
    prepare_plan_tables(c, plan_lde(logN, log_expansion));
    const LdeArgs L = lde_args(c, d_vectors, 1ull << (log_len - log_depth), (u32)planes, logN, d_tmp, d_planes);
    if (launch_lde(L, c->stream) != 0) return fail(c, WHIRGPU_E_INVALID, "LDE launch");
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? WHIRGPU_OK : cuda_fail(c, e, "LDE");
}

whirgpu_status whirgpu_rs_commit_batch(whirgpu_ctx* c, const uint64_t* vectors, int location, size_t count,
                                       uint32_t log_len, uint32_t log_expansion, uint32_t log_depth, uint8_t* roots) {
    if (!c || !vectors || !roots || count == 0 || count > 65535) return WHIRGPU_E_INVALID;
    if (!shape_ok(log_len, log_expansion, log_depth)) return fail(c, WHIRGPU_E_INVALID, "rs_commit shape");
    const u64 planes = (u64)count << log_depth;
    if (planes > 65535) return fail(c, WHIRGPU_E_INVALID, "too many planes");
    const u32 logN = log_len - log_depth + log_expansion;
    const u64 N = 1ull << logN;
    const u64 in_words = count << log_len;
    prepare_plan_tables(c, plan_lde(logN, log_expansion));
    const u64 node_words = (2 * N) * 8;  // 32-bit words of one tree's node array
    const size_t bytes = (location == WHIRGPU_INPUT_DEVICE ? 0 : in_words * 8) + 2 * planes * N * 8 +
                         count * node_words * 4 + 256;
    char* ws = nullptr;
    whirgpu_status s = kernel_scratch(c, bytes, &ws);
    if (s != WHIRGPU_OK) return s;
    u64* tmp = reinterpret_cast<u64*>(ws);
    u64* out = tmp + planes * N;
    u32* nodes = reinterpret_cast<u32*>(out + planes * N);
    const u64* src = vectors;
    if (location != WHIRGPU_INPUT_DEVICE) {
        u64* in = reinterpret_cast<u64*>(nodes + count * node_words);
        cudaError_t e = cudaMemcpyAsync(in, vectors, in_words * 8, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "input copy");
        src = in;
    }
    const LdeArgs L = lde_args(c, src, 1ull << (log_len - log_depth), (u32)planes, logN, tmp, out);
    if (launch_lde(L, c->stream) != 0) return fail(c, WHIRGPU_E_INVALID, "LDE launch");
    const u32 depth = 1u << log_depth;
    if (launch_leaves_batch(out, N, depth, 1, nodes, (u32)count, (u64)depth * N, node_words, 0, c->stream) != 0)
        return fail(c, WHIRGPU_E_INVALID, "leaf launch");
    if (launch_merkle_batch(nodes, logN, (u32)count, node_words, c->stream) != 0)
        return fail(c, WHIRGPU_E_INVALID, "merkle launch");
    // root of tree k: the last node of its array (level logN), 32 bytes
    const u64 root_word = ((2ull << logN) - 2) * 8;
    for (size_t k = 0; k < count; ++k) {
        cudaError_t e = cudaMemcpyAsync(roots + 32 * k, nodes + k * node_words + root_word, 32, cudaMemcpyDeviceToHost,
                                        c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "root copy");
    }
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? WHIRGPU_OK : cuda_fail(c, e, "rs_commit");
}

// ---- pass-plan autotuner --------------------------------------------------
whirgpu_status whirgpu_ntt_autotune(whirgpu_ctx* c, uint32_t log_n, uint32_t log_expansion, uint32_t planes,
                                    uint32_t reps, whirgpu_ntt_plan* best, double* best_us, uint32_t* tried) {
    if (!c || !best || planes == 0 || planes > 65535 || log_n > TW_LOG || log_expansion > log_n || reps == 0)
        return WHIRGPU_E_INVALID;
    const u64 N = 1ull << log_n, m = N >> log_expansion;
    const size_t bytes = planes * m * 8 + 2 * planes * N * 8 + 256;
    char* ws = nullptr;
    whirgpu_status s = kernel_scratch(c, bytes, &ws);
    if (s != WHIRGPU_OK) return s;
    u64* tmp = reinterpret_cast<u64*>(ws);
    u64* out = tmp + planes * N;
    u64* src = out + planes * N;
    unsigned long long* dig = reinterpret_cast<unsigned long long*>(src + planes * m);
    k_fill_canonical<<<4 * device_sms(), 256, 0, c->stream>>>(src, planes * m, 0x5EED0000ull + log_n);
    const LdeArgs L = lde_args(c, src, m, planes, log_n, tmp, out);

    auto digest = [&](unsigned long long* h) -> bool {
        cudaMemsetAsync(dig, 0, 8, c->stream);
        k_digest<<<4 * device_sms(), 256, 0, c->stream>>>(out, planes * N, dig);
        return cudaMemcpyAsync(h, dig, 8, cudaMemcpyDeviceToHost, c->stream) == cudaSuccess &&
               cudaStreamSynchronize(c->stream) == cudaSuccess;
    };
    // Candidates: every radix split, and columns per CTA in {auto, 1..4} per pass
    // (three-pass plans with the automatic columns only), each with one tile per
    // CTA and pipelined.
    std::vector<LdePlan> cand;
    auto add = [&](LdePlan p) {
        p.logN = log_n;
        if (lde_plan_valid(p)) cand.push_back(p);
    };
    const u32 A = LDE_W_AUTO;
    const u32 wopts[] = {A, 1, 2, 3, 4};
    for (u32 pp = 0; pp <= 1; ++pp)
        for (u32 mb = 2; mb <= 4; ++mb) {
            if (log_n <= 11) add(LdePlan{log_n, 1, {log_n, 0, 0}, {A, A, A}, mb, pp});
            for (u32 r0 = 1; r0 < log_n && r0 <= 11; ++r0) {
                const u32 r1 = log_n - r0;
                if (r1 > 11) continue;
                for (u32 w0 : wopts)
                    for (u32 w1 : wopts) add(LdePlan{log_n, 2, {r0, r1, 0}, {w0, w1, A}, mb, pp});
            }
            if (log_n >= 12)
                for (u32 r0 = 1; r0 <= 11; ++r0)
                    for (u32 r1 = 1; r1 <= 11 && r0 + r1 < log_n; ++r1) {
                        const u32 r2 = log_n - r0 - r1;
                        if (r2 >= 1 && r2 <= 11) add(LdePlan{log_n, 3, {r0, r1, r2}, {A, A, A}, mb, pp});
                    }
        }
    if (cand.empty()) return fail(c, WHIRGPU_E_INVALID, "no valid plan");

    unsigned long long want = 0;
    prepare_plan_tables(c, default_plan_lde(log_n));
    if (launch_lde_plan(L, default_plan_lde(log_n), c->stream) != 0 || !digest(&want))
        return fail(c, WHIRGPU_E_CUDA, "reference LDE");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best_t = 1e30;
    LdePlan best_p = default_plan_lde(log_n);
    uint32_t rejected = 0;
    whirgpu_status result = WHIRGPU_OK;
    for (const LdePlan& p : cand) {
        prepare_plan_tables(c, p);  // the plans are timed as proofs run them
        cudaMemsetAsync(out, 0, planes * N * 8, c->stream);
        unsigned long long got = 0;
        if (launch_lde_plan(L, p, c->stream) != 0 || !digest(&got)) { result = fail(c, WHIRGPU_E_CUDA, "candidate"); break; }
        if (got != want) {  // never chosen; counted for the caller
            ++rejected;
            continue;
        }
        std::vector<float> ts;
        for (u32 r = 0; r < reps; ++r) {
            cudaEventRecord(e0, c->stream);
            launch_lde_plan(L, p, c->stream);
            cudaEventRecord(e1, c->stream);
            cudaEventSynchronize(e1);
            float t = 0;
            cudaEventElapsedTime(&t, e0, e1);
            ts.push_back(t);
        }
        std::sort(ts.begin(), ts.end());
        const double med = 1000.0 * ts[ts.size() / 2];
        if (med < best_t) { best_t = med; best_p = p; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (result != WHIRGPU_OK) return result;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "autotune");
    lde_install_plan(log_expansion, best_p);
    best->log_n = log_n;
    best->log_expansion = log_expansion;
    best->npass = best_p.npass;
    best->min_blocks = best_p.minb;
    best->pipelined = best_p.pipe;
    for (int k = 0; k < 3; ++k) {
        best->log_radix[k] = best_p.logR[k];
        best->log_cols[k] = best_p.logW[k];
    }
    if (best_us) *best_us = best_t;
    if (tried) *tried = (uint32_t)cand.size();
    if (rejected) return fail(c, WHIRGPU_E_DEVICE, std::to_string(rejected) + " LDE plans disagreed with the built-in plan");
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_ntt_set_plan(const whirgpu_ntt_plan* p) {
    if (!p) return WHIRGPU_E_INVALID;
    LdePlan q{};
    q.logN = p->log_n;
    q.npass = p->npass;
    q.minb = p->min_blocks;
    q.pipe = p->pipelined;
    for (int k = 0; k < 3; ++k) {
        q.logR[k] = k < (int)p->npass ? p->log_radix[k] : 0;
        q.logW[k] = k < (int)p->npass ? p->log_cols[k] : LDE_W_AUTO;
    }
    if (p->npass != 0 && !lde_plan_valid(q)) return WHIRGPU_E_INVALID;
    lde_install_plan(p->log_expansion, q);
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_ntt_get_plan(uint32_t log_n, uint32_t log_expansion, whirgpu_ntt_plan* out) {
    if (!out || log_n > TW_LOG) return WHIRGPU_E_INVALID;
    const LdePlan p = plan_lde(log_n, log_expansion);
    out->log_n = log_n;
    out->log_expansion = log_expansion;
    out->npass = p.npass;
    out->min_blocks = p.minb;
    out->pipelined = p.pipe;
    for (int k = 0; k < 3; ++k) {
        out->log_radix[k] = p.logR[k];
        out->log_cols[k] = p.logW[k];
    }
    return WHIRGPU_OK;
}

void whirgpu_ntt_clear_plans(void) { lde_clear_plans(); }

size_t whirgpu_ntt_list_plans(whirgpu_ntt_plan* out, size_t cap) {
    std::vector<u32> keys(cap);
    std::vector<LdePlan> plans(cap);
    const size_t n = lde_installed_plans(keys.data(), plans.data(), cap);
    for (size_t i = 0; i < n && i < cap; ++i) {
        out[i].log_n = keys[i] >> 8;
        out[i].log_expansion = keys[i] & 0xFF;
        out[i].npass = plans[i].npass;
        out[i].min_blocks = plans[i].minb;
        out[i].pipelined = plans[i].pipe;
        for (int k = 0; k < 3; ++k) {
            out[i].log_radix[k] = plans[i].logR[k];
            out[i].log_cols[k] = plans[i].logW[k];
        }
    }
    return n;
}

// Plan files: {"plans": [{"log_n": 22, "log_expansion": 2, "npass": 2,
//   "log_radix": [11, 11, 0], "log_cols": [2, 2, 255], "min_blocks": 3}, ...]} --
// the objects of the "plans" array are read by key (min_blocks optional);
// anything else in the file is ignored.
static bool read_int_field(const std::string& obj, const char* key, long* out) {
    const std::string k = std::string("\"") + key + "\"";
    size_t p = obj.find(k);
    if (p == std::string::npos) return false;
    p = obj.find(':', p + k.size());
    if (p == std::string::npos) return false;
    char* end = nullptr;
    *out = std::strtol(obj.c_str() + p + 1, &end, 10);
    return end != obj.c_str() + p + 1;
}
static bool read_triple(const std::string& obj, const char* key, long v[3]) {
    const std::string k = std::string("\"") + key + "\"";
    size_t p = obj.find(k);
    if (p == std::string::npos) return false;
    p = obj.find('[', p);
    if (p == std::string::npos) return false;
    const char* s = obj.c_str() + p + 1;
    for (int i = 0; i < 3; ++i) {
        char* end = nullptr;
        v[i] = std::strtol(s, &end, 10);
        if (end == s) return false;
        s = end;
        while (*s == ' ' || *s == ',' || *s == '\n' || *s == '\t') ++s;
    }
    return true;
}

whirgpu_status whirgpu_ntt_load_plans(const char* path, size_t* loaded) {
    if (loaded) *loaded = 0;
    if (!path) return WHIRGPU_E_INVALID;
    FILE* f = std::fopen(path, "rb");
    if (!f) return WHIRGPU_E_INVALID;
    std::string text;
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, k);
    std::fclose(f);
    size_t p = text.find("\"plans\"");
    if (p == std::string::npos) return WHIRGPU_E_INVALID;
    size_t n = 0;
    for (p = text.find('{', p); p != std::string::npos; p = text.find('{', p + 1)) {
        const size_t q = text.find('}', p);
        if (q == std::string::npos) break;
        const std::string obj = text.substr(p, q - p + 1);
        long ln, lx, np, r[3], w[3];
        if (!read_int_field(obj, "log_n", &ln) || !read_int_field(obj, "log_expansion", &lx) ||
            !read_int_field(obj, "npass", &np) || !read_triple(obj, "log_radix", r) || !read_triple(obj, "log_cols", w))
            continue;
        long mb = 0, pp = 0;
        read_int_field(obj, "min_blocks", &mb);  // optional
        read_int_field(obj, "pipelined", &pp);   // optional
        whirgpu_ntt_plan pl{};
        pl.min_blocks = (uint32_t)mb;
        pl.pipelined = (uint32_t)pp;
        pl.log_n = (uint32_t)ln;
        pl.log_expansion = (uint32_t)lx;
        pl.npass = (uint32_t)np;
        for (int i = 0; i < 3; ++i) {
            pl.log_radix[i] = (uint32_t)r[i];
            pl.log_cols[i] = (uint32_t)w[i];
        }
        if (whirgpu_ntt_set_plan(&pl) == WHIRGPU_OK) ++n;
        p = q;
    }
    if (loaded) *loaded = n;
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_ntt_save_plans(const char* path) {
    if (!path) return WHIRGPU_E_INVALID;
    std::vector<whirgpu_ntt_plan> v(whirgpu_ntt_list_plans(nullptr, 0));
    whirgpu_ntt_list_plans(v.data(), v.size());
    FILE* f = std::fopen(path, "wb");
    if (!f) return WHIRGPU_E_INVALID;
    std::fprintf(f, "{\"plans\": [\n");
    for (size_t i = 0; i < v.size(); ++i) {
        const auto& p = v[i];
        std::fprintf(f,
                     "  {\"log_n\": %u, \"log_expansion\": %u, \"npass\": %u, \"log_radix\": [%u, %u, %u], "
                     "\"log_cols\": [%u, %u, %u], \"min_blocks\": %u, \"pipelined\": %u}%s\n",
                     p.log_n, p.log_expansion, p.npass, p.log_radix[0], p.log_radix[1], p.log_radix[2], p.log_cols[0],
                     p.log_cols[1], p.log_cols[2], p.min_blocks, p.pipelined, i + 1 < v.size() ? "," : "");
    }
    std::fprintf(f, "]}\n");
    std::fclose(f);
    return WHIRGPU_OK;
}

// Plans shipped beside the library (ntt_plans.json next to libwhirgpu.so), or
// the file named by WHIRGPU_NTT_PLANS, are installed once per process.
static void load_default_plans_once() {
    const char* env = std::getenv("WHIRGPU_NTT_PLANS");
    if (env && *env) {
        whirgpu_ntt_load_plans(env, nullptr);
        return;
    }
    Dl_info info{};
    if (dladdr(reinterpret_cast<void*>(&whirgpu_ntt_load_plans), &info) && info.dli_fname) {
        std::string dir(info.dli_fname);
        const size_t slash = dir.rfind('/');
        dir = slash == std::string::npos ? std::string(".") : dir.substr(0, slash);
        whirgpu_ntt_load_plans((dir + "/ntt_plans.json").c_str(), nullptr);
    }
}

void whirgpu_ntt_load_default_plans(void) {
    static std::once_flag once;
    std::call_once(once, load_default_plans_once);
}

}  // extern "C"
