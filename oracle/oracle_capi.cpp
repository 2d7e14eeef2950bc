// oracle_capi.cpp -- TEST INFRASTRUCTURE ONLY: C entry points of the CPU
// oracle (whir_oracle.hpp) for the Python tests (ctypes).  Never linked into,
// or called by, the product library.
#include "whir_oracle.hpp"

#include <cstring>
#include <exception>
#include <new>

using namespace oracle;

namespace {
Params make_params(u64 rho, u64 k, u64 sec, u64 powb, int unique) {
    Params p;
    p.starting_log_inv_rate = rho;
    p.initial_folding_factor = k;
    p.folding_factor = k;
    p.security_level = sec;
    p.pow_bits = powb;
    p.unique_decoding = unique != 0;
    p.batch_size = 1;
    return p;
}
std::vector<E3> read_e3(const u64* w, size_t n) {
    std::vector<E3> v(n);
    for (size_t i = 0; i < n; ++i) for (int c = 0; c < 3; ++c) v[i].c[c] = w[3 * i + c];
    return v;
}
}  // namespace

extern "C" {

// Codeword order of every later commitment and opening: 0 natural (the C++
// reference), 1 coset-major (the Rust crate without rs_in_order).
void oracle_set_coset_major(int on) { coset_major_order() = on != 0; }
u64 oracle_transpose_permute(u64 k, u64 rows, u64 cols) { return transpose_permute(k, rows, cols); }
void oracle_blake3(const u8* d, size_t n, u8* out) { Hash h = blake3(d, n); std::memcpy(out, h.data(), 32); }
void oracle_sha3_256(const u8* d, size_t n, u8* out) { sha3_256(d, n, out); }
void oracle_sha3_512(const u8* d, size_t n, u8* out) { sha3_512(d, n, out); }
void oracle_shake128(const u8* d, size_t n, u8* out, size_t m) { shake128(d, n, out, m); }
void oracle_keccak_f1600(u64* s) { keccak_f1600(s); }

u64 oracle_fmul(u64 a, u64 b) { return fmul(a, b); }
u64 oracle_fadd(u64 a, u64 b) { return fadd(a, b); }
u64 oracle_fsub(u64 a, u64 b) { return fsub(a, b); }
u64 oracle_fpow(u64 a, u64 e) { return fpow(a, e); }
size_t oracle_indices(const u8* ent, u64 N, u64 count, int dedup, u64* out) {
    auto v = indices_from_entropy(ent, N, count, dedup != 0);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    return v.size();
}
u64 oracle_root_of_unity(u64 n) { return root_of_unity(n); }
void oracle_e3_mul(const u64* a, const u64* b, u64* out) {
    E3 x, y;
    for (int i = 0; i < 3; ++i) { x.c[i] = a[i]; y.c[i] = b[i]; }
    E3 r = x * y;
    for (int i = 0; i < 3; ++i) out[i] = r.c[i];
}

void oracle_ntt(u64* data, size_t n) {
    std::vector<u64> v(data, data + n);
    ntt_inplace(v);
    std::memcpy(data, v.data(), n * 8);
}
// RS encode of one base vector into a row-major N x depth matrix.
void oracle_rs_encode_base(const u64* v, size_t len, u64 N, u64 depth, u64* out) {
    std::vector<u64> in(v, v + len);
    auto m = rs_encode_base(in, N, depth);
    std::memcpy(out, m.data(), m.size() * 8);
}
// RS encode of one Ext3 vector (AoS, 3 words per element) into AoS rows.
void oracle_rs_encode_e3(const u64* v, size_t len, u64 N, u64 depth, u64* out) {
    auto m = rs_encode_e3(read_e3(v, len), N, depth);
    std::memcpy(out, m.data(), m.size() * 24);
}
// Matrix-commitment root of one base vector (irs_commit.hpp:402-470 with one
// vector): RS encode into N x depth rows, BLAKE3 leaves, Merkle root.
void oracle_rs_commit_root(const u64* v, size_t len, u64 N, u64 depth, u8* root_out) {
    std::vector<u64> in(v, v + len);
    auto m = rs_encode_base(in, N, depth);
    auto lv = leaves_base(m, depth);
    auto nodes = merkle_build(lv);
    std::memcpy(root_out, nodes.back().data(), 32);
}
// Merkle root (and optionally the node array) of `n` 32-byte leaves.
void oracle_merkle_root(const u8* leaves, size_t n, u8* root_out, u8* nodes_out) {
    std::vector<Hash> lv(n);
    for (size_t i = 0; i < n; ++i) std::memcpy(lv[i].data(), leaves + 32 * i, 32);
    auto nodes = merkle_build(lv);
    std::memcpy(root_out, nodes.back().data(), 32);
    if (nodes_out) for (size_t i = 0; i < nodes.size(); ++i) std::memcpy(nodes_out + 32 * i, nodes[i].data(), 32);
}
// Merkle opening hints; returns the number of 32-byte hints written.
size_t oracle_merkle_open(const u8* leaves, size_t n, const u64* idx, size_t nidx, u8* out, size_t cap) {
    std::vector<Hash> lv(n);
    for (size_t i = 0; i < n; ++i) std::memcpy(lv[i].data(), leaves + 32 * i, 32);
    auto nodes = merkle_build(lv);
    auto hints = merkle_open(nodes, layers_for(n), std::vector<u64>(idx, idx + nidx));
    for (size_t i = 0; i < hints.size() && i < cap; ++i) std::memcpy(out + 32 * i, hints[i].data(), 32);
    return hints.size();
}
u64 oracle_find_nonce(const u8* ch, u64 threshold) { return find_nonce(ch, threshold); }
u64 oracle_find_nonce_sha2(const u8* ch, u64 threshold) { return find_nonce(ch, threshold, Engine::Sha2); }
void oracle_sha256(const u8* d, size_t n, u8* out) {
    Hash h = sha256(d, n);
    std::memcpy(out, h.data(), 32);
}
// Merkle root / opening hints with SHA-256 nodes.
void oracle_merkle_root_sha2(const u8* leaves, size_t n, u8* root_out) {
    std::vector<Hash> lv(n);
    for (size_t i = 0; i < n; ++i) std::memcpy(lv[i].data(), leaves + 32 * i, 32);
    auto nodes = merkle_build(lv, Engine::Sha2);
    std::memcpy(root_out, nodes.back().data(), 32);
}
size_t oracle_merkle_open_sha2(const u8* leaves, size_t n, const u64* idx, size_t nidx, u8* out, size_t cap) {
    std::vector<Hash> lv(n);
    for (size_t i = 0; i < n; ++i) std::memcpy(lv[i].data(), leaves + 32 * i, 32);
    auto nodes = merkle_build(lv, Engine::Sha2);
    auto hints = merkle_open(nodes, layers_for(n), std::vector<u64>(idx, idx + nidx));
    for (size_t i = 0; i < hints.size() && i < cap; ++i) std::memcpy(out + 32 * i, hints[i].data(), 32);
    return hints.size();
}

// Opaque transcript for the per-primitive pins (base/Ext3 challenges).
void* oracle_tx_new(void) { return new (std::nothrow) Transcript(); }
void oracle_tx_free(void* t) { delete static_cast<Transcript*>(t); }
void oracle_tx_absorb(void* t, const u8* d, size_t n) { static_cast<Transcript*>(t)->absorb(d, n); }
void oracle_tx_message(void* t, const u8* d, size_t n) { static_cast<Transcript*>(t)->message_bytes(d, n); }
void oracle_tx_squeeze(void* t, u8* out, size_t n) { static_cast<Transcript*>(t)->squeeze(out, n); }
u64 oracle_tx_challenge_base(void* t) { return static_cast<Transcript*>(t)->challenge_base(); }
void oracle_tx_challenge_e3(void* t, u64* out) {
    E3 e = static_cast<Transcript*>(t)->challenge_e3();
    for (int i = 0; i < 3; ++i) out[i] = e.c[i];
}
size_t oracle_tx_narg(void* t, u8* out, size_t cap) {
    auto& v = static_cast<Transcript*>(t)->narg;
    if (out) std::memcpy(out, v.data(), std::min(cap, v.size()));
    return v.size();
}

void oracle_cli_domain_separator(u64 rho, u64 k, u64 sec, u64 powb, int unique, u8* out96) {
    DomainSep ds = cli_domain_separator(make_params(rho, k, sec, powb, unique));
    std::memcpy(out96, ds.protocol_id, 64);
    std::memcpy(out96 + 64, ds.session_id, 32);
}

// Schedule of Config::from_params as a flat u64 array:
//   [n_rounds, init_N, init_q, init_ood, init_sc_pow, skip_pow,
//    per round: vec, N, q, ood, pow, sc_pow,  final_size, final_rounds, final_pow, final_sc_pow]
size_t oracle_whir_config(u64 n, u64 rho, u64 k, u64 sec, u64 powb, int unique, u64* out, size_t cap) {
    try {
        WhirCfg c = whir_from_params(1ull << n, make_params(rho, k, sec, powb, unique));
        std::vector<u64> v{c.rounds.size(), c.initial.codeword_length, c.initial.in_domain, c.initial.out_domain,
                           c.initial_sumcheck.pow_threshold, c.initial_skip_pow};
        for (auto& r : c.rounds) {
            v.insert(v.end(), {r.irs.vector_size, r.irs.codeword_length, r.irs.in_domain, r.irs.out_domain,
                               r.pow_threshold, r.sumcheck.pow_threshold});
        }
        v.insert(v.end(), {c.final_sumcheck.initial_size, c.final_sumcheck.num_rounds, c.final_pow,
                           c.final_sumcheck.pow_threshold});
        for (size_t i = 0; i < v.size() && i < cap; ++i) out[i] = v[i];
        return v.size();
    } catch (const std::exception&) {
        return 0;
    }
}

// MLE of a base vector (2^n entries) at an Ext3 point (n coordinates).
void oracle_mle_eval_base(const u64* v, u64 n, const u64* point, u64* out) {
    std::vector<u64> vec(v, v + (1ull << n));
    E3 r = mle_eval_base(vec, read_e3(point, n));
    for (int i = 0; i < 3; ++i) out[i] = r.c[i];
}

// Whole commit + prove with the CLI domain separator and MLE-point forms.
// Returns 0 on success; narg/hints lengths are written to lens[0], lens[1]
// (the buffers receive min(cap, len) bytes).
int oracle_whir_prove(u64 n, u64 rho, u64 k, u64 sec, u64 powb, int unique, const u64* coeffs,
                      const u64* points, size_t npoints, const u64* evals, u8* narg, size_t narg_cap,
                      u8* hints, size_t hints_cap, u64* lens, int sha2) {
    try {
        Params p = make_params(rho, k, sec, powb, unique);
        if (sha2) std::memcpy(p.hash_id, SHA2_ENGINE_ID, 32);
        std::vector<u64> v(coeffs, coeffs + (1ull << n));
        Statement st;
        for (size_t i = 0; i < npoints; ++i) st.mle_points.push_back(read_e3(points + 3 * n * i, n));
        st.evaluations = read_e3(evals, npoints);
        ProofOut o = prove(p, v, st, cli_domain_separator(p));
        lens[0] = o.narg.size();
        lens[1] = o.hints.size();
        std::memcpy(narg, o.narg.data(), std::min(narg_cap, o.narg.size()));
        std::memcpy(hints, o.hints.data(), std::min(hints_cap, o.hints.size()));
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// Commit + prove with a statement of mixed forms: kinds[f] = 0 MultilinearExtension
// (n Ext3 coordinates), 1 dense Covector (2^n Ext3 values); form_data holds the
// forms' words back to back in form order.  evals: nforms * V values, form-major.
// flags: bit 0 SHA-2 engine, bit 1 Identity<Goldilocks> target (base-field
// values given as (x, 0, 0)).
int oracle_whir_prove_forms(u64 n, u64 rho, u64 k, u64 sec, u64 powb, int unique, u64 batch_size, u64 num_witnesses,
                            const u64* coeffs, const int* kinds, size_t nforms, const u64* form_data, const u64* evals,
                            u8* narg, size_t narg_cap, u8* hints, size_t hints_cap, u64* lens, int sha2) {
    try {
        Params p = make_params(rho, k, sec, powb, unique);
        p.batch_size = batch_size;
        if (sha2 & 1) std::memcpy(p.hash_id, SHA2_ENGINE_ID, 32);
        const int deg = (sha2 & 2) ? 1 : 3;
        const u64 V = batch_size * num_witnesses, size = 1ull << n;
        std::vector<std::vector<u64>> vs(V);
        for (u64 j = 0; j < V; ++j) vs[j].assign(coeffs + j * size, coeffs + (j + 1) * size);
        Statement st;
        const u64* d = form_data;
        for (size_t f = 0; f < nforms; ++f) {
            if (kinds[f] == 0) {
                st.mle_points.push_back(read_e3(d, n));
                d += 3 * n;
            } else {
                st.covectors.push_back(read_e3(d, size));
                d += 3 * size;
            }
            st.dense.push_back(kinds[f] != 0);
        }
        st.evaluations = read_e3(evals, nforms * V);
        ProofOut o = prove_multi(p, vs, num_witnesses, st, cli_domain_separator(p), deg);
        lens[0] = o.narg.size();
        lens[1] = o.hints.size();
        std::memcpy(narg, o.narg.data(), std::min(narg_cap, o.narg.size()));
        std::memcpy(hints, o.hints.data(), std::min(hints_cap, o.hints.size()));
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// Commit + prove for a Config given field by field (the reference's golden
// dumpers build it so, cpp/tests/dump_whir.cpp:121-148) and a given domain
// separator.  cfg words:
//   [0..4] initial committer: vector_size, codeword_length, depth, in_domain, out_domain
//   [5..7] initial sumcheck rounds, its PoW threshold, the skip-PoW threshold
//   [8] R, then per round 8 words: vector_size, codeword_length, depth, in_domain,
//       out_domain, PoW threshold, sumcheck rounds, sumcheck PoW threshold
//   then final sumcheck rounds, its PoW threshold, the final PoW threshold.
// deg: 3 Basefield<GoldilocksExt3>, 1 Identity<Goldilocks>.  eval_point
// receives the FinalClaim evaluation point (3 words per coordinate).
int oracle_whir_prove_config(const u64* cfg, size_t cfg_len, int deg, int sha2, const u8* ds96, u64 batch_size,
                             u64 num_witnesses, const u64* coeffs, const int* kinds, size_t nforms,
                             const u64* form_data, const u64* evals, u8* narg, size_t narg_cap, u8* hints,
                             size_t hints_cap, u64* lens, u64* eval_point, size_t eval_point_cap) {
    try {
        if (cfg_len < 12) return 2;
        WhirCfg c;
        auto irs = [&](const u64* w) {
            IrsCfg r;
            r.num_vectors = 1;
            r.vector_size = w[0];
            r.codeword_length = w[1];
            r.depth = w[2];
            r.in_domain = w[3];
            r.out_domain = w[4];
            return r;
        };
        c.initial = irs(cfg);
        c.initial.num_vectors = batch_size;
        c.initial_sumcheck = {cfg[0], cfg[5], cfg[6]};
        c.initial_skip_pow = cfg[7];
        const u64 R = cfg[8];
        if (cfg_len != 12 + 8 * R) return 2;
        u64 size = cfg[0] >> cfg[5];
        for (u64 r = 0; r < R; ++r) {
            const u64* w = cfg + 9 + 8 * r;
            RoundCfg rc;
            rc.irs = irs(w);
            rc.pow_threshold = w[5];
            rc.sumcheck = {w[0], w[6], w[7]};
            c.rounds.push_back(rc);
            size = w[0] >> w[6];
        }
        const u64* f = cfg + 9 + 8 * R;
        c.final_sumcheck = {size, f[0], f[1]};
        c.final_pow = f[2];
        const u64 V = batch_size * num_witnesses, vsize = cfg[0];
        std::vector<std::vector<u64>> vs(V);
        for (u64 j = 0; j < V; ++j) vs[j].assign(coeffs + j * vsize, coeffs + (j + 1) * vsize);
        u64 n = 0;
        while ((1ull << n) < vsize) ++n;
        Statement st;
        const u64* d = form_data;
        for (size_t k = 0; k < nforms; ++k) {
            if (kinds[k] == 0) {
                st.mle_points.push_back(read_e3(d, n));
                d += 3 * n;
            } else {
                st.covectors.push_back(read_e3(d, vsize));
                d += 3 * vsize;
            }
            st.dense.push_back(kinds[k] != 0);
        }
        st.evaluations = read_e3(evals, nforms * V);
        DomainSep ds;
        std::memcpy(ds.protocol_id, ds96, 64);
        std::memcpy(ds.session_id, ds96 + 64, 32);
        ProofOut o = prove_cfg(c, sha2 ? Engine::Sha2 : Engine::Blake3, deg, batch_size, vs, num_witnesses, st, ds);
        lens[0] = o.narg.size();
        lens[1] = o.hints.size();
        lens[2] = o.evaluation_point.size();
        std::memcpy(narg, o.narg.data(), std::min(narg_cap, o.narg.size()));
        std::memcpy(hints, o.hints.data(), std::min(hints_cap, o.hints.size()));
        for (size_t k = 0; k < o.evaluation_point.size() && k < eval_point_cap; ++k)
            for (int j = 0; j < 3; ++j) eval_point[3 * k + j] = o.evaluation_point[k].c[j];
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// Commit of num_witnesses witnesses of batch_size vectors each, then one
// prove over all of them.  coeffs: num_witnesses * batch_size vectors of 2^n
// words, back to back; evals: npoints * num_vectors Ext3 values, form-major.
int oracle_whir_prove_multi(u64 n, u64 rho, u64 k, u64 sec, u64 powb, int unique, u64 batch_size, u64 num_witnesses,
                            const u64* coeffs, const u64* points, size_t npoints, const u64* evals, u8* narg,
                            size_t narg_cap, u8* hints, size_t hints_cap, u64* lens, int sha2) {
    try {
        Params p = make_params(rho, k, sec, powb, unique);
        p.batch_size = batch_size;
        if (sha2) std::memcpy(p.hash_id, SHA2_ENGINE_ID, 32);
        const u64 V = batch_size * num_witnesses, size = 1ull << n;
        std::vector<std::vector<u64>> vs(V);
        for (u64 j = 0; j < V; ++j) vs[j].assign(coeffs + j * size, coeffs + (j + 1) * size);
        Statement st;
        for (size_t i = 0; i < npoints; ++i) st.mle_points.push_back(read_e3(points + 3 * n * i, n));
        st.evaluations = read_e3(evals, npoints * V);
        ProofOut o = prove_multi(p, vs, num_witnesses, st, cli_domain_separator(p));
        lens[0] = o.narg.size();
        lens[1] = o.hints.size();
        std::memcpy(narg, o.narg.data(), std::min(narg_cap, o.narg.size()));
        std::memcpy(hints, o.hints.data(), std::min(hints_cap, o.hints.size()));
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

}  // extern "C"
