// prover.cu -- workspace layout and kernel schedule of commit + prove.
//
// The order of steps is the reference's (cpp/include/whir/protocols/whir/
// whir.hpp:303-309 and whir_prover.hpp:56-407) over Goldilocks vectors with
// Ext3 challenges, for nwit initial commitments of batch_size vectors each:
//   commit:  per commitment: RS encode (batch_size * 2^k planes) -> leaves ->
//            Merkle root (message) -> OOD points / values of its vectors
//   prove:   OOD completion across commitments, vector + constraint RLC,
//            covector (and the combined vector), initial sumcheck,
//            per round: commit folded vector, PoW, open previous commitment(s),
//                       STIR RLC + covector update, sumcheck;
//            final vector, final PoW, final opening, final sumcheck.
#include <algorithm>
#include <stdexcept>

#include "launch.h"
#include "prover.h"
#include "state.cuh"

namespace wg {

static_assert(MAX_FORMS == 8, "ProofPlan::dense and CovInitArgs::dense hold MAX_FORMS pointers");

namespace {
size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
struct Bump {
    size_t cur = 0;
    size_t take(size_t bytes) {
        size_t o = cur;
        cur = align_up(cur + bytes, 256);
        return o;
    }
};
uint32_t ilog2(uint64_t v) {
    uint32_t k = 0;
    while ((1ull << k) < v) ++k;
    return k;
}
}  // namespace

ProofPlan make_plan(uint32_t n, const ProtocolParams& params, int n_forms, size_t ds_len, uint32_t nwit) {
    return make_plan(make_schedule(n, params), params, n_forms, ds_len, nwit);
}

ProofPlan make_plan(const WhirSchedule& sched, const ProtocolParams& params, int n_forms, size_t ds_len, uint32_t nwit) {
    validate_schedule(sched);
    if (params.field_degree < 1 || params.field_degree > 3) throw std::invalid_argument("field degree must be 1, 2 or 3");
    const uint32_t n = ilog2(sched.initial.vector_size);
    ProofPlan p;
    p.sch = sched;
    p.params = params;
    p.n = n;
    p.n_forms = n_forms;
    const uint32_t deg = (uint32_t)params.field_degree;  // words per target-field element
    if (n_forms < 0 || n_forms > MAX_FORMS) throw std::invalid_argument("too many statement forms");
    if (params.batch_size == 0 || nwit == 0) throw std::invalid_argument("no committed vectors");
    if (nwit > (uint32_t)MAX_WITNESSES) throw std::invalid_argument("too many witnesses");
    if (params.batch_size * nwit > (uint64_t)MAX_VECTORS) throw std::invalid_argument("too many committed vectors");
    p.nwit = nwit;
    p.nvec = (uint32_t)params.batch_size * nwit;
    const uint32_t batch = (uint32_t)params.batch_size;
    const WhirSchedule& s = p.sch;
    auto check_irs = [&params](const IrsSchedule& c, uint32_t row_elems, uint32_t ncomp) {
        const uint64_t N = c.codeword_length;
        if (N == 0 || (N & (N - 1))) throw std::invalid_argument("codeword length must be a power of two");
        if (ilog2(N) > TW_LOG) throw std::invalid_argument("codeword length above 2^26");
        if (c.depth > (uint64_t)MAX_DEPTH) throw std::invalid_argument("folding factor too large");
        if (params.hash == 0 && (uint64_t)row_elems * ncomp * 8 > 16384)
            throw std::invalid_argument("rows above 16 BLAKE3 chunks");
        if (c.in_domain > (uint64_t)MAX_QUERIES) throw std::invalid_argument("too many in-domain samples");
        if (c.out_domain > (uint64_t)MAX_OOD) throw std::invalid_argument("too many out-of-domain samples");
        if (N % c.message_length() != 0) throw std::invalid_argument("codeword length not a multiple of message length");
    };
    check_irs(s.initial, (uint32_t)s.initial.depth * batch, 1);
    for (const auto& r : s.rounds) check_irs(r.irs, (uint32_t)r.irs.depth, deg);
    if ((size_t)n > (size_t)MAX_SC_ROUNDS) throw std::invalid_argument("too many variables");
    if (s.rounds.size() + nwit > (size_t)MAX_COMMITS) throw std::invalid_argument("too many rounds");

    Bump b;
    const uint64_t size = 1ull << n;
    p.off_coeffs = b.take((size_t)p.nvec * size * 8);
    // One vector: round 0 reads the base coefficients and the first fold
    // writes half the size.  Several vectors, or no initial round: the
    // covector pass writes the (combined, lifted) vector at full size.
    p.full_vector = p.nvec > 1 || s.initial_sumcheck.num_rounds == 0;
    p.a_plane_words = p.full_vector ? size : std::max<uint64_t>(size / 2, 1);
    p.off_a = b.take(3 * p.a_plane_words * 8);
    p.cov_plane_words = size;
    p.off_cov = b.take(3 * size * 8);
    size_t tmp_words = 0;
    auto commit_of = [&](const IrsSchedule& c, uint32_t row_elems, uint32_t ncomp) {
        CommitBuffers cb;
        cb.N = c.codeword_length;
        cb.logN = ilog2(cb.N);
        cb.logX = cb.logN - ilog2(c.message_length());
        if (params.coset_major) cb.perm_log_e = cb.logN - ilog2(c.message_length());
        cb.depth = row_elems;
        cb.ncomp = ncomp;
        tmp_words = std::max(tmp_words, (size_t)cb.N * cb.depth * ncomp);
        return cb;
    };
    {  // initial commitments: planes side by side, then node arrays side by side
        CommitBuffers cb = commit_of(s.initial, (uint32_t)s.initial.depth * batch, 1);
        p.init_planes_stride = align_up((size_t)cb.N * cb.depth * 8, 256);
        p.init_nodes_stride = align_up((2 * cb.N - 1) * 32, 256);
        const size_t planes0 = b.take(p.init_planes_stride * nwit);
        const size_t nodes0 = b.take(p.init_nodes_stride * nwit);
        for (uint32_t w = 0; w < nwit; ++w) {
            cb.planes = planes0 + w * p.init_planes_stride;
            cb.nodes = nodes0 + w * p.init_nodes_stride;
            p.commits.push_back(cb);
        }
    }
    for (const auto& r : s.rounds) {
        CommitBuffers cb = commit_of(r.irs, (uint32_t)r.irs.depth, deg);
        cb.planes = b.take((size_t)cb.N * cb.depth * deg * 8);
        cb.nodes = b.take((2 * cb.N - 1) * 32);
        p.commits.push_back(cb);
    }
    p.off_tmp = b.take(tmp_words * 8);
    p.off_sc_scratch = b.take(sumcheck_scratch_bytes());
    p.ood_values = std::max<uint32_t>((uint32_t)s.initial.out_domain * p.nvec, (uint32_t)MAX_OOD);
    p.off_ood_scratch = b.take(ood_scratch_bytes(1ull << n, p.ood_values));
    const int init_ood = (int)(s.initial.out_domain * nwit);
    size_t cov_scratch = cov_init_scratch_bytes(n, n_forms, init_ood);
    cov_scratch = std::max(cov_scratch, tsc_scratch_bytes(n, (uint32_t)s.initial_sumcheck.num_rounds, n_forms + init_ood));
    for (size_t r = 0; r < s.rounds.size(); ++r) {
        const IrsSchedule& prev = r == 0 ? s.initial : s.rounds[r - 1].irs;
        const int npts = (int)(s.rounds[r].irs.out_domain + prev.in_domain);
        cov_scratch = std::max(cov_scratch, cov_acc_scratch_bytes(s.rounds[r].irs.vector_size, npts));
    }
    p.off_cov_scratch = b.take(cov_scratch);
    p.off_tx = b.take(sizeof(TxState));
    p.off_scalars = b.take(sizeof(ProofScalars));

    // Proof stream sizes.
    size_t narg = 0, hints = 0;
    const uint64_t esz = 8ull * deg;  // bytes of a target-field element message
    auto commit_narg = [esz](const IrsSchedule& c, uint64_t vectors) { return 32 + esz * c.out_domain * vectors; };
    auto pow_narg = [](uint64_t thr) { return thr == ~0ull ? 0 : 8; };
    auto sumcheck_narg = [&](const SumcheckSchedule& sc) { return sc.num_rounds * (2 * esz + pow_narg(sc.pow_threshold)); };
    auto open_hints = [](const IrsSchedule& c, uint64_t vectors, uint32_t ncomp, uint64_t commitments) {
        const uint64_t logN = ilog2(c.codeword_length);
        const uint64_t merkle = std::min<uint64_t>(c.in_domain * logN, c.codeword_length);
        return commitments * (8 + c.in_domain * c.depth * vectors * 8 * ncomp + 32 * merkle);
    };
    narg += nwit * commit_narg(s.initial, batch);
    narg += esz * s.initial.out_domain * nwit * (p.nvec - batch);  // OOD completion
    // initial sumcheck, or (no constraint) the skip-PoW: added below per variant
    const size_t narg_initial_constrained = sumcheck_narg(s.initial_sumcheck);
    const size_t narg_initial_free = pow_narg(s.initial_skip_pow);
    size_t sc_rounds = s.initial_sumcheck.num_rounds;
    for (size_t r = 0; r < s.rounds.size(); ++r) {
        narg += commit_narg(s.rounds[r].irs, 1) + pow_narg(s.rounds[r].pow_threshold) + sumcheck_narg(s.rounds[r].sumcheck);
        hints += r == 0 ? open_hints(s.initial, batch, 1, nwit) : open_hints(s.rounds[r - 1].irs, 1, deg, 1);
        sc_rounds += s.rounds[r].sumcheck.num_rounds;
    }
    narg += esz * s.final_sumcheck.initial_size + pow_narg(s.final_pow) + sumcheck_narg(s.final_sumcheck);
    hints += s.rounds.empty() ? open_hints(s.initial, batch, 1, nwit) : open_hints(s.rounds.back().irs, 1, deg, 1);
    sc_rounds += s.final_sumcheck.num_rounds;
    p.narg_len_constrained = narg + narg_initial_constrained;
    p.narg_len_free = narg + narg_initial_free;
    p.narg_len = std::max(p.narg_len_constrained, p.narg_len_free);  // stream capacity until the forms are known
    p.hints_cap = hints;
    p.total_sumcheck_rounds = sc_rounds;
    p.off_narg = b.take(p.narg_len + 64);
    p.off_hints = b.take(hints + 64);
    p.ds_cap = std::max<size_t>(ds_len, 96);
    p.off_ds = b.take(p.ds_cap);
    p.off_points = b.take((size_t)std::max(n_forms, 1) * n * 24 + 64);
    p.total_bytes = b.cur;
    return p;
}

void plan_set_forms(ProofPlan& p, int n_forms) {
    p.n_forms = n_forms;
    p.narg_len = n_forms + p.sch.initial.out_domain > 0 ? p.narg_len_constrained : p.narg_len_free;
}

TxState* plan_tx(const ProofPlan& p, char* ws) { return p.tx_ext ? p.tx_ext : reinterpret_cast<TxState*>(ws + p.off_tx); }
ProofScalars* plan_scalars(const ProofPlan& p, char* ws) { return reinterpret_cast<ProofScalars*>(ws + p.off_scalars); }

namespace {

struct Ctx {
    const ProofPlan& p;
    char* ws;
    const DeviceTables& tw;
    cudaStream_t st;
    Timer* timer;
    TxState* tx() const { return plan_tx(p, ws); }
    ProofScalars* sc() const { return plan_scalars(p, ws); }
    uint64_t* w(size_t off) const { return reinterpret_cast<uint64_t*>(ws + off); }
    uint64_t* a(int c) const { return w(p.off_a) + (size_t)c * p.a_plane_words; }
    uint64_t* cov(int c) const { return w(p.off_cov) + (size_t)c * p.cov_plane_words; }
};

#define WG_TRY(x)                 \
    do {                          \
        int _rc = (x);            \
        if (_rc != 0) return _rc; \
    } while (0)

// Launch `x` bracketed by the family timer when timing is on.
#define WG_TIMED(c, fam, x)                                \
    do {                                                   \
        if ((c).timer) (c).timer->begin((fam), (c).st);    \
        int _rc = (x);                                     \
        if ((c).timer) (c).timer->end((fam), (c).st);      \
        if (_rc != 0) return _rc;                          \
    } while (0)

// RS encode + leaves + Merkle of commitment `ci` whose message is `vectors`
// vectors (src planes, vsize words each, consecutive), then the OOD values of
// those vectors at the commitment's points, stored at out[j * out_stride + v].
int commit_vectors(const Ctx& c, int ci, const uint64_t* const src[3], uint32_t ncomp, uint64_t vsize,
                   uint32_t vectors, int n_ood, E3* out, uint32_t out_stride) {
    const CommitBuffers& cb = c.p.commits[ci];
    const uint32_t fold_depth = cb.depth / vectors;
    LdeArgs L{};
    for (int k = 0; k < 3; ++k) L.src[k] = src[k] ? src[k] : src[0];
    L.m = vsize / fold_depth;
    L.depth = cb.depth;
    L.planes = cb.depth * ncomp;
    L.logN = cb.logN;
    L.tmp = c.w(c.p.off_tmp);
    L.out = c.w(cb.planes);
    L.tw_stage = c.tw.tw_stage;
    L.tw_hi = c.tw.tw_hi;
    L.tw_lo = c.tw.tw_lo;
    L.tables = c.tw.lde;
    WG_TIMED(c, FAM_NTT, launch_lde(L, c.st));
    uint32_t* nodes = reinterpret_cast<uint32_t*>(c.ws + cb.nodes);
    WG_TIMED(c, FAM_LEAF, launch_leaves(c.w(cb.planes), cb.N, cb.depth, ncomp, nodes, c.p.params.hash, c.st,
                                        cb.perm_log_e));
    WG_TIMED(c, FAM_MERKLE, launch_merkle(nodes, cb.logN, c.tx(), c.sc(), ci, n_ood, c.p.params.hash, c.st));
    OodArgs o{};
    for (int k = 0; k < 3; ++k) o.v[k] = src[k] ? src[k] : src[0];
    o.ext3 = ncomp != 1;  // Ext2 vectors are read as (c0, c1, c2 = 0) planes
    o.ext2 = c.p.params.field_degree == 2;
    o.size = vsize;
    o.nvec = vectors;
    o.vec_stride = vsize;
    o.pts = &c.sc()->ood_pts[ci][0];
    o.n_ood = n_ood;
    o.out = out;
    o.out_stride = out_stride;
    o.tx = c.tx();
    o.scratch = c.ws + c.p.off_ood_scratch;
    o.scratch_values = c.p.ood_values;
    WG_TIMED(c, FAM_OOD, launch_ood(o, c.st));
    return 0;
}

// `rounds` sumcheck rounds on (a, cov) of size `size`.  `base_first`: the
// vector is still the base-field coefficient array (first sumcheck only).
// Leaves a, cov folded to size >> rounds when `fold_after` is set.
int sumcheck(const Ctx& c, const SumcheckSchedule& s, uint64_t size, bool base_first, int& r_slot, bool fold_after) {
    if (s.num_rounds > 0) {  // small sumchecks: one single-CTA kernel for every round
        SumcheckArgs a{};
        a.a_base = base_first ? c.w(c.p.off_coeffs) : nullptr;
        for (int k = 0; k < 3; ++k) { a.a_in[k] = c.a(k); a.a_out[k] = c.a(k); a.b[k] = c.cov(k); }
        a.size = size;
        a.r_slot = r_slot;
        a.pow_threshold = s.pow_threshold;
        a.hash = c.p.params.hash;
        a.tx = c.tx();
        a.sc = c.sc();
        a.ext2 = c.p.params.field_degree == 2;
        int rc = 1;
        WG_TIMED(c, FAM_SUMCHECK, (rc = launch_sumcheck_small(a, (int)s.num_rounds, fold_after ? 1 : 0, c.st)) < 0 ? rc : 0);
        if (rc == 0) {
            r_slot += (int)s.num_rounds;
            return 0;
        }
    }
    for (uint64_t t = 0; t < s.num_rounds; ++t) {
        SumcheckArgs a{};
        const bool from_base = base_first && t <= 1;
        a.a_base = from_base ? c.w(c.p.off_coeffs) : nullptr;
        for (int k = 0; k < 3; ++k) { a.a_in[k] = c.a(k); a.a_out[k] = c.a(k); a.b[k] = c.cov(k); }
        a.size = size >> t;
        a.fold = t > 0;
        a.fold_r = r_slot - 1;
        a.r_slot = r_slot;
        a.pow_threshold = s.pow_threshold;
        a.hash = c.p.params.hash;
        a.tx = c.tx();
        a.sc = c.sc();
        a.ext2 = c.p.params.field_degree == 2;
        a.scratch = c.ws + c.p.off_sc_scratch;
        if (base_first && t == 0) a.a_base = c.w(c.p.off_coeffs);
        WG_TIMED(c, FAM_SUMCHECK, launch_sumcheck_round(a, c.st));
        ++r_slot;
    }
    if (fold_after && s.num_rounds > 0) {
        SumcheckArgs a{};
        const bool from_base = base_first && s.num_rounds == 1;
        a.a_base = from_base ? c.w(c.p.off_coeffs) : nullptr;
        for (int k = 0; k < 3; ++k) { a.a_in[k] = c.a(k); a.a_out[k] = c.a(k); a.b[k] = c.cov(k); }
        a.size = size >> s.num_rounds;
        a.fold_r = r_slot - 1;
        a.sc = c.sc();
        a.ext2 = c.p.params.field_degree == 2;
        WG_TIMED(c, FAM_SUMCHECK, launch_fold(a, c.st));
    }
    return 0;
}

}  // namespace

int enqueue_commit(const ProofPlan& p, char* ws, uint32_t ds_len, const DeviceTables& tw, cudaStream_t st,
                   Timer* timer, bool init_tx) {
    Ctx c{p, ws, tw, st, timer};
    if (init_tx)
        WG_TIMED(c, FAM_TX, launch_tx_init(c.tx(), reinterpret_cast<const unsigned char*>(ws + p.off_ds), ds_len,
                          reinterpret_cast<unsigned char*>(ws + p.off_narg), p.narg_len + 64,
                          reinterpret_cast<unsigned char*>(ws + p.off_hints), p.hints_cap + 64, c.sc(),
                          (unsigned)p.params.field_degree, st));
    const uint64_t size = 1ull << p.n;
    const uint32_t batch = (uint32_t)p.params.batch_size;
    const int ood = (int)p.sch.initial.out_domain;
    for (uint32_t w = 0; w < p.nwit; ++w) {
        const uint64_t* src[3] = {c.w(p.off_coeffs) + (size_t)w * batch * size, nullptr, nullptr};
        E3* out = &c.sc()->init_ood_mat[(size_t)w * ood * p.nvec + (size_t)w * batch];
        WG_TRY(commit_vectors(c, (int)w, src, 1, size, batch, ood, out, p.nvec));
    }
    return 0;
}

int enqueue_prove(const ProofPlan& p, char* ws, const DeviceTables& tw, cudaStream_t st, Timer* timer) {
    Ctx c{p, ws, tw, st, timer};
    const WhirSchedule& s = p.sch;
    const int ood0 = (int)s.initial.out_domain;
    const uint32_t W = p.nwit, V = p.nvec, batch = (uint32_t)p.params.batch_size;
    const uint64_t size0 = 1ull << p.n;
    // OOD completion (whir_prover.hpp:92-120): the other commitments' vectors
    // at each commitment's points, sent in order.
    if (W > 1 && ood0 > 0) {
        for (uint32_t w = 0; w < W; ++w) {
            OodArgs o{};
            o.v[0] = o.v[1] = o.v[2] = c.w(p.off_coeffs);
            o.ext3 = 0;
            o.size = size0;
            o.nvec = V;
            o.vec_stride = size0;
            o.skip_lo = w * batch;
            o.skip_hi = (w + 1) * batch;
            o.pts = &c.sc()->ood_pts[w][0];
            o.n_ood = ood0;
            o.out = &c.sc()->init_ood_mat[(size_t)w * ood0 * V];
            o.out_stride = V;
            o.tx = c.tx();
            o.scratch = ws + p.off_ood_scratch;
            o.scratch_values = p.ood_values;
            o.ext2 = p.params.field_degree == 2;
            WG_TIMED(c, FAM_OOD, launch_ood(o, st));
        }
    }
    WG_TIMED(c, FAM_TX, launch_constraint_rlc(c.tx(), c.sc(), p.n_forms, (int)W, ood0, (int)V, st));
    const bool has_constraints = p.n_forms + ood0 > 0;
    int r_slot = 0;
    // One base-field vector whose covector is MLE forms and OOD points only:
    // the initial sumcheck by block evaluation (k_sc_tensor.cu) never writes
    // the 2^n covector and leaves a, cov folded exactly as the rounds below do.
    const uint32_t k0 = (uint32_t)s.initial_sumcheck.num_rounds;
    const bool tensor = has_constraints && V == 1 && !p.full_vector && p.dense_mask == 0 &&
                        p.params.field_degree != 2 && s.initial_sumcheck.pow_threshold == ~0ull &&
                        tsc_applicable(p.n, k0, p.n_forms + ood0 * (int)W);
    if (tensor) {
        TscArgs ta{};
        ta.coeffs = c.w(p.off_coeffs);
        ta.n = p.n;
        ta.k = k0;
        ta.points = c.w(p.off_points);
        ta.n_forms = p.n_forms;
        ta.n_ood = ood0 * (int)W;
        ta.sc = c.sc();
        ta.tx = c.tx();
        ta.r_slot = r_slot;
        for (int k = 0; k < 3; ++k) { ta.a_out[k] = c.a(k); ta.cov_out[k] = c.cov(k); }
        ta.scratch = ws + p.off_cov_scratch;
        ta.scratch_bytes = p.off_tx - p.off_cov_scratch;  // the covector scratch region
        WG_TIMED(c, FAM_SUMCHECK, launch_tsc(ta, st));
        r_slot += (int)k0;
    } else {  // covector (zero without constraints) and, with several vectors, the combined vector
        CovInitArgs ci{};
        for (int k = 0; k < 3; ++k) { ci.cov[k] = c.cov(k); ci.vec_out[k] = c.a(k); }
        ci.logS = p.n;
        ci.points = c.w(p.off_points);
        ci.n_forms = p.n_forms;
        ci.n_ood = ood0 * (int)W;
        ci.sc = c.sc();
        ci.scratch = ws + p.off_cov_scratch;
        ci.nvec = V;
        ci.write_vec = p.full_vector;
        ci.vecs = c.w(p.off_coeffs);
        ci.dense_mask = p.dense_mask;
        for (int f = 0; f < 8; ++f) ci.dense[f] = p.dense[f];
        ci.ext2 = p.params.field_degree == 2;
        ci.tx = c.tx();
        WG_TIMED(c, FAM_COV, launch_cov_init(ci, st));
    }
    if (tensor) {
        // done above
    } else if (has_constraints) {
        WG_TRY(sumcheck(c, s.initial_sumcheck, size0, !p.full_vector, r_slot, true));
    } else {
        // No constraint (unique decoding, no forms; whir_prover.hpp:211-218): the
        // folding randomness is squeezed directly, the skip-PoW keeps the
        // transcript in step, and the vector is folded once per challenge (the
        // zero covector folds to zero).
        const int k = (int)s.initial_sumcheck.num_rounds;
        WG_TIMED(c, FAM_TX, launch_squeeze_challenges(c.tx(), c.sc(), 0, k, st));
        WG_TIMED(c, FAM_POW, launch_pow(c.tx(), c.sc(), s.initial_skip_pow, MAX_COMMITS + 1, c.p.params.hash, st));
        for (int t = 0; t < k; ++t) {
            SumcheckArgs a{};
            a.a_base = (!p.full_vector && t == 0) ? c.w(p.off_coeffs) : nullptr;
            for (int q = 0; q < 3; ++q) { a.a_in[q] = c.a(q); a.a_out[q] = c.a(q); a.b[q] = c.cov(q); }
            a.size = size0 >> (t + 1);
            a.fold_r = t;
            a.sc = c.sc();
            a.ext2 = p.params.field_degree == 2;
            WG_TIMED(c, FAM_SUMCHECK, launch_fold(a, st));
        }
        r_slot = k;
    }

    uint64_t vsize = size0 >> s.initial_sumcheck.num_rounds;
    for (size_t r = 0; r < s.rounds.size(); ++r) {
        const RoundSchedule& rc = s.rounds[r];
        const int ci = (int)(W + r);
        // base-field rounds commit the c0 plane only, Ext2 rounds c0 and c1 (c2 is zero)
        const uint32_t deg = (uint32_t)p.params.field_degree;
        const uint64_t* src[3] = {c.a(0), deg >= 2 ? c.a(1) : nullptr, deg >= 2 ? c.a(2) : nullptr};
        WG_TRY(commit_vectors(c, ci, src, deg, vsize, 1, (int)rc.irs.out_domain, &c.sc()->ood_vals[ci][0], 1));
        WG_TIMED(c, FAM_POW, launch_pow(c.tx(), c.sc(), rc.pow_threshold, ci, c.p.params.hash, st));
        // open the previous commitment (the first round: every initial commitment)
        const IrsSchedule& prev = r == 0 ? s.initial : s.rounds[r - 1].irs;
        const CommitBuffers& pb = p.commits[r == 0 ? 0 : ci - 1];
        OpenArgs oa{};
        oa.tx = c.tx();
        oa.sc = c.sc();
        oa.planes = c.w(pb.planes);
        oa.nodes = reinterpret_cast<const uint32_t*>(ws + pb.nodes);
        oa.nwit = r == 0 ? W : 1;
        oa.planes_stride = r == 0 ? p.init_planes_stride / 8 : 0;
        oa.nodes_stride = r == 0 ? p.init_nodes_stride / 4 : 0;
        oa.N = pb.N;
        oa.logN = pb.logN;
        oa.depth = pb.depth;
        oa.ncomp = pb.ncomp;
        oa.q = (uint32_t)prev.in_domain;
        oa.gen = gl_pow_host(7, (GL_P - 1) / pb.N);  // w_N = 7^((p-1)/N)
        oa.perm_log_e = pb.perm_log_e;
        oa.stir = 1;
        oa.use_vrlc = r == 0 && V > 1;
        oa.ood_offset = (int)rc.irs.out_domain;
        const uint32_t prev_fold = (uint32_t)(r == 0 ? s.initial_sumcheck.num_rounds : s.rounds[r - 1].sumcheck.num_rounds);
        oa.fold = prev_fold;
        oa.r_offset = r_slot - (int)prev_fold;
        WG_TIMED(c, FAM_OPEN, launch_open(oa, st));
        WG_TIMED(c, FAM_TX, launch_stir_rlc(c.tx(), c.sc(), ci, (int)rc.irs.out_domain, (int)prev.in_domain, st));
        CovAccArgs ca{};
        for (int k = 0; k < 3; ++k) ca.cov[k] = c.cov(k);
        ca.size = vsize;
        ca.n_ext = (int)rc.irs.out_domain;
        ca.n_base = (int)prev.in_domain;
        ca.sc = c.sc();
        ca.scratch = ws + p.off_cov_scratch;
        ca.ext2 = p.params.field_degree == 2;
        WG_TIMED(c, FAM_COV, launch_cov_accumulate(ca, st));
        WG_TRY(sumcheck(c, rc.sumcheck, vsize, false, r_slot, true));
        vsize >>= rc.sumcheck.num_rounds;
    }

    // final vector, PoW, opening, sumcheck
    WG_TIMED(c, FAM_TX, launch_send_vector(c.tx(), c.a(0), c.a(1), c.a(2), vsize, st));
    WG_TIMED(c, FAM_POW, launch_pow(c.tx(), c.sc(), s.final_pow, (int)(W + s.rounds.size()), c.p.params.hash, st));
    {
        const bool initial = s.rounds.empty();
        const IrsSchedule& last = initial ? s.initial : s.rounds.back().irs;
        const CommitBuffers& lb = initial ? p.commits[0] : p.commits.back();
        OpenArgs oa{};
        oa.tx = c.tx();
        oa.sc = c.sc();
        oa.planes = c.w(lb.planes);
        oa.nodes = reinterpret_cast<const uint32_t*>(ws + lb.nodes);
        oa.nwit = initial ? W : 1;
        oa.planes_stride = initial ? p.init_planes_stride / 8 : 0;
        oa.nodes_stride = initial ? p.init_nodes_stride / 4 : 0;
        oa.N = lb.N;
        oa.logN = lb.logN;
        oa.depth = lb.depth;
        oa.ncomp = lb.ncomp;
        oa.q = (uint32_t)last.in_domain;
        oa.gen = 1;
        oa.stir = 0;
        oa.perm_log_e = lb.perm_log_e;
        WG_TIMED(c, FAM_OPEN, launch_open(oa, st));
    }
    if (s.final_sumcheck.num_rounds > 0) WG_TRY(sumcheck(c, s.final_sumcheck, vsize, false, r_slot, false));
    return 0;
}

}  // namespace wg
