// params.h -- WHIR round schedule derived from ProtocolParameters.
//
// Restates Config<M>::from_params (cpp/include/whir/protocols/whir/whir.hpp:118-224)
// and irs_commit::Config::from_params (cpp/include/whir/protocols/irs_commit.hpp:192-324)
// for M = Basefield<GoldilocksExt3> (192-bit target field).  The security
// formulas are floating point and decide sample counts and PoW thresholds, so
// every expression keeps the reference's operation order (no fast-math).
#pragma once
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace wg {

struct ProtocolParams {  // whir::ProtocolParameters (cpp/include/whir/parameters.hpp:25-34)
    bool unique_decoding = false;
    uint64_t starting_log_inv_rate = 1;
    uint64_t initial_folding_factor = 4;
    uint64_t folding_factor = 4;
    uint64_t security_level = 100;
    uint64_t pow_bits = 20;
    uint64_t batch_size = 1;
    int hash = 0;  // engine of hash_id: 0 BLAKE3, 1 SHA-256 (leaves, Merkle, PoW)
    // Not a ProtocolParameters field but the embedding M of Config<M>: the
    // target field's degree over Goldilocks, 3 for Basefield<GoldilocksExt3>
    // (field_size_bits 192), 2 for Basefield<GoldilocksExt2> (128), 1 for
    // Identity<Goldilocks> (64).
    int field_degree = 3;
    // Codeword row order (not a ProtocolParameters field either): 0 natural, as
    // the C++ reference commits (mod_ntt.hpp:49-130); 1 coset-major, as the
    // Rust crate commits without its rs_in_order feature
    // (rust/src/algebra/ntt/cooley_tukey.rs:375-480): committed row k is the
    // natural row k / m + (k mod m) N / m for message length m.
    int coset_major = 0;
};

struct IrsSchedule {
    uint64_t vector_size = 0, depth = 0, codeword_length = 0;
    double johnson_slack = 0.0;
    uint64_t in_domain = 0, out_domain = 0;
    uint64_t message_length() const { return vector_size / depth; }
    double rate() const { return (double)message_length() / (double)codeword_length; }
    bool unique() const { return out_domain == 0 && johnson_slack == 0.0; }
    double list_size() const { return unique() ? 1.0 : 1.0 / (2.0 * johnson_slack * std::sqrt(rate())); }
    double rbr_queries() const {
        const double per = unique() ? ((1.0 + rate()) * 0.5) : (std::sqrt(rate()) + johnson_slack);
        return (double)in_domain * (-std::log2(per));
    }
    double fold_prox_gaps(double field_bits) const {
        const double lir = -std::log2(rate());
        const double logk = std::log2((double)message_length());
        double err;
        if (unique()) err = logk + lir;
        else {
            constexpr double LOG2_10 = 3.321928094887362;
            err = 7.0 * LOG2_10 + 3.5 * lir + 2.0 * logk;
        }
        return field_bits - err;
    }
    static IrsSchedule make(double security, bool ud, uint64_t vsize, uint64_t depth, double rate, double field_bits) {
        IrsSchedule c;
        c.vector_size = vsize;
        c.depth = depth;
        const uint64_t ml = vsize / depth;
        c.codeword_length = (uint64_t)std::ceil((double)ml / rate);
        const double ar = (double)ml / (double)c.codeword_length;
        c.johnson_slack = ud ? 0.0 : std::sqrt(ar) / 20.0;
        if (ud) {
            c.out_domain = 0;
        } else {
            const double L = 1.0 / (2.0 * c.johnson_slack * std::sqrt(ar));
            const double lc2 = L * (L - 1.0) / 2.0;
            const double lps = field_bits - std::log2((double)(vsize - 1));
            c.out_domain = (uint64_t)std::ceil((security + std::log2(lc2)) / lps);
            if (c.out_domain < 1) c.out_domain = 1;
        }
        const double per = ud ? ((1.0 + ar) * 0.5) : (std::sqrt(ar) + c.johnson_slack);
        c.in_domain = (uint64_t)std::ceil(security / (-std::log2(per)));
        return c;
    }
};

struct SumcheckSchedule {
    uint64_t initial_size = 0, num_rounds = 0, pow_threshold = ~0ull;
};
struct RoundSchedule {
    IrsSchedule irs;
    SumcheckSchedule sumcheck;
    uint64_t pow_threshold = ~0ull;
};
struct WhirSchedule {
    uint64_t num_variables = 0;
    IrsSchedule initial;
    SumcheckSchedule initial_sumcheck;
    uint64_t initial_skip_pow = ~0ull;
    std::vector<RoundSchedule> rounds;
    SumcheckSchedule final_sumcheck;
    uint64_t final_pow = ~0ull;
};

inline uint64_t pow_threshold(double bits) {
    return bits <= 0.0 ? ~0ull : (uint64_t)std::ceil(std::exp2(64.0 - bits));
}

// Throws std::invalid_argument for parameters the reference would assert on.
inline WhirSchedule make_schedule(uint64_t num_variables, const ProtocolParams& p) {
    if (num_variables >= 40) throw std::invalid_argument("num_variables too large");
    if (p.initial_folding_factor == 0 || p.folding_factor == 0) throw std::invalid_argument("folding factor must be >= 1");
    if (num_variables < p.initial_folding_factor) throw std::invalid_argument("num_variables < initial folding factor");
    if (p.pow_bits > p.security_level) throw std::invalid_argument("pow_bits > security_level");
    if (p.batch_size == 0) throw std::invalid_argument("batch_size must be >= 1");
    const uint64_t size = 1ull << num_variables;
    WhirSchedule c;
    c.num_variables = num_variables;
    const double security = (double)p.security_level;
    const double psec = (double)(p.security_level - p.pow_bits);
    const double fbits = 64.0 * p.field_degree;  // Target::field_size_bits: 64, 128 (Ext2), 192 (Ext3)
    uint64_t lir = p.starting_log_inv_rate;
    uint64_t nv = num_variables;
    const double irate = std::pow(0.5, (double)p.starting_log_inv_rate);
    c.initial = IrsSchedule::make(psec, p.unique_decoding, size, 1ull << p.initial_folding_factor, irate, fbits);
    const double start_fold = std::max(
        security - std::min(c.initial.fold_prox_gaps(fbits), fbits - std::log2(c.initial.list_size()) - 1.0), 0.0);
    const double skip =
        std::max(security - (c.initial.fold_prox_gaps(fbits) + std::log2((double)p.initial_folding_factor)), 0.0);
    c.initial_sumcheck = {size, p.initial_folding_factor, pow_threshold(start_fold)};
    c.initial_skip_pow = pow_threshold(skip);
    uint64_t rd = 0, ids = c.initial.in_domain;
    double qe = c.initial.rbr_queries();
    nv -= p.initial_folding_factor;
    while (nv >= p.folding_factor) {
        const uint64_t rff = rd == 0 ? p.initial_folding_factor : p.folding_factor;
        const uint64_t nli = lir + (rff - 1);
        const double rr = std::pow(0.5, (double)nli);
        RoundSchedule rc;
        rc.irs = IrsSchedule::make(psec, p.unique_decoding, 1ull << nv, 1ull << p.folding_factor, rr, fbits);
        const double ll = std::log2(rc.irs.list_size());
        const uint64_t cnt = rc.irs.out_domain + ids;
        const double cbe = fbits - (std::log2((double)cnt) + ll + 1.0);
        const double pb = std::max(security - std::min(qe, cbe), 0.0);
        const double fpb = std::max(security - std::min(rc.irs.fold_prox_gaps(fbits), fbits - ll - 1.0), 0.0);
        rc.sumcheck = {1ull << nv, p.folding_factor, pow_threshold(fpb)};
        rc.pow_threshold = pow_threshold(pb);
        ++rd;
        nv -= p.folding_factor;
        lir = nli;
        ids = rc.irs.in_domain;
        qe = rc.irs.rbr_queries();
        c.rounds.push_back(rc);
    }
    const double rbr_e = c.rounds.empty() ? c.initial.rbr_queries() : c.rounds.back().irs.rbr_queries();
    const double fpb2 = std::max(security - rbr_e, 0.0);
    const double ffpb = std::max(security - fbits + 1.0, 0.0);
    c.final_sumcheck = {1ull << nv, nv, pow_threshold(ffpb)};
    c.final_pow = pow_threshold(fpb2);
    return c;
}

// Structural checks of a schedule given field by field (a Config built by the
// caller, as the reference's golden dumpers do): the shapes the prove order
// relies on.  Each commitment's depth is 2^(rounds of the sumcheck that
// follows it), so the STIR rows match the eq weights of the folding randomness
// (whir_prover.hpp:283-310); sizes chain from round to round.  Throws
// std::invalid_argument.
inline void validate_schedule(const WhirSchedule& s) {
    auto pow2 = [](uint64_t v) { return v && !(v & (v - 1)); };
    auto irs_ok = [&](const IrsSchedule& c, uint64_t vsize, uint64_t rounds, const char* what) {
        if (c.vector_size != vsize) throw std::invalid_argument(std::string(what) + ": vector size does not chain");
        if (rounds >= 64 || c.depth != (1ull << rounds))
            throw std::invalid_argument(std::string(what) + ": depth != 2^(sumcheck rounds)");
        if (!pow2(c.codeword_length) || c.depth > vsize || c.codeword_length % (vsize / c.depth) != 0)
            throw std::invalid_argument(std::string(what) + ": codeword length");
    };
    if (!pow2(s.initial.vector_size)) throw std::invalid_argument("vector size must be a power of two");
    irs_ok(s.initial, s.initial.vector_size, s.initial_sumcheck.num_rounds, "initial committer");
    if (s.initial_sumcheck.initial_size != s.initial.vector_size)
        throw std::invalid_argument("initial sumcheck size != vector size");
    uint64_t size = s.initial.vector_size >> s.initial_sumcheck.num_rounds;
    for (const RoundSchedule& r : s.rounds) {
        irs_ok(r.irs, size, r.sumcheck.num_rounds, "round committer");
        if (r.sumcheck.initial_size != size) throw std::invalid_argument("round sumcheck size does not chain");
        size >>= r.sumcheck.num_rounds;
    }
    if (s.final_sumcheck.initial_size != size || (s.final_sumcheck.num_rounds < 64 && (size >> s.final_sumcheck.num_rounds) == 0) ||
        s.final_sumcheck.num_rounds >= 64)
        throw std::invalid_argument("final sumcheck does not fit the folded vector");
}

}  // namespace wg
