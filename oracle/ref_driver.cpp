// ref_driver.cpp -- test infrastructure, NOT product code.
//
// Runs the *unmodified* reference C++ WHIR prover (hxd77/WhirPlonk, the
// header-only library under cpp/include/whir, compiled in place by
// oracle/Makefile) on an input file written by the test harness, and writes
// the proof bytes.  It is the "reference" arm of the oracle: the Python tests
// use it to pin the CPU restatement in oracle/whir_oracle.hpp, bench.py uses it
// as the timed reference CPU prover.
//
// Call chain mirrored from the reference CLI `run_pcs` (cpp/main.cpp:292-467):
//   Config<M>::from_params (whir.hpp:118), M = Basefield<GoldilocksExt3>, or
//   Identity<Goldilocks> with --field1 (the CLI's --field Goldilocks1), or
//   Basefield<GoldilocksExt2> with --field2 (--field Goldilocks2)
//   ProverState::from_ds(ds, Empty)               (transcript.hpp:605)
//   config.commit / config.prove                   (whir.hpp:303, whir_prover.hpp:56)
// with the domain separator of `make_rust_cli_domain_separator`
// (cpp/main.cpp:203-215), re-stated here because main.cpp is not a header.
//
// Input file (little endian), written by oracle/refio.py:
//   u32 magic 0x49524857 ('WHRI'), u32 version 1, 2 or 3
//   u64 num_variables, folding_factor, starting_log_inv_rate,
//       security_level, pow_bits, num_points (= number of linear forms)
//   versions 2, 3: u64 batch_size, num_witnesses (version 1: both 1)
//   versions 1, 2: num_points * num_variables * 3 u64   MLE points (Ext3 coords)
//   version 3: per form u64 kind, then kind 0: num_variables * 3 u64 (an MLE
//              point), kind 1: 2^num_variables * 3 u64 (a dense Covector)
//   V * 2^num_variables u64              coefficients of the V = batch_size *
//                                        num_witnesses vectors (canonical, < p)
// The V vectors are committed as num_witnesses witnesses of batch_size
// vectors each, in order, then proven together.
// Output file:
//   u64 narg_len, narg bytes, u64 hints_len, hint bytes,
//   num_points * V * 3 u64 evaluations (form-major),
//   f64 commit_ms, f64 prove_ms, f64 verify_ok
#include "whir/algebra/embedding.hpp"
#include "whir/algebra/goldilocks.hpp"
#include "whir/algebra/goldilocks_ext2.hpp"
#include "whir/algebra/goldilocks_ext3.hpp"
#include "whir/algebra/linear_form.hpp"
#include "whir/hash/blake3_engine.hpp"
#include "whir/hash/sha2_engine.hpp"
#include "whir/parameters.hpp"
#include "whir/protocols/whir/whir.hpp"
#include "whir/transcript/transcript.hpp"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <span>
#include <string>
#include <type_traits>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;
using Source = ::whir::algebra::Goldilocks;
using M3 = ::whir::algebra::Basefield<::whir::algebra::GoldilocksExt3>;  // --field Goldilocks3 (default)
using M1 = ::whir::algebra::Identity<::whir::algebra::Goldilocks>;       // --field Goldilocks1
using M2 = ::whir::algebra::Basefield<::whir::algebra::GoldilocksExt2>;  // --field Goldilocks2

[[noreturn]] void die(const char* msg) {
    std::fprintf(stderr, "ref_driver: %s\n", msg);
    std::exit(2);
}

std::vector<std::uint8_t> read_file(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) die("cannot open input");
    std::vector<std::uint8_t> buf;
    std::uint8_t tmp[1 << 16];
    std::size_t got;
    while ((got = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
    std::fclose(f);
    return buf;
}

struct Reader {
    const std::vector<std::uint8_t>& b;
    std::size_t pos = 0;
    std::uint64_t u64() {
        if (pos + 8 > b.size()) die("truncated input");
        std::uint64_t v;
        std::memcpy(&v, b.data() + pos, 8);
        pos += 8;
        return v;
    }
    std::uint32_t u32() {
        if (pos + 4 > b.size()) die("truncated input");
        std::uint32_t v;
        std::memcpy(&v, b.data() + pos, 4);
        pos += 4;
        return v;
    }
};

// CBOR map of ProtocolParameters, key order and encodings as the reference
// CLI writes them (cpp/main.cpp:174-198).
void cbor_params(std::vector<std::uint8_t>& out, const ::whir::ProtocolParameters& p) {
    namespace tx = ::whir::transcript;
    out.push_back(0xA8);  // map of 8 pairs
    tx::cbor_write_text(out, "unique_decoding");
    out.push_back(p.unique_decoding ? 0xF5 : 0xF4);
    tx::cbor_write_text(out, "starting_log_inv_rate");
    tx::cbor_write_uint(out, p.starting_log_inv_rate);
    tx::cbor_write_text(out, "initial_folding_factor");
    tx::cbor_write_uint(out, p.initial_folding_factor);
    tx::cbor_write_text(out, "folding_factor");
    tx::cbor_write_uint(out, p.folding_factor);
    tx::cbor_write_text(out, "security_level");
    tx::cbor_write_uint(out, p.security_level);
    tx::cbor_write_text(out, "pow_bits");
    tx::cbor_write_uint(out, p.pow_bits);
    tx::cbor_write_text(out, "batch_size");
    tx::cbor_write_uint(out, p.batch_size);
    tx::cbor_write_text(out, "hash_id");
    tx::cbor_array_header(out, 32);
    for (auto byte : p.hash_id.bytes()) tx::cbor_write_uint(out, byte);
}

::whir::transcript::DomainSeparator cli_domain_separator(const ::whir::ProtocolParameters& p) {
    ::whir::transcript::DomainSeparator ds;
    std::vector<std::uint8_t> cbor;
    cbor_params(cbor, p);
    sha3_512_hash(cbor.data(), cbor.size(), ds.protocol_id.data());
    std::vector<std::uint8_t> sess;
    ::whir::transcript::cbor_write_text(sess, "Example at src/bin/main.rs:133");
    sha3_256_hash(sess.data(), sess.size(), ds.session_id.data());
    return ds;
}

void put_u64(FILE* f, std::uint64_t v) { std::fwrite(&v, 8, 1, f); }
void put_f64(FILE* f, double v) { std::fwrite(&v, 8, 1, f); }

// Target-field element from three input words (c0 c1 c2); a base-field target
// takes c0 and requires c1 = c2 = 0.
template <typename T>
T make_target(std::uint64_t a, std::uint64_t b, std::uint64_t c) {
    if constexpr (std::is_same_v<T, ::whir::algebra::Goldilocks>) {
        if (b || c) die("base-field target given an extension element");
        return T::from_u64(a);
    } else if constexpr (std::is_same_v<T, ::whir::algebra::GoldilocksExt2>) {
        if (c) die("quadratic-extension target given a cubic element");
        return T(Source::from_u64(a), Source::from_u64(b));
    } else {
        return T(Source::from_u64(a), Source::from_u64(b), Source::from_u64(c));
    }
}
template <typename T>
void put_target(FILE* f, const T& e) {
    if constexpr (std::is_same_v<T, ::whir::algebra::Goldilocks>) {
        put_u64(f, e.as_canonical_u64());
        put_u64(f, 0);
        put_u64(f, 0);
    } else if constexpr (std::is_same_v<T, ::whir::algebra::GoldilocksExt2>) {
        put_u64(f, e.c0().as_canonical_u64());
        put_u64(f, e.c1().as_canonical_u64());
        put_u64(f, 0);
    } else {
        put_u64(f, e.c0().as_canonical_u64());
        put_u64(f, e.c1().as_canonical_u64());
        put_u64(f, e.c2().as_canonical_u64());
    }
}

// Parsed input file and flags.
struct Job {
    std::size_t n = 0, k = 0, rho = 0, sec = 0, powb = 0, npts = 0, batch = 1, nwit = 1;
    std::vector<bool> dense;
    std::vector<std::vector<std::uint64_t>> forms;  // 3 words per element
    std::vector<std::vector<Source>> vecs;
    bool do_verify = false, print_cfg = false, config_only = false, use_sha2 = false, unique = false;
    int reps = 1;
    const char* out_path = nullptr;
};

}  // namespace

template <typename M>
int run(const Job& j) {
    using Target = typename M::Target;
    const std::size_t n = j.n, npts = j.npts, batch = j.batch, nwit = j.nwit, size = std::size_t{1} << n;
    const auto& vecs = j.vecs;
    const int reps = j.reps;
    std::vector<std::vector<Target>> points(npts);
    for (std::size_t f = 0; f < npts; ++f)
        for (std::size_t e = 0; e < j.forms[f].size() / 3; ++e)
            points[f].push_back(make_target<Target>(j.forms[f][3 * e], j.forms[f][3 * e + 1], j.forms[f][3 * e + 2]));
    auto make_form = [&](std::size_t f) -> std::unique_ptr<::whir::algebra::LinearForm<Target>> {
        if (j.dense[f]) return std::make_unique<::whir::algebra::Covector<Target>>(points[f]);
        return std::make_unique<::whir::algebra::MultilinearExtension<Target>>(points[f]);
    };
    ::whir::ProtocolParameters params;
    params.security_level = j.sec;
    params.pow_bits = j.powb;
    params.initial_folding_factor = j.k;
    params.folding_factor = j.k;
    params.unique_decoding = j.unique;
    params.starting_log_inv_rate = j.rho;
    params.batch_size = batch;
    params.hash_id = j.use_sha2 ? ::whir::hash::ENGINE_ID_SHA2 : ::whir::hash::ENGINE_ID_BLAKE3;

    auto config = ::whir::protocols::whir::Config<M>::from_params(size, params);
    if (j.print_cfg) {
        std::printf("initial codeword %zu q %zu ood %zu\n",
            config.initial_committer.codeword_length,
            config.initial_committer.in_domain_samples,
            config.initial_committer.out_domain_samples);
        std::printf("initial sumcheck pow_threshold %llu\n",
            (unsigned long long)config.initial_sumcheck.round_pow.threshold_val);
        for (std::size_t r = 0; r < config.round_configs.size(); ++r) {
            const auto& rc = config.round_configs[r];
            std::printf("round %zu vec %zu codeword %zu q %zu ood %zu pow %llu sc_pow %llu\n", r,
                rc.irs_committer.vector_size, rc.irs_committer.codeword_length,
                rc.irs_committer.in_domain_samples, rc.irs_committer.out_domain_samples,
                (unsigned long long)rc.pow.threshold_val,
                (unsigned long long)rc.sumcheck.round_pow.threshold_val);
        }
        std::printf("final size %zu rounds %zu pow %llu sc_pow %llu\n",
            config.final_sumcheck.initial_size, config.final_sumcheck.num_rounds,
            (unsigned long long)config.final_pow.threshold_val,
            (unsigned long long)config.final_sumcheck.round_pow.threshold_val);
        if (j.config_only) return 0;
    }

    M emb{};
    std::vector<Target> evaluations;  // form-major, as Config::prove expects (whir_prover.hpp:77)
    for (std::size_t f = 0; f < npts; ++f) {
        for (const auto& vec : vecs) {
            if (j.dense[f]) {
                ::whir::algebra::Covector<Target> cv(points[f]);
                evaluations.push_back(cv.template evaluate<M>(emb, std::span<const Source>{vec}));
            } else {
                ::whir::algebra::MultilinearExtension<Target> lf(points[f]);
                evaluations.push_back(lf.template evaluate<M>(emb, std::span<const Source>{vec}));
            }
        }
    }
    auto ds = cli_domain_separator(params);
    ::whir::transcript::Empty instance;
    std::vector<std::span<const Source>> spans;
    for (const auto& vec : vecs) spans.push_back(std::span<const Source>{vec});

    ::whir::transcript::ProverState::Proof proof;
    double commit_ms = 0, prove_ms = 0;
    for (int rep = 0; rep < reps; ++rep) {
        std::vector<std::unique_ptr<::whir::algebra::LinearForm<Target>>> forms;
        for (std::size_t f = 0; f < npts; ++f) forms.push_back(make_form(f));
        auto ps = ::whir::transcript::ProverState::from_ds(ds, instance);
        auto t0 = Clock::now();
        std::vector<::whir::protocols::irs_commit::Witness<Source, Target>> wits;
        for (std::size_t w = 0; w < nwit; ++w) {
            std::span<const std::span<const Source>> mine{spans.data() + w * batch, batch};
            wits.push_back(config.commit(ps, mine));
        }
        auto t1 = Clock::now();
        config.prove(ps, spans,
            std::span<const ::whir::protocols::irs_commit::Witness<Source, Target>>{wits},
            std::move(forms), std::span<const Target>{evaluations});
        auto t2 = Clock::now();
        proof = std::move(ps).proof();
        commit_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        prove_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
        if (reps > 1) std::printf("rep %d commit_ms %.3f prove_ms %.3f\n", rep, commit_ms, prove_ms);
    }

    double verify_ok = -1.0;
    if (j.do_verify) {
        auto vs = ::whir::transcript::VerifierState::from_ds(ds, instance, proof);
        std::vector<::whir::protocols::irs_commit::Commitment<Target>> comms;
        for (std::size_t w = 0; w < nwit; ++w) comms.push_back(config.receive_commitment(vs));
        std::vector<const ::whir::protocols::irs_commit::Commitment<Target>*> cp;
        for (const auto& cm : comms) cp.push_back(&cm);
        auto claim = config.verify(vs, cp, std::span<const Target>{evaluations});
        std::vector<std::unique_ptr<::whir::algebra::LinearForm<Target>>> vforms;
        std::vector<const ::whir::algebra::LinearForm<Target>*> refs;
        for (std::size_t f = 0; f < npts; ++f) {
            vforms.push_back(make_form(f));
            refs.push_back(vforms.back().get());
        }
        verify_ok = (claim.verify(refs) && vs.check_eof()) ? 1.0 : 0.0;
    }

    FILE* f = std::fopen(j.out_path, "wb");
    if (!f) die("cannot open output");
    put_u64(f, proof.narg_string.size());
    std::fwrite(proof.narg_string.data(), 1, proof.narg_string.size(), f);
    put_u64(f, proof.hints.size());
    std::fwrite(proof.hints.data(), 1, proof.hints.size(), f);
    for (const auto& e : evaluations) put_target(f, e);
    put_f64(f, commit_ms);
    put_f64(f, prove_ms);
    put_f64(f, verify_ok);
    std::fclose(f);
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: ref_driver INPUT OUTPUT [--verify] [--reps R] [--config] [--sha2] [--unique] [--field1 | --field2]\n");
        return 2;
    }
    Job j;
    j.out_path = argv[2];
    bool field1 = false, field2 = false;
    for (int i = 3; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--verify")) j.do_verify = true;
        else if (!std::strcmp(argv[i], "--config")) j.print_cfg = true;
        else if (!std::strcmp(argv[i], "--config-only")) j.print_cfg = j.config_only = true;
        else if (!std::strcmp(argv[i], "--sha2")) j.use_sha2 = true;
        else if (!std::strcmp(argv[i], "--unique")) j.unique = true;
        else if (!std::strcmp(argv[i], "--field1")) field1 = true;
        else if (!std::strcmp(argv[i], "--field2")) field2 = true;
        else if (!std::strcmp(argv[i], "--reps") && i + 1 < argc) j.reps = std::atoi(argv[++i]);
        else die("bad flag");
    }
    auto buf = read_file(argv[1]);
    Reader rd{buf};
    if (rd.u32() != 0x49524857u) die("bad magic");
    const std::uint32_t version = rd.u32();
    if (version < 1u || version > 3u) die("bad version");
    const std::size_t n = rd.u64();
    const std::size_t k = rd.u64();
    const std::size_t rho = rd.u64();
    const std::size_t sec = rd.u64();
    const std::size_t powb = rd.u64();
    const std::size_t npts = rd.u64();
    const std::size_t batch = version >= 2u ? rd.u64() : 1;
    const std::size_t nwit = version >= 2u ? rd.u64() : 1;
    if (n >= 40) die("num_variables too large");
    if (batch == 0 || nwit == 0 || batch * nwit > 64) die("bad vector count");
    const std::size_t nvec = batch * nwit;

    const std::size_t size = std::size_t{1} << n;
    j.n = n; j.k = k; j.rho = rho; j.sec = sec; j.powb = powb; j.npts = npts; j.batch = batch; j.nwit = nwit;
    j.dense.assign(npts, false);
    j.forms.resize(npts);  // MLE point, or the covector's values
    for (std::size_t f = 0; f < npts; ++f) {
        if (version == 3u) {
            const std::uint64_t kind = rd.u64();
            if (kind > 1) die("bad form kind");
            j.dense[f] = kind == 1;
        }
        j.forms[f].resize(3 * (j.dense[f] ? size : n));
        for (auto& w : j.forms[f]) w = rd.u64();
    }
    j.vecs.assign(nvec, std::vector<Source>(size));
    for (auto& vec : j.vecs)
        for (auto& v : vec) v = Source::from_u64(rd.u64());
    return field1 ? run<M1>(j) : field2 ? run<M2>(j) : run<M3>(j);
}

