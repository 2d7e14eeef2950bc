// ref_zk_driver.cpp -- test infrastructure, NOT product code.
//
// Runs the *unmodified* reference zero-knowledge WHIR prover (hxd77/WhirPlonk
// cpp/include/whir/protocols/whir_zk, compiled in place by oracle/Makefile) on
// an input file written by oracle/refio.py and writes the proof bytes, the
// same way cpp/tests/dump_whir_zk.cpp drives it:
//   ZkConfig<Goldilocks>::from_params[_with_policy] (whir_zk.hpp:95-105, 279-305)
//   DeterministicRng(seed, "WHIR_ZK:mask")            (deterministic_rng.hpp)
//   config.commit / config.prove                      (whir_zk_impl.hpp:42-330)
// The domain separator is the CLI one of the parameters (cpp/main.cpp:174-215)
// rather than the canonical ZK configuration's: the ZK prover takes any.
//
// Input file (little endian):
//   u32 magic 0x4B5A4857 ('WHZK'), u32 version 1
//   u64 num_variables, folding_factor, starting_log_inv_rate, security_level,
//       pow_bits, num_forms, num_polynomials, hash (0 BLAKE3, 1 SHA-2),
//       no_pow (1: every PoW threshold of both inner configs disabled, as the
//       reference's dumper does), q_delta_1, q_delta_2, t1, t2 (all 0: the
//       policy from_params derives), seed (the RNG seed's first 8 bytes, LE)
//   per form: u64 kind (0 MultilinearExtension: n coordinates, 1 Covector:
//       2^n values), then its words (one u64 per base-field element)
//   num_polynomials * 2^n u64 coefficients
// Output file:
//   u64 narg_len, narg bytes, u64 hints_len, hint bytes,
//   num_forms * num_polynomials u64 evaluations (form-major), f64 verify_ok,
//   u64 num_blinding_variables, u64 blinded initial q, u64 blinding batch size,
//   f64 milliseconds of commit + prove (wall clock, the reference's own threads)
#include "whir/algebra/embedding.hpp"
#include "whir/algebra/goldilocks.hpp"
#include "whir/algebra/linear_form.hpp"
#include "whir/deterministic_rng.hpp"
#include "whir/hash/blake3_engine.hpp"
#include "whir/hash/sha2_engine.hpp"
#include "whir/parameters.hpp"
#include "whir/protocols/whir_zk/whir_zk.hpp"
#include "whir/transcript/transcript.hpp"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <span>
#include <string>
#include <vector>

namespace {

using F = ::whir::algebra::Goldilocks;

[[noreturn]] void die(const char* msg) {
    std::fprintf(stderr, "ref_zk_driver: %s\n", msg);
    std::exit(2);
}

struct Reader {
    std::vector<std::uint8_t> b;
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

void cbor_params(std::vector<std::uint8_t>& out, const ::whir::ProtocolParameters& p) {
    namespace tx = ::whir::transcript;
    out.push_back(0xA8);
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

void disable_whir_pow(::whir::protocols::whir::Config<::whir::algebra::Identity<F>>& config) {
    config.initial_sumcheck.round_pow.threshold_val = UINT64_MAX;
    config.initial_skip_pow.threshold_val = UINT64_MAX;
    for (auto& round : config.round_configs) {
        round.sumcheck.round_pow.threshold_val = UINT64_MAX;
        round.pow.threshold_val = UINT64_MAX;
    }
    config.final_sumcheck.round_pow.threshold_val = UINT64_MAX;
    config.final_pow.threshold_val = UINT64_MAX;
}

void put_u64(FILE* f, std::uint64_t v) { std::fwrite(&v, 8, 1, f); }

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: ref_zk_driver INPUT OUTPUT [--verify]\n");
        return 2;
    }
    const bool do_verify = argc > 3 && !std::strcmp(argv[3], "--verify");
    Reader rd;
    {
        FILE* f = std::fopen(argv[1], "rb");
        if (!f) die("cannot open input");
        std::uint8_t tmp[1 << 16];
        std::size_t got;
        while ((got = std::fread(tmp, 1, sizeof(tmp), f)) > 0) rd.b.insert(rd.b.end(), tmp, tmp + got);
        std::fclose(f);
    }
    if (rd.u32() != 0x4B5A4857u) die("bad magic");
    if (rd.u32() != 1u) die("bad version");
    const std::size_t n = rd.u64(), k = rd.u64(), rho = rd.u64(), sec = rd.u64(), powb = rd.u64();
    const std::size_t nforms = rd.u64(), npolys = rd.u64(), hash = rd.u64(), no_pow = rd.u64();
    const std::size_t q1 = rd.u64(), q2 = rd.u64(), t1 = rd.u64(), t2 = rd.u64();
    const std::uint64_t seed64 = rd.u64();
    if (n >= 32 || npolys == 0) die("bad sizes");
    const std::size_t size = std::size_t{1} << n;
    std::vector<bool> dense(nforms);
    std::vector<std::vector<F>> data(nforms);
    for (std::size_t f = 0; f < nforms; ++f) {
        dense[f] = rd.u64() == 1;
        data[f].resize(dense[f] ? size : n);
        for (auto& v : data[f]) v = F::from_u64(rd.u64());
    }
    std::vector<std::vector<F>> polys(npolys, std::vector<F>(size));
    for (auto& p : polys)
        for (auto& v : p) v = F::from_u64(rd.u64());

    ::whir::ProtocolParameters params;
    params.unique_decoding = false;
    params.security_level = sec;
    params.pow_bits = powb;
    params.initial_folding_factor = k;
    params.folding_factor = k;
    params.starting_log_inv_rate = rho;
    params.batch_size = 1;
    params.hash_id = hash ? ::whir::hash::ENGINE_ID_SHA2 : ::whir::hash::ENGINE_ID_BLAKE3;

    using Zk = ::whir::protocols::whir_zk::ZkConfig<F>;
    Zk config;
    if (q1 || q2 || t1 || t2) {
        ::whir::protocols::whir_zk::BlindingSizePolicy policy;
        policy.q_delta_1 = q1;
        policy.q_delta_2 = q2;
        policy.t1 = t1;
        policy.t2 = t2;
        policy.sumcheck_round_degree = 3;
        config = Zk::from_params_with_policy(size, params, npolys, policy);
    } else {
        config = Zk::from_params(size, params, npolys);
    }
    if (no_pow) {
        disable_whir_pow(config.blinded_commitment);
        disable_whir_pow(config.blinding_commitment);
    }

    auto make_form = [&](std::size_t f) -> std::unique_ptr<::whir::algebra::LinearForm<F>> {
        if (dense[f]) return std::make_unique<::whir::algebra::Covector<F>>(data[f]);
        return std::make_unique<::whir::algebra::MultilinearExtension<F>>(data[f]);
    };
    ::whir::algebra::Identity<F> emb;
    std::vector<F> evaluations;  // form-major
    for (std::size_t f = 0; f < nforms; ++f)
        for (const auto& p : polys) {
            if (dense[f]) evaluations.push_back(::whir::algebra::Covector<F>(data[f]).evaluate(emb, std::span<const F>{p}));
            else evaluations.push_back(::whir::algebra::MultilinearExtension<F>(data[f]).template evaluate<
                                       ::whir::algebra::Identity<F>>(emb, std::span<const F>{p}));
        }

    auto ds = cli_domain_separator(params);
    ::whir::transcript::Empty instance;
    auto ps = ::whir::transcript::ProverState::from_ds(ds, instance);
    std::array<std::uint8_t, 32> seed{};
    for (int i = 0; i < 8; ++i) seed[i] = static_cast<std::uint8_t>(seed64 >> (8 * i));
    ::whir::DeterministicRng rng(seed, "WHIR_ZK:mask");
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::span<const F>> spans;
    for (const auto& p : polys) spans.push_back(std::span<const F>{p});
    auto witness = config.commit(ps, spans, rng);
    std::vector<F> flat;
    for (const auto& p : polys) flat.insert(flat.end(), p.begin(), p.end());
    std::vector<std::unique_ptr<::whir::algebra::LinearForm<F>>> forms;
    for (std::size_t f = 0; f < nforms; ++f) forms.push_back(make_form(f));
    config.prove(ps, std::span<const F>{flat}, std::move(witness), std::move(forms), std::span<const F>{evaluations},
                 rng);
    auto proof = std::move(ps).proof();
    const double prove_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

    double verify_ok = -1.0;
    if (do_verify) {
        auto vs = ::whir::transcript::VerifierState::from_ds(ds, instance, proof);
        auto commitment = config.receive_commitments(vs, npolys);
        std::vector<std::unique_ptr<::whir::algebra::LinearForm<F>>> vforms;
        std::vector<const ::whir::algebra::LinearForm<F>*> refs;
        for (std::size_t f = 0; f < nforms; ++f) {
            vforms.push_back(make_form(f));
            refs.push_back(vforms.back().get());
        }
        const bool ok = config.verify(vs, std::span<const ::whir::algebra::LinearForm<F>*>{refs},
                                      std::span<const F>{evaluations}, commitment);
        verify_ok = (ok && vs.check_eof()) ? 1.0 : 0.0;
    }

    FILE* f = std::fopen(argv[2], "wb");
    if (!f) die("cannot open output");
    put_u64(f, proof.narg_string.size());
    std::fwrite(proof.narg_string.data(), 1, proof.narg_string.size(), f);
    put_u64(f, proof.hints.size());
    std::fwrite(proof.hints.data(), 1, proof.hints.size(), f);
    for (const auto& e : evaluations) put_u64(f, e.as_canonical_u64());
    std::fwrite(&verify_ok, 8, 1, f);
    put_u64(f, config.num_blinding_variables());
    put_u64(f, config.blinded_commitment.initial_committer.in_domain_samples);
    put_u64(f, config.blinding_commitment.initial_committer.num_vectors);
    std::fwrite(&prove_ms, 8, 1, f);
    std::fclose(f);
    return 0;
}
