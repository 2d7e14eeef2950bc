"""Host-side checks of the C ABI library (no GPU needed): the shared library
loads and exports every symbol include/whirgpu.h declares, and its host logic
(parameter schedule, domain separator, seeded sampler) agrees with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from whirplonk_b200 import ProtocolParameters, _lib, cli_domain_separator, sample_goldilocks
from whirplonk_b200.whir import Config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_header_symbols_exported():
    L = _lib.load()
    with open(os.path.join(ROOT, "include", "whirgpu.h")) as f:
        hdr = f.read()
    declared = sorted(set(re.findall(r"\b(whirgpu_[a-z0-9_]+)\s*\(", hdr)))
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(L, name), f"{name} declared in whirgpu.h but not exported"
    assert sorted(_lib.EXPORTED) == declared


PARAM_GRID = [
    (n, k, rho, sec, pb)
    for (n, k, rho, sec, pb) in [
        (18, 4, 1, 100, 20), (24, 4, 2, 100, 20), (24, 4, 3, 100, 20), (20, 4, 1, 128, 20), (12, 4, 1, 100, 20),
        (14, 2, 2, 80, 10), (16, 3, 3, 100, 0), (9, 1, 1, 64, 16), (22, 4, 1, 100, 20), (4, 4, 1, 100, 20),
        (13, 5, 2, 100, 20), (17, 4, 3, 90, 30), (21, 4, 2, 128, 0),
    ]
]


@pytest.mark.parametrize("n,k,rho,sec,pb", PARAM_GRID)
def test_schedule_matches_oracle(oracle, n, k, rho, sec, pb):
    params = ProtocolParameters.cli(security_level=sec, pow_bits=pb, folding_factor=k, log_inv_rate=rho)
    cfg = Config.from_params(1 << n, params)
    assert cfg.schedule == oracle.whir_config(n, rho, k, sec, pb)


def test_schedule_rejects_bad_params():
    with pytest.raises(ValueError):
        Config.from_params(1 << 3, ProtocolParameters.cli(folding_factor=4))  # n < k
    with pytest.raises(ValueError):
        Config.from_params(3, ProtocolParameters.cli())


@pytest.mark.parametrize("rho,k,sec,pb", [(1, 4, 100, 20), (2, 4, 100, 20), (3, 2, 128, 0)])
def test_domain_separator_matches_oracle(oracle, rho, k, sec, pb):
    params = ProtocolParameters.cli(security_level=sec, pow_bits=pb, folding_factor=k, log_inv_rate=rho)
    ds = cli_domain_separator(params)
    assert ds.protocol_id + ds.session_id == oracle.domain_separator(rho, k, sec, pb)


def test_chacha20_block_rfc8439():
    """RFC 8439 block function against the `cryptography` package's ChaCha20."""
    cr = pytest.importorskip("cryptography.hazmat.primitives.ciphers")
    L = _lib.load()
    rng = np.random.default_rng(7)
    for _ in range(4):
        key = bytes(rng.integers(0, 256, 32, dtype=np.uint8))
        nonce = bytes(rng.integers(0, 256, 12, dtype=np.uint8))
        counter = int(rng.integers(0, 2**32 - 2))
        out = ctypes.create_string_buffer(64)
        L.whirgpu_chacha20_block(key, counter, nonce, out)
        full_nonce = counter.to_bytes(4, "little") + nonce
        enc = cr.Cipher(cr.algorithms.ChaCha20(key, full_nonce), mode=None).encryptor()
        assert out.raw == enc.update(bytes(64))


def test_numpy_sampler_matches_library():
    """oracle/chacha.py (the benchmark's reference-arm sampler, no GPU library)
    draws the same words as whirgpu_sample_goldilocks, and its block function
    gives the RFC 8439 section 2.3.2 test vector."""
    import struct

    from oracle.chacha import chacha20_blocks
    from oracle.chacha import sample_goldilocks as np_sample

    for seed, count in [(1, 1), (11, 100), (1024, 1 << 16), (12345678901234567, 3000), (2**64 - 1, 77)]:
        assert (np_sample(seed, count) == sample_goldilocks(seed, count)).all(), (seed, count)
    key = struct.unpack("<8I", bytes(range(32)))
    nonce = struct.unpack("<3I", bytes.fromhex("000000090000004a00000000"))
    blk = chacha20_blocks(key, 1, 1, nonce)[0].tobytes()
    assert blk.hex() == (
        "10f1e7e4d13b5915500fdd1fa32071c4c7d1f4c733c068030422aa9ac3d46c4e"
        "d2826446079faa0914c2d705d98b02a2b5129cd1de164eb9cbd083e8a2503c4e")


def test_sampler_is_seeded_uniform_and_canonical():
    a = sample_goldilocks(123, 1 << 14)
    b = sample_goldilocks(123, 1 << 14)
    c = sample_goldilocks(124, 1 << 14)
    assert (a == b).all() and not (a == c).all()
    assert (a < np.uint64(0xFFFFFFFF00000001)).all()
    # prefix property: a shorter draw is a prefix of a longer one
    assert (sample_goldilocks(123, 100) == a[:100]).all()
    # crude uniformity: top bits spread
    top = (a >> np.uint64(60)).astype(np.int64)
    assert np.bincount(top, minlength=16).min() > (1 << 14) / 16 * 0.8


def test_ntt_plan_table_roundtrip(tmp_path):
    """Plan install / validation / save / load are host-only."""
    import ctypes

    from whirplonk_b200 import _lib

    L = _lib.load()
    L.whirgpu_ntt_clear_plans()
    good = _lib.NttPlan(20, 3, 2, (9, 11, 0), (4, 2, 255))
    piped = _lib.NttPlan(21, 2, 2, (11, 10, 0), (1, 2, 255), 3, 1)
    assert L.whirgpu_ntt_set_plan(ctypes.byref(good)) == _lib.OK
    assert L.whirgpu_ntt_set_plan(ctypes.byref(piped)) == _lib.OK
    for bad in [_lib.NttPlan(20, 3, 2, (8, 11, 0), (255, 255, 255)),   # radices do not sum to log_n
                _lib.NttPlan(24, 1, 2, (12, 12, 0), (255, 255, 255)),  # radix above 2^11
                _lib.NttPlan(22, 1, 1, (22, 0, 0), (255, 255, 255)),   # one pass above 2^11
                _lib.NttPlan(20, 3, 2, (9, 11, 0), (7, 0, 255)),       # too many columns
                _lib.NttPlan(20, 3, 2, (9, 11, 0), (4, 2, 255), 3, 2)]:  # pipelined is 0 or 1
        assert L.whirgpu_ntt_set_plan(ctypes.byref(bad)) == _lib.E_INVALID
    out = _lib.NttPlan()
    assert L.whirgpu_ntt_get_plan(20, 3, ctypes.byref(out)) == _lib.OK
    assert out.as_dict() == good.as_dict()
    assert L.whirgpu_ntt_get_plan(20, 2, ctypes.byref(out)) == _lib.OK  # untuned: built-in split
    assert out.npass == 2 and list(out.log_radix)[:2] == [10, 10]
    path = str(tmp_path / "plans.json")
    assert L.whirgpu_ntt_save_plans(path.encode()) == _lib.OK
    L.whirgpu_ntt_clear_plans()
    assert L.whirgpu_ntt_list_plans(None, 0) == 0
    n = ctypes.c_size_t()
    assert L.whirgpu_ntt_load_plans(path.encode(), ctypes.byref(n)) == _lib.OK and n.value == 2
    assert L.whirgpu_ntt_get_plan(20, 3, ctypes.byref(out)) == _lib.OK and out.as_dict() == good.as_dict()
    assert L.whirgpu_ntt_get_plan(21, 2, ctypes.byref(out)) == _lib.OK and out.as_dict() == piped.as_dict()
    import json

    plans = {(p["log_n"], p["log_expansion"]): p for p in json.load(open(path))["plans"]}
    assert plans[(20, 3)]["log_radix"] == [9, 11, 0] and plans[(20, 3)]["pipelined"] == 0
    assert plans[(21, 2)]["pipelined"] == 1
    L.whirgpu_ntt_clear_plans()
