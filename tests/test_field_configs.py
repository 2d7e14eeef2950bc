"""Config<M>::from_params (whir.hpp:118-224) for every target field the
reference CLI accepts (Goldilocks1/2/3): whirgpu_config_from_params (host only)
against the reference's own derivation printed by oracle/_ref/ref_driver --config."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from oracle.refio import REF_DRIVER, ref_available, write_input
from whirplonk_b200 import FIELD_GOLDILOCKS1, FIELD_GOLDILOCKS2, FIELD_GOLDILOCKS3, Config, ProtocolParameters

FLAGS = {FIELD_GOLDILOCKS1: ["--field1"], FIELD_GOLDILOCKS2: ["--field2"], FIELD_GOLDILOCKS3: []}


def reference_config(n, k, rho, sec, pb, field):
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        pt = np.zeros((1, n, 3), dtype=np.uint64)
        write_input(inp, n, k, rho, sec, pb, pt, np.zeros(1 << n, dtype=np.uint64))
        text = subprocess.run([REF_DRIVER, inp, out, "--config-only"] + FLAGS[field], check=True, capture_output=True,
                              text=True, timeout=60).stdout
    init = re.search(r"initial codeword (\d+) q (\d+) ood (\d+)", text).groups()
    sc_pow = re.search(r"initial sumcheck pow_threshold (\d+)", text).group(1)
    rounds = re.findall(r"round \d+ vec (\d+) codeword (\d+) q (\d+) ood (\d+) pow (\d+) sc_pow (\d+)", text)
    final = re.search(r"final size (\d+) rounds (\d+) pow (\d+) sc_pow (\d+)", text).groups()
    return [int(x) for x in init], int(sc_pow), [[int(x) for x in r] for r in rounds], [int(x) for x in final]


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("field", [FIELD_GOLDILOCKS1, FIELD_GOLDILOCKS2, FIELD_GOLDILOCKS3])
@pytest.mark.parametrize("n,k,rho,sec,pb", [(18, 4, 1, 100, 20), (22, 4, 2, 80, 16), (14, 3, 3, 60, 10)])
def test_config_from_params_matches_reference(field, n, k, rho, sec, pb):
    p = ProtocolParameters(False, rho, k, k, sec, pb, 1)
    c = Config.from_params(1 << n, p, field).cconfig if field != FIELD_GOLDILOCKS3 else None
    init, sc_pow, rounds, final = reference_config(n, k, rho, sec, pb, field)
    if c is None:  # the Ext3 path: the same derivation through whirgpu_config_from_params
        from whirplonk_b200 import _lib
        import ctypes

        c = _lib.WhirConfig()
        pc = p.to_c()
        _lib.check(_lib.load().whirgpu_config_from_params(ctypes.byref(pc), n, field, ctypes.byref(c)))
    ic = c.initial_committer
    assert [ic.codeword_length, ic.in_domain_samples, ic.out_domain_samples] == init
    assert c.initial_sumcheck.pow_threshold == sc_pow
    assert c.num_rounds == len(rounds)
    for r, ref in enumerate(rounds):
        rc = c.round_configs[r]
        assert [rc.irs_committer.vector_size, rc.irs_committer.codeword_length, rc.irs_committer.in_domain_samples,
                rc.irs_committer.out_domain_samples, rc.pow_threshold, rc.sumcheck.pow_threshold] == ref
    assert [int(c.final_sumcheck.num_rounds), int(c.final_pow), int(c.final_sumcheck.pow_threshold)] == \
        [final[1], final[2], final[3]]
