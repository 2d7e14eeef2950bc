"""Seeded inputs of the mixed-form statement fixtures ("forms" in
reference_proofs.json): shared by make_fixtures.py and the tests."""
from whirplonk_b200 import sample_goldilocks


def form_inputs(n, seed, kinds, nvec, base_field=False, ext2=False):
    """Coefficients (nvec, 2^n) and the linear forms: ("mle", (n, 3)) or
    ("covector", (2^n, 3)) canonical words, in statement order.  With
    base_field (an Identity<Goldilocks> target) the forms' values are (x, 0, 0),
    with ext2 (a GoldilocksExt2 target) (x, y, 0)."""
    coeffs = sample_goldilocks(seed, nvec << n).reshape(nvec, 1 << n)
    forms = []
    for f, kind in enumerate(kinds):
        if kind == "mle":
            d = sample_goldilocks(seed + 5000 + f, n * 3).reshape(n, 3)
        else:
            d = sample_goldilocks(seed + 6000 + f, 3 << n).reshape(1 << n, 3)
        if base_field:
            d[:, 1:] = 0
        if ext2:
            d[:, 2] = 0
        forms.append((kind, d))
    return coeffs, forms
