"""Seeded inputs of the mixed-form statement fixtures ("forms" in
reference_proofs.json): shared by make_fixtures.py and the tests."""
from whirplonk_b200 import sample_goldilocks


def form_inputs(n, seed, kinds, nvec):
    """Coefficients (nvec, 2^n) and the linear forms: ("mle", (n, 3)) or
    ("covector", (2^n, 3)) canonical words, in statement order."""
    coeffs = sample_goldilocks(seed, nvec << n).reshape(nvec, 1 << n)
    forms = []
    for f, kind in enumerate(kinds):
        if kind == "mle":
            forms.append(("mle", sample_goldilocks(seed + 5000 + f, n * 3).reshape(n, 3)))
        else:
            forms.append(("covector", sample_goldilocks(seed + 6000 + f, 3 << n).reshape(1 << n, 3)))
    return coeffs, forms
