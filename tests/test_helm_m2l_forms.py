"""The algebra behind the two forms of the tiled Helmholtz M2L, on CPU.

h2dmploc weights the Toeplitz term T[i - j] M_j by rs^e with
e = |i| + |j| - |i - j|.  The tiled kernel (csrc/helmholtz.cu,
helm_m2l_tile_kernel) uses
  * a case split of that weight: 1 when i and j differ in sign or one is 0,
    rs^(2 |j|) when they share a sign and |j| <= |i|, rs^(2 |i|) otherwise;
  * the scaled form: T_q rs^-|q| against M_j rs^|j|, the sum times rs^|i|.
Both are checked here against the per-term weight."""
import numpy as np
import pytest


def weight_case_split(i, j, pw):
    same = (i > 0 and j > 0) or (i < 0 and j < 0)
    if not same:
        return pw[0]
    return pw[2 * abs(j)] if abs(j) <= abs(i) else pw[2 * abs(i)]


@pytest.mark.parametrize("p,rs", [(5, 0.3), (20, 0.06), (40, 1.0)])
def test_case_split_equals_the_exponent_weight(p, rs):
    pw = rs ** np.arange(2 * p + 1)
    for i in range(-p, p + 1):
        for j in range(-p, p + 1):
            e = abs(i) + abs(j) - abs(i - j)
            assert weight_case_split(i, j, pw) == pw[e]


@pytest.mark.parametrize("p,rs", [(6, 0.4), (20, 0.06), (30, 1.0)])
def test_scaled_form_equals_weighted_sum(p, rs):
    rng = np.random.default_rng(p)
    T = rng.standard_normal(4 * p + 1) + 1j * rng.standard_normal(4 * p + 1)  # T[q], q = -2p..2p
    M = rng.standard_normal(2 * p + 1) + 1j * rng.standard_normal(2 * p + 1)  # M[j], j = -p..p
    q = np.arange(-2 * p, 2 * p + 1)
    j = np.arange(-p, p + 1)
    Ts = T * rs ** (-np.abs(q).astype(float))
    Ms = M * rs ** np.abs(j).astype(float)
    for i in range(-p, p + 1):
        e = abs(i) + np.abs(j) - np.abs(i - j)
        ref = np.sum(T[i - j + 2 * p] * rs ** e.astype(float) * M)
        got = rs ** abs(i) * np.sum(Ts[i - j + 2 * p] * Ms)
        assert abs(got - ref) <= 1e-12 * max(1.0, np.sum(np.abs(T[i - j + 2 * p] * M)))
