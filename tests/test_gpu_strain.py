"""ComputeStrain.m on the GPU against the oracle: every method and strain type
on a random displacement field."""
import numpy as np
import pytest

from oracle import strain as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", [0, 1, 2, 3])
@pytest.mark.parametrize("stype", [0, 1, 2])
def test_compute_strain_matches_oracle(aldic, method, stype):
    rng = np.random.default_rng(method * 3 + stype)
    M, N, h = 23, 17, 8.0
    U = rng.standard_normal(2 * M * N)
    F = 0.05 * rng.standard_normal(4 * M * N)
    para = {"MethodToComputeStrain": method, "StrainType": stype, "PlaneFitRad": 2, "winstepsize": h}
    r = aldic.ComputeStrain(U, F, {"M": M, "N": N}, para)
    fs, ff = S.compute_strain(M, N, h, method, 2 if method == 2 else 1, stype, U, F)
    np.testing.assert_allclose(r["FStrain"], fs, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(r["FStrainFinite"], ff, rtol=1e-12, atol=1e-13)
    rad = {0: 0, 1: 1, 2: 2, 3: 1}[method]
    w = r["FStrainWorld"].reshape(-1, 4)
    assert len(w) == (M - 2 * rad) * (N - 2 * rad)
    k = rad * M + rad
    # the world-frame copy is the finite strain itself, interior ring removed, slots 1, 2 negated
    np.testing.assert_array_equal(w[0], r["FStrainFinite"].reshape(-1, 4)[k] * [1, -1, -1, 1])
