"""The exact finite-torus energy of the 2D Ising model (oracle/exact2d.py)
pinned by the transfer matrix and by enumeration, and the reference's own
EMCS loop (oracle/_ref, random-site Metropolis + Wolff on mt19937_64)
agreeing with it at L = 64, beta_c."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import exact2d as X  # noqa: E402
from oracle import stats as S  # noqa: E402

BETA_C = 0.44068679


@pytest.mark.parametrize("L", [4, 6, 8])
@pytest.mark.parametrize("K", [0.2, BETA_C, 0.7])
def test_kaufman_equals_transfer_matrix(L, K):
    assert abs(X.kaufman_energy(L, K) - X.transfer_energy(L, K)) < 1e-8


def test_kaufman_equals_enumeration_L4():
    for K in (0.1, BETA_C, 1.0):
        assert abs(X.kaufman_energy(4, K) - X.brute_energy(4, K)) < 1e-8


def test_kaufman_approaches_onsager_at_criticality():
    # e(beta_c) -> -sqrt(2) for L -> infinity, with O(1/L) corrections
    e64, e256 = X.kaufman_energy(64, BETA_C), X.kaufman_energy(256, BETA_C)
    assert abs(e256 + np.sqrt(2)) < abs(e64 + np.sqrt(2)) < 0.02


def test_reference_emcs_matches_exact_energy():
    from oracle.oracle import RefHarness, ref_path
    if not os.path.exists(ref_path()):
        pytest.skip("reference harness not built")
    obs, _ = RefHarness().emcs_ising2d(64, -1.0, BETA_C, 2024, 1, 1, 1000, 10000)
    e, de = S.mean_err(obs[:, 0])
    exact = X.kaufman_energy(64, BETA_C)
    assert abs(e - exact) < 2 * de, (e, de, exact)
