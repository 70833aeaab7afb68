"""The grouped mode's penalised one-voxel update (safeguarded Newton on the
reference's equation and bracket) against the reference's own solvers
(penalties.cpp:61-154, restated in oracle/port.cpp) on random inputs."""
import numpy as np
import pytest

import ctbb_icd_b200 as C
import oracle_util as O

pytestmark = pytest.mark.gpu

BISECTION_HALF_WIDTH = 1e-8  # penalties.cpp:131: stop when (b - a) / 2 < 1e-8


def _cases(n, seed, mu=0.192, spread=0.02):
    """Voxel + 8 neighbours around water, with edges (large jumps), flat
    patches (equal neighbours), voxels at the volume border (neighbours
    missing) and alpha = 0 (a voxel no ray of the window reaches)."""
    rng = np.random.default_rng(seed)
    x9 = rng.normal(mu, spread, (n, 9)).astype(np.float32)
    k = n // 8
    x9[:k, 1:] = x9[:k, :1]                                                # flat
    x9[k:2 * k, 1:5] += np.float32(0.2)                                    # an edge through the voxel
    x9[2 * k:3 * k] = np.abs(rng.normal(0.0, 1e-4, (k, 9))).astype(np.float32)  # near-zero (air)
    miss = rng.random((n, 8)) < 0.1
    miss[3 * k:4 * k, :3] = True                                           # first row of a slice
    x9[:, 1:][miss] = np.nan
    alpha = rng.uniform(0.5, 40.0, n)
    alpha[4 * k:4 * k + k // 4] = 0.0
    beta = alpha * rng.normal(0.0, 0.01, n)
    beta[5 * k:6 * k] = alpha[5 * k:6 * k] * rng.normal(0.0, 0.3, k)        # large steps
    return alpha, beta, x9


@pytest.mark.parametrize("lam,delta", [(0.1, 9.6e-4), (0.5, 0.005), (5.0, 0.05), (1e3, 0.005)])
def test_edge_preserving_step_matches_reference_bisection(ctx, lam, delta):
    alpha, beta, x9 = _cases(40000, seed=int(lam * 10) + 1)
    gpu = C.penalty_steps(ctx, C.PENALTY_EDGE_PRESERVING, lam, delta, alpha, beta, x9)
    ref = O.port_penalty_steps(C.PENALTY_EDGE_PRESERVING, lam, delta, alpha, beta, x9)
    assert np.all(np.isfinite(gpu))
    assert np.all(gpu[alpha == 0.0] == 0.0)  # penalties.cpp:101-102
    err = np.abs(gpu - ref)
    assert err.max() <= BISECTION_HALF_WIDTH * 1.001, (err.max(), int(err.argmax()))


@pytest.mark.parametrize("lam", [0.1, 1e3])
def test_quadratic_step_matches_reference(ctx, lam):
    alpha, beta, x9 = _cases(40000, seed=7)
    gpu = C.penalty_steps(ctx, C.PENALTY_QUADRATIC, lam, 0.0, alpha, beta, x9)
    ref = O.port_penalty_steps(C.PENALTY_QUADRATIC, lam, 0.0, alpha, beta, x9)
    # closed form; only the neighbour summation order differs
    assert np.allclose(gpu, ref, rtol=1e-12, atol=1e-15)
