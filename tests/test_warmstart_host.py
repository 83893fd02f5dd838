"""Host-side helpers of the learned warm start (numpy only, no GPU):
parameter normalisation, the nearest-neighbour visiting order used to
generate training states, and the factor / proposal algebra that turns a
network output into an initial state and a deflation space."""
import numpy as np

from quac_b200 import warmstart as WS


def test_normalize_maps_the_sweep_box_to_unit_cube():
    lo, hi = WS.RANGES[:, 0], WS.RANGES[:, 1]
    assert np.allclose(WS.normalize(lo[None, :]), -1.0)
    assert np.allclose(WS.normalize(hi[None, :]), 1.0)
    th = WS.sweep_params(200, seed=1)
    z = WS.normalize(th)
    assert z.shape == (200, 4) and np.all(np.abs(z) <= 1.0 + 1e-12)


def test_sweep_params_fixed_columns_and_seed():
    a = WS.sweep_params(50, seed=7, fixed={2: 0.1, 3: 5e-3})
    b = WS.sweep_params(50, seed=7, fixed={2: 0.1, 3: 5e-3})
    assert np.array_equal(a, b)
    assert np.all(a[:, 2] == 0.1) and np.all(a[:, 3] == 5e-3)
    assert not np.array_equal(a, WS.sweep_params(50, seed=8, fixed={2: 0.1, 3: 5e-3}))


def test_nn_chain_is_a_greedy_permutation():
    th = WS.sweep_params(40, seed=3)
    order = WS.nn_chain(th)
    assert order[0] == 0 and sorted(order) == list(range(40))
    z = WS.normalize(th)
    for k in range(1, len(order)):
        left = order[k:]
        d = np.sum((z[left] - z[order[k - 1]]) ** 2, axis=1)
        assert np.isclose(d[0], d.min())


def _random_rho(rng, D, rank):
    A = rng.normal(size=(D, rank)) + 1j * rng.normal(size=(D, rank))
    rho = A @ A.conj().T
    return rho / np.trace(rho).real


def test_factors_reproduce_low_rank_states():
    rng = np.random.default_rng(5)
    D = 24
    rho = _random_rho(rng, D, 6)
    F = WS.factors_from_rho(rho.reshape(-1, order="F"), D, 16)
    assert F.shape == (D, 16)
    assert np.linalg.norm(F @ F.conj().T - rho) < 1e-12 * np.linalg.norm(rho)
    # a full-rank state is truncated to its leading r eigenpairs
    full = _random_rho(rng, D, D)
    F4 = WS.factors_from_rho(full.reshape(-1, order="F"), D, 4)
    w = np.sort(np.linalg.eigvalsh(full))[::-1]
    assert np.allclose(np.sort(np.linalg.eigvalsh(F4 @ F4.conj().T))[::-1][:4], w[:4])


def test_proposal_is_a_state_and_an_orthonormal_subspace():
    rng = np.random.default_rng(6)
    D, r, kd = 20, 8, 5
    F = rng.normal(size=(D, r)) + 1j * rng.normal(size=(D, r))
    x0, U = WS.proposal_from_factors(F, kd)
    R = x0.reshape(D, D, order="F")
    assert abs(np.trace(R) - 1.0) < 1e-12
    assert np.abs(R - R.conj().T).max() < 1e-14
    assert np.linalg.eigvalsh(R).min() > -1e-12
    assert U.shape == (D, kd) and np.allclose(U.conj().T @ U, np.eye(kd), atol=1e-12)
    # U spans the kd leading directions of F F^H
    w, V = np.linalg.eigh(F @ F.conj().T)
    lead = V[:, np.argsort(-w)[:kd]]
    assert np.allclose(U @ (U.conj().T @ lead), lead, atol=1e-10)
    # a zero proposal falls back to the maximally mixed state
    x0z, _ = WS.proposal_from_factors(np.zeros((D, r), complex), kd)
    assert np.allclose(x0z.reshape(D, D, order="F"), np.eye(D) / D)
