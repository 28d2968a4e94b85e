"""Host-side helpers of the measurement scripts (no GPU): the block sums that map a fine gradient to
the coarse grid in closure_study, and the kinetic energy of a flattened state."""
import numpy as np
import torch

from public_b200 import closure_study


def test_block_sum_matches_fortran_blocks():
    n, r = 8, 2
    rng = np.random.default_rng(0)
    g = rng.standard_normal((n, n, n, 5))                      # (i, j, k, v), Fortran flattening
    flat = torch.from_numpy(np.ascontiguousarray(g.ravel(order="F")))
    got = closure_study.block_sum(flat, n, r).numpy().reshape((n // r,) * 3 + (5,), order="F")
    want = g.reshape(n // r, r, n // r, r, n // r, r, 5).sum(axis=(1, 3, 5))
    assert np.allclose(got, want, rtol=1e-14, atol=1e-13)


def test_kinetic_energy_of_flat_state():
    n = 4
    rng = np.random.default_rng(1)
    q = rng.uniform(0.5, 1.5, (n, n, n, 5))
    flat = torch.from_numpy(np.ascontiguousarray(q.ravel(order="F")))
    want = 0.1 * np.sum((q[..., 1] ** 2 + q[..., 2] ** 2 + q[..., 3] ** 2) / (2 * q[..., 0]))
    assert abs(closure_study.kinetic_energy(flat, 0.1) - want) < 1e-12 * want
