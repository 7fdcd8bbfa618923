"""The neighbour-list invariant the solver's rebuild rule relies on, checked on
the CPU in FP32: lists of radius 2h + skin built at positions x0 hold every
pair within 2h of the current positions while no particle has moved more than
skin / 2 since the build (|r_now| <= |r_build| + |dx_i| + |dx_j|).  The solver
rebuilds before the measured displacement (plus 2.5 steps of drift) reaches
skin / 2, and tests the support exactly on every list entry."""
import numpy as np
import pytest


def pairs_within(pos, radius):
    d = pos[:, None, :] - pos[None, :, :]
    r2 = np.einsum("ijk,ijk->ij", d, d, dtype=np.float32)
    np.fill_diagonal(r2, np.inf)
    return r2 < np.float32(radius) ** 2


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("skin_h", [0.1, 0.3])
def test_lists_cover_the_support_within_half_the_skin(seed, skin_h):
    rng = np.random.default_rng(seed)
    dx, h = 0.01, 0.013
    n_side = 9
    g = np.arange(n_side, dtype=np.float32) * np.float32(dx)
    x0 = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    x0 += rng.uniform(-0.1 * dx, 0.1 * dx, x0.shape).astype(np.float32)
    skin = skin_h * h
    lists = pairs_within(x0, 2 * h + skin)
    # every particle moves by less than half the skin, in a random direction
    u = rng.normal(size=x0.shape)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    mag = rng.uniform(0.0, 0.49 * skin, size=(len(x0), 1))
    x1 = (x0 + (u * mag).astype(np.float32)).astype(np.float32)
    support = pairs_within(x1, 2 * h)
    assert support.sum() > 0
    assert not (support & ~lists).any()


def test_a_larger_move_can_break_the_lists():
    """Beyond skin / 2 per particle the invariant no longer holds: two
    particles just outside the list radius that approach each other by more
    than the skin end up in support without a list entry."""
    h, skin = 0.013, 0.3 * 0.013
    x0 = np.array([[0.0, 0.0, 0.0], [2 * h + 1.01 * skin, 0.0, 0.0]], dtype=np.float32)
    assert not pairs_within(x0, 2 * h + skin)[0, 1]
    x1 = x0 + np.array([[0.6 * skin, 0, 0], [-0.6 * skin, 0, 0]], dtype=np.float32)
    assert pairs_within(x1, 2 * h)[0, 1]
