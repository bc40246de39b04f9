"""The tracer-particle oracle (oracle/particles.py) against the reference's
own src/Particle.cpp, built in place (oracle/_ref): identical positions and
energies to the last bit, on a non-cubic grid, through many periodic wraps."""
import numpy as np
import pytest


def _velocity(shape, seed, scale):
    r = np.random.default_rng(seed)
    return [scale * (r.standard_normal(shape) + 1j * r.standard_normal(shape)) for _ in range(3)]


def test_particle_oracle_matches_the_reference_bit_for_bit(oracle):
    from oracle import particles as PO
    if not oracle.have_ref():
        pytest.skip("reference build (oracle/_ref) not present")
    u = _velocity((12, 8, 16), 3, 2.0)
    K = 0.05
    loc0, loc_ref, e_ref = oracle.ref_particles(7, 500, u, K, 40)
    assert np.all((loc0 >= 0) & (loc0 <= 2 * np.pi))
    loc = loc0
    for _ in range(40):
        loc, v = PO.move(loc, u, K)
    assert np.array_equal(loc, loc_ref)
    assert np.array_equal(PO.energy(v), e_ref)


def test_particle_oracle_upper_cell_and_wrap():
    """Positions in the last cell use cell n - 2 (extrapolation, no periodic
    wrap of the stencil); steps past 2 pi or below 0 wrap around."""
    from oracle import particles as PO
    n = 8
    u = [np.ones((n, n, n), dtype=complex) * c for c in (1.0, -2.0, 0.5)]
    loc = np.array([[2 * np.pi - 1e-3, 0.1, 3.0]])
    new, v = PO.move(loc, u, 0.01)
    assert np.allclose(v, [[1.0, -2.0, 0.5]])
    assert np.isclose(new[0, 0], 2 * np.pi - 1e-3 + 0.01 - 2 * np.pi)
    assert np.isclose(new[0, 1], 0.1 - 0.02)
    new, v = PO.move(np.array([[0.005, 0.005, 0.005]]), u, 0.01)
    assert np.isclose(new[0, 1], 2 * np.pi + 0.005 - 0.02)
