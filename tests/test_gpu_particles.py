"""Tracer particles on the GPU (sns_particles_move) against the particle
oracle and the reference's own src/Particle.cpp: positions and velocities
equal to the last bit (FP64 arithmetic in the reference's order)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _velocity(shape, seed, scale):
    r = np.random.default_rng(seed)
    return [scale * (r.standard_normal(shape) + 1j * r.standard_normal(shape)) for _ in range(3)]


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_particles_match_the_oracle_bit_for_bit(sns, cuda, dtype):
    from oracle import particles as PO
    u = _velocity((12, 8, 16), 5, 2.0)
    if dtype == torch.complex64:
        u = [x.astype(np.complex64).astype(np.complex128) for x in u]
    ud = [torch.from_numpy(x).to(cuda, dtype) for x in u]
    tr = sns.Tracers.uniform(3000, seed=1, device=cuda)
    loc = tr.pos.cpu().numpy()
    for _ in range(40):
        tr.move(ud, 0.05)
        loc, v = PO.move(loc, u, 0.05)
    assert np.array_equal(tr.pos.cpu().numpy(), loc)
    assert np.array_equal(tr.vel.cpu().numpy(), v)
    assert np.allclose(tr.energy().cpu().numpy(), PO.energy(v), rtol=1e-15, atol=0)


def test_particles_match_the_reference_build(sns, oracle, cuda):
    if not oracle.have_ref():
        pytest.skip("reference build (oracle/_ref) not present")
    u = _velocity((8, 16, 12), 6, 1.5)
    loc0, loc_ref, e_ref = oracle.ref_particles(11, 700, u, 0.04, 25)
    tr = sns.Tracers(torch.from_numpy(loc0).to(cuda))
    ud = [torch.from_numpy(x).to(cuda) for x in u]
    for _ in range(25):
        tr.move(ud, 0.04)
    assert np.array_equal(tr.pos.cpu().numpy(), loc_ref)
    assert np.array_equal(tr.energy().cpu().numpy(), e_ref)


def test_tracers_follow_a_running_stepper(sns, cuda):
    """Advection through an NSStepper's velocity (inverse-transformed on the
    device) agrees with the oracle fed by numpy's inverse of the same V."""
    from oracle import particles as PO
    from spectral_upcxx_b200 import ic
    n, dt = 32, 1e-3
    V0 = ic.solenoidal_spectrum_hat(n, 2, cuda)
    st = sns.NSStepper((n, n, n), 1 / 400, dt, torch.complex128, device=cuda)
    st.bootstrap(V0, sns.curl(V0))
    tr = sns.Tracers.uniform(2000, seed=3, device=cuda)
    loc = tr.pos.cpu().numpy()
    for _ in range(10):
        st.step(1)
        u = [np.fft.ifftn(x.cpu().numpy()) for x in st.velocity()]
        tr.advect(st, dt)
        loc, v = PO.move(loc, u, dt)
    got = tr.pos.cpu().numpy()
    assert np.abs(got - loc).max() < 1e-12
    assert np.all((got > 0) & (got < 2 * np.pi))
    st.close()


def test_particles_reject_bad_arguments(sns, cuda):
    tr = sns.Tracers.uniform(10, device=cuda)
    u = [torch.zeros((4, 4, 1), dtype=torch.complex128, device=cuda) for _ in range(3)]
    with pytest.raises(sns.SNSError):
        tr.move(u, 0.1)
