"""Device spectral operators and element-wise arithmetic against the oracle
and the reference's golden vectors (complex128: rel L2 <= 1e-12; complex64:
rel L2 <= 2e-6, <= 5e-6 for the cross product which runs 9 transforms)."""
import os

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = {torch.complex128: 1e-12, torch.complex64: 2e-6}
DT = [torch.complex128, torch.complex64]


def dev(a, dtype, device):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def host(t):
    return t.detach().cpu().to(torch.complex128).numpy()


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "operators.npz"))


@pytest.mark.parametrize("dtype", DT)
def test_operators_golden(sns, cuda, gold, dtype):
    tol = TOL[dtype]
    v = [dev(gold[f"v{d}"], dtype, cuda) for d in range(3)]
    w = [dev(gold[f"w{d}"], dtype, cuda) for d in range(3)]
    for d, x in enumerate(sns.gradient(v[0])):
        assert rel_l2(host(x), gold[f"grad{d}"]) < tol
    assert rel_l2(host(sns.laplacian(v[0])), gold["lap"]) < tol
    t = v[0].clone()
    sns.laplacian_inverse(t, 0.0, 1.0)
    assert rel_l2(host(t), gold["ilap_0_1"]) < tol
    t = v[0].clone()
    sns.laplacian_inverse(t, 1.0, -0.25)
    assert rel_l2(host(t), gold["ilap_1_m0.25"]) < tol
    for d, x in enumerate(sns.curl(v)):
        assert rel_l2(host(x), gold[f"curl{d}"]) < tol
    assert rel_l2(host(sns.divergence(v)), gold["div"]) < tol
    for d, x in enumerate(sns.vector_laplacian(v)):
        assert rel_l2(host(x), gold[f"vlap{d}"]) < tol
    for d, x in enumerate(sns.cross(v, w)):
        assert rel_l2(host(x), gold[f"cross{d}"]) < tol * 2.5
    avg = sns.average(v[0])
    assert abs(avg - float(gold["average_v0"])) / float(gold["average_v0"]) < tol


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("shape", [(16, 16, 16), (8, 16, 32), (64, 32, 16)])
def test_operators_match_oracle(sns, oracle, cuda, dtype, shape):
    from spectral_upcxx_b200 import ic
    tol = TOL[dtype]
    v = [oracle.forward(ic.uniform_complex(shape, 60 + d)) for d in range(3)]
    w = [oracle.forward(ic.uniform_complex(shape, 70 + d)) for d in range(3)]
    tv = [dev(x, dtype, cuda) for x in v]
    tw = [dev(x, dtype, cuda) for x in w]
    for a, b in zip(sns.curl(tv), oracle.curl(v)):
        assert rel_l2(host(a), b) < tol
    assert rel_l2(host(sns.divergence(tv)), oracle.divergence(v)) < tol
    for a, b in zip(sns.cross(tv, tw), oracle.cross(v, w)):
        assert rel_l2(host(a), b) < tol * 2.5
    t = tv[1].clone()
    sns.zero_high_modes(t)
    assert rel_l2(host(t), oracle.zero_high_modes(host(tv[1]))) == 0.0


@pytest.mark.parametrize("dtype", DT)
def test_elementwise(sns, oracle, cuda, dtype):
    from spectral_upcxx_b200 import ic
    a = ic.uniform_complex((8, 8, 8), 1)
    b = ic.uniform_complex((8, 8, 8), 2)
    ta, tb = dev(a, dtype, cuda), dev(b, dtype, cuda)
    tol = TOL[dtype]
    assert rel_l2(host(sns.axpby(1.0, ta, 1.0, tb)), a + b) < tol
    assert rel_l2(host(sns.axpby(1.0, ta, -1.0, tb)), a - b) < tol
    assert rel_l2(host(sns.axpby(2.5, ta)), 2.5 * a) < tol
    assert rel_l2(host(sns.mul(ta, tb)), a * b) < tol


@pytest.mark.parametrize("dtype", DT)
def test_average_large(sns, cuda, dtype):
    n = 256
    g = torch.Generator(device=cuda).manual_seed(4)
    x = torch.complex(torch.rand((n, n, n), device=cuda, generator=g, dtype=torch.float64),
                      torch.rand((n, n, n), device=cuda, generator=g, dtype=torch.float64))
    exp = torch.mean(torch.abs(x)).item()
    got = sns.average(x.to(dtype))
    assert abs(got - exp) / exp < (1e-12 if dtype == torch.complex128 else 1e-6)
