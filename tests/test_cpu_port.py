"""The tuned CPU port (oracle/cpu_port.cpp), the CPU baseline that bench.py
times, against the oracle: vmult to 1e-13 relative for the heat operator with
k(T) on perturbed cells, the constant-coefficient heat operator on uniform
cells (Dirichlet faces) and the advection-diffusion operator with the vortex
velocity on uniform and perturbed cells, degrees 1-4; the diagonal; CG +
Jacobi iteration counts."""
import numpy as np
import pytest

from oracle import cpu_port as P
from oracle import oracle as O

TOL = 1e-13


def rng(s):
    return np.random.Generator(np.random.PCG64(s))


def _mask(om, nc, p):
    from meltpooldg_b200.operators import boundary_mask
    return boundary_mask(nc, p)


def relerr(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_heat_kT_perturbed(p):
    nc = (5, 4, 3)
    V = O.box_vertices(3, nc, (0, 0, 0), (1, 1, 1), 0.1, 2)
    om = O.Mesh(3, p, nc, V)
    mask = _mask(om, nc, p)
    T = rng(3).uniform(300, 3000, om.n_dofs)
    src = rng(p).uniform(-1, 1, om.n_dofs)
    port = P.PortOperator(V, nc, p, mask, uniform=False, kind=0, dt=1e-3, rho_cp=2.0, k0=1.5, k_alpha=1e-3,
                          temperature=T)
    got = port.vmult(np.zeros(om.n_dofs), src)
    oop = O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, k_alpha=1e-3, temperature=T, dirichlet=mask)
    assert relerr(got, O.vmult(om, oop, src)) < TOL
    assert relerr(port.diagonal(), O.diagonal(om, oop)) < TOL


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("perturb", [0.0, 0.1])
def test_advdiff_vortex(p, perturb):
    nc = (4, 3, 5)
    V = O.box_vertices(3, nc, (0, 0, 0), (1, 1, 1), perturb, 4)
    om = O.Mesh(3, p, nc, V)
    src = rng(10 + p).uniform(-1, 1, om.n_dofs)
    port = P.PortOperator(V, nc, p, None, uniform=perturb == 0.0, kind=1, dt=1e-3, theta=0.5,
                          diffusivity=1e-3, velocity="vortex")
    got = port.vmult(np.zeros(om.n_dofs), src)
    oop = O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-3, vel_kind=O.VEL_VORTEX)
    assert relerr(got, O.vmult(om, oop, src)) < TOL


@pytest.mark.parametrize("p", [2, 3])
def test_uniform_heat_cg_jacobi(p):
    nc = (6, 6, 6)
    V = O.box_vertices(3, nc, (0, 0, 0), (1, 1, 1))
    om = O.Mesh(3, p, nc, V)
    mask = _mask(om, nc, p)
    port = P.PortOperator(V, nc, p, mask, uniform=True, kind=0, dt=1e-3, rho_cp=1.0, k0=1.0)
    oop = O.Operator(O.HEAT, 1e-3, rho_cp=1.0, k0=1.0, dirichlet=mask)
    src = rng(1).uniform(-1, 1, om.n_dofs)
    assert relerr(port.vmult(np.zeros(om.n_dofs), src), O.vmult(om, oop, src)) < TOL
    b = rng(5).uniform(-1, 1, om.n_dofs)
    b[mask == 1] = 0.0
    x, it, res = port.cg_jacobi(b, rel_tol=1e-10, abs_tol=0.0)
    xo, it_o, _, ok = O.cg(om, oop, b, inv_diag=O.inverse_diagonal(om, oop), rel_tol=1e-10, abs_tol=0.0)
    assert ok and it == it_o
    assert relerr(x, xo) < 1e-9
