"""GPU tests of the discrete adjoint (FP64): the dot-product test of the linear
map (initial state -> seismograms) and central finite differences of an L2
waveform misfit along random directions in (lambda, mu, rho)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model(nx=8, nz=8, nr=9, sources=True, nst=12):
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=nx, nz=nz, nr=nr, nstations=nst, nr_aware_dt=True)
    if not sources:
        m.ms_elem = np.zeros(0, np.int32)
        m.ms_nu = np.zeros(0, np.int32)
        m.ms_pat_off = np.zeros(0, np.int64)
        m.ms_pattern = np.zeros(0, np.complex128)
        m.ms_stf = []
    return m


def test_adjoint_dot_product(built):
    """<R Phi(u0, v0), r> == <u0, ubar0(r)> + <v0, vbar0(r)> in FP64 (real inner
    products over the stored complex modes), over several checkpoint segments."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = _model(sources=False)
    rng = np.random.default_rng(0)
    u0 = meshgen.random_displacement(m, seed=1)
    v0 = meshgen.random_displacement(m, seed=2) * 50.0
    nsteps = 230
    with Solver(m, "fp64") as s:
        s.set_field(u0, "displ")
        s.set_field(v0, "veloc")
        s.forward_checkpointed(nsteps, 64)
        seis = s.seismograms()
        r = rng.normal(size=seis.shape)
        g = s.adjoint(r)
    lhs = float(np.sum(seis * r))
    rhs = float(np.sum(np.real(np.conj(u0) * g["displ0"])) + np.sum(np.real(np.conj(v0) * g["veloc0"])))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1e-300), (lhs, rhs)


def test_adjoint_gradient_matches_finite_differences(built):
    """Misfit J = 1/2 |d(m) - d_obs|^2 (L2 waveform difference at the receivers
    against synthetics in the unperturbed model): autograd gradient vs central
    finite differences along random directions in lambda, mu and rho."""
    import torch
    from axisem3d_b200 import meshgen
    from axisem3d_b200.autograd import seismograms
    base = _model(nx=8, nz=8, nr=9)
    pert = meshgen.blob_model(base, amp=0.05, seed=3)
    nsteps = 300
    ne = base.n_solid_elements
    mods0 = base.se_moduli.reshape(ne, 2, 25)
    with torch.no_grad():
        obs = seismograms(torch.tensor(mods0[:, 0]), torch.tensor(mods0[:, 1]),
                          torch.tensor(base.meta_rho), base, nsteps, 50)
    mods = pert.se_moduli.reshape(ne, 2, 25)
    lam = torch.tensor(mods[:, 0].copy(), requires_grad=True)
    mu = torch.tensor(mods[:, 1].copy(), requires_grad=True)
    rho = torch.tensor(pert.meta_rho.copy(), requires_grad=True)

    def misfit(l_, m_, r_):
        d = seismograms(l_, m_, r_, base, nsteps, 50)
        return 0.5 * torch.sum((d - obs) ** 2)

    J = misfit(lam, mu, rho)
    J.backward()
    grads = (lam.grad.numpy(), mu.grad.numpy(), rho.grad.numpy())
    rng = np.random.default_rng(7)
    scales = (np.abs(mods[:, 0]).mean(), np.abs(mods[:, 1]).mean(), pert.meta_rho.mean())
    def fd_at(eps, dirs):
        with torch.no_grad():
            jp = misfit(*(torch.tensor(x + eps * d) for x, d in
                          zip((mods[:, 0], mods[:, 1], pert.meta_rho), dirs))).item()
            jm = misfit(*(torch.tensor(x - eps * d) for x, d in
                          zip((mods[:, 0], mods[:, 1], pert.meta_rho), dirs))).item()
        return (jp - jm) / (2 * eps)

    # ten random directions; central differences at eps and eps/2, Richardson-extrapolated
    # (error O(eps^4)): the O(eps^2) term alone is ~1e-5 of J' here, because the misfit's
    # first derivative is small next to its higher ones
    for k in range(10):
        dirs = [rng.normal(size=(ne, 25)) * sc for sc in scales]
        eps = 1e-4
        f1, f2 = fd_at(eps, dirs), fd_at(eps / 2, dirs)
        fd = (4 * f2 - f1) / 3
        an = sum(float(np.sum(g * d)) for g, d in zip(grads, dirs))
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-300), (k, f1, f2, fd, an)
