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


def _fd_check(misfit_at, grad_dot, dirs_fn, ndir=10, eps=1e-4, tol=1e-6, seed=7):
    """Central differences at eps and eps/2, Richardson-extrapolated (error O(eps^4)), along
    `ndir` random directions, against the adjoint gradient."""
    rng = np.random.default_rng(seed)
    for k in range(ndir):
        d = dirs_fn(rng)
        f1 = (misfit_at(eps, d) - misfit_at(-eps, d)) / (2 * eps)
        f2 = (misfit_at(eps / 2, d) - misfit_at(-eps / 2, d)) / eps
        fd = (4 * f2 - f1) / 3
        an = grad_dot(d)
        assert abs(fd - an) <= tol * max(abs(an), 1e-300), (k, f1, f2, fd, an)


def _no_sources(m):
    m.ms_elem = np.zeros(0, np.int32)
    m.ms_nu = np.zeros(0, np.int32)
    m.ms_pat_off = np.zeros(0, np.int64)
    m.ms_pattern = np.zeros(0, np.complex128)
    m.ms_stf = []
    return m


def test_adjoint_dot_product_on_the_adjoint_workload_mesh(built):
    """The FP64 dot-product test on the adjoint workload's own mesh (200 x 200 quads, nr = 9,
    50 receivers): 600 steps, checkpoint every 100."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = _no_sources(meshgen.cartesian_model(nx=200, nz=200, nr=9, nstations=50, nr_aware_dt=True))
    rng = np.random.default_rng(0)
    u0 = meshgen.random_displacement(m, seed=1)
    v0 = meshgen.random_displacement(m, seed=2) * 50.0
    with Solver(m, "fp64") as s:
        s.set_field(u0, "displ")
        s.set_field(v0, "veloc")
        s.forward_checkpointed(600, 100)
        seis = s.seismograms()
        r = rng.normal(size=seis.shape)
        g = s.adjoint(r)
    lhs = float(np.sum(seis * r))
    rhs = float(np.sum(np.real(np.conj(u0) * g["displ0"])) + np.sum(np.real(np.conj(v0) * g["veloc0"])))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1e-300), (lhs, rhs)


def test_adjoint_gradient_on_the_adjoint_workload_mesh(built):
    """The autograd gradient of the L2 waveform misfit against Richardson-extrapolated central
    differences along ten random directions, on the adjoint workload's mesh (200 x 200 quads,
    nr = 9, 50 surface receivers, 5 % Gaussian blob in mu and rho): 1000 steps, checkpoint
    every 100."""
    import torch
    from axisem3d_b200 import meshgen
    from axisem3d_b200.autograd import seismograms
    base = meshgen.cartesian_model(nx=200, nz=200, nr=9, nstations=50, nr_aware_dt=True)
    pert = meshgen.blob_model(base, amp=0.05, seed=3)
    nsteps = 1000
    ne = base.n_solid_elements
    mods0 = base.se_moduli.reshape(ne, 2, 25)
    with torch.no_grad():
        obs = seismograms(torch.tensor(mods0[:, 0]), torch.tensor(mods0[:, 1]),
                          torch.tensor(base.meta_rho), base, nsteps, 100)
    mods = pert.se_moduli.reshape(ne, 2, 25)
    x0 = (mods[:, 0].copy(), mods[:, 1].copy(), pert.meta_rho.copy())
    lam, mu, rho = (torch.tensor(x, requires_grad=True) for x in x0)

    def misfit(l_, m_, r_):
        d = seismograms(l_, m_, r_, base, nsteps, 100)
        return 0.5 * torch.sum((d - obs) ** 2)

    J = misfit(lam, mu, rho)
    J.backward()
    grads = (lam.grad.numpy(), mu.grad.numpy(), rho.grad.numpy())
    assert J.item() > 0
    scales = tuple(float(np.abs(x).mean()) for x in x0)

    def misfit_at(eps, dirs):
        with torch.no_grad():
            return misfit(*(torch.tensor(x + eps * d) for x, d in zip(x0, dirs))).item()

    _fd_check(misfit_at, lambda dirs: sum(float(np.sum(g * d)) for g, d in zip(grads, dirs)),
              lambda rng: [rng.normal(size=(ne, 25)) * sc for sc in scales], ndir=10)


def _model3d(base, lam3, mu3, rho3):
    """The 3-D parameterisation of a uniform-nr isotropic model: per-slice lambda, mu (3-D
    elements, [2][nr][25] each) and per-slice density, assembled into per-slice point masses
    (Mass3D, Material::getMass per slice)."""
    import copy
    m = copy.copy(base)
    ne = base.n_solid_elements
    nr = int(base.se_nr[0])
    m.se_is3d = np.ones(ne, np.uint8)
    m.se_moduli = np.stack([lam3, mu3], axis=1).reshape(-1)
    m.se_mat_off = np.arange(ne, dtype=np.int64) * 2 * nr * 25
    ifact = base.se_geom[:, 5, :]
    mass = np.zeros((len(base.sp_nr), nr))
    for k in range(nr):
        np.add.at(mass[:, k], base.se_pts.ravel(), (rho3[:, k, :] * ifact).ravel())
    m.sp_mass = mass.ravel()
    m.sp_mass_nr = np.full(len(base.sp_nr), nr, np.int32)
    m.sp_mass_off = np.arange(len(base.sp_nr), dtype=np.int64) * nr
    return m


def test_adjoint_per_slice_gradient(built):
    """Per-slice sensitivities (the gradient w.r.t. the values of lambda, mu and rho at every
    slice phi_k = 2 pi k / nr of every element point; a real DFT over k gives them per Fourier
    mode): their sums over the slices equal the 1-D gradient, and central differences of the
    misfit along random 3-D directions -- runs of 3-D elements with per-slice moduli and
    Mass3D masses -- match them."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    base = _model(nx=8, nz=8, nr=9)
    pert = meshgen.blob_model(base, amp=0.05, seed=3)
    nsteps = 300
    ne, nr = base.n_solid_elements, 9
    with Solver(base, "fp64") as s:
        s.run(nsteps)
        obs = s.seismograms()
    with Solver(pert, "fp64") as s:
        s.forward_checkpointed(nsteps, 50)
        d = s.seismograms()
        g = s.adjoint(d - obs, slices=True)
    g3 = np.stack(g["moduli_slices"])                     # (ne, 2, nr, 25)
    gm3 = np.stack(g["mass_slices"])                      # (npoints, nr)
    assert np.allclose(g3.sum(axis=2), g["moduli"], rtol=1e-9, atol=1e-12 * np.abs(g["moduli"]).max())
    assert np.allclose(gm3.sum(axis=1), g["mass"], rtol=1e-9, atol=1e-12 * np.abs(g["mass"]).max())
    # dJ/drho at (element, slice, point) through the per-slice masses
    ifact = base.se_geom[:, 5, :]
    grho3 = gm3[base.se_pts].transpose(0, 2, 1) * ifact[:, None, :]      # (ne, nr, 25)
    mods = pert.se_moduli.reshape(ne, 2, 25)
    x0 = [np.repeat(mods[:, 0][:, None, :], nr, axis=1), np.repeat(mods[:, 1][:, None, :], nr, axis=1),
          np.repeat(pert.meta_rho[:, None, :], nr, axis=1)]
    # the 3-D path at slice-constant values is the 1-D run (odd nr)
    with Solver(_model3d(base, *x0), "fp64") as s:
        s.run(nsteps)
        assert np.linalg.norm(s.seismograms() - d) <= 1e-10 * np.linalg.norm(d)

    def misfit_at(eps, dirs):
        m3 = _model3d(base, *(x + eps * dd for x, dd in zip(x0, dirs)))
        with Solver(m3, "fp64") as s:
            s.run(nsteps)
            r = s.seismograms() - obs
        return 0.5 * float(np.sum(r * r))

    grads = (g3[:, 0], g3[:, 1], grho3)
    scales = tuple(float(np.abs(x).mean()) for x in x0)
    _fd_check(misfit_at, lambda dirs: sum(float(np.sum(gg * dd)) for gg, dd in zip(grads, dirs)),
              lambda rng: [rng.normal(size=(ne, nr, 25)) * sc for sc in scales], ndir=6)
