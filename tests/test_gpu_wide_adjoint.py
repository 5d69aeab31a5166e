"""GPU tests of the discrete adjoint on transversely isotropic and 21-Cij elements (FP64,
phi-constant moduli, SPZ and RTZ frames): the dot-product test of the linear map
(initial state -> seismograms) and the moduli gradient of an L2 waveform misfit against
central finite differences along random directions."""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NMOD = {0: 2, 1: 5, 2: 21}


def _wide_model(kind, rtz, sources, nx=8, nz=8, nr=9, seed=5, att=None):
    """The 8 x 8, nr = 9 box with its elements made TI ("tiso"), 21-Cij ("aniso") or a mix of
    isotropic, TI and 21-Cij elements ("mixed"), or left isotropic ("iso"): the isotropic
    background's moduli with seeded 3 % perturbations (TI: each of A, C, F, L, N; 21 Cij: a
    positive-definite symmetric one). With rtz the TI and 21-Cij elements take their moduli in
    the RTZ frame at smooth per-point polar angles. att = "full" or "cg4": 3 SLS with
    Q_mu = 120 (the unrelaxed moduli of the background), CG4 taking dlambda, dmu at its four
    points."""
    from axisem3d_b200 import _lib as L
    from axisem3d_b200 import meshgen
    sls = dict(meshgen.default_sls(3), qkappa=57823.0, qmu=120.0) if att else None
    m = meshgen.cartesian_model(nx=nx, nz=nz, nr=nr, nstations=12, nr_aware_dt=True, attenuation=sls)
    m.dt = meshgen.round_dt(m.dt * 0.9)       # headroom for the stiffer perturbed moduli
    if att:
        a, b, g = meshgen.att_alpha_beta_gamma(sls["w"], sls["y"], m.dt)
        m.att_alpha, m.att_beta, m.att_gamma = a, b, g
        if att == "cg4":
            ne_ = m.n_solid_elements
            am = m.se_att_moduli.reshape(ne_, 2, 25)[:, :, meshgen.CG4_POINTS]
            m.se_att = np.full(ne_, L.AXG_ATT_CG4, np.int32)
            m.se_att_off = np.arange(ne_, dtype=np.int64) * 8
            m.se_att_moduli = np.ascontiguousarray(am).ravel()
    if not sources:
        m.ms_elem = np.zeros(0, np.int32)
        m.ms_nu = np.zeros(0, np.int32)
        m.ms_pat_off = np.zeros(0, np.int64)
        m.ms_pattern = np.zeros(0, np.complex128)
        m.ms_stf = []
    rng = np.random.default_rng(seed)
    ne = m.n_solid_elements
    iso = m.se_moduli.reshape(ne, 2, 25)
    codes = {"iso": [L.AXG_ISO] * ne, "tiso": [L.AXG_TISO] * ne, "aniso": [L.AXG_ANISO] * ne,
             "mixed": [(L.AXG_ISO, L.AXG_TISO, L.AXG_ANISO)[e % 3] for e in range(ne)]}[kind]
    pool, off = [], []
    o = 0
    for e in range(ne):
        lam, mu = iso[e, 0], iso[e, 1]
        if codes[e] == L.AXG_ISO:
            mods = np.stack([lam, mu])
        elif codes[e] == L.AXG_TISO:
            base = np.stack([lam + 2 * mu, lam + 2 * mu, lam, mu, mu])
            mods = base * (1.0 + 0.03 * rng.uniform(-1.0, 1.0, base.shape))
        else:
            mods = np.stack(meshgen.aniso_moduli_from(lam, mu, rng, 0.03))
        off.append(o)
        o += mods.size
        pool.append(mods.ravel())
    m.se_rheo = np.array(codes, np.int32)
    m.se_mat_off = np.array(off, np.int64)
    m.se_moduli = np.concatenate(pool)
    if rtz:
        m.se_rtz = np.ones(ne, np.uint8)
        sz = m.sp_coords[m.se_pts]                      # (ne, 25, 2)
        m.se_theta = 0.4 + 0.6 * sz[..., 0] / 100e3 - 0.3 * sz[..., 1] / 100e3
    return m


def _flat(g):
    return np.concatenate([np.ravel(x) for x in g]) if isinstance(g, list) else np.ravel(g)


@pytest.mark.parametrize("kind,rtz", [("tiso", False), ("aniso", True), ("mixed", True)])
def test_wide_adjoint_dot_product(built, kind, rtz):
    """<R Phi(u0, v0), r> == <u0, ubar0(r)> + <v0, vbar0(r)> in FP64 over several checkpoint
    segments, for TI, 21-Cij (RTZ frame) and mixed-rheology models."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = _wide_model(kind, rtz, sources=False)
    rng = np.random.default_rng(0)
    u0 = meshgen.random_displacement(m, seed=1)
    v0 = meshgen.random_displacement(m, seed=2) * 50.0
    with Solver(m, "fp64") as s:
        s.set_field(u0, "displ")
        s.set_field(v0, "veloc")
        s.forward_checkpointed(230, 64)
        seis = s.seismograms()
        r = rng.normal(size=seis.shape)
        g = s.adjoint(r)
    assert np.all(np.isfinite(seis)) and float(np.max(np.abs(seis))) > 0
    lhs = float(np.sum(seis * r))
    rhs = float(np.sum(np.real(np.conj(u0) * g["displ0"])) + np.sum(np.real(np.conj(v0) * g["veloc0"])))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1e-300), (lhs, rhs)
    # the gradient comes back in each element's own moduli layout
    gm = g["moduli"]
    nm = [NMOD[int(c)] for c in m.se_rheo]
    if kind == "mixed":
        assert isinstance(gm, list) and [x.shape for x in gm] == [(k, 25) for k in nm]
    else:
        assert gm.shape == (m.n_solid_elements, nm[0], 25)


@pytest.mark.parametrize("kind,rtz", [("tiso", True), ("aniso", False), ("mixed", True)])
def test_wide_adjoint_moduli_gradient(built, kind, rtz):
    """Misfit J = 1/2 |d(C) - d_obs|^2 at the receivers (d_obs: the unperturbed model's
    synthetics): the adjoint gradient by every modulus of every element point against central
    differences at eps and eps/2, Richardson-extrapolated, along six random directions."""
    from axisem3d_b200.solver import Solver
    base = _wide_model(kind, rtz, sources=True)
    nsteps, interval = 300, 50

    def run(model):
        with Solver(model, "fp64") as s:
            s.forward_checkpointed(nsteps, interval)
            return s.seismograms()

    obs = run(base)
    rng = np.random.default_rng(11)
    x0 = base.se_moduli * (1.0 + 0.02 * rng.uniform(-1.0, 1.0, base.se_moduli.shape))

    def model_at(x):
        m = copy.deepcopy(base)
        m.se_moduli = x
        return m

    with Solver(model_at(x0), "fp64") as s:
        s.forward_checkpointed(nsteps, interval)
        d = s.seismograms()
        g = s.adjoint(d - obs)
    grad = _flat(g["moduli"])
    assert grad.shape == x0.shape
    J0 = 0.5 * float(np.sum((d - obs) ** 2))
    assert J0 > 0

    def misfit_at(eps, dirv):
        return 0.5 * float(np.sum((run(model_at(x0 + eps * dirv)) - obs) ** 2))

    scale = float(np.mean(np.abs(x0)))
    eps = 1e-4
    for k in range(6):
        dirv = rng.normal(size=x0.shape) * scale
        f1 = (misfit_at(eps, dirv) - misfit_at(-eps, dirv)) / (2 * eps)
        f2 = (misfit_at(eps / 2, dirv) - misfit_at(-eps / 2, dirv)) / eps
        fd = (4 * f2 - f1) / 3
        an = float(np.dot(grad, dirv))
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-300), (k, f1, f2, fd, an)


def _att_grad(model, gm):
    """The adjoint's dlambda, dmu rows (the last two of each attenuating element) in the layout
    of model.se_att_moduli: [2][25] per element (FULL), [2][4] at the CG4 points (CG4)."""
    from axisem3d_b200 import _lib as L
    from axisem3d_b200 import meshgen
    rows = gm if isinstance(gm, list) else list(gm)
    out = []
    for e, r in enumerate(rows):
        d = r[-2:]
        out.append((d[:, meshgen.CG4_POINTS] if model.se_att[e] == L.AXG_ATT_CG4 else d).ravel())
    return np.concatenate(out)


@pytest.mark.parametrize("kind,rtz,att", [("iso", False, "full"), ("tiso", True, "full"),
                                          ("aniso", True, "cg4"), ("mixed", True, "full")])
def test_attenuation_adjoint_dot_product(built, kind, rtz, att):
    """The dot-product test through the SLS recursion (FULL and CG4; checkpoints hold the
    memory variables, each segment is recomputed from them): <R Phi(u0, v0), r> ==
    <u0, ubar0(r)> + <v0, vbar0(r)> in FP64 over several checkpoint segments."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = _wide_model(kind, rtz, sources=False, att=att)
    rng = np.random.default_rng(0)
    u0 = meshgen.random_displacement(m, seed=1)
    v0 = meshgen.random_displacement(m, seed=2) * 50.0
    with Solver(m, "fp64") as s:
        s.set_field(u0, "displ")
        s.set_field(v0, "veloc")
        s.forward_checkpointed(230, 64)
        seis = s.seismograms()
        r = rng.normal(size=seis.shape)
        g = s.adjoint(r)
        # the adjoint leaves the handle in the state after the forward run, SLS memory included
        d_end = s.get_field("displ")
        s.run(5)
        d_more = s.get_field("displ")
    with Solver(m, "fp64") as s2:
        s2.set_field(u0, "displ")
        s2.set_field(v0, "veloc")
        s2.run(230)
        ref_end = s2.get_field("displ")
        s2.run(5)
        ref_more = s2.get_field("displ")
    # equal up to the order of the atomic scatter-adds
    assert np.linalg.norm(d_end - ref_end) <= 1e-11 * np.linalg.norm(ref_end)
    assert np.linalg.norm(d_more - ref_more) <= 1e-11 * np.linalg.norm(ref_more)
    lhs = float(np.sum(seis * r))
    rhs = float(np.sum(np.real(np.conj(u0) * g["displ0"])) + np.sum(np.real(np.conj(v0) * g["veloc0"])))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1e-300), (lhs, rhs)


@pytest.mark.parametrize("kind,rtz,att", [("iso", False, "full"), ("tiso", True, "cg4")])
def test_attenuation_adjoint_moduli_gradient(built, kind, rtz, att):
    """The gradient by the unrelaxed moduli and by dlambda, dmu of every attenuating element
    point against Richardson-extrapolated central differences of the L2 waveform misfit along
    six random directions."""
    from axisem3d_b200.solver import Solver
    base = _wide_model(kind, rtz, sources=True, att=att)
    nsteps, interval = 300, 50
    nm = base.se_moduli.size

    def model_at(x):
        m = copy.deepcopy(base)
        m.se_moduli = x[:nm].copy()
        m.se_att_moduli = x[nm:].copy()
        return m

    def run(model):
        with Solver(model, "fp64") as s:
            s.forward_checkpointed(nsteps, interval)
            return s.seismograms()

    obs = run(base)
    rng = np.random.default_rng(13)
    xb = np.concatenate([base.se_moduli, base.se_att_moduli])
    x0 = xb * (1.0 + 0.02 * rng.uniform(-1.0, 1.0, xb.shape))
    with Solver(model_at(x0), "fp64") as s:
        s.forward_checkpointed(nsteps, interval)
        d = s.seismograms()
        g = s.adjoint(d - obs)
    gm = g["moduli"]
    rows = gm if isinstance(gm, list) else list(gm)
    grad = np.concatenate([np.concatenate([r[:-2].ravel() for r in rows]), _att_grad(base, gm)])
    assert grad.shape == x0.shape
    assert float(np.max(np.abs(_att_grad(base, gm)))) > 0

    def misfit_at(eps, dirv):
        return 0.5 * float(np.sum((run(model_at(x0 + eps * dirv)) - obs) ** 2))

    # directions scaled per block: the attenuation moduli are a few % of the elastic ones
    sc = np.concatenate([np.full(nm, np.mean(np.abs(x0[:nm]))), np.full(x0.size - nm, np.mean(np.abs(x0[nm:])))])
    eps = 1e-4
    for k in range(6):
        dirv = rng.normal(size=x0.shape) * sc
        f1 = (misfit_at(eps, dirv) - misfit_at(-eps, dirv)) / (2 * eps)
        f2 = (misfit_at(eps / 2, dirv) - misfit_at(-eps / 2, dirv)) / eps
        fd = (4 * f2 - f1) / 3
        an = float(np.dot(grad, dirv))
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-300), (k, f1, f2, fd, an)
    # the attenuation moduli alone
    dirv = np.zeros_like(x0)
    dirv[nm:] = rng.normal(size=x0.size - nm) * sc[nm:]
    f1 = (misfit_at(eps, dirv) - misfit_at(-eps, dirv)) / (2 * eps)
    f2 = (misfit_at(eps / 2, dirv) - misfit_at(-eps / 2, dirv)) / eps
    fd = (4 * f2 - f1) / 3
    an = float(np.dot(grad, dirv))
    assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-300), (f1, f2, fd, an)


def test_wide_adjoint_rejects_slices_and_3d_moduli(built):
    """Per-slice sensitivities stay isotropic and elastic; 3-D (per-slice) TI moduli stay
    undifferentiated (3-D elements must be isotropic and elastic)."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import EngineError, Solver
    m = _wide_model("tiso", False, sources=False)
    with Solver(m, "fp64") as s:
        s.set_field(meshgen.random_displacement(m, seed=1), "displ")
        s.forward_checkpointed(20, 10)
        r = np.zeros_like(s.seismograms())
        with pytest.raises(EngineError, match="per-slice sensitivities need isotropic"):
            s.adjoint(r, slices=True)
    from axisem3d_b200 import _lib as L
    m3 = meshgen.cartesian_model(nx=4, nz=4, nr=5, nstations=4)
    ne = m3.n_solid_elements
    lam, mu = m3.se_moduli.reshape(ne, 2, 25)[0, :, 0]
    m3.se_is3d = np.ones(ne, np.uint8)
    m3.se_rheo = np.full(ne, L.AXG_TISO, np.int32)
    m3.se_moduli = np.tile(np.repeat(np.array([lam + 2 * mu, lam + 2 * mu, lam, mu, mu]), 5 * 25), ne)
    m3.se_mat_off = np.arange(ne, dtype=np.int64) * 5 * 5 * 25
    with Solver(m3, "fp64") as s:
        with pytest.raises(EngineError, match="3-D elements must be isotropic"):
            s.forward_checkpointed(10, 5)


def _model3d_elastic(nr, sources, seed=7, pert=0.05):
    """The 8 x 8 box with 3-D isotropic elements: lambda, mu per (slice, point) with seeded
    5 % perturbations around the background (a 3-D model), 1-D masses."""
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=8, nz=8, nr=nr, nstations=12, nr_aware_dt=True)
    m.dt = meshgen.round_dt(m.dt * 0.9)
    if not sources:
        m.ms_elem = np.zeros(0, np.int32)
        m.ms_nu = np.zeros(0, np.int32)
        m.ms_pat_off = np.zeros(0, np.int64)
        m.ms_pattern = np.zeros(0, np.complex128)
        m.ms_stf = []
    ne = m.n_solid_elements
    rng = np.random.default_rng(seed)
    iso = m.se_moduli.reshape(ne, 2, 1, 25)
    m3 = np.repeat(iso, nr, axis=2) * (1.0 + pert * rng.uniform(-1.0, 1.0, (ne, 2, nr, 25)))
    m.se_is3d = np.ones(ne, np.uint8)
    m.se_moduli = m3.ravel()
    m.se_mat_off = np.arange(ne, dtype=np.int64) * 2 * nr * 25
    return m


@pytest.mark.parametrize("nr", [9, 8])
def test_3d_moduli_adjoint_dot_product(built, nr):
    """The dot-product test on a 3-D model (per-slice moduli couple the Fourier modes; the
    transpose is W K W^-1 with the azimuthal weights, the Nyquist mode of the even nr
    included): <R Phi(u0, v0), r> == <u0, ubar0(r)> + <v0, vbar0(r)> in FP64."""
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import Solver
    m = _model3d_elastic(nr, sources=False)
    rng = np.random.default_rng(0)
    u0 = meshgen.random_displacement(m, seed=1)
    v0 = meshgen.random_displacement(m, seed=2) * 50.0
    with Solver(m, "fp64") as s:
        s.set_field(u0, "displ")
        s.set_field(v0, "veloc")
        s.forward_checkpointed(230, 64)
        seis = s.seismograms()
        r = rng.normal(size=seis.shape)
        g = s.adjoint(r)
    assert np.all(np.isfinite(seis)) and float(np.max(np.abs(seis))) > 0
    lhs = float(np.sum(seis * r))
    rhs = float(np.sum(np.real(np.conj(u0) * g["displ0"])) + np.sum(np.real(np.conj(v0) * g["veloc0"])))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1e-300), (lhs, rhs)


def test_3d_moduli_adjoint_per_slice_gradient(built):
    """On a 3-D background (per-slice lambda, mu): the per-slice sensitivities against
    Richardson-extrapolated central differences of the L2 waveform misfit along six random
    per-slice directions, and their sums over the slices against the gradient by a
    phi-constant change."""
    from axisem3d_b200.solver import Solver
    nr = 9
    base = _model3d_elastic(nr, sources=True, seed=7)
    ne = base.n_solid_elements
    nsteps, interval = 300, 50

    def run(model):
        with Solver(model, "fp64") as s:
            s.forward_checkpointed(nsteps, interval)
            return s.seismograms()

    obs = run(base)
    rng = np.random.default_rng(17)
    x0 = base.se_moduli * (1.0 + 0.02 * rng.uniform(-1.0, 1.0, base.se_moduli.shape))

    def model_at(x):
        m = copy.deepcopy(base)
        m.se_moduli = x
        return m

    with Solver(model_at(x0), "fp64") as s:
        s.forward_checkpointed(nsteps, interval)
        d = s.seismograms()
        g = s.adjoint(d - obs, slices=True)
    g3 = np.stack(g["moduli_slices"])                    # (ne, 2, nr, 25)
    assert g3.shape == (ne, 2, nr, 25)
    assert np.allclose(g3.sum(axis=2), g["moduli"], rtol=1e-9, atol=1e-12 * np.abs(g["moduli"]).max())
    grad = g3.ravel()

    def misfit_at(eps, dirv):
        return 0.5 * float(np.sum((run(model_at(x0 + eps * dirv)) - obs) ** 2))

    scale = float(np.mean(np.abs(x0)))
    eps = 1e-4
    for k in range(6):
        dirv = rng.normal(size=x0.shape) * scale
        f1 = (misfit_at(eps, dirv) - misfit_at(-eps, dirv)) / (2 * eps)
        f2 = (misfit_at(eps / 2, dirv) - misfit_at(-eps / 2, dirv)) / eps
        fd = (4 * f2 - f1) / 3
        an = float(np.dot(grad, dirv))
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-300), (k, f1, f2, fd, an)
