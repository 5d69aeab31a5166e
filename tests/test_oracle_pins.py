"""CPU tests: the oracle pinned against the reference's tables and analytic
invariants, and the C-ABI library's exports (no GPU needed)."""
import json
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "spectral_npol4.json")


def _golden():
    with open(GOLDEN) as f:
        return json.load(f)["tables"]


def test_spectral_tables_python_match_reference():
    import spectral
    g = _golden()
    t = spectral.tables()
    for k, v in g.items():
        assert np.array_equal(np.asarray(v), t[k]), k


def test_spectral_tables_engine_match_reference(built):
    from axisem3d_b200.solver import spectral_tables
    g = _golden()
    t = spectral_tables()
    for k, v in g.items():
        assert np.array_equal(np.asarray(v), t[k]), k


def test_capi_exports_every_declared_symbol(built):
    import ctypes
    hdr = open(os.path.join(ROOT, "include", "axg.h")).read()
    names = sorted(set(re.findall(r"\b(axg_[a-z0-9_]+)\s*\(", hdr)))
    assert len(names) > 30
    lib = ctypes.CDLL(os.path.join(ROOT, "axisem3d_b200", "libaxg.so"))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from axisem3d_b200 import _lib
    assert set(_lib.SIGNATURES) == set(names)


def test_capi_rejects_bad_config(built):
    import ctypes as C
    from axisem3d_b200 import _lib as L
    lib = L.lib()
    h = C.c_void_p()
    cfg = L.axg_config()
    cfg.precision = 7
    cfg.dt = 1.0
    assert lib.axg_create(C.byref(cfg), C.byref(h)) == L.AXG_E_ARG
    cfg.precision = L.AXG_FP32
    cfg.dt = -1.0
    assert lib.axg_create(C.byref(cfg), C.byref(h)) == L.AXG_E_ARG


def test_quad_geometry_linear_square(built):
    """dsdxii etc. of an axis-aligned 2 x 2 square and the integral factor w_i w_j detJ s."""
    from axisem3d_b200.solver import quad_geometry, spectral_tables
    g, sz = quad_geometry([10., 0., 12., 0., 12., 2., 10., 2.], axial=False)
    t = spectral_tables()
    assert np.allclose(g[0], 1.0) and np.allclose(g[3], 1.0)     # dsdxii = dzdeta = 1 (J = I)
    assert np.allclose(g[1], 0.0) and np.allclose(g[2], 0.0)
    w = np.outer(t["wGLL"], t["wGLL"]).ravel()
    assert np.allclose(g[5], w * sz[0])
    assert np.allclose(g[4], 1.0 / sz[0])


def test_att_moduli_matches_numpy_restatement(built):
    from axisem3d_b200 import meshgen
    from axisem3d_b200.solver import att_moduli
    sls = meshgen.default_sls(3)
    kp = np.linspace(1e11, 2e11, 7)
    mu = np.linspace(5e10, 7e10, 7)
    qk = np.full(7, 57823.0)
    qm = np.linspace(80, 600, 7)
    k2, m2, dk, dm = att_moduli(sls["w"], sls["y"], sls["fmin"], sls["fmax"], sls["fref"], qk, qm, kp, mu)
    kna, kd, kat = meshgen.att_factors(qk, sls)
    mna, md, mat = meshgen.att_factors(qm, sls)
    assert np.allclose(k2, kp * kat, rtol=1e-14) and np.allclose(m2, mu * mat, rtol=1e-14)
    assert np.allclose(dk, kp * kd, rtol=1e-14) and np.allclose(dm, mu * md, rtol=1e-14)


# ------------------------------------------------------------ oracle invariants ---
def _models():
    from axisem3d_b200 import meshgen
    return {
        "cartesian_iso_1d": meshgen.cartesian_model(nx=4, nz=4, nr=5),
        "tiso_3d_full": meshgen.microbench_model(n_elem=24, nr_max=24, seed=3),
        "iso_3d_axial": meshgen.microbench_model(n_elem=24, nr_max=16, seed=4, rheology="iso",
                                                 axial_column=True),
        "aniso_3d": meshgen.microbench_model(n_elem=24, nr_max=16, seed=5, rheology="aniso",
                                             attenuation=None),
    }


def _stiff(o, u, fresh=True):
    """One stiffness evaluation; fresh=True clears the attenuation memory first."""
    if fresh:
        o.reset_attenuation()
    o.set_field(u, "displ")
    o.set_field(np.zeros_like(u), "stiff")
    o.compute_stiffness()
    return o.get_field("stiff")


@pytest.mark.parametrize("name", ["cartesian_iso_1d", "tiso_3d_full", "iso_3d_axial", "aniso_3d"])
def test_oracle_rigid_body_motion_has_no_stiffness(built, name):
    """Rigid translation along z and rotation about z (mode 0) produce zero strain,
    hence zero stiffness force, in every rheology and on the axis."""
    import oracle as O
    m = _models()[name]
    o = O.Oracle(m, "fp64")
    nu = np.asarray(m.sp_nr) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    ref = np.linalg.norm(_stiff(o, __import__("axisem3d_b200").meshgen.random_displacement(m)))
    u = np.zeros((int(nu.sum()), 3), complex)
    u[first, 2] = 1.0                        # translation along z
    f = _stiff(o, u.ravel())
    assert np.linalg.norm(f) < 1e-11 * ref
    u = np.zeros((int(nu.sum()), 3), complex)
    u[first, 1] = m.sp_coords[:, 0] / np.max(m.sp_coords[:, 0])   # rotation about z: u_phi = omega s
    f = _stiff(o, u.ravel())
    assert np.linalg.norm(f) < 1e-11 * ref


SYM_CASES = {
    # name: (builder kwargs, Nyquist weight of the element transform)
    "cartesian_iso_1d": (None, 2.0),
    "tiso_1d_varying_nr": (dict(n_elem=30, nr_max=24, seed=3, is3d=False, attenuation=None), 2.0),
    "tiso_3d_even_nr": (dict(n_elem=30, nr_min=8, nr_max=8, seed=3, attenuation=None), 4.0),
    "aniso_3d_odd_nr": (dict(n_elem=30, nr_min=9, nr_max=9, seed=5, rheology="aniso",
                             attenuation=None), 2.0),
    "iso_3d_axial_even_nr": (dict(n_elem=30, nr_min=6, nr_max=6, seed=4, rheology="iso",
                                  axial_column=True, attenuation=None), 4.0),
}


@pytest.mark.parametrize("name", sorted(SYM_CASES))
def test_oracle_stiffness_is_self_adjoint(built, name):
    """<v, K u>_w == <u, K v>_w with the azimuthal weights w_0 = 1, w_a = 2, and
    w_Nyquist = 4 where a 3-D element's transform halves/doubles its Nyquist mode
    (SolverFFTW.hpp:101-172). With even-nr 3-D elements of different nr sharing a
    point the reference's operator is not self-adjoint in any one such inner
    product, so those cases use a uniform nr."""
    import oracle as O
    from axisem3d_b200 import meshgen
    kw, wn = SYM_CASES[name]
    m = meshgen.cartesian_model(nx=4, nz=4, nr=5) if kw is None else meshgen.microbench_model(**kw)
    o = O.Oracle(m, "fp64")
    u = meshgen.random_displacement(m, seed=11)
    v = meshgen.random_displacement(m, seed=12)
    nr = np.asarray(m.sp_nr)
    nu = nr // 2 + 1
    w = np.concatenate([np.where(np.arange(k) == 0, 1.0,
                                 np.where((np.arange(k) == k - 1) & (r % 2 == 0) & (k > 1), wn, 2.0))
                        for k, r in zip(nu, nr)])
    w = np.repeat(w, 3)
    ku, kv = _stiff(o, u), _stiff(o, v)
    a = np.sum(w * np.real(np.conj(v) * ku))
    b = np.sum(w * np.real(np.conj(u) * kv))
    assert abs(a - b) <= 1e-12 * np.linalg.norm(ku) * np.linalg.norm(v) * 4


def test_oracle_3d_constant_slices_equal_1d(built):
    """A 3-D element whose slices all carry the same moduli gives the 1-D result
    (the Fourier <-> slice transforms are an exact round trip). Odd nr: for even
    nr the slice transform drops the imaginary part of the Nyquist mode, which
    the in-Fourier path keeps."""
    import oracle as O
    from axisem3d_b200 import meshgen
    m1 = meshgen.microbench_model(n_elem=20, nr_min=11, nr_max=11, seed=7, is3d=False, attenuation=None)
    m3 = meshgen.microbench_model(n_elem=20, nr_min=11, nr_max=11, seed=7, is3d=False, attenuation=None)
    ne = m1.n_solid_elements
    mods = m1.se_moduli.reshape(ne, 5, 25)
    chunks, off = [], []
    o_ = 0
    for e in range(ne):
        nrs = int(m1.se_nr[e])
        chunks.append(np.repeat(mods[e][:, None, :], nrs, axis=1).ravel())
        off.append(o_)
        o_ += chunks[-1].size
    m3.se_moduli = np.concatenate(chunks)
    m3.se_mat_off = np.array(off, np.int64)
    m3.se_is3d = np.ones(ne, np.uint8)
    u = meshgen.random_displacement(m1, seed=5)
    f1 = _stiff(O.Oracle(m1, "fp64"), u)
    f3 = _stiff(O.Oracle(m3, "fp64"), u)
    assert np.linalg.norm(f3 - f1) <= 1e-13 * np.linalg.norm(f1)


def test_oracle_sls_relaxes_to_relaxed_moduli(built):
    """Held strain: the SLS memory variables converge to sum_l m_l = dsigma, so the
    stress relaxes to the one of (lambda - dlambda, mu - dmu) without attenuation
    (steady state of Attenuation::updateMem*, AttBuilder::setAlphaBetaGamma)."""
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.microbench_model(n_elem=12, nr_max=9, seed=9, rheology="iso", is3d=False)
    # fast relaxation so that steady state is reached in a few hundred evaluations
    sls = meshgen.default_sls(3, fmin=5.0, fmax=50.0)
    from axisem3d_b200.solver import att_alpha_beta_gamma
    m.att_alpha, m.att_beta, m.att_gamma = att_alpha_beta_gamma(sls["w"], sls["y"], 0.01)
    u = meshgen.random_displacement(m, seed=3)
    o = O.Oracle(m, "fp64")
    for _ in range(600):
        f = _stiff(o, u, fresh=False)
    ne = m.n_solid_elements
    relaxed = meshgen.microbench_model(n_elem=12, nr_max=9, seed=9, rheology="iso", is3d=False)
    mods = relaxed.se_moduli.reshape(ne, 2, 25).copy()
    am = m.se_att_moduli.reshape(ne, 2, 25)
    mods -= am
    relaxed.se_moduli = mods.ravel()
    relaxed.se_att = None
    relaxed.nsls = 0
    fr = _stiff(O.Oracle(relaxed, "fp64"), u)
    assert np.linalg.norm(f - fr) <= 1e-9 * np.linalg.norm(fr)


def test_oracle_fp32_close_to_fp64(built):
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.microbench_model(n_elem=40, nr_max=32, seed=2)
    u = meshgen.random_displacement(m, seed=1)
    f64 = _stiff(O.Oracle(m, "fp64"), u)
    f32 = _stiff(O.Oracle(m, "fp32"), u)
    assert np.linalg.norm(f32 - f64) <= 1e-5 * np.linalg.norm(f64)


def test_spherical_mapping_geometry(built):
    """MappingSpherical: GLL points of a shell quad lie on their circles, the four
    orientations of the same quad give the same points and the same integral factor."""
    from axisem3d_b200 import _lib as L
    from axisem3d_b200.solver import quad_geometry
    r0, r1, t0, t1 = 4.0e6, 4.2e6, 0.3, 0.35
    P = lambda t, r: (r * np.sin(t), r * np.cos(t))  # noqa: E731
    n = [P(t0, r0), P(t1, r0), P(t1, r1), P(t0, r1)]
    g, sz = quad_geometry(np.array(n).ravel(), False, L.AXG_MAP_SPHERICAL)
    r = np.hypot(sz[0], sz[1]).reshape(5, 5)
    assert np.allclose(r[:, 0], r0, rtol=1e-13) and np.allclose(r[:, 4], r1, rtol=1e-13)
    ref = {tuple(np.round(p, 3)) for p in sz.T}
    for rot in range(1, 4):
        nn = n[rot:] + n[:rot]
        g2, sz2 = quad_geometry(np.array(nn).ravel(), False, L.AXG_MAP_SPHERICAL)
        assert {tuple(np.round(p, 3)) for p in sz2.T} == ref
        assert np.isclose(np.sum(g2[5]), np.sum(g[5]), rtol=1e-12)
    assert np.all(g[5] > 0)


def test_absorbing_boundaries_drain_energy():
    """Clayton conditions plus a sponge on two edges (with the halved step that
    Quad::computeDt takes on Clayton quads) stay stable and leave less motion behind
    than reflecting edges at the same step."""
    import oracle as O
    from axisem3d_b200 import meshgen
    m_abc = meshgen.cartesian_model(nx=10, nz=10, nr=3, absorbing=True)
    m_ref = meshgen.cartesian_model(nx=10, nz=10, nr=3)
    m_ref.dt = m_abc.dt
    late = []
    for m in (m_ref, m_abc):
        o = O.Oracle(m, "fp64", threads=4)
        o.run(3000)
        late.append(np.linalg.norm(o.get_field("veloc")))
        assert np.isfinite(late[-1])
    assert late[1] < 0.6 * late[0], late


def test_ocean_and_mass3d_reduce_to_mass1d():
    """MassOceanLoad1D with no ocean mass, and Mass3D with the same mass on every slice,
    act as Mass1D (to rounding): five steps of the oracle in FP64."""
    import oracle as O
    from axisem3d_b200 import meshgen
    base = meshgen.cartesian_model(nx=5, nz=5, nr=6)
    u0 = meshgen.random_displacement(base, seed=4) * 1e-3

    def run(m):
        o = O.Oracle(m, "fp64")
        o.set_field(u0, "displ")
        o.run(5)
        return o.get_field("displ")

    ref = run(base)
    oc = meshgen.cartesian_model(nx=5, nz=5, nr=6)
    meshgen.add_ocean_load(oc, 5, 5, 100e3, tilt=0.4, seed=3)
    oc.ocean_load = (oc.ocean_load[0], np.zeros(len(oc.ocean_load[0])), oc.ocean_load[2])
    m3 = meshgen.with_mass3d(base, amp=0.0, seed=1)
    for m in (oc, m3):
        d = run(m)
        assert np.linalg.norm(d - ref) <= 1e-13 * np.linalg.norm(ref)


def test_scanning_peak_and_mode_count():
    """Scanning1D on a prescribed history: a displacement whose Fourier series fills modes
    0..3 equally, with amplitudes 1, 2, 3, 2, 1 at five scans, has one energy peak (found at
    the scan after the maximum) that needs 4 modes: every point reports nr = 2 * 4 + 1."""
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=3, nz=3, nr=16)
    m.ms_elem = np.zeros(0, np.int32)
    m.ms_nu = np.zeros(0, np.int32)
    m.ms_pat_off = np.zeros(0, np.int64)
    m.ms_pattern = np.zeros(0, np.complex128)
    m.ms_stf = []
    m.scanning = dict(tol_fourier_h1=1e-2, rel_tol_h1=0.1, abs_tol_h1=1e-12, max_num_peaks=10, interval=1)
    o = O.Oracle(m, "fp64")
    nu = 16 // 2 + 1
    pattern = np.zeros((len(m.sp_nr), nu, 3), np.complex128)
    pattern[:, :4, :] = 1.0 + 0.5j
    for t, amp in enumerate((1.0, 2.0, 3.0, 2.0, 1.0)):
        o.set_field((amp * pattern).ravel(), "displ")
        o.record_stations(t)
    s_nr, _ = o.scanning_nr()
    assert np.all(s_nr == 9), np.unique(s_nr)


def test_ocean_load3d_reduces_to_1d():
    """MassOceanLoad3D with the same ocean mass on every slice and a vertical normal equals
    MassOceanLoad1D with theta = 0 (to rounding): five oracle steps in FP64."""
    import oracle as O
    from axisem3d_b200 import meshgen
    m1 = meshgen.cartesian_model(nx=5, nz=5, nr=6)
    meshgen.add_ocean_load(m1, 5, 5, 100e3)
    m3 = meshgen.cartesian_model(nx=5, nz=5, nr=6)
    pts, mo, _ = m1.ocean_load
    nr = np.asarray(m3.sp_nr)[pts]
    off = np.concatenate([[0], np.cumsum(nr)[:-1]]).astype(np.int64)
    nrm = np.zeros((int(nr.sum()), 3))
    nrm[:, 2] = 1.0
    m3.ocean_load3d = (pts, off, np.repeat(mo, nr), nrm)
    u0 = meshgen.random_displacement(m1, seed=4) * 1e-3
    out = []
    for m in (m1, m3):
        o = O.Oracle(m, "fp64")
        o.set_field(u0, "displ")
        o.run(5)
        out.append(o.get_field("displ"))
    assert np.linalg.norm(out[1] - out[0]) <= 1e-12 * np.linalg.norm(out[0])


PRT_CASES = {
    # name: (model builder, 3-D PRT factors)
    "cartesian_iso_1d_full": (lambda m: m.cartesian_model(nx=4, nz=4, nr=6, attenuation=dict(
        m.default_sls(3), qkappa=57823.0, qmu=120.0)), False),
    "tiso_3d_full_prt3d": (lambda m: m.microbench_model(n_elem=40, nr_max=24, seed=21), True),
    "sph_aniso_rtz": (lambda m: m.spherical_model(n_theta=16, n_solid_layers=4, n_fluid_layers=2, nr_max=24,
                                                  rheology="aniso", attenuation=None), False),
}


@pytest.mark.parametrize("name", sorted(PRT_CASES))
def test_identity_prt_equals_no_prt(built, name):
    """PRT factors of the identity (X0 = X3 = |J| = 1, X1 = X2 = 0) give the stiffness of the
    same elements without PRT (two evaluations, attenuation memory included): the
    9-component gradient, RTZ and quadrature of the PRT branch against the 6-component ones."""
    import copy
    import oracle as O
    from axisem3d_b200 import meshgen
    build, three_d = PRT_CASES[name]
    m = build(meshgen)
    u = meshgen.random_displacement(m, seed=5)
    mi = copy.copy(m)
    meshgen.add_prt(mi, amp=0.0, three_d=three_d)
    out = []
    for mm in (m, mi):
        o = O.Oracle(mm, "fp64")
        o.set_field(u, "displ")
        for _ in range(2):
            o.set_field(np.zeros_like(u), "stiff")
            o.compute_stiffness()
        out.append(o.get_field("stiff"))
    assert np.linalg.norm(out[1] - out[0]) <= 1e-14 * np.linalg.norm(out[0])


def test_prt_stiffness_is_self_adjoint(built):
    """With PRT factors (undulatedToSpherical6 scaled by |J| is the transpose of
    sphericalToUndulated6), the stiffness stays self-adjoint under the azimuthal weights."""
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=4, nz=4, nr=5)
    meshgen.add_prt(m, amp=0.08, seed=9)
    o = O.Oracle(m, "fp64")
    u = meshgen.random_displacement(m, seed=11)
    v = meshgen.random_displacement(m, seed=12)
    nu = np.asarray(m.sp_nr) // 2 + 1
    w = np.repeat(np.concatenate([np.where(np.arange(k) == 0, 1.0, 2.0) for k in nu]), 3)
    ku, kv = _stiff(o, u), _stiff(o, v)
    a = np.sum(w * np.real(np.conj(v) * ku))
    b = np.sum(w * np.real(np.conj(u) * kv))
    assert abs(a - b) <= 1e-12 * np.linalg.norm(ku) * np.linalg.norm(v) * 4


def _fluid3d(m):
    import copy
    m3 = copy.copy(m)
    nr = np.asarray(m.fe_nr)
    K = np.asarray(m.fe_moduli).reshape(-1, 25)
    m3.fe_is3d = np.ones(len(nr), np.uint8)
    m3.fe_moduli = np.concatenate([
        (np.tile(K[e], (nr[e], 1)) * (1 + 0.02 * np.sin(np.arange(nr[e])))[:, None]).ravel()
        for e in range(len(nr))])
    m3.fe_mat_off = np.concatenate([[0], np.cumsum(nr * 25)[:-1]]).astype(np.int64)
    return m3


@pytest.mark.parametrize("three_d", [False, True])
def test_identity_fluid_prt_equals_no_prt(built, three_d):
    """Identity PRT factors on the fluid elements of a spherical shell (RTZ frame on) give the
    fluid stiffness without PRT; 3-D fluid elements with per-slice K and 3-D factors too."""
    import copy
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.spherical_model(n_theta=16, n_solid_layers=4, n_fluid_layers=2, nr_max=24)
    if three_d:
        m = _fluid3d(m)
    uf = meshgen.random_displacement(m, seed=6, solid=False)
    out = []
    for mm in (m, meshgen.add_prt_fluid(copy.copy(m), amp=0.0, three_d=three_d)):
        o = O.Oracle(mm, "fp64")
        o.set_field(uf, "displ", solid=False)
        o.compute_stiffness()
        out.append(o.get_field("stiff", solid=False))
    assert np.linalg.norm(out[1] - out[0]) <= 1e-14 * np.linalg.norm(out[0])


@pytest.mark.parametrize("nm", ["GLL", "GLJ"])
def test_reference_tables_are_exact_on_polynomials(nm):
    """The reference's own 12-decimal tables (spectrals.hpp:73-102, as text in the golden file):
    G(j, i) = l_j'(x_i) differentiates every polynomial of degree <= 4 at the nodes, and the
    weights integrate degree <= 7 exactly, against dx (GLL) or (1 + x) dx (GLJ, the axial
    direction), to the tables' rounding."""
    t = _golden()
    x, w = np.asarray(t["p" + nm]), np.asarray(t["w" + nm])
    G = np.asarray(t["g" + nm]).reshape(5, 5)
    for k in range(5):
        dp = k * x ** (k - 1) if k else np.zeros_like(x)
        assert np.abs((x ** k) @ G - dp).max() < 1e-10, k
    for k in range(8):
        exact = (1 - (-1) ** (k + 1)) / (k + 1)
        if nm == "GLJ":
            exact += (1 - (-1) ** (k + 2)) / (k + 2)
        assert abs(w @ x ** k - exact) < 1e-11, k


def _axial_projection(f, mode):
    """AxialBoundary::apply (AxialBoundary.cpp:21-51) on one mode of axis points' forces:
    mode 0 keeps z; mode 1 keeps t = (f_s - i f_phi) / 2 as f_s = t, f_phi = i t; higher
    modes vanish."""
    f = f.copy()
    if mode == 0:
        f[:, :2] = 0
    elif mode == 1:
        t = 0.5 * (f[:, 0] - 1j * f[:, 1])
        f[:, 0], f[:, 1], f[:, 2] = t, 1j * t, 0
    else:
        f[:] = 0
    return f


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("rheology", ["iso", "tiso"])
def test_oracle_patch_test_uniform_strain(built, rheology, mode):
    """Patch test of gradient, stress and quadrature together: a Cartesian-linear field has
    uniform strain, so in a homogeneous isotropic or z-axis TI medium the stress is constant
    and divergence-free and the assembled force vanishes at every point off the outer boundary
    of the box, the axis points included (after their axial projection); the boundary points
    carry the traction. Mode 0: u_x = a x, u_y = a y, u_z = b z, i.e. u_s = a s, u_z = b z.
    Mode 1 (the azimuthal derivative terms and the axis rows of the gradient): the shear
    u_x = a z, u_z = b x, i.e. u_s = a z cos phi, u_phi = -a z sin phi, u_z = b s cos phi, whose
    mode-1 coefficients (u = 2 Re(c e^{i phi})) are a z / 2, i a z / 2 and b s / 2. The
    absolute scale too: <u, K u> (azimuthal weight 1 / 2) equals sigma : e times the integral
    of s ds dz over the box (1e-10)."""
    import oracle as O
    from axisem3d_b200 import _lib as L
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=6, nz=5, nr=5)
    ne = m.n_solid_elements
    if rheology == "tiso":
        lam, mu = m.se_moduli.reshape(ne, 2, 25)[0, :, 0]
        A, Cc, F, Lm, N = (lam + 2 * mu) * 1.08, (lam + 2 * mu) * 0.95, lam * 1.1, mu * 0.9, mu * 1.05
        m.se_rheo = np.full(ne, L.AXG_TISO, np.int32)
        m.se_moduli = np.tile(np.repeat(np.array([A, Cc, F, Lm, N]), 25), ne)
        m.se_mat_off = np.arange(ne, dtype=np.int64) * 125
    o = O.Oracle(m, "fp64")
    nu = np.asarray(m.sp_nr) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    s, z = m.sp_coords[:, 0], m.sp_coords[:, 1]
    u = np.zeros((int(nu.sum()), 3), complex)
    rows = first + mode
    if mode == 0:
        u[rows, 0] = 1e-3 * s
        u[rows, 2] = -2e-3 * z
    else:
        u[rows, 0] = 0.5e-3 * z
        u[rows, 1] = 0.5e-3j * z
        u[rows, 2] = 0.7e-3 * s
    width, height = s.max(), -z.min()
    tol = 1e-9 * max(width, height)
    axis = s < tol
    boundary = (np.abs(s - width) < tol) | (np.abs(z) < tol) | (np.abs(z + height) < tol)

    def force(u):
        f = _stiff(o, u.ravel()).reshape(-1, 3)
        g = f[rows].copy()
        g[axis] = _axial_projection(g[axis], mode)
        return f, g

    f_all, f = force(u)
    fb = np.linalg.norm(f[boundary])
    assert fb > 0 and np.any(~boundary & axis)        # axis points among the interior
    assert np.linalg.norm(f[~boundary]) <= 1e-10 * fb, np.linalg.norm(f[~boundary]) / fb
    # the other modes stay zero (phi-constant medium: the modes decouple)
    assert np.linalg.norm(np.delete(f_all, rows, axis=0)) == 0
    # the energy scale: <u, K u> with the azimuthal weight (1 for mode 0, 2 for mode 1) is the
    # strain energy density sigma : e of the uniform strain times the box's integral of s ds dz
    # (the integral factor carries s; the engine's Fourier-space operator is the energy per 2 pi)
    if rheology == "iso":
        lam, mu = m.se_moduli.reshape(ne, 2, 25)[0, :, 0]
        A = Cc = lam + 2 * mu
        F, Lm, N = lam, mu, mu
    if mode == 0:
        ea, eb = 1e-3, -2e-3             # e_ss = e_phiphi = ea, e_zz = eb
        density = 4 * A * ea * ea - 4 * N * ea * ea + 4 * F * ea * eb + Cc * eb * eb
    else:
        density = Lm * (1e-3 + 1.4e-3) ** 2    # gamma_xz = a + b
    uKu = -(1.0 if mode == 0 else 2.0) * float(np.sum(np.real(np.conj(u.ravel()) * f_all.ravel())))
    assert abs(uKu - density * width ** 2 / 2 * height) <= 1e-10 * abs(uKu), uKu / (density * width ** 2 / 2 * height)
    # the same field with a quadratic term in z is not a patch: the check has teeth
    u[rows, 2] += 1e-8 * z ** 2
    assert np.linalg.norm(force(u)[1][~boundary]) > 1e-6 * fb


def _shell_patch_residuals(n_theta, n_solid_layers, n_fluid_layers, bump):
    """Interior / boundary force norms of the shell patch fields (solid, fluid); bump > 0
    multiplies the fields by 1 + bump (r / r_surface)^2 (non-uniform strain)."""
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.spherical_model(n_theta=n_theta, n_solid_layers=n_solid_layers,
                                n_fluid_layers=n_fluid_layers, nr_max=24, three_d=False, attenuation=None)
    ne, nf = m.n_solid_elements, m.n_fluid_elements
    m.se_moduli = np.tile(np.concatenate([np.full(25, 1.3e11), np.full(25, 0.7e11)]), ne)
    m.se_mat_off = np.arange(ne, dtype=np.int64) * 50
    m.fe_moduli = np.full(nf * 25, float(np.mean(m.fe_moduli)))
    o = O.Oracle(m, "fp64")
    r_cmb, r_top, r_surf = 3480e3, 3600e3, 6371e3

    def rows(nr):
        nu = np.asarray(nr) // 2 + 1
        return np.concatenate([[0], np.cumsum(nu)[:-1]]), int(nu.sum())

    out = []
    for solid, ndim, coords, edges in ((True, 3, m.sp_coords, (r_top, r_surf)),
                                       (False, 1, m.fp_coords, (r_cmb, r_top))):
        first, _ = rows(m.sp_nr if solid else m.fp_nr)
        s, z = coords[:, 0], coords[:, 1]
        r = np.hypot(s, z)
        g = 1.0 + bump * (r / r_surf) ** 2
        boundary = np.zeros(len(r), bool)
        for e in edges:
            boundary |= np.abs(r - e) < 1e-6 * r_surf
        axis = s < 1e-9 * r_surf
        assert np.any(~boundary) and np.any(~boundary & axis)
        us = np.zeros((rows(m.sp_nr)[1], 3), complex)
        uf = np.zeros(rows(m.fp_nr)[1], complex)
        if solid:
            us[first, 0] = 1e-4 * s * g
            us[first, 2] = 1e-4 * z * g
        else:
            uf[first] = 1e3 * z * g
        o.reset_attenuation()
        o.set_field(us.ravel(), "displ")
        o.set_field(np.zeros_like(us.ravel()), "stiff")
        o.set_field(uf, "displ", solid=False)
        o.set_field(np.zeros_like(uf), "stiff", solid=False)
        o.compute_stiffness()
        f = np.asarray(o.get_field("stiff", solid=solid)).reshape(-1, ndim)[first]
        if solid:
            f[axis, :2] = 0            # mode 0 on the axis keeps z (AxialBoundary.cpp:21-51)
        fb = np.linalg.norm(f[boundary])
        assert fb > 0
        out.append(np.linalg.norm(f[~boundary]) / fb)
    return out


def test_oracle_patch_test_spherical_shell(built):
    """The patch test on curved (spherically mapped) quads, solid and fluid, in the shell with
    homogeneous moduli: the uniform dilatation u = a x (u_s = a s, u_z = a z, mode 0) against
    the solid force off the outer surface and the solid-fluid boundary, the linear potential
    chi = b z against the fluid force off the core-mantle and solid-fluid boundaries, axis points
    included. A linear field is not a polynomial of the reference coordinates on a curved quad,
    so the force is small rather than zero: the residual (1e-7 solid, 2e-8 fluid on this mesh)
    falls by more than 10x (22x, 13x) when the mesh is refined twice over, and a field with
    non-uniform strain leaves a force over 1e4 times larger."""
    coarse = _shell_patch_residuals(24, 6, 3, 0.0)
    fine = _shell_patch_residuals(48, 12, 6, 0.0)
    bumped = _shell_patch_residuals(24, 6, 3, 0.5)
    for k in range(2):
        assert coarse[k] < 1e-6, coarse
        assert fine[k] < coarse[k] / 10, (coarse, fine)
        assert bumped[k] > 1e4 * coarse[k], (coarse, bumped)


def test_oracle_newmark_conserves_discrete_energy(built):
    """Energy pin of the whole step (stiffness, axial projection, 1/M, Newmark): without
    sources, attenuation or absorbing boundaries the reference's update (v += h/2 (a_{n-1} +
    a_n); u += h v + h^2/2 a_n, NewmarkTimeScheme.hpp:47-59, velocity Verlet) conserves
    E_n = 1/2 <v, M v> + 1/2 <u, K u> - h^2/8 <a, M a> exactly for a linear system, with
    <u, K u> = -<u, M a> and the azimuthal weights (1 for mode 0, 2 for the others) making the
    Fourier-space products the physical ones. Over 400 steps E stays within 1e-13 (1e-15
    measured), while 1/2 <v, M v> + 1/2 <u, K u> alone moves by 9 %."""
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=8, nz=8, nr=5, nstations=4)
    m.ms_elem = np.zeros(0, np.int32)
    m.ms_nu = np.zeros(0, np.int32)
    m.ms_pat_off = np.zeros(0, np.int64)
    m.ms_pattern = np.zeros(0, np.complex128)
    m.ms_stf = []
    nu = np.asarray(m.sp_nr) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    axis = np.asarray(m.sp_axial) != 0
    mode = np.concatenate([np.arange(k) for k in nu])
    point = np.repeat(np.arange(len(nu)), nu)
    w = np.where(mode == 0, 1.0, 2.0)[:, None]
    mass = np.asarray(m.sp_mass)[point][:, None]

    def project(f):
        f = f.reshape(-1, 3).copy()
        for al in range(int(nu.max())):
            rows = first[axis & (nu > al)] + al
            f[rows] = _axial_projection(f[rows], al)
        f[mode == 0] = f[mode == 0].real        # mode 0 of a real field
        return f.ravel()

    u0 = project(meshgen.random_displacement(m, seed=3))
    v0 = project(meshgen.random_displacement(m, seed=4)) * 200.0
    o = O.Oracle(m, "fp64")
    o.set_field(u0, "displ")
    o.set_field(v0, "veloc")
    h = m.dt

    def dot(x, y):
        return float(np.sum(w * np.real(np.conj(x.reshape(-1, 3)) * y.reshape(-1, 3))))

    a_prev = np.zeros_like(u0)
    E, E_plain = [], []
    for t in range(400):
        o.apply_sources(t)
        o.compute_stiffness()
        o.apply_bc_before_assembly()
        o.apply_bc_after_assembly()
        o.stiff_to_accel()
        # stiff_to_accel leaves a_n in the stiffness field (SolidPoint::computeStiffToAccel);
        # the acceleration field still holds a_{n-1} until the update
        u, v, a = o.get_field("displ"), o.get_field("veloc"), o.get_field("stiff")
        assert np.array_equal(o.get_field("accel"), a_prev)
        vh = v + h / 2 * (a_prev + a)
        Ma = (mass * a.reshape(-1, 3)).ravel()
        uKu = -dot(u, Ma)
        E.append(0.5 * dot(vh, (mass * vh.reshape(-1, 3)).ravel()) + 0.5 * uKu - h * h / 8 * dot(a, Ma))
        E_plain.append(0.5 * dot(vh, (mass * vh.reshape(-1, 3)).ravel()) + 0.5 * uKu)
        o.newmark_update()
        a_prev = a
    E, E_plain = np.array(E), np.array(E_plain)
    assert E[0] > 0
    assert np.abs(E - E[0]).max() <= 1e-13 * E[0], np.abs(E - E[0]).max() / E[0]
    assert np.abs(E_plain - E_plain[0]).max() > 1e-3 * E_plain[0]


@pytest.mark.parametrize("alpha", [2, 3, 4])
@pytest.mark.parametrize("rheology", ["iso", "tiso"])
def test_oracle_antiplane_patch_higher_modes(built, rheology, alpha):
    """The patch test in the higher Fourier modes: the anti-plane field u_z = Re((x + i y)^a)
    / W^a = (s / W)^a cos(a phi) is harmonic, so in a homogeneous isotropic or z-axis TI medium
    (sigma_xz, sigma_yz = L grad u_z) it is in equilibrium and leaves no force off the box's
    outer boundary, the axis included (all modes a >= 2 vanish there). (s / W)^a with a <= 4 is
    in the element basis and the weak form's integrands stay within the GLL / GLJ rules'
    degree 7, so the check is exact to round-off: it pins the a^2 / s terms of the gradient and
    the quadrature and their axis rows. Scale: <u, K u> (weight 2) = L a H / 2."""
    import oracle as O
    from axisem3d_b200 import _lib as L
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=6, nz=5, nr=9)
    ne = m.n_solid_elements
    lam, mu = m.se_moduli.reshape(ne, 2, 25)[0, :, 0]
    shear = mu
    if rheology == "tiso":
        A, Cc, F, Lm, N = (lam + 2 * mu) * 1.08, (lam + 2 * mu) * 0.95, lam * 1.1, mu * 0.9, mu * 1.05
        m.se_rheo = np.full(ne, L.AXG_TISO, np.int32)
        m.se_moduli = np.tile(np.repeat(np.array([A, Cc, F, Lm, N]), 25), ne)
        m.se_mat_off = np.arange(ne, dtype=np.int64) * 125
        shear = Lm
    o = O.Oracle(m, "fp64")
    nu = np.asarray(m.sp_nr) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    rows = first + alpha
    s, z = m.sp_coords[:, 0], m.sp_coords[:, 1]
    width, height = s.max(), -z.min()
    u = np.zeros((int(nu.sum()), 3), complex)
    u[rows, 2] = 0.5 * (s / width) ** alpha         # u_z = 2 Re(c e^{i a phi})
    f_all = _stiff(o, u.ravel()).reshape(-1, 3)
    f = f_all[rows].copy()
    eps = 1e-9 * max(width, height)
    axis = s < eps
    boundary = (np.abs(s - width) < eps) | (np.abs(z) < eps) | (np.abs(z + height) < eps)
    f[axis] = _axial_projection(f[axis], alpha)
    fb = np.linalg.norm(f[boundary])
    assert fb > 0 and np.any(~boundary & axis)
    assert np.linalg.norm(f[~boundary]) <= 1e-10 * fb, np.linalg.norm(f[~boundary]) / fb
    assert np.linalg.norm(np.delete(f_all, rows, axis=0)) == 0
    uKu = -2.0 * float(np.sum(np.real(np.conj(u.ravel()) * f_all.ravel())))
    want = shear * alpha * height / 2
    assert abs(uKu - want) <= 1e-10 * want, uKu / want


def _fluid_box(nr=9):
    """The plain forward box with every element made a fluid element (scalar potential) of
    homogeneous 1/rho, no solid elements, sources or stations."""
    import copy
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=6, nz=5, nr=nr, nstations=1)
    f = copy.copy(m)
    ne = m.n_solid_elements
    f.fe_nr, f.fe_pts, f.fe_axial, f.fe_geom = m.se_nr, m.se_pts, m.se_axial, m.se_geom
    f.fe_is3d = np.zeros(ne, np.uint8)
    f.fe_mat_off = np.arange(ne, dtype=np.int64) * 25
    f.fe_moduli = np.full(ne * 25, 1.0 / 2700.0)
    f.fp_nr, f.fp_mass, f.fp_axial = m.sp_nr, m.sp_mass, m.sp_axial
    f.fp_surface = np.zeros(len(m.sp_nr), np.uint8)
    f.fp_coords = m.sp_coords
    f.se_nr = np.zeros(0, np.int32)
    f.se_pts = np.zeros((0, 25), np.int32)
    f.se_axial = np.zeros(0, np.uint8)
    f.se_geom = np.zeros((0, 6, 25))
    f.se_rheo = np.zeros(0, np.int32)
    f.se_is3d = np.zeros(0, np.uint8)
    f.se_mat_off = np.zeros(0, np.int64)
    f.se_moduli = np.zeros(0)
    f.meta_rho = None
    f.sp_nr = np.zeros(0, np.int32)
    f.sp_mass = np.zeros(0)
    f.sp_axial = np.zeros(0, np.uint8)
    f.sp_coords = np.zeros((0, 2))
    f.ms_elem = np.zeros(0, np.int32)
    f.ms_nu = np.zeros(0, np.int32)
    f.ms_pat_off = np.zeros(0, np.int64)
    f.ms_pattern = np.zeros(0, np.complex128)
    f.ms_stf = []
    f.st_elem = np.zeros(0, np.int32)
    f.st_w = np.zeros((0, 25))
    f.st_phi = np.zeros(0)
    return f


@pytest.mark.parametrize("alpha", [0, 1, 2, 3, 4])
def test_oracle_fluid_patch_test(built, alpha):
    """The fluid element's patch test: in a homogeneous fluid the weak form of div(grad chi / rho)
    leaves no force off the box's outer boundary for a harmonic potential, exactly for one in
    the element basis: chi = z / H (mode 0) and chi = (s / W)^a cos(a phi) = Re((x + i y)^a) / W^a
    (modes 1-4), axis points included (mode >= 1 of a fluid axis point is projected out).
    Scale: <chi, K chi> (azimuthal weight 1 / 2) = (1 / rho) times the integral of |grad chi|^2
    s ds dz over the box per 2 pi: W^2 / (2 H) for mode 0, a H / 2 for mode a."""
    import oracle as O
    m = _fluid_box()
    o = O.Oracle(m, "fp64")
    nu = np.asarray(m.fp_nr) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    rows = first + alpha
    s, z = m.fp_coords[:, 0], m.fp_coords[:, 1]
    width, height = s.max(), -z.min()
    chi = np.zeros(int(nu.sum()), complex)
    chi[rows] = z / height if alpha == 0 else 0.5 * (s / width) ** alpha
    o.set_field(chi, "displ", solid=False)
    o.set_field(np.zeros_like(chi), "stiff", solid=False)
    o.compute_stiffness()
    f_all = o.get_field("stiff", solid=False)
    f = f_all[rows].copy()
    eps = 1e-9 * max(width, height)
    axis = s < eps
    boundary = (np.abs(s - width) < eps) | (np.abs(z) < eps) | (np.abs(z + height) < eps)
    if alpha >= 1:
        f[axis] = 0                          # AxialBoundary: fluid modes >= 1 vanish on the axis
    fb = np.linalg.norm(f[boundary])
    assert fb > 0 and np.any(~boundary & axis)
    assert np.linalg.norm(f[~boundary]) <= 1e-10 * fb, np.linalg.norm(f[~boundary]) / fb
    assert np.linalg.norm(np.delete(f_all, rows)) == 0
    kk = -(1.0 if alpha == 0 else 2.0) * float(np.sum(np.real(np.conj(chi) * f_all)))
    want = (width ** 2 / (2 * height) if alpha == 0 else alpha * height / 2) / 2700.0
    assert abs(kk - want) <= 1e-10 * want, kk / want


def test_oracle_station_records_the_analytic_field(built):
    """Station recording (Station::interpolate, computeFourierAtPhiExp, eigen_tools.hpp:78-106):
    with a displacement whose Fourier coefficients are polynomials of degree <= 4 in s and in
    z (inside the element basis, GLJ rows on the axis), a station at any (xi, eta, phi) of any
    element records the field's value there, u(s, z, phi) = Re c_0 + 2 sum_a Re(c_a e^{i a phi}),
    to round-off: on and off the axis, at interior and edge positions."""
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=6, nz=5, nr=5, nstations=1)
    nu = np.asarray(m.sp_nr) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    s, z = m.sp_coords[:, 0], m.sp_coords[:, 1]
    width, height = s.max(), -z.min()

    def coeffs(s, z):
        x, y = s / width, z / height
        return [np.asarray(1.0 + 0.5 * x - 2.0 * y ** 2 + x ** 3 * y, complex),
                (x - 0.3 * x ** 2 * y) + 1j * (0.7 * x * y ** 2 - x ** 4),
                (x ** 2 + 0.2 * y ** 4) * (0.5 - 1.5j)]

    u = np.zeros((int(nu.sum()), 3), complex)
    for al, c in enumerate(coeffs(s, z)):
        for comp, scale in enumerate((1.0, -0.4, 2.5)):
            u[first + al, comp] = scale * (c if al else c.real)
    rng = np.random.default_rng(5)
    ne, nz_ = m.n_solid_elements, 5
    picks = [(0, -1.0, 0.3), (0, 0.2, -0.7), (7, 0.5, 0.5), (12, -0.9, 1.0), (29, 1.0, -1.0), (3, 0.0, 0.0)]
    st_e, st_w, st_phi, where = [], [], [], []
    for e, xi, eta in picks:
        axial = bool(m.se_axial[e])
        st_e.append(e)
        st_w.append(meshgen.inplane_weights(xi, eta, axial))
        st_phi.append(rng.uniform(0, 2 * np.pi))
        i, j = divmod(e, nz_)
        h_s, h_z = width / 6, height / 5
        where.append(((i + (xi + 1) / 2) * h_s, -height + (j + (eta + 1) / 2) * h_z))
    m.st_elem = np.array(st_e, np.int32)
    m.st_w = np.array(st_w)
    m.st_phi = np.array(st_phi)
    o = O.Oracle(m, "fp64")
    o.set_field(u.ravel(), "displ")
    o.record_stations(0)
    got = o.seismograms()[0]
    for k, ((ss, zz), phi) in enumerate(zip(where, st_phi)):
        c = coeffs(np.array(ss), np.array(zz))
        for comp, scale in enumerate((1.0, -0.4, 2.5)):
            want = scale * (c[0].real + sum(2 * np.real(c[al] * np.exp(1j * al * phi)) for al in (1, 2)))
            assert abs(got[k, comp] - want) <= 1e-12 * (1 + abs(want)), (k, comp, got[k, comp], want)


def test_oracle_moment_source_does_the_moment_tensors_work(built):
    """The moment-tensor source (Mechanism::release for a source on the axis, Mechanism.cpp:
    131-222, injected through SolidElement::addMomentSource, SolidElement.cpp:273-356): its
    nodal force does on any uniform-strain virtual displacement du the work M : e(du) at the
    source, up to one common factor (the STF value, 2 pi, sign). With the azimuthal weights
    (1 for mode 0, 2 for the others), the ratios of <du, F> over seven Cartesian-linear fields
    in modes 0, 1 and 2 equal those of M_zz, M_xx + M_yy, M_xz (twice: du_x = z and du_z = x),
    M_yz, M_xx - M_yy and 2 M_xy, with (x, y, z) = (theta, phi, r) of the source frame at the
    axis: a pin of the pattern's mode structure and of the quadrature without integration."""
    import oracle as O
    from axisem3d_b200 import meshgen
    m = meshgen.cartesian_model(nx=6, nz=5, nr=5, nstations=1)
    mrr, mtt, mpp, mrt, mrp, mtp = m.meta["moment"]
    Mxx, Myy, Mzz, Mxz, Myz, Mxy = mtt, mpp, mrr, mrt, mrp, mtp
    o = O.Oracle(m, "fp64")
    step = int(round(2.5 / m.dt))                     # near the Ricker's peak
    o.apply_sources(step)
    F = o.get_field("stiff").reshape(-1, 3)
    assert np.abs(F).max() > 0
    nu = np.asarray(m.sp_nr) // 2 + 1
    first = np.concatenate([[0], np.cumsum(nu)[:-1]])
    s, z = m.sp_coords[:, 0], m.sp_coords[:, 1]

    def work(mode, cs, cp, cz):
        du = np.zeros_like(F)
        du[first + mode, 0], du[first + mode, 1], du[first + mode, 2] = cs, cp, cz
        return (1.0 if mode == 0 else 2.0) * float(np.sum(np.real(np.conj(du) * F)))

    zero = np.zeros_like(s)
    fields = [
        (work(0, zero, zero, z), Mzz),                        # du_z = z
        (work(0, s, zero, zero), Mxx + Myy),                  # du = (x, y, 0)
        (work(1, z / 2, 1j * z / 2, zero), Mxz),              # du_x = z
        (work(1, zero, zero, s / 2), Mxz),                    # du_z = x
        (work(1, -1j * z / 2, z / 2, zero), Myz),             # du_y = z
        (work(2, s / 2, 1j * s / 2, zero), Mxx - Myy),        # du = (x, -y, 0)
        (work(2, -1j * s / 2, s / 2, zero), 2 * Mxy),         # du = (y, x, 0)
    ]
    k = fields[0][0] / fields[0][1]
    assert k != 0 and all(abs(w) > 0 for _, w in fields)
    scale = max(abs(w) for _, w in fields)
    for i, (got, want) in enumerate(fields):
        assert abs(got - k * want) <= 1e-10 * abs(k) * scale, (i, got / k, want)
