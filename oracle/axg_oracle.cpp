// axg_oracle.cpp -- CPU restatement of AxiSEM3D's per-time-step loop (nPol = 4).
//
// TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA engine in
// axisem3d_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline load it. It is never part of the product path.
//
// Parity status: the reference ships no tests, fixtures or golden vectors for
// this path and cannot be compiled in this container (Eigen, Boost, FFTW3,
// METIS, NetCDF and MPI are absent). The restatement is therefore pinned only
// on the reference's GLL/GLJ tables (tests/golden/spectral_npol4.json) and on
// analytic invariants (polynomial gradients, symmetry of the stiffness
// operator, FFT round trips, closed-form SLS relaxation): parity unpinned
// against reference outputs.
//
// Each step follows the reference files cited beside it, in the reference's
// operation order, with a direct DFT in place of FFTW (same normalisation and
// Nyquist conventions, SOLVER/src/core/fft/SolverFFTW.hpp:101-172). Templated
// on the working precision: Real = double is the FP64 oracle; Real = float
// follows the reference's default single-precision build.
//
// Inputs are the structs of include/axg.h, so the same model feeds the oracle
// and the engine.

#include "../include/axg.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <map>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

namespace {

constexpr int P = 5;
constexpr int N = 25;

// ---------------------------------------------------------------------------
// GLL / GLJ tables for nPol = 4, generated from their definitions (see
// spectral_tables() below); must equal spectrals.hpp:73-102 to 12 decimals.
// ---------------------------------------------------------------------------
struct Spectral {
    double G_GLL[P][P];   // G(j, i) = l_j'(x_i), row-major (GradientQuadrature sG_GLL)
    double G_GLJ[P][P];
};

Spectral gSpectral;
bool gSpectralSet = false;

// ------------------------------- small types --------------------------------
template <class R> using Cx = std::complex<R>;
template <class R> struct CM { Cx<R> a[P][P]; };       // CMatPP_RM
template <class R> struct RM { R a[P][P]; };            // RMatPP_RM

template <class R>
struct Ops {                    // GradientQuadrature operands (cast to Real)
    RM<R> dsdxii, dsdeta, dzdxii, dzdeta, inv_s;
    RM<R> dsdxii_if, dsdeta_if, dzdxii_if, dzdeta_if, inv_s_if;
    bool axial;
};

template <class R>
struct GMat {
    RM<R> G_GLL, G_GLJ, GT_GLL, GT_GLJ;
};

// ---------------------------------------------------------------------------
// Gradient / quadrature (SOLVER/src/core/element/grad/GradientQuadrature.hpp)
// ---------------------------------------------------------------------------
template <class R>
struct Grad {
    const Ops<R> &o;
    const GMat<R> &g;
    const RM<R> &GTxi() const { return o.axial ? g.GT_GLJ : g.GT_GLL; }
    const RM<R> &Gxi() const { return o.axial ? g.G_GLJ : g.G_GLL; }

    // computeGrad_dSdZ (GradientQuadrature.hpp:404-418)
    void dSdZ(const CM<R> &F, CM<R> &dS, CM<R> &dZ) const {
        const RM<R> &GT = GTxi();
        for (int i = 0; i < P; i++) {
            for (int j = 0; j < P; j++) {
                Cx<R> X = 0, Y = 0;
                for (int k = 0; k < P; k++) {
                    X += GT.a[i][k] * F.a[k][j];
                    Y += F.a[i][k] * g.G_GLL.a[k][j];
                }
                dS.a[i][j] = X * o.dzdeta.a[i][j] + Y * o.dzdxii.a[i][j];
                dZ.a[i][j] = X * o.dsdeta.a[i][j] + Y * o.dsdxii.a[i][j];
            }
        }
    }
    // computeGrad_1overS_setTo / _addTo (GradientQuadrature.hpp:421-459)
    void overS(const CM<R> &A, CM<R> &AoS, bool add) const {
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                Cx<R> v = A.a[i][j] * o.inv_s.a[i][j];
                AoS.a[i][j] = add ? AoS.a[i][j] + v : v;
            }
        if (o.axial) {
            const RM<R> &GT = GTxi();
            for (int j = 0; j < P; j++) {
                Cx<R> X = 0, Y = 0;
                for (int k = 0; k < P; k++) {
                    X += GT.a[0][k] * A.a[k][j];
                    Y += A.a[0][k] * g.G_GLL.a[k][j];
                }
                Cx<R> v = X * o.dzdeta.a[0][j] + Y * o.dzdxii.a[0][j];
                AoS.a[0][j] = add ? AoS.a[0][j] + v : v;
            }
        }
    }
    // computeQuad_dSdZ (GradientQuadrature.hpp:462-478)
    void quad_dSdZ(const CM<R> &dS, const CM<R> &dZ, CM<R> &F, bool integrate) const {
        const RM<R> &sx = integrate ? o.dsdxii_if : o.dsdxii;
        const RM<R> &se = integrate ? o.dsdeta_if : o.dsdeta;
        const RM<R> &zx = integrate ? o.dzdxii_if : o.dzdxii;
        const RM<R> &ze = integrate ? o.dzdeta_if : o.dzdeta;
        CM<R> X, Y;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                X.a[i][j] = dS.a[i][j] * ze.a[i][j] + dZ.a[i][j] * se.a[i][j];
                Y.a[i][j] = dS.a[i][j] * zx.a[i][j] + dZ.a[i][j] * sx.a[i][j];
            }
        const RM<R> &G = Gxi();
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                Cx<R> a = 0, b = 0;
                for (int k = 0; k < P; k++) {
                    a += G.a[i][k] * X.a[k][j];
                    b += Y.a[i][k] * g.GT_GLL.a[k][j];
                }
                F.a[i][j] = a + b;
            }
    }
    // computeQuad_1overS_addTo (GradientQuadrature.hpp:481-500)
    void quad_overS(const CM<R> &A, CM<R> &F, bool integrate) const {
        const RM<R> &os = integrate ? o.inv_s_if : o.inv_s;
        const RM<R> &zx = integrate ? o.dzdxii_if : o.dzdxii;
        const RM<R> &ze = integrate ? o.dzdeta_if : o.dzdeta;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) F.a[i][j] -= A.a[i][j] * os.a[i][j];
        if (o.axial) {
            const RM<R> &G = Gxi();
            Cx<R> X0[P], Y0[P];
            for (int j = 0; j < P; j++) {
                X0[j] = A.a[0][j] * ze.a[0][j];
                Y0[j] = A.a[0][j] * zx.a[0][j];
            }
            for (int i = 0; i < P; i++)
                for (int j = 0; j < P; j++) F.a[i][j] -= G.a[i][0] * X0[j];
            for (int j = 0; j < P; j++) {
                Cx<R> b = 0;
                for (int k = 0; k < P; k++) b += Y0[k] * g.GT_GLL.a[k][j];
                F.a[0][j] -= b;
            }
        }
    }
    static Cx<R> ia(int alpha, const Cx<R> &x) { return Cx<R>((R)0, (R)alpha) * x; }

    // computeGrad6 (GradientQuadrature.hpp:207-231)
    void grad6(const CM<R> u[3], CM<R> e[6], int alpha) const {
        dSdZ(u[0], e[0], e[4]);
        dSdZ(u[1], e[5], e[3]);
        dSdZ(u[2], e[1], e[2]);
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) e[4].a[i][j] += e[1].a[i][j];
        CM<R> A0, A1, A2;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                A0.a[i][j] = ia(alpha, u[0].a[i][j]) - u[1].a[i][j];
                A1.a[i][j] = ia(alpha, u[1].a[i][j]) + u[0].a[i][j];
                A2.a[i][j] = ia(alpha, u[2].a[i][j]);
            }
        overS(A0, e[5], true);
        overS(A1, e[1], false);
        overS(A2, e[3], true);
    }
    // computeQuad6 / computeQuad6_NoIntegration (GradientQuadrature.hpp:294-324, 363-390)
    void quad6(const CM<R> s[6], CM<R> f[3], int alpha, bool integrate) const {
        quad_dSdZ(s[0], s[4], f[0], integrate);
        quad_dSdZ(s[5], s[3], f[1], integrate);
        quad_dSdZ(s[4], s[2], f[2], integrate);
        CM<R> A0, A1, A2;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                A0.a[i][j] = ia(alpha, s[5].a[i][j]) - s[1].a[i][j];
                A1.a[i][j] = ia(alpha, s[1].a[i][j]) + s[5].a[i][j];
                A2.a[i][j] = ia(alpha, s[3].a[i][j]);
            }
        quad_overS(A0, f[0], integrate);
        quad_overS(A1, f[1], integrate);
        quad_overS(A2, f[2], integrate);
    }
    // computeGrad9 (GradientQuadrature.hpp:181-205): ui_j with j = d/ds, 1/s terms, d/dz
    void grad9(const CM<R> u[3], CM<R> g[9], int alpha) const {
        dSdZ(u[0], g[0], g[2]);
        dSdZ(u[1], g[3], g[5]);
        dSdZ(u[2], g[6], g[8]);
        CM<R> A0, A1, A2;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                A0.a[i][j] = ia(alpha, u[0].a[i][j]) - u[1].a[i][j];
                A1.a[i][j] = ia(alpha, u[1].a[i][j]) + u[0].a[i][j];
                A2.a[i][j] = ia(alpha, u[2].a[i][j]);
            }
        overS(A0, g[1], false);
        overS(A1, g[4], false);
        overS(A2, g[7], false);
    }
    // computeQuad9 (GradientQuadrature.hpp:258-292)
    void quad9(const CM<R> s[9], CM<R> f[3], int alpha) const {
        quad_dSdZ(s[0], s[2], f[0], true);
        quad_dSdZ(s[3], s[5], f[1], true);
        quad_dSdZ(s[6], s[8], f[2], true);
        CM<R> A0, A1, A2;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                A0.a[i][j] = ia(alpha, s[1].a[i][j]) - s[4].a[i][j];
                A1.a[i][j] = ia(alpha, s[4].a[i][j]) + s[1].a[i][j];
                A2.a[i][j] = ia(alpha, s[7].a[i][j]);
            }
        quad_overS(A0, f[0], true);
        quad_overS(A1, f[1], true);
        quad_overS(A2, f[2], true);
    }
    // computeGrad3 (GradientQuadrature.hpp:163-175)
    void grad3(const CM<R> &p, CM<R> q[3], int alpha) const {
        dSdZ(p, q[0], q[2]);
        CM<R> A;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) A.a[i][j] = ia(alpha, p.a[i][j]);
        overS(A, q[1], false);
    }
    // computeQuad3 (GradientQuadrature.hpp:234-252)
    void quad3(const CM<R> q[3], CM<R> &f, int alpha) const {
        quad_dSdZ(q[0], q[2], f, true);
        CM<R> A;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) A.a[i][j] = ia(alpha, q[1].a[i][j]);
        quad_overS(A, f, true);
    }
};

// ---------------------------------------------------------------------------
// Direct real DFT with FFTW's conventions (SolverFFTW.hpp:101-172)
// ---------------------------------------------------------------------------
template <class R>
struct Twiddle {
    int nr = 0;
    std::vector<R> c, s;   // cos / sin (2 pi j / nr), j in [0, nr)
    void set(int n) {
        nr = n; c.resize(n); s.resize(n);
        for (int j = 0; j < n; j++) {
            double ang = 2.0 * M_PI * (double)j / (double)n;
            double cv = std::cos(ang), sv = std::sin(ang);
            // exact values on the quarter points, as an FFT's trivial twiddles
            if (4 * j == n) { cv = 0; sv = 1; }
            else if (2 * j == n) { cv = -1; sv = 0; }
            else if (4 * j == 3 * n) { cv = 0; sv = -1; }
            c[j] = (R)cv; s[j] = (R)sv;
        }
    }
};

// computeC2R: r_k = Re c_0 + 2 sum_{a>=1} Re(c_a e^{i a phi_k}) (Nyquist doubled)
template <class R>
void c2r(const Cx<R> *c, int nu, R *r, int nr, const Twiddle<R> &tw) {
    for (int k = 0; k < nr; k++) {
        R acc = c[0].real();
        int j = 0;
        for (int a = 1; a < nu; a++) {
            j += k; if (j >= nr) j -= nr;
            acc += (R)2 * (c[a].real() * tw.c[j] - c[a].imag() * tw.s[j]);
        }
        r[k] = acc;
    }
}
// computeR2C: c_a = (1/nr) sum_k r_k e^{-i a phi_k}, Nyquist halved
template <class R>
void r2c(const R *r, int nr, Cx<R> *c, int nu, const Twiddle<R> &tw) {
    R inv = (R)(1.0 / nr);
    for (int a = 0; a < nu; a++) {
        R re = 0, im = 0;
        int j = 0;
        for (int k = 0; k < nr; k++) {
            R x = r[k] * inv;
            re += x * tw.c[j];
            im -= x * tw.s[j];
            j += a; if (j >= nr) j -= nr;
        }
        if (a == 0) im = 0;
        if (nr % 2 == 0 && a == nr / 2) { re *= (R)0.5; im = 0; }
        c[a] = Cx<R>(re, im);
    }
}

// ---------------------------------------------------------------------------
// model storage
// ---------------------------------------------------------------------------
template <class R>
struct PointSet {
    int n = 0, ndim = 3;
    std::vector<int> nr, nu, off;
    std::vector<int> mass_nr;
    std::vector<std::vector<R>> inv_mass;    // 1 or nr values
    std::vector<double> mass1;               // 1-D mass (double), for MassOceanLoad1D
    std::vector<int> ocean;                  // index into ocean_c, -1 = none
    std::vector<std::array<R, 4>> ocean_c;   // (ss, zz, sz, pp)
    std::vector<int> ocean3;                 // index into ocean3_c, -1 = none
    std::vector<std::vector<R>> ocean3_c;    // [nr][4]: 1/m, k_s, k_phi, k_z
    std::vector<std::vector<double>> mass3;  // the point's masses per slice (or one)
    std::vector<uint8_t> axial, surface;
    std::vector<Cx<R>> stiff, displ, veloc, accel;
    size_t total = 0;
    void build(int count, const int32_t *nr_, const int32_t *mnr, const int64_t *moff,
               const double *mass, const uint8_t *ax, const uint8_t *surf, int nd) {
        n = count; ndim = nd;
        nr.assign(nr_, nr_ + n); nu.resize(n); off.resize(n);
        mass_nr.resize(n); inv_mass.resize(n); mass1.assign(n, 0.0); ocean.assign(n, -1); ocean_c.clear();
        ocean3.assign(n, -1); ocean3_c.clear(); mass3.assign(n, {});
        axial.assign(n, 0); surface.assign(n, 0);
        size_t o = 0;
        for (int p = 0; p < n; p++) {
            nu[p] = nr[p] / 2 + 1; off[p] = (int)o; o += nu[p];
            mass_nr[p] = mnr ? mnr[p] : 1;
            int64_t mo = moff ? moff[p] : p;
            inv_mass[p].resize(mass_nr[p]);
            // Mass1D / Mass3D store (Real)(1 / mass)  (Mass1D.hpp:19-21, Mass3D.hpp:19-20)
            for (int k = 0; k < mass_nr[p]; k++) inv_mass[p][k] = (R)(1.0 / mass[mo + k]);
            mass1[p] = mass[mo];
            mass3[p].assign(mass + mo, mass + mo + mass_nr[p]);
            if (ax) axial[p] = ax[p];
            if (surf) surface[p] = surf[p];
        }
        total = o;
        stiff.assign(total * ndim, Cx<R>(0));
        displ = veloc = accel = stiff;
    }
};

template <class R>
struct SolidElem {
    int nr, nu;
    int pts[N];
    Ops<R> ops;
    int rheo, is3d, att, rtz;
    int nslice;
    std::vector<R> mod;            // [nmod][nslice][25]
    std::vector<R> mod2;           // derived: 2 mu (ISO) or -2 N (TI), [nslice][25]
    std::vector<R> dlam, dmu, dmu2;// [nslice][npa]
    // attenuation state
    std::vector<Cx<R>> dstressF;   // [nu][6][npa]
    std::vector<Cx<R>> memF;       // [nsls][nu][6][npa]
    std::vector<R> dstressC;       // [nr][6][npa]
    std::vector<R> memC;           // [nsls][nr][6][npa]
    R sin1[N], cos1[N], sin2[N], cos2[N];
    // PRT: X0..X3 then X0|J|..X3|J|, [8][xns][25]
    int prt = 0, prt3 = 0;
    std::vector<R> X;
};

template <class R>
struct FluidElem {
    int nr, nu;
    int pts[N];
    Ops<R> ops;
    int is3d, nslice;
    std::vector<R> K;              // [nslice][25]
    // PRT: X0..X3 then X0|J|..X3|J| [8][xns][25]; RTZ frame sin / cos of theta
    int prt = 0, prt3 = 0, rtz = 0;
    std::vector<R> X;
    R sin1[N], cos1[N];
};

template <class R>
struct MomentSrc {
    int elem, nu;
    std::vector<Cx<R>> pattern;    // [nu][6][25]
    axg_stf stf;
};
template <class R>
struct ForceSrc {
    int elem, nu;
    std::vector<Cx<R>> pattern;    // [nu][3][25]
    axg_stf stf;
};

template <class R>
struct PressureSrc {
    int elem, nu;
    std::vector<Cx<R>> pattern;    // [nu][25]
    axg_stf stf;
};

struct Station {
    int elem;
    double w[N];
    double phi;
};

// GaussianSTF::getValue (GaussianSTF.hpp:35-58), double then cast to Real
double stf_value(const axg_stf &s, double time) {
    const double invSqrtPi = 1. / std::sqrt(M_PI);
    const double f = s.decay_factor / s.half_duration;
    double t = time - s.time_shift;
    double ft = f * t;
    switch (s.derivative_order) {
        case -1: return std::erf(ft) * 0.5 + 0.5;
        case 0: return invSqrtPi * f * std::exp(-ft * ft);
        case 1: return invSqrtPi * std::pow(f, 3) * std::exp(-ft * ft) * (-2. * t);
        case 2: return invSqrtPi * std::pow(f, 3) * std::exp(-ft * ft) * (4. * ft * ft - 2.);
    }
    throw std::runtime_error("GaussianSTF::getValue || Unsupported derivative order.");
}

// StreamSTF::getValue (StreamSTF.cpp:63-93) / NetCDF_STF::getValue (NetCDF_STF.cpp:92-140),
// vector_tools::linearInterpSorted (vector_tools.hpp:23-66): samples in Real, combined in
// double
struct StfTable {
    std::vector<double> t, v;
    int padding = 0, pad_first = 0;
    double left = 0, right = 0;
};
template <class R>
R stf_table_value(const StfTable &tb, double time) {
    const size_t n = tb.t.size();
    if (tb.pad_first && tb.padding) {
        if (time < tb.t.front()) return (R)tb.left;
        if (time > tb.t.back()) return (R)tb.right;
    }
    const double tol = (tb.t.back() - tb.t.front()) * 1e-12;
    if (time < tb.t.front() - tol || time > tb.t.back() + tol) {
        if (!tb.padding) throw std::runtime_error("StreamSTF::getValue || Time is out of range with padding disabled.");
        return (R)(time < tb.t.front() ? tb.left : tb.right);
    }
    size_t i1 = (size_t)(std::upper_bound(tb.t.begin(), tb.t.end(), time) - tb.t.begin());
    if (i1 == 0) i1++;
    else if (i1 == n) i1--;
    const size_t i0 = i1 - 1;
    const double f1 = (time - tb.t[i0]) / (tb.t[i1] - tb.t[i0]), f0 = 1. - f1;
    return (R)(f0 * (double)(R)tb.v[i0] + f1 * (double)(R)tb.v[i1]);
}

int nmod_of(int rheo) { return rheo == AXG_ISO ? 2 : (rheo == AXG_TISO ? 5 : 21); }

// ---------------------------------------------------------------------------
// the oracle solver
// ---------------------------------------------------------------------------
struct OracleBase {
    virtual ~OracleBase() = default;
    std::string err;
    virtual void set_solid_points(const axg_solid_points *) = 0;
    virtual void set_fluid_points(const axg_fluid_points *) = 0;
    virtual void set_solid_elements(const axg_solid_elements *) = 0;
    virtual void set_fluid_elements(const axg_fluid_elements *) = 0;
    virtual void set_solid_fluid(const axg_solid_fluid *) = 0;
    virtual void set_moment_sources(const axg_moment_sources *) = 0;
    virtual void set_force_sources(const axg_force_sources *) = 0;
    virtual void set_pressure_sources(const axg_pressure_sources *) = 0;
    virtual void set_solid_fluid3d(int n, const int *sp_, const int *fp_, const int64_t *off, const double *nu3,
                                   const double *na3, const double *mf) = 0;
    virtual void set_stf_table(int kind, int index, int n, const double *t, const double *v, int padding,
                               double left, double right, int pad_first) = 0;
    virtual void set_stations(const axg_stations *, int) = 0;
    virtual void set_clayton(int solid, const axg_clayton *) = 0;
    virtual void set_sponge(int solid, int n, const int32_t *pt, const double *g) = 0;
    virtual void set_ocean_load(int n, const int32_t *pt, const double *mo, const double *theta) = 0;
    virtual void set_ocean_load3d(int n, const int32_t *pt, const int64_t *off, const double *mo,
                                  const double *normal) = 0;
    virtual void set_clayton3d(int solid, const axg_clayton3d *c) = 0;
    virtual void set_scanning(const axg_scanning *s) = 0;
    virtual void set_prt_fluid(int n, const int32_t *elem, const int64_t *off, const uint8_t *x3d, const double *x,
                               const double *theta) = 0;
    virtual void set_prt(int n, const int32_t *elem, const int64_t *off, const uint8_t *x3d, const double *x) = 0;
    virtual void scanning_nr(int32_t *s, int32_t *f) = 0;
    virtual void set_sponge3d(int solid, int n, const int32_t *pt, const int64_t *off, const double *g) = 0;
    virtual void apply_sources(int tstep) = 0;
    virtual void compute_stiffness(int nthreads) = 0;
    // the elements of one part only (part 0 / 1 per element from set_element_parts): the
    // order of a rank that hides its exchange behind the elements off the shared points
    virtual void compute_stiffness_part(int nthreads, int part) = 0;
    void set_element_parts(const uint8_t *s, int ns, const uint8_t *f, int nf) {
        se_part.assign(s ? s : nullptr, s ? s + ns : nullptr);
        fe_part.assign(f ? f : nullptr, f ? f + nf : nullptr);
    }
    std::vector<uint8_t> se_part, fe_part;
    virtual void bc_before() = 0;
    virtual void bc_after() = 0;
    virtual void stiff_to_accel() = 0;
    virtual void newmark() = 0;
    virtual void record(int tstep) = 0;
    virtual void run(int nsteps, int nthreads) = 0;
    virtual void get_field(int solid, int which, double *out) = 0;
    virtual void set_field(int solid, int which, const double *in) = 0;
    virtual int64_t field_size(int solid) = 0;
    virtual int get_seismograms(double *out) = 0;
    virtual void reset_attenuation() = 0;
    int step = 0;
};

template <class R>
struct Oracle : OracleBase {
    axg_config cfg;
    GMat<R> gm;
    R alphaA[AXG_MAX_SLS], betaA[AXG_MAX_SLS], gammaA[AXG_MAX_SLS];
    PointSet<R> sp, fp;
    std::vector<SolidElem<R>> se;
    std::vector<FluidElem<R>> fe;
    // coupling
    struct Couple { int s, f; R nsu, nzu, nsa_m, nza_m; };
    std::vector<Couple> sf;
    std::vector<MomentSrc<R>> msrc;
    std::vector<ForceSrc<R>> fsrc;
    std::vector<PressureSrc<R>> psrc;
    // SolidFluidCoupling3D: pairs, per-slice unassembled normal and assembled normal / fluid mass
    struct Cp3 { int s, f; std::vector<R> nu3, na3; };
    std::vector<Cp3> cp3;
    void set_solid_fluid3d(int n, const int *sp_, const int *fp_, const int64_t *off, const double *nu3,
                           const double *na3, const double *mf) override {
        cp3.resize(n);
        for (int i = 0; i < n; i++) {
            Cp3 &c = cp3[i];
            c.s = sp_[i]; c.f = fp_[i];
            const int nr = sp.nr[c.s];
            prepare_twiddle(nr);
            c.nu3.resize((size_t)nr * 3); c.na3.resize((size_t)nr * 3);
            for (int k = 0; k < nr; k++)
                for (int d = 0; d < 3; d++) {
                    c.nu3[(size_t)k * 3 + d] = (R)nu3[(off[i] + k) * 3 + d];
                    c.na3[(size_t)k * 3 + d] = (R)(na3[(off[i] + k) * 3 + d] / mf[off[i] + k]);
                }
        }
    }
    // SolidFluidCoupling3D::coupleSolidToFluid / coupleFluidToSolid (SolidFluidCoupling3D.cpp:40-94)
    void couple3d() {
        for (auto &c : cp3) {
            const int nr = sp.nr[c.s], nu = nr / 2 + 1;
            const Twiddle<R> &t = twiddle(nr);
            std::vector<Cx<R>> cb(nu);
            std::vector<R> ur((size_t)3 * nr), fr(nr);
            for (int d = 0; d < 3; d++) {
                for (int a = 0; a < nu; a++) cb[a] = sp.displ[((size_t)sp.off[c.s] + a) * 3 + d];
                c2r(cb.data(), nu, &ur[(size_t)d * nr], nr, t);
            }
            for (int k = 0; k < nr; k++)
                fr[k] = c.nu3[3 * k] * ur[k] + c.nu3[3 * k + 1] * ur[nr + k] + c.nu3[3 * k + 2] * ur[2 * nr + k];
            r2c(fr.data(), nr, cb.data(), nu, t);
            Cx<R> *fs = &fp.stiff[(size_t)fp.off[c.f]];
            for (int a = 0; a < nu; a++) fs[a] += cb[a];
            for (int a = 0; a < nu; a++) cb[a] = fs[a];
            c2r(cb.data(), nu, fr.data(), nr, t);
            Cx<R> *ss = &sp.stiff[(size_t)sp.off[c.s] * 3];
            for (int d = 0; d < 3; d++) {
                for (int k = 0; k < nr; k++) ur[(size_t)d * nr + k] = fr[k] * c.na3[3 * k + d];
                r2c(&ur[(size_t)d * nr], nr, cb.data(), nu, t);
                for (int a = 0; a < nu; a++) ss[a * 3 + d] -= cb[a];
            }
        }
    }
    std::map<int, StfTable> stf_tab[3];   // moment, force, pressure sources with a table STF
    R src_stf(int kind, int i, const axg_stf &g, double t) const {
        auto it = stf_tab[kind].find(i);
        return it == stf_tab[kind].end() ? (R)stf_value(g, t) : stf_table_value<R>(it->second, t);
    }
    void set_stf_table(int kind, int index, int n, const double *t, const double *v, int padding, double left,
                       double right, int pad_first) override {
        StfTable tb;
        tb.t.assign(t, t + n);
        tb.v.assign(v, v + n);
        tb.padding = padding; tb.left = left; tb.right = right; tb.pad_first = pad_first;
        stf_tab[kind][index] = tb;
    }
    std::vector<Cx<R>> pressure;          // FluidPoint mPressureSource, per fluid point mode
    std::vector<Station> st;
    int rec_interval = 1;
    std::vector<double> seis;   // [nrec][nst][3]
    int nrec = 0;
    std::vector<Twiddle<R>> tw;  // by nr
    // absorbing boundaries
    struct ClaytonS { int p; R ss, zz, sz, pp; };
    struct ClaytonF { int p; R c; };
    std::vector<ClaytonS> cls;
    std::vector<ClaytonF> clf;
    std::vector<std::pair<int, R>> sgs, sgf;
    // 3-D Clayton (per slice: rsa, k_s, k_phi, k_z for solid points; area / rho vp for fluid)
    struct Clayton3 { int p; std::vector<R> c; };
    std::vector<Clayton3> cl3s, cl3f;
    struct Sponge3 { int p; std::vector<R> g; };
    std::vector<Sponge3> sg3s, sg3f;

    explicit Oracle(const axg_config *c) : cfg(*c) {
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                gm.G_GLL.a[i][j] = (R)gSpectral.G_GLL[i][j];
                gm.G_GLJ.a[i][j] = (R)gSpectral.G_GLJ[i][j];
                gm.GT_GLL.a[j][i] = (R)gSpectral.G_GLL[i][j];
                gm.GT_GLJ.a[j][i] = (R)gSpectral.G_GLJ[i][j];
            }
        for (int l = 0; l < cfg.nsls; l++) {
            alphaA[l] = (R)cfg.att_alpha[l];
            betaA[l] = (R)cfg.att_beta[l];
            gammaA[l] = (R)cfg.att_gamma[l];
        }
    }

    // twiddle tables are built up front (prepare_twiddles) so that the worker
    // threads of compute_stiffness only read them
    const Twiddle<R> &twiddle(int nr) const {
        if ((int)tw.size() <= nr || tw[nr].nr != nr)
            throw std::runtime_error("Oracle::twiddle || table for nr not prepared.");
        return tw[nr];
    }
    void prepare_twiddle(int nr) {
        if ((int)tw.size() <= nr) tw.resize(nr + 1);
        if (tw[nr].nr != nr) tw[nr].set(nr);
    }

    static void make_ops(const double *g, bool axial, Ops<R> &o) {
        // GradientQuadrature constructor (GradientQuadrature.hpp:122-137):
        // plain operators cast to Real; _IF products formed in double, then cast
        const double *dsdxii = g, *dsdeta = g + 25, *dzdxii = g + 50, *dzdeta = g + 75,
                     *invs = g + 100, *ifact = g + 125;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                int q = i * P + j;
                o.dsdxii.a[i][j] = (R)dsdxii[q];
                o.dsdeta.a[i][j] = (R)dsdeta[q];
                o.dzdxii.a[i][j] = (R)dzdxii[q];
                o.dzdeta.a[i][j] = (R)dzdeta[q];
                o.inv_s.a[i][j] = (R)invs[q];
                o.dsdxii_if.a[i][j] = (R)(dsdxii[q] * ifact[q]);
                o.dsdeta_if.a[i][j] = (R)(dsdeta[q] * ifact[q]);
                o.dzdxii_if.a[i][j] = (R)(dzdxii[q] * ifact[q]);
                o.dzdeta_if.a[i][j] = (R)(dzdeta[q] * ifact[q]);
                o.inv_s_if.a[i][j] = (R)(invs[q] * ifact[q]);
            }
        o.axial = axial;
    }

    void set_solid_points(const axg_solid_points *p) override {
        sp.build(p->count, p->nr, p->mass_nr, p->mass_offset, p->mass, p->axial, nullptr, 3);
        for (int q = 0; q < sp.n; q++)
            if (sp.mass_nr[q] > 1) prepare_twiddle(sp.nr[q]);
    }
    void set_fluid_points(const axg_fluid_points *p) override {
        fp.build(p->count, p->nr, p->mass_nr, p->mass_offset, p->mass, p->axial, p->surface, 1);
        for (int q = 0; q < fp.n; q++)
            if (fp.mass_nr[q] > 1) prepare_twiddle(fp.nr[q]);
    }

    void set_solid_elements(const axg_solid_elements *e) override {
        se.resize(e->count);
        for (int i = 0; i < e->count; i++) {
            SolidElem<R> &el = se[i];
            el.nr = e->nr[i]; el.nu = el.nr / 2 + 1;
            for (int q = 0; q < N; q++) el.pts[q] = e->points[(size_t)i * N + q];
            make_ops(e->geometry + (size_t)i * 150, e->axial[i] != 0, el.ops);
            el.rheo = e->rheology[i];
            el.is3d = e->is3d ? e->is3d[i] : 0;
            el.att = e->attenuation ? e->attenuation[i] : AXG_ATT_NONE;
            el.rtz = e->rtz ? e->rtz[i] : 0;
            el.nslice = el.is3d ? el.nr : 1;
            if (el.is3d) prepare_twiddle(el.nr);
            int nm = nmod_of(el.rheo);
            size_t cnt = (size_t)nm * el.nslice * N;
            el.mod.resize(cnt);
            const double *m = e->moduli + e->mat_offset[i];
            for (size_t q = 0; q < cnt; q++) el.mod[q] = (R)m[q];
            // derived 2 mu (Isotropic.hpp:34) / -2 N (TransverselyIsotropic.hpp:37),
            // formed in double then cast
            if (el.rheo == AXG_ISO) {
                el.mod2.resize((size_t)el.nslice * N);
                for (size_t q = 0; q < el.mod2.size(); q++)
                    el.mod2[q] = (R)(m[(size_t)1 * el.nslice * N + q] * 2.);
            } else if (el.rheo == AXG_TISO) {
                el.mod2.resize((size_t)el.nslice * N);
                for (size_t q = 0; q < el.mod2.size(); q++)
                    el.mod2[q] = (R)(m[(size_t)4 * el.nslice * N + q] * (-2.));
            }
            if (el.rtz) {
                // CoordTransformSpherical constructor (CoordTransformSpherical.hpp:43-48)
                for (int q = 0; q < N; q++) {
                    double t = e->theta[(size_t)i * N + q];
                    el.sin1[q] = (R)std::sin(t); el.cos1[q] = (R)std::cos(t);
                    el.sin2[q] = (R)std::sin(2. * t); el.cos2[q] = (R)std::cos(2. * t);
                }
            }
            if (el.att != AXG_ATT_NONE) {
                int npa = el.att == AXG_ATT_FULL ? N : 4;
                size_t na = (size_t)el.nslice * npa;
                const double *a = e->att_moduli + e->att_offset[i];
                el.dlam.resize(na); el.dmu.resize(na); el.dmu2.resize(na);
                for (size_t q = 0; q < na; q++) {
                    el.dlam[q] = (R)a[q];
                    el.dmu[q] = (R)a[na + q];
                    el.dmu2[q] = (R)(a[na + q] * 2.);
                }
                int ns = cfg.nsls;
                if (!el.is3d) {
                    el.dstressF.assign((size_t)el.nu * 6 * npa, Cx<R>(0));
                    el.memF.assign((size_t)ns * el.nu * 6 * npa, Cx<R>(0));
                } else {
                    el.dstressC.assign((size_t)el.nr * 6 * npa, 0);
                    el.memC.assign((size_t)ns * el.nr * 6 * npa, 0);
                }
            }
        }
    }

    void reset_attenuation() override {
        for (auto &el : se) {
            std::fill(el.dstressF.begin(), el.dstressF.end(), Cx<R>(0));
            std::fill(el.memF.begin(), el.memF.end(), Cx<R>(0));
            std::fill(el.dstressC.begin(), el.dstressC.end(), R(0));
            std::fill(el.memC.begin(), el.memC.end(), R(0));
        }
    }

    void set_fluid_elements(const axg_fluid_elements *e) override {
        fe.resize(e->count);
        for (int i = 0; i < e->count; i++) {
            FluidElem<R> &el = fe[i];
            el.nr = e->nr[i]; el.nu = el.nr / 2 + 1;
            for (int q = 0; q < N; q++) el.pts[q] = e->points[(size_t)i * N + q];
            make_ops(e->geometry + (size_t)i * 150, e->axial[i] != 0, el.ops);
            el.is3d = e->is3d ? e->is3d[i] : 0;
            el.nslice = el.is3d ? el.nr : 1;
            if (el.is3d) prepare_twiddle(el.nr);
            el.K.resize((size_t)el.nslice * N);
            const double *m = e->moduli + e->mat_offset[i];
            for (size_t q = 0; q < el.K.size(); q++) el.K[q] = (R)m[q];
        }
    }

    void set_solid_fluid(const axg_solid_fluid *c) override {
        sf.resize(c->count);
        for (int i = 0; i < c->count; i++) {
            // SolidFluidCoupling1D constructor: normals cast to Real, assembled
            // normals divided by the fluid mass in double
            sf[i].s = c->solid_point[i]; sf[i].f = c->fluid_point[i];
            sf[i].nsu = (R)c->ns_unassembled[i];
            sf[i].nzu = (R)c->nz_unassembled[i];
            sf[i].nsa_m = (R)(c->ns_assembled[i] / c->mass_fluid[i]);
            sf[i].nza_m = (R)(c->nz_assembled[i] / c->mass_fluid[i]);
        }
    }

    void set_moment_sources(const axg_moment_sources *s) override {
        msrc.resize(s->count);
        for (int i = 0; i < s->count; i++) {
            msrc[i].elem = s->element[i]; msrc[i].nu = s->nu[i];
            msrc[i].pattern.resize((size_t)msrc[i].nu * 6 * N);
            const double *pp = s->pattern + 2 * s->pattern_offset[i];
            for (size_t q = 0; q < msrc[i].pattern.size(); q++)
                msrc[i].pattern[q] = Cx<R>((R)pp[2 * q], (R)pp[2 * q + 1]);
            msrc[i].stf = s->stf[i];
        }
    }
    void set_force_sources(const axg_force_sources *s) override {
        fsrc.resize(s->count);
        for (int i = 0; i < s->count; i++) {
            fsrc[i].elem = s->element[i]; fsrc[i].nu = s->nu[i];
            fsrc[i].pattern.resize((size_t)fsrc[i].nu * 3 * N);
            const double *pp = s->pattern + 2 * s->pattern_offset[i];
            for (size_t q = 0; q < fsrc[i].pattern.size(); q++)
                fsrc[i].pattern[q] = Cx<R>((R)pp[2 * q], (R)pp[2 * q + 1]);
            fsrc[i].stf = s->stf[i];
        }
    }
    void set_pressure_sources(const axg_pressure_sources *s) override {
        psrc.resize(s->count);
        for (int i = 0; i < s->count; i++) {
            psrc[i].elem = s->element[i]; psrc[i].nu = s->nu[i];
            psrc[i].pattern.resize((size_t)psrc[i].nu * N);
            const double *pp = s->pattern + 2 * s->pattern_offset[i];
            for (size_t q = 0; q < psrc[i].pattern.size(); q++)
                psrc[i].pattern[q] = Cx<R>((R)pp[2 * q], (R)pp[2 * q + 1]);
            psrc[i].stf = s->stf[i];
        }
    }
    void set_stations(const axg_stations *s, int interval) override {
        st.resize(s->count);
        for (int i = 0; i < s->count; i++) {
            st[i].elem = s->element[i];
            for (int q = 0; q < N; q++) st[i].w[q] = s->weights[(size_t)i * N + q];
            st[i].phi = s->phi[i];
        }
        rec_interval = interval > 0 ? interval : 1;
    }

    // ClaytonSolid1D / ClaytonFluid1D constructors (coefficients in double, cast)
    void set_clayton(int solid, const axg_clayton *c) override {
        for (int i = 0; i < c->count; i++) {
            if (solid) {
                double ct = std::cos(c->theta[i]), st = std::sin(c->theta[i]);
                double rsa = c->rho_vs[i] * c->area[i], rpa = c->rho_vp[i] * c->area[i];
                cls.push_back({c->point[i], (R)(rsa * ct * ct + rpa * st * st), (R)(rsa * st * st + rpa * ct * ct),
                               (R)((rpa - rsa) * ct * st), (R)rsa});
            } else {
                clf.push_back({c->point[i], (R)(c->area[i] / c->rho_vp[i])});
            }
        }
    }
    // PRT constructor (PRT.hpp): X0..X3 cast, X_k |J| formed in double then cast
    void set_prt(int n, const int32_t *elem, const int64_t *off, const uint8_t *x3d, const double *x) override {
        for (int i = 0; i < n; i++) {
            SolidElem<R> &el = se[elem[i]];
            el.prt = 1;
            el.prt3 = x3d[i];
            const size_t xs = (size_t)(el.prt3 ? el.nr : 1) * N;
            const double *xv = x + off[i];
            el.X.resize(8 * xs);
            for (int c = 0; c < 4; c++)
                for (size_t j = 0; j < xs; j++) {
                    el.X[c * xs + j] = (R)xv[c * xs + j];
                    el.X[(4 + c) * xs + j] = (R)(xv[c * xs + j] * xv[4 * xs + j]);
                }
        }
    }
    void set_prt_fluid(int n, const int32_t *elem, const int64_t *off, const uint8_t *x3d, const double *x,
                       const double *theta) override {
        for (int i = 0; i < n; i++) {
            FluidElem<R> &el = fe[elem[i]];
            el.prt = 1;
            el.prt3 = x3d[i];
            const size_t xs = (size_t)(el.prt3 ? el.nr : 1) * N;
            const double *xv = x + off[i];
            el.X.resize(8 * xs);
            for (int c = 0; c < 4; c++)
                for (size_t j = 0; j < xs; j++) {
                    el.X[c * xs + j] = (R)xv[c * xs + j];
                    el.X[(4 + c) * xs + j] = (R)(xv[c * xs + j] * xv[4 * xs + j]);
                }
            el.rtz = theta != nullptr;
            if (theta)
                for (int q = 0; q < N; q++) {
                    el.sin1[q] = (R)std::sin(theta[(size_t)i * N + q]);
                    el.cos1[q] = (R)std::cos(theta[(size_t)i * N + q]);
                }
        }
    }
    // ClaytonSolid3D / ClaytonFluid3D constructors (in double, cast); after the points
    void set_clayton3d(int solid, const axg_clayton3d *c) override {
        for (int i = 0; i < c->count; i++) {
            const int p = c->point[i];
            const int nr = solid ? sp.nr[p] : fp.nr[p];
            Clayton3 x{p, {}};
            for (int k = 0; k < nr; k++) {
                const int64_t q = c->offset[i] + k;
                if (solid) {
                    const double sk = std::sqrt((c->rho_vp[q] - c->rho_vs[q]) * c->area[q]);
                    x.c.push_back((R)(c->rho_vs[q] * c->area[q]));
                    for (int d = 0; d < 3; d++) x.c.push_back((R)(sk * c->normal[q * 3 + d]));
                } else {
                    x.c.push_back((R)(c->area[q] / c->rho_vp[q]));
                }
            }
            prepare_twiddle(nr);
            (solid ? cl3s : cl3f).push_back(std::move(x));
        }
    }
    // Sponge 3-D constructor: gamma cast to Real
    void set_sponge3d(int solid, int n, const int32_t *pt, const int64_t *off, const double *g) override {
        for (int i = 0; i < n; i++) {
            const int nr = solid ? sp.nr[pt[i]] : fp.nr[pt[i]];
            Sponge3 x{pt[i], {}};
            for (int k = 0; k < nr; k++) x.g.push_back((R)g[off[i] + k]);
            prepare_twiddle(nr);
            (solid ? sg3s : sg3f).push_back(std::move(x));
        }
    }
    // MassOceanLoad3D constructor (MassOceanLoad3D.cpp: in double, cast); after set_solid_points
    void set_ocean_load3d(int n, const int32_t *pt, const int64_t *off, const double *mo,
                          const double *normal) override {
        for (int i = 0; i < n; i++) {
            const int p = pt[i], nr = sp.nr[p];
            std::vector<R> c;
            for (int k = 0; k < nr; k++) {
                const double mass = sp.mass3[p][sp.mass_nr[p] > 1 ? k : 0];
                const double m0 = mo[off[i] + k];
                const double sk = std::sqrt(m0 / (mass * (mass + m0)));
                c.push_back((R)(1.0 / mass));
                for (int d = 0; d < 3; d++) c.push_back((R)(sk * normal[(off[i] + k) * 3 + d]));
            }
            sp.ocean3[p] = (int)sp.ocean3_c.size();
            sp.ocean3_c.push_back(std::move(c));
            prepare_twiddle(nr);
        }
    }
    // MassOceanLoad1D constructor (coefficients in double, cast); after set_solid_points
    void set_ocean_load(int n, const int32_t *pt, const double *mo, const double *theta) override {
        for (int i = 0; i < n; i++) {
            const int p = pt[i];
            const double mass = sp.mass1[p], mv = mass + mo[i];
            const double ct = std::cos(theta[i]), st = std::sin(theta[i]);
            sp.ocean[p] = (int)sp.ocean_c.size();
            sp.ocean_c.push_back({(R)(1. / mass * ct * ct + 1. / mv * st * st),
                                  (R)(1. / mass * st * st + 1. / mv * ct * ct),
                                  (R)((1. / mv - 1. / mass) * ct * st), (R)(1 / mass)});
        }
    }
    void set_sponge(int solid, int n, const int32_t *pt, const double *g) override {
        for (int i = 0; i < n; i++) (solid ? sgs : sgf).push_back({pt[i], (R)g[i]});
    }

    // ------------------------------ sources ------------------------------
    double time_of(int tstep) const {
        // t accumulated as in NewmarkTimeScheme::solve (t += mDt)
        double t = cfg.t0;
        for (int i = 0; i < tstep; i++) t += cfg.dt;
        return t;
    }
    void apply_sources(int tstep) override {
        double t = time_of(tstep);
        // FluidPressure::apply -> FluidElement::addPressureSource -> FluidPoint::
        // addPressureSource (FluidPoint.hpp:113-119): kept until computeStiffToAccel
        if (!psrc.empty() && pressure.size() != fp.total) pressure.assign(fp.total, Cx<R>(0, 0));
        for (size_t si = 0; si < psrc.size(); si++) {
            auto &s = psrc[si];
            FluidElem<R> &el = fe[s.elem];
            R v = src_stf(2, (int)si, s.stf, t);
            for (int q = 0; q < N; q++) {
                int p = el.pts[q];
                int numin = std::min(fp.nu[p], s.nu);
                for (int a = 0; a < numin; a++) pressure[(size_t)fp.off[p] + a] += s.pattern[(size_t)a * N + q] * v;
            }
        }
        // SolidMoment::apply -> SolidElement::addMomentSource (SolidElement.cpp:273-356)
        for (size_t si = 0; si < msrc.size(); si++) {
            auto &s = msrc[si];
            SolidElem<R> &el = se[s.elem];
            R v = src_stf(0, (int)si, s.stf, t);
            int nu_co = std::min(el.nu, s.nu);
            std::vector<CM<R>> stress(6);
            Grad<R> g{el.ops, gm};
            for (int a = 0; a < nu_co; a++) {
                CM<R> sig[6], f[3];
                for (int d = 0; d < 6; d++)
                    for (int q = 0; q < N; q++)
                        sig[d].a[q / P][q % P] = -(s.pattern[((size_t)a * 6 + d) * N + q] * v);
                g.quad6(sig, f, a, false);
                for (int q = 0; q < N; q++) {
                    int p = el.pts[q];
                    if (a < sp.nu[p])
                        for (int c = 0; c < 3; c++)
                            sp.stiff[((size_t)sp.off[p] + a) * 3 + c] -= f[c].a[q / P][q % P];
                }
            }
        }
        // SolidForce::apply -> SolidPoint::addForceSource (SolidPoint.hpp:112-119)
        for (size_t si = 0; si < fsrc.size(); si++) {
            auto &s = fsrc[si];
            SolidElem<R> &el = se[s.elem];
            R v = src_stf(1, (int)si, s.stf, t);
            for (int q = 0; q < N; q++) {
                int p = el.pts[q];
                int numin = std::min(sp.nu[p], s.nu);
                for (int a = 0; a < numin; a++)
                    for (int c = 0; c < 3; c++)
                        sp.stiff[((size_t)sp.off[p] + a) * 3 + c] +=
                            s.pattern[((size_t)a * 3 + c) * N + q] * v;
            }
        }
    }

    // ------------------------------ rheology ------------------------------
    // Isotropic::strainToStress (Isotropic.hpp:154-170) on one point
    template <class T>
    static void iso(const T e[6], T s[6], R lam, R mu, R mu2) {
        T sii = (e[0] + e[1] + e[2]) * lam;
        s[0] = sii + e[0] * mu2;
        s[1] = sii + e[1] * mu2;
        s[2] = sii + e[2] * mu2;
        s[3] = e[3] * mu; s[4] = e[4] * mu; s[5] = e[5] * mu;
    }
    // TransverselyIsotropic::strainToStress (TransverselyIsotropic.hpp:160-180)
    template <class T>
    static void tiso(const T e[6], T s[6], R A, R C, R F, R L, R Nn, R mN2) {
        T t3 = e[0] + e[1];
        T t4 = t3 * A + e[2] * F;
        s[0] = t4 + e[1] * mN2;
        s[1] = t4 + e[0] * mN2;
        s[2] = t3 * F + e[2] * C;
        s[3] = e[3] * L; s[4] = e[4] * L; s[5] = e[5] * Nn;
    }
    // Anisotropic::strainToStress (Anisotropic.hpp:202-274)
    template <class T>
    static void aniso(const T e[6], T s[6], const R c[21]) {
        static const int idx[6][6] = {{0, 1, 2, 3, 4, 5}, {1, 6, 7, 8, 9, 10},
                                      {2, 7, 11, 12, 13, 14}, {3, 8, 12, 15, 16, 17},
                                      {4, 9, 13, 16, 18, 19}, {5, 10, 14, 17, 19, 20}};
        for (int i = 0; i < 6; i++) {
            T acc = e[0] * c[idx[i][0]];
            for (int j = 1; j < 6; j++) acc = acc + e[j] * c[idx[i][j]];
            s[i] = acc;
        }
    }

    template <class T>
    void elastic(const SolidElem<R> &el, int slice, int q, const T e[6], T s[6]) const {
        size_t ns = (size_t)el.nslice * N, o = (size_t)slice * N + q;
        if (el.rheo == AXG_ISO) {
            iso(e, s, el.mod[o], el.mod[ns + o], el.mod2[o]);
        } else if (el.rheo == AXG_TISO) {
            tiso(e, s, el.mod[o], el.mod[ns + o], el.mod[2 * ns + o], el.mod[3 * ns + o],
                 el.mod[4 * ns + o], el.mod2[o]);
        } else {
            R c[21];
            for (int k = 0; k < 21; k++) c[k] = el.mod[k * ns + o];
            aniso(e, s, c);
        }
    }

    // AttenuationFull::apply / AttenuationCG4::apply on one point of one mode or slice
    // (AttenuationFull.hpp:189-207, AttenuationCG4.hpp:309-330, Attenuation.hpp:92-134)
    template <class T>
    void attenuate(const T e[6], T s[6], T *dst, T *mem, size_t memStride, R dl, R dm,
                   R dm2) const {
        int ns = cfg.nsls;
        for (int l = 0; l < ns; l++)
            for (int d = 0; d < 6; d++) s[d] -= mem[l * memStride + d];
        for (int l = 0; l < ns; l++)
            for (int d = 0; d < 6; d++)
                mem[l * memStride + d] = alphaA[l] * mem[l * memStride + d] + betaA[l] * dst[d];
        T nd[6];
        iso(e, nd, dl, dm, dm2);
        for (int d = 0; d < 6; d++) dst[d] = nd[d];
        for (int l = 0; l < ns; l++)
            for (int d = 0; d < 6; d++) mem[l * memStride + d] += gammaA[l] * dst[d];
    }

    // CoordTransformSpherical::transformSPZ_RTZ6 / transformRTZ_SPZ6
    // (CoordTransformSpherical.hpp:186-255) on one point of one mode
    static void spz_rtz6(Cx<R> e[6], R s1, R c1, R s2, R c2) {
        const R half = (R).5;
        Cx<R> s02 = e[0] + e[2], d02 = e[0] - e[2];
        e[0] = (s02 + d02 * c2 - e[4] * s2) * half;
        e[2] = s02 - e[0];
        e[4] = e[4] * c2 + d02 * s2;
        Cx<R> t3 = e[3];
        e[3] = t3 * c1 + e[5] * s1;
        e[5] = e[5] * c1 - t3 * s1;
    }
    static void rtz_spz6(Cx<R> s[6], R s1, R c1, R s2, R c2) {
        const R half = (R).5;
        Cx<R> s02 = s[0] + s[2], d02 = s[0] - s[2];
        s[0] = (s02 + d02 * c2) * half + s[4] * s2;
        s[2] = s02 - s[0];
        s[4] = s[4] * c2 - d02 * s2 * half;
        Cx<R> t3 = s[3];
        s[3] = t3 * c1 - s[5] * s1;
        s[5] = s[5] * c1 + t3 * s1;
    }

    // PRT::sphericalToUndulated6 / undulatedToSpherical6 (PRT/PRT.hpp)
    template <class V>
    static void sph2und(const V g[9], V u[6], R X0, R X1, R X2, R X3) {
        u[0] = g[0] * X0 + g[2] * X1;
        u[1] = g[4] * X0 + g[5] * X2;
        u[2] = g[8] * X3;
        u[3] = g[7] * X0 + g[8] * X2 + g[5] * X3;
        u[4] = g[6] * X0 + g[8] * X1 + g[2] * X3;
        u[5] = (g[3] + g[1]) * X0 + g[5] * X1 + g[2] * X2;
    }
    template <class V>
    static void und2sph(const V u[6], V g[9], R X0, R X1, R X2, R X3) {
        g[0] = u[0] * X0;
        g[1] = u[5] * X0;
        g[2] = u[0] * X1 + u[4] * X3 + u[5] * X2;
        g[3] = g[1];
        g[4] = u[1] * X0;
        g[5] = u[1] * X2 + u[3] * X3 + u[5] * X1;
        g[6] = u[4] * X0;
        g[7] = u[3] * X0;
        g[8] = u[2] * X3 + u[3] * X2 + u[4] * X1;
    }
    // CoordTransformSpherical::transformSPZ_RTZ9 / transformRTZ_SPZ9 (CoordTransformSpherical.hpp:102-183)
    static void rtz9(Cx<R> n[9], R s1, R c1, R s2, R c2, bool to_rtz) {
        const R half = (R).5;
        const Cx<R> s08 = n[0] + n[8], d08 = n[0] - n[8], s26 = n[2] + n[6], d26 = n[2] - n[6];
        if (to_rtz) {
            n[0] = (s08 + d08 * c2 - s26 * s2) * half;
            n[2] = (d26 + s26 * c2 + d08 * s2) * half;
        } else {
            n[0] = (s08 + d08 * c2 + s26 * s2) * half;
            n[2] = (d26 + s26 * c2 - d08 * s2) * half;
        }
        n[6] = n[2] - d26;
        n[8] = s08 - n[0];
        const Cx<R> t1 = n[1], t3 = n[3];
        if (to_rtz) {
            n[1] = t1 * c1 - n[7] * s1;
            n[7] = n[7] * c1 + t1 * s1;
            n[3] = t3 * c1 - n[5] * s1;
            n[5] = n[5] * c1 + t3 * s1;
        } else {
            n[1] = t1 * c1 + n[7] * s1;
            n[7] = n[7] * c1 - t1 * s1;
            n[3] = t3 * c1 + n[5] * s1;
            n[5] = n[5] * c1 - t3 * s1;
        }
    }
    // attenuation of one (point, mode) (complex V) or (point, slice) (real V) of an element's
    // state, the same steps as solid_element's
    template <class V>
    void att_at(SolidElem<R> &el, int a_or_k, int q, const V e[6], V s[6]) {
        static const int cg4pt[4] = {6, 8, 16, 18};
        const int npa = el.att == AXG_ATT_CG4 ? 4 : N;
        int kk = q;
        if (el.att == AXG_ATT_CG4) {
            kk = -1;
            for (int j = 0; j < 4; j++)
                if (cg4pt[j] == q) kk = j;
            if (kk < 0) return;
        }
        V dst[6], mem[AXG_MAX_SLS * 6];
        if constexpr (std::is_same<V, Cx<R>>::value) {
            const size_t memStride = (size_t)el.nu * 6 * npa;
            for (int d = 0; d < 6; d++) {
                dst[d] = el.dstressF[((size_t)a_or_k * 6 + d) * npa + kk];
                for (int l = 0; l < cfg.nsls; l++) mem[l * 6 + d] = el.memF[l * memStride + ((size_t)a_or_k * 6 + d) * npa + kk];
            }
            attenuate(e, s, dst, mem, 6, el.dlam[kk], el.dmu[kk], el.dmu2[kk]);
            for (int d = 0; d < 6; d++) {
                el.dstressF[((size_t)a_or_k * 6 + d) * npa + kk] = dst[d];
                for (int l = 0; l < cfg.nsls; l++) el.memF[l * memStride + ((size_t)a_or_k * 6 + d) * npa + kk] = mem[l * 6 + d];
            }
        } else {
            const size_t memStride = (size_t)el.nr * 6 * npa;
            for (int d = 0; d < 6; d++) {
                dst[d] = el.dstressC[((size_t)a_or_k * 6 + d) * npa + kk];
                for (int l = 0; l < cfg.nsls; l++) mem[l * 6 + d] = el.memC[l * memStride + ((size_t)a_or_k * 6 + d) * npa + kk];
            }
            const size_t ao = (size_t)a_or_k * npa + kk;
            attenuate(e, s, dst, mem, 6, el.dlam[ao], el.dmu[ao], el.dmu2[ao]);
            for (int d = 0; d < 6; d++) {
                el.dstressC[((size_t)a_or_k * 6 + d) * npa + kk] = dst[d];
                for (int l = 0; l < cfg.nsls; l++) el.memC[l * memStride + ((size_t)a_or_k * 6 + d) * npa + kk] = mem[l * 6 + d];
            }
        }
    }
    // SolidElement::displToStiff, PRT branch (SolidElement.cpp:113-161)
    void solid_element_prt(SolidElem<R> &el, std::vector<Cx<R>> &elemStiff) {
        const int nu = el.nu, nr = el.nr;
        std::vector<CM<R>> U((size_t)nu * 3), G((size_t)nu * 9);
        for (int q = 0; q < N; q++) {
            int p = el.pts[q];
            for (int a = 0; a < nu; a++)
                for (int c = 0; c < 3; c++)
                    U[(size_t)a * 3 + c].a[q / P][q % P] =
                        a < sp.nu[p] ? sp.displ[((size_t)sp.off[p] + a) * 3 + c] : Cx<R>(0);
        }
        Grad<R> g{el.ops, gm};
        for (int a = 0; a < nu; a++) g.grad9(&U[(size_t)a * 3], &G[(size_t)a * 9], a);
        auto at = [&](int a, int d, int q) -> Cx<R> & { return G[(size_t)a * 9 + d].a[q / P][q % P]; };
        if (el.rtz)
            for (int a = 0; a < nu; a++)
                for (int q = 0; q < N; q++) {
                    Cx<R> n[9];
                    for (int d = 0; d < 9; d++) n[d] = at(a, d, q);
                    rtz9(n, el.sin1[q], el.cos1[q], el.sin2[q], el.cos2[q], true);
                    for (int d = 0; d < 9; d++) at(a, d, q) = n[d];
                }
        const int xns = el.prt3 ? nr : 1;
        const size_t xs = (size_t)xns * N;
        auto X = [&](int c, int k, int q) { return el.X[c * xs + (size_t)k * N + q]; };
        if (!el.is3d) {
            for (int a = 0; a < nu; a++)
                for (int q = 0; q < N; q++) {
                    Cx<R> n[9], eu[6], su[6];
                    for (int d = 0; d < 9; d++) n[d] = at(a, d, q);
                    sph2und(n, eu, X(0, 0, q), X(1, 0, q), X(2, 0, q), X(3, 0, q));
                    elastic(el, 0, q, eu, su);
                    if (el.att != AXG_ATT_NONE) att_at(el, a, q, eu, su);
                    und2sph(su, n, X(4, 0, q), X(5, 0, q), X(6, 0, q), X(7, 0, q));
                    for (int d = 0; d < 9; d++) at(a, d, q) = n[d];
                }
        } else {
            const Twiddle<R> &t = twiddle(nr);
            std::vector<R> gc((size_t)nr * 9 * N);
            std::vector<Cx<R>> cbuf(nu);
            std::vector<R> rbuf(nr);
            for (int d = 0; d < 9; d++)
                for (int q = 0; q < N; q++) {
                    for (int a = 0; a < nu; a++) cbuf[a] = at(a, d, q);
                    c2r(cbuf.data(), nu, rbuf.data(), nr, t);
                    for (int k = 0; k < nr; k++) gc[((size_t)k * 9 + d) * N + q] = rbuf[k];
                }
            for (int k = 0; k < nr; k++)
                for (int q = 0; q < N; q++) {
                    R n[9], eu[6], su[6];
                    for (int d = 0; d < 9; d++) n[d] = gc[((size_t)k * 9 + d) * N + q];
                    const int kx = el.prt3 ? k : 0;
                    sph2und(n, eu, X(0, kx, q), X(1, kx, q), X(2, kx, q), X(3, kx, q));
                    elastic(el, k, q, eu, su);
                    if (el.att != AXG_ATT_NONE) att_at(el, k, q, eu, su);
                    und2sph(su, n, X(4, kx, q), X(5, kx, q), X(6, kx, q), X(7, kx, q));
                    for (int d = 0; d < 9; d++) gc[((size_t)k * 9 + d) * N + q] = n[d];
                }
            for (int d = 0; d < 9; d++)
                for (int q = 0; q < N; q++) {
                    for (int k = 0; k < nr; k++) rbuf[k] = gc[((size_t)k * 9 + d) * N + q];
                    r2c(rbuf.data(), nr, cbuf.data(), nu, t);
                    for (int a = 0; a < nu; a++) at(a, d, q) = cbuf[a];
                }
        }
        if (el.rtz)
            for (int a = 0; a < nu; a++)
                for (int q = 0; q < N; q++) {
                    Cx<R> n[9];
                    for (int d = 0; d < 9; d++) n[d] = at(a, d, q);
                    rtz9(n, el.sin1[q], el.cos1[q], el.sin2[q], el.cos2[q], false);
                    for (int d = 0; d < 9; d++) at(a, d, q) = n[d];
                }
        elemStiff.resize((size_t)nu * 3 * N);
        for (int a = 0; a < nu; a++) {
            CM<R> f[3];
            g.quad9(&G[(size_t)a * 9], f, a);
            for (int c = 0; c < 3; c++)
                for (int q = 0; q < N; q++) elemStiff[((size_t)a * 3 + c) * N + q] = f[c].a[q / P][q % P];
        }
    }

    // ----------------------- SolidElement::computeStiff -----------------------
    void solid_element(SolidElem<R> &el, std::vector<Cx<R>> &elemStiff,
                       std::vector<CM<R>> &S, std::vector<CM<R>> &E) {
        if (el.prt) { solid_element_prt(el, elemStiff); return; }
        int nu = el.nu, nr = el.nr;
        // collectDisplFromPoints (SolidElement.cpp:101-109, SolidPoint.hpp:82-98)
        std::vector<CM<R>> U((size_t)nu * 3);
        for (int q = 0; q < N; q++) {
            int p = el.pts[q];
            for (int a = 0; a < nu; a++)
                for (int c = 0; c < 3; c++)
                    U[(size_t)a * 3 + c].a[q / P][q % P] =
                        a < sp.nu[p] ? sp.displ[((size_t)sp.off[p] + a) * 3 + c] : Cx<R>(0);
        }
        Grad<R> g{el.ops, gm};
        E.resize((size_t)nu * 6);
        S.resize((size_t)nu * 6);
        for (int a = 0; a < nu; a++) g.grad6(&U[(size_t)a * 3], &E[(size_t)a * 6], a);
        if (el.rtz)
            for (int a = 0; a < nu; a++)
                for (int q = 0; q < N; q++) {
                    Cx<R> e[6];
                    for (int d = 0; d < 6; d++) e[d] = E[(size_t)a * 6 + d].a[q / P][q % P];
                    spz_rtz6(e, el.sin1[q], el.cos1[q], el.sin2[q], el.cos2[q]);
                    for (int d = 0; d < 6; d++) E[(size_t)a * 6 + d].a[q / P][q % P] = e[d];
                }
        int npa = el.att == AXG_ATT_CG4 ? 4 : N;
        static const int cg4pt[4] = {6, 8, 16, 18};   // (1,1) (1,3) (3,1) (3,3)
        if (!el.is3d) {
            // strainToStress_FR per mode (1D material, _1D_FR case)
            for (int a = 0; a < nu; a++)
                for (int q = 0; q < N; q++) {
                    Cx<R> e[6], s[6];
                    for (int d = 0; d < 6; d++) e[d] = E[(size_t)a * 6 + d].a[q / P][q % P];
                    elastic(el, 0, q, e, s);
                    for (int d = 0; d < 6; d++) S[(size_t)a * 6 + d].a[q / P][q % P] = s[d];
                }
            if (el.att != AXG_ATT_NONE) {
                size_t memStride = (size_t)nu * 6 * npa;   // between SLS
                for (int a = 0; a < nu; a++)
                    for (int k = 0; k < npa; k++) {
                        int q = el.att == AXG_ATT_FULL ? k : cg4pt[k];
                        Cx<R> e[6], s[6], dst[6], mem[AXG_MAX_SLS * 6];
                        for (int d = 0; d < 6; d++) {
                            e[d] = E[(size_t)a * 6 + d].a[q / P][q % P];
                            s[d] = S[(size_t)a * 6 + d].a[q / P][q % P];
                            dst[d] = el.dstressF[((size_t)a * 6 + d) * npa + k];
                            for (int l = 0; l < cfg.nsls; l++)
                                mem[l * 6 + d] = el.memF[l * memStride + ((size_t)a * 6 + d) * npa + k];
                        }
                        attenuate(e, s, dst, mem, 6, el.dlam[k], el.dmu[k], el.dmu2[k]);
                        for (int d = 0; d < 6; d++) {
                            S[(size_t)a * 6 + d].a[q / P][q % P] = s[d];
                            el.dstressF[((size_t)a * 6 + d) * npa + k] = dst[d];
                            for (int l = 0; l < cfg.nsls; l++)
                                el.memF[l * memStride + ((size_t)a * 6 + d) * npa + k] = mem[l * 6 + d];
                        }
                    }
            }
        } else {
            // gFFT_N6.computeC2R -> strainToStress_CD -> attenuation -> computeR2C
            const Twiddle<R> &t = twiddle(nr);
            std::vector<R> ec((size_t)nr * 6 * N), sc((size_t)nr * 6 * N);
            std::vector<Cx<R>> cbuf(nu);
            std::vector<R> rbuf(nr);
            for (int d = 0; d < 6; d++)
                for (int q = 0; q < N; q++) {
                    for (int a = 0; a < nu; a++) cbuf[a] = E[(size_t)a * 6 + d].a[q / P][q % P];
                    c2r(cbuf.data(), nu, rbuf.data(), nr, t);
                    for (int k = 0; k < nr; k++) ec[((size_t)k * 6 + d) * N + q] = rbuf[k];
                }
            for (int k = 0; k < nr; k++)
                for (int q = 0; q < N; q++) {
                    R e[6], s[6];
                    for (int d = 0; d < 6; d++) e[d] = ec[((size_t)k * 6 + d) * N + q];
                    elastic(el, k, q, e, s);
                    for (int d = 0; d < 6; d++) sc[((size_t)k * 6 + d) * N + q] = s[d];
                }
            if (el.att != AXG_ATT_NONE) {
                size_t memStride = (size_t)nr * 6 * npa;
                for (int k = 0; k < nr; k++)
                    for (int kk = 0; kk < npa; kk++) {
                        int q = el.att == AXG_ATT_FULL ? kk : cg4pt[kk];
                        R e[6], s[6], dst[6], mem[AXG_MAX_SLS * 6];
                        for (int d = 0; d < 6; d++) {
                            e[d] = ec[((size_t)k * 6 + d) * N + q];
                            s[d] = sc[((size_t)k * 6 + d) * N + q];
                            dst[d] = el.dstressC[((size_t)k * 6 + d) * npa + kk];
                            for (int l = 0; l < cfg.nsls; l++)
                                mem[l * 6 + d] = el.memC[l * memStride + ((size_t)k * 6 + d) * npa + kk];
                        }
                        size_t ao = (size_t)k * npa + kk;
                        attenuate(e, s, dst, mem, 6, el.dlam[ao], el.dmu[ao], el.dmu2[ao]);
                        for (int d = 0; d < 6; d++) {
                            sc[((size_t)k * 6 + d) * N + q] = s[d];
                            el.dstressC[((size_t)k * 6 + d) * npa + kk] = dst[d];
                            for (int l = 0; l < cfg.nsls; l++)
                                el.memC[l * memStride + ((size_t)k * 6 + d) * npa + kk] = mem[l * 6 + d];
                        }
                    }
            }
            for (int d = 0; d < 6; d++)
                for (int q = 0; q < N; q++) {
                    for (int k = 0; k < nr; k++) rbuf[k] = sc[((size_t)k * 6 + d) * N + q];
                    r2c(rbuf.data(), nr, cbuf.data(), nu, t);
                    for (int a = 0; a < nu; a++) S[(size_t)a * 6 + d].a[q / P][q % P] = cbuf[a];
                }
        }
        if (el.rtz)
            for (int a = 0; a < nu; a++)
                for (int q = 0; q < N; q++) {
                    Cx<R> s[6];
                    for (int d = 0; d < 6; d++) s[d] = S[(size_t)a * 6 + d].a[q / P][q % P];
                    rtz_spz6(s, el.sin1[q], el.cos1[q], el.sin2[q], el.cos2[q]);
                    for (int d = 0; d < 6; d++) S[(size_t)a * 6 + d].a[q / P][q % P] = s[d];
                }
        elemStiff.resize((size_t)nu * 3 * N);
        for (int a = 0; a < nu; a++) {
            CM<R> f[3];
            g.quad6(&S[(size_t)a * 6], f, a, true);
            for (int c = 0; c < 3; c++)
                for (int q = 0; q < N; q++)
                    elemStiff[((size_t)a * 3 + c) * N + q] = f[c].a[q / P][q % P];
        }
    }

    // PRT::sphericalToUndulated3 / undulatedToSpherical3 (PRT.hpp:313-371) as written there
    template <class V>
    static void sph2und3(const V g[3], V u[3], R X0, R X1, R X2, R X3) {
        (void)X2;
        u[0] = g[0] * X0 + g[2] * X1;
        u[1] = g[1] * X0 + g[2] * X1;
        u[2] = g[2] * X3;
    }
    template <class V>
    static void und2sph3(const V u[3], V g[3], R X0, R X1, R X2, R X3) {
        g[0] = u[0] * X0;
        g[1] = u[1] * X0;
        g[2] = u[0] * X1 + u[1] * X2 + u[2] * X3;
    }
    // transformSPZ_RTZ3 / transformRTZ_SPZ3 (CoordTransformSpherical.hpp:54-100)
    static void rtz3(Cx<R> g[3], R s1, R c1, bool to_rtz) {
        const Cx<R> u0 = g[0];
        if (to_rtz) { g[0] = u0 * c1 - g[2] * s1; g[2] = g[2] * c1 + u0 * s1; }
        else { g[0] = u0 * c1 + g[2] * s1; g[2] = g[2] * c1 - u0 * s1; }
    }
    // FluidElement::displToStiff, PRT branch (FluidElement.cpp:101-148)
    void fluid_element_prt(const FluidElem<R> &el, std::vector<Cx<R>> &elemStiff) {
        const int nu = el.nu, nr = el.nr;
        std::vector<CM<R>> X(nu), Q((size_t)nu * 3);
        for (int q = 0; q < N; q++) {
            int p = el.pts[q];
            for (int a = 0; a < nu; a++)
                X[a].a[q / P][q % P] = a < fp.nu[p] ? fp.displ[(size_t)fp.off[p] + a] : Cx<R>(0);
        }
        Grad<R> g{el.ops, gm};
        for (int a = 0; a < nu; a++) g.grad3(X[a], &Q[(size_t)a * 3], a);
        auto at = [&](int a, int c, int q) -> Cx<R> & { return Q[(size_t)a * 3 + c].a[q / P][q % P]; };
        if (el.rtz)
            for (int a = 0; a < nu; a++)
                for (int q = 0; q < N; q++) {
                    Cx<R> v[3] = {at(a, 0, q), at(a, 1, q), at(a, 2, q)};
                    rtz3(v, el.sin1[q], el.cos1[q], true);
                    for (int c = 0; c < 3; c++) at(a, c, q) = v[c];
                }
        const int xns = el.prt3 ? nr : 1;
        const size_t xs = (size_t)xns * N;
        auto XF = [&](int c, int k, int q) { return el.X[c * xs + (size_t)k * N + q]; };
        if (!el.is3d) {
            for (int a = 0; a < nu; a++)
                for (int q = 0; q < N; q++) {
                    Cx<R> v[3] = {at(a, 0, q), at(a, 1, q), at(a, 2, q)}, u[3];
                    sph2und3(v, u, XF(0, 0, q), XF(1, 0, q), XF(2, 0, q), XF(3, 0, q));
                    for (int c = 0; c < 3; c++) u[c] *= el.K[q];
                    und2sph3(u, v, XF(4, 0, q), XF(5, 0, q), XF(6, 0, q), XF(7, 0, q));
                    for (int c = 0; c < 3; c++) at(a, c, q) = v[c];
                }
        } else {
            const Twiddle<R> &t = twiddle(nr);
            std::vector<R> gc((size_t)nr * 3 * N);
            std::vector<Cx<R>> cbuf(nu);
            std::vector<R> rbuf(nr);
            for (int c = 0; c < 3; c++)
                for (int q = 0; q < N; q++) {
                    for (int a = 0; a < nu; a++) cbuf[a] = at(a, c, q);
                    c2r(cbuf.data(), nu, rbuf.data(), nr, t);
                    for (int k = 0; k < nr; k++) gc[((size_t)k * 3 + c) * N + q] = rbuf[k];
                }
            for (int k = 0; k < nr; k++)
                for (int q = 0; q < N; q++) {
                    const int kx = el.prt3 ? k : 0;
                    R v[3] = {gc[((size_t)k * 3) * N + q], gc[((size_t)k * 3 + 1) * N + q], gc[((size_t)k * 3 + 2) * N + q]}, u[3];
                    sph2und3(v, u, XF(0, kx, q), XF(1, kx, q), XF(2, kx, q), XF(3, kx, q));
                    for (int c = 0; c < 3; c++) u[c] *= el.K[(size_t)k * N + q];
                    und2sph3(u, v, XF(4, kx, q), XF(5, kx, q), XF(6, kx, q), XF(7, kx, q));
                    for (int c = 0; c < 3; c++) gc[((size_t)k * 3 + c) * N + q] = v[c];
                }
            for (int c = 0; c < 3; c++)
                for (int q = 0; q < N; q++) {
                    for (int k = 0; k < nr; k++) rbuf[k] = gc[((size_t)k * 3 + c) * N + q];
                    r2c(rbuf.data(), nr, cbuf.data(), nu, t);
                    for (int a = 0; a < nu; a++) at(a, c, q) = cbuf[a];
                }
        }
        if (el.rtz)
            for (int a = 0; a < nu; a++)
                for (int q = 0; q < N; q++) {
                    Cx<R> v[3] = {at(a, 0, q), at(a, 1, q), at(a, 2, q)};
                    rtz3(v, el.sin1[q], el.cos1[q], false);
                    for (int c = 0; c < 3; c++) at(a, c, q) = v[c];
                }
        elemStiff.resize((size_t)nu * N);
        for (int a = 0; a < nu; a++) {
            CM<R> f;
            g.quad3(&Q[(size_t)a * 3], f, a);
            for (int q = 0; q < N; q++) elemStiff[(size_t)a * N + q] = f.a[q / P][q % P];
        }
    }

    // ----------------------- FluidElement::computeStiff -----------------------
    void fluid_element(const FluidElem<R> &el, std::vector<Cx<R>> &elemStiff) {
        if (el.prt) { fluid_element_prt(el, elemStiff); return; }
        int nu = el.nu, nr = el.nr;
        std::vector<CM<R>> X(nu), Q((size_t)nu * 3);
        for (int q = 0; q < N; q++) {
            int p = el.pts[q];
            for (int a = 0; a < nu; a++)
                X[a].a[q / P][q % P] = a < fp.nu[p] ? fp.displ[(size_t)fp.off[p] + a] : Cx<R>(0);
        }
        Grad<R> g{el.ops, gm};
        for (int a = 0; a < nu; a++) g.grad3(X[a], &Q[(size_t)a * 3], a);
        // Acoustic::strainToStress (Acoustic.hpp:85-92)
        if (!el.is3d) {
            for (int a = 0; a < nu; a++)
                for (int c = 0; c < 3; c++)
                    for (int q = 0; q < N; q++) Q[(size_t)a * 3 + c].a[q / P][q % P] *= el.K[q];
        } else {
            const Twiddle<R> &t = twiddle(nr);
            std::vector<Cx<R>> cbuf(nu);
            std::vector<R> rbuf(nr);
            for (int c = 0; c < 3; c++)
                for (int q = 0; q < N; q++) {
                    for (int a = 0; a < nu; a++) cbuf[a] = Q[(size_t)a * 3 + c].a[q / P][q % P];
                    c2r(cbuf.data(), nu, rbuf.data(), nr, t);
                    for (int k = 0; k < nr; k++) rbuf[k] *= el.K[(size_t)k * N + q];
                    r2c(rbuf.data(), nr, cbuf.data(), nu, t);
                    for (int a = 0; a < nu; a++) Q[(size_t)a * 3 + c].a[q / P][q % P] = cbuf[a];
                }
        }
        elemStiff.resize((size_t)nu * N);
        for (int a = 0; a < nu; a++) {
            CM<R> f;
            g.quad3(&Q[(size_t)a * 3], f, a);
            for (int q = 0; q < N; q++) elemStiff[(size_t)a * N + q] = f.a[q / P][q % P];
        }
    }

    void compute_stiffness(int nthreads) override { stiffness_of(nthreads, -1); }
    void compute_stiffness_part(int nthreads, int part) override {
        if (part < 0 || part > 1) throw std::runtime_error("axo_compute_stiffness_part || part must be 0 or 1.");
        stiffness_of(nthreads, part);
    }
    // part < 0: every element
    void stiffness_of(int nthreads, int part) {
        // elements are computed in parallel, assembled serially in element order
        // (Domain::computeStiffness, Domain.cpp:298-308)
        auto in_s = [&](int i) {
            return part < 0 || (int)(se_part.size() == se.size() ? se_part[i] : 0) == part;
        };
        auto in_f = [&](int i) {
            return part < 0 || (int)(fe_part.size() == fe.size() ? fe_part[i] : 0) == part;
        };
        int ne = (int)se.size();
        if (nthreads < 1) nthreads = 1;
        int chunk = 256;
        for (int base = 0; base < ne; base += chunk * nthreads) {
            int hi = std::min(ne, base + chunk * nthreads);
            std::vector<std::vector<Cx<R>>> out(hi - base);
            auto work = [&](int t) {
                std::vector<CM<R>> S, E;
                for (int i = base + t; i < hi; i += nthreads)
                    if (in_s(i)) solid_element(se[i], out[i - base], S, E);
            };
            if (nthreads == 1) work(0);
            else {
                std::vector<std::thread> th;
                for (int t = 0; t < nthreads; t++) th.emplace_back(work, t);
                for (auto &x : th) x.join();
            }
            for (int i = base; i < hi; i++) {
                if (!in_s(i)) continue;
                // addStiffToPoints -> SolidPoint::gatherStiffFromElement (SolidPoint.hpp:101-109)
                const SolidElem<R> &el = se[i];
                const std::vector<Cx<R>> &f = out[i - base];
                for (int q = 0; q < N; q++) {
                    int p = el.pts[q];
                    for (int a = 0; a < sp.nu[p]; a++)
                        for (int c = 0; c < 3; c++)
                            sp.stiff[((size_t)sp.off[p] + a) * 3 + c] -= f[((size_t)a * 3 + c) * N + q];
                }
            }
        }
        std::vector<Cx<R>> f;
        for (size_t i = 0; i < fe.size(); i++) {
            if (!in_f((int)i)) continue;
            const FluidElem<R> &el = fe[i];
            fluid_element(el, f);
            for (int q = 0; q < N; q++) {
                int p = el.pts[q];
                for (int a = 0; a < fp.nu[p]; a++) fp.stiff[(size_t)fp.off[p] + a] -= f[(size_t)a * N + q];
            }
        }
    }

    // AbsorbingBoundary::applyClayton, then SolidFluidCoupling::apply
    // (Domain::applyBC_BeforeAssemblingStiff, Domain.cpp:313-317)
    void bc_before() override {
        for (auto &c : cls) {
            Cx<R> *f = &sp.stiff[(size_t)sp.off[c.p] * 3];
            const Cx<R> *v = &sp.veloc[(size_t)sp.off[c.p] * 3];
            for (int a = 0; a < sp.nu[c.p]; a++) {
                f[a * 3 + 0] -= (c.ss * v[a * 3 + 0] + c.sz * v[a * 3 + 2]);
                f[a * 3 + 2] -= (c.sz * v[a * 3 + 0] + c.zz * v[a * 3 + 2]);
                f[a * 3 + 1] -= c.pp * v[a * 3 + 1];
            }
        }
        for (auto &c : clf)
            for (int a = 0; a < fp.nu[c.p]; a++)
                fp.stiff[(size_t)fp.off[c.p] + a] -= fp.veloc[(size_t)fp.off[c.p] + a] * c.c;
        // ClaytonSolid3D::apply / ClaytonFluid3D::apply (ABC/ClaytonSolid3D.cpp, ClaytonFluid3D.cpp)
        for (int solid = 1; solid >= 0; solid--) {
            PointSet<R> &ps = solid ? sp : fp;
            const int nd = ps.ndim;
            for (auto &c : (solid ? cl3s : cl3f)) {
                const int nr = ps.nr[c.p], nu = ps.nu[c.p];
                const Twiddle<R> &t = twiddle(nr);
                Cx<R> *f = &ps.stiff[(size_t)ps.off[c.p] * nd];
                const Cx<R> *v = &ps.veloc[(size_t)ps.off[c.p] * nd];
                std::vector<Cx<R>> cb(nu);
                std::vector<R> vr((size_t)nd * nr), ar((size_t)nd * nr);
                for (int d = 0; d < nd; d++) {
                    for (int a = 0; a < nu; a++) cb[a] = v[a * nd + d];
                    c2r(cb.data(), nu, &vr[(size_t)d * nr], nr, t);
                }
                for (int k = 0; k < nr; k++) {
                    if (nd == 3) {
                        const R *q = &c.c[(size_t)4 * k];
                        const R v0 = vr[k], v1 = vr[nr + k], v2 = vr[2 * nr + k];
                        const R dot = v0 * q[1] + v1 * q[2] + v2 * q[3];
                        ar[k] = q[0] * v0 + dot * q[1];
                        ar[nr + k] = q[0] * v1 + dot * q[2];
                        ar[2 * nr + k] = q[0] * v2 + dot * q[3];
                    } else {
                        ar[k] = vr[k] * c.c[k];
                    }
                }
                for (int d = 0; d < nd; d++) {
                    r2c(&ar[(size_t)d * nr], nr, cb.data(), nu, t);
                    for (int a = 0; a < nu; a++) f[a * nd + d] -= cb[a];
                }
            }
        }
        for (auto &c : sf) {
            int nus = sp.nu[c.s], nuf = fp.nu[c.f];
            int nu = std::min(nus, nuf);
            (void)nu;
            for (int a = 0; a < nuf; a++) {
                fp.stiff[(size_t)fp.off[c.f] + a] += c.nsu * sp.displ[((size_t)sp.off[c.s] + a) * 3 + 0];
                fp.stiff[(size_t)fp.off[c.f] + a] += c.nzu * sp.displ[((size_t)sp.off[c.s] + a) * 3 + 2];
            }
            for (int a = 0; a < nus; a++) {
                sp.stiff[((size_t)sp.off[c.s] + a) * 3 + 0] -= c.nsa_m * fp.stiff[(size_t)fp.off[c.f] + a];
                sp.stiff[((size_t)sp.off[c.s] + a) * 3 + 2] -= c.nza_m * fp.stiff[(size_t)fp.off[c.f] + a];
            }
        }
        couple3d();
    }

    // AxialBoundary::apply (AxialBoundary.cpp:21-51), FluidSurfaceBoundary::apply
    void bc_after() override {
        const Cx<R> cJ((R)0, (R)1);
        const R half = (R).5;
        for (int p = 0; p < sp.n; p++) {
            if (!sp.axial[p]) continue;
            Cx<R> *f = &sp.stiff[(size_t)sp.off[p] * 3];
            int nu = sp.nu[p] - 1;
            f[0] = 0; f[1] = 0;
            if (nu >= 1) {
                f[3 + 0] = (f[3 + 0] - cJ * f[3 + 1]) * half;
                f[3 + 1] = cJ * f[3 + 0];
                f[3 + 2] = 0;
                for (int a = 2; a <= nu; a++)
                    for (int c = 0; c < 3; c++) f[a * 3 + c] = 0;
            }
        }
        for (int p = 0; p < fp.n; p++) {
            if (fp.axial[p])
                for (int a = 1; a < fp.nu[p]; a++) fp.stiff[(size_t)fp.off[p] + a] = 0;
        }
        for (int p = 0; p < fp.n; p++) {
            if (fp.surface[p])
                for (int a = 0; a < fp.nu[p]; a++) fp.stiff[(size_t)fp.off[p] + a] = 0;
        }
    }

    // SolidPoint/FluidPoint::computeStiffToAccel (SolidPoint.cpp:28-36, FluidPoint.cpp:28-54)
    void points_to_accel(PointSet<R> &ps) {
        int nd = ps.ndim;
        for (int p = 0; p < ps.n; p++) {
            Cx<R> *f = &ps.stiff[(size_t)ps.off[p] * nd];
            int nu = ps.nu[p], nr = ps.nr[p];
            if (nr % 2 == 0)
                for (int c = 0; c < nd; c++) f[(nu - 1) * nd + c].imag(0);
            if (ps.ocean3.size() && ps.ocean3[p] >= 0) {
                // MassOceanLoad3D::computeAccel (MassOceanLoad3D.cpp)
                const std::vector<R> &c = ps.ocean3_c[ps.ocean3[p]];
                const Twiddle<R> &t = twiddle(nr);
                std::vector<Cx<R>> cb(nu);
                std::vector<R> fr((size_t)3 * nr);
                for (int d = 0; d < 3; d++) {
                    for (int a = 0; a < nu; a++) cb[a] = f[a * 3 + d];
                    c2r(cb.data(), nu, &fr[(size_t)d * nr], nr, t);
                }
                for (int k = 0; k < nr; k++) {
                    const R f0 = fr[k], f1 = fr[nr + k], f2 = fr[2 * nr + k];
                    const R *q = &c[(size_t)4 * k];
                    const R dot = f0 * q[1] + f1 * q[2] + f2 * q[3];
                    fr[k] = q[0] * f0 - dot * q[1];
                    fr[nr + k] = q[0] * f1 - dot * q[2];
                    fr[2 * nr + k] = q[0] * f2 - dot * q[3];
                }
                for (int d = 0; d < 3; d++) {
                    r2c(&fr[(size_t)d * nr], nr, cb.data(), nu, t);
                    for (int a = 0; a < nu; a++) f[a * 3 + d] = cb[a];
                }
            } else if (ps.ocean.size() && ps.ocean[p] >= 0) {
                // MassOceanLoad1D::computeAccel (MassOceanLoad1D.hpp)
                const std::array<R, 4> &c = ps.ocean_c[ps.ocean[p]];
                for (int a = 0; a < nu; a++) {
                    const Cx<R> s0 = f[a * 3 + 0];
                    f[a * 3 + 0] = c[0] * s0 + c[2] * f[a * 3 + 2];
                    f[a * 3 + 2] = c[2] * s0 + c[1] * f[a * 3 + 2];
                    f[a * 3 + 1] *= c[3];
                }
            } else if (ps.mass_nr[p] == 1) {
                R im = ps.inv_mass[p][0];
                for (int q = 0; q < nu * nd; q++) f[q] *= im;
            } else {
                // Mass3D::computeAccel (Mass3D.cpp:41-68)
                const Twiddle<R> &t = twiddle(nr);
                std::vector<Cx<R>> cb(nu);
                std::vector<R> rb(nr);
                for (int c = 0; c < nd; c++) {
                    for (int a = 0; a < nu; a++) cb[a] = f[a * nd + c];
                    c2r(cb.data(), nu, rb.data(), nr, t);
                    for (int k = 0; k < nr; k++) rb[k] *= ps.inv_mass[p][k];
                    r2c(rb.data(), nr, cb.data(), nu, t);
                    for (int a = 0; a < nu; a++) f[a * nd + c] = cb[a];
                }
            }
        }
    }
    // computeStiffToAccel on all points, then the sponge
    // (Domain::applyBC_AfterComputingAccel, Sponge::apply, ABC/Sponge.hpp:74-98)
    void stiff_to_accel() override {
        points_to_accel(sp);
        points_to_accel(fp);
        // FluidPoint::computeStiffToAccel (FluidPoint.cpp:42-48): the pressure source is added
        // to the new acceleration and zeroed for the next step
        for (size_t i = 0; i < pressure.size(); i++) {
            fp.stiff[i] += pressure[i];
            pressure[i] = Cx<R>(0, 0);
        }
        const R two = 2;
        for (auto &g : sgs) {
            size_t o = (size_t)sp.off[g.first] * 3;
            for (int q = 0; q < sp.nu[g.first] * 3; q++)
                sp.stiff[o + q] -= (two * g.second) * sp.veloc[o + q] + (g.second * g.second) * sp.displ[o + q];
        }
        for (auto &g : sgf) {
            size_t o = (size_t)fp.off[g.first];
            for (int q = 0; q < fp.nu[g.first]; q++)
                fp.stiff[o + q] -= (two * g.second) * fp.veloc[o + q] + (g.second * g.second) * fp.displ[o + q];
        }
        // Sponge::apply, 3-D branch (ABC/Sponge.hpp:74-98)
        for (int solid = 1; solid >= 0; solid--) {
            PointSet<R> &ps = solid ? sp : fp;
            const int nd = ps.ndim;
            for (auto &g : (solid ? sg3s : sg3f)) {
                const int nr = ps.nr[g.p], nu = ps.nu[g.p];
                const Twiddle<R> &t = twiddle(nr);
                const size_t o = (size_t)ps.off[g.p] * nd;
                std::vector<Cx<R>> cb(nu);
                std::vector<R> sr(nr), vr(nr), ur(nr);
                for (int d = 0; d < nd; d++) {
                    for (int a = 0; a < nu; a++) cb[a] = ps.stiff[o + a * nd + d];
                    c2r(cb.data(), nu, sr.data(), nr, t);
                    for (int a = 0; a < nu; a++) cb[a] = ps.veloc[o + a * nd + d];
                    c2r(cb.data(), nu, vr.data(), nr, t);
                    for (int a = 0; a < nu; a++) cb[a] = ps.displ[o + a * nd + d];
                    c2r(cb.data(), nu, ur.data(), nr, t);
                    for (int k = 0; k < nr; k++) sr[k] -= (two * g.g[k]) * vr[k] + (g.g[k] * g.g[k]) * ur[k];
                    r2c(sr.data(), nr, cb.data(), nu, t);
                    for (int a = 0; a < nu; a++) ps.stiff[o + a * nd + d] = cb[a];
                }
            }
        }
    }

    // NewmarkTimeScheme::update (NewmarkTimeScheme.hpp:47-71)
    void newmark_points(PointSet<R> &ps) {
        const R dt = (R)cfg.dt;
        const R half_dt = (R)(.5 * cfg.dt);
        const R half_dt_dt = (R)(.5 * cfg.dt * cfg.dt);
        size_t n = ps.total * ps.ndim;
        for (size_t q = 0; q < n; q++) {
            ps.veloc[q] += half_dt * (ps.accel[q] + ps.stiff[q]);
            ps.accel[q] = ps.stiff[q];
            ps.displ[q] += dt * ps.veloc[q] + half_dt_dt * ps.accel[q];
            ps.stiff[q] = 0;
        }
    }
    void newmark() override {
        newmark_points(sp);
        newmark_points(fp);
    }

    // StationSolid::record, displacement channel (StationSolid.cpp:58-66, Station.hpp:53-72)
    // ---------------- wavefield scanning (Scanning1D, Point.hpp:106-198) ----------------
    struct Scan1D {
        R h2p = 0, h2pp = 0;
        std::map<R, int> cand;
    };
    bool scan_on = false;
    R scan_tf = 0, scan_rel = 0, scan_abs = 0;
    int scan_peaks = 1, scan_interval = 1;
    std::vector<int> scan_pts[2];            // [fluid, solid]
    std::vector<std::vector<Scan1D>> scan_st[2];
    void set_scanning(const axg_scanning *s) override {
        scan_on = true;
        scan_tf = (R)(s->tol_fourier_h1 * s->tol_fourier_h1);
        scan_rel = (R)(s->rel_tol_h1 * s->rel_tol_h1);
        scan_abs = (R)(s->abs_tol_h1 * s->abs_tol_h1);
        scan_peaks = std::min(s->max_num_peaks, AXG_SCAN_MAX_PEAKS);
        scan_interval = s->interval;
        for (int solid = 1; solid >= 0; solid--) {
            const PointSet<R> &ps = solid ? sp : fp;
            const int n = solid ? s->n_solid : s->n_fluid;
            const int32_t *pts = solid ? s->solid_points : s->fluid_points;
            scan_pts[solid].clear();
            if (n < 0) for (int p = 0; p < ps.n; p++) scan_pts[solid].push_back(p);
            else for (int i = 0; i < n; i++) scan_pts[solid].push_back(pts[i]);
            scan_st[solid].assign(scan_pts[solid].size(), std::vector<Scan1D>(ps.ndim));
        }
    }
    static void scan_one(Scan1D &sc, const Cx<R> *f, int stride, int nu, R tf, R rel, R abs_, int peaks) {
        R l2 = 0;
        for (int a = 0; a < nu; a++) l2 += f[a * stride].real() * f[a * stride].real() + f[a * stride].imag() * f[a * stride].imag();
        const R n0 = f[0].real() * f[0].real() + f[0].imag() * f[0].imag();
        const R h2 = (R)((double)l2 - .5 * (double)n0);
        const R maxh2 = sc.cand.empty() ? (R)0 : sc.cand.rbegin()->first;
        if (!(h2 > abs_ && h2 > rel * maxh2 && sc.h2p > h2 && sc.h2p > sc.h2pp)) {
            sc.h2pp = sc.h2p;
            sc.h2p = h2;
            return;
        }
        const R absf = h2 * tf;
        int nn = 1;
        R head = 0;
        for (; nn < nu; nn++) {
            head += f[(nn - 1) * stride].real() * f[(nn - 1) * stride].real() +
                    f[(nn - 1) * stride].imag() * f[(nn - 1) * stride].imag();
            if (l2 - head < absf) break;
        }
        auto it = sc.cand.find(h2);
        if (it != sc.cand.end()) {
            it->second = std::max(it->second, nn);
        } else {
            if (maxh2 < h2) sc.cand.erase(sc.cand.begin(), sc.cand.lower_bound(rel * h2));
            sc.cand.insert({h2, nn});
        }
        if ((int)sc.cand.size() > peaks) sc.cand.erase(sc.cand.begin());
        sc.h2pp = sc.h2p;
        sc.h2p = h2;
    }
    void scan(int tstep) {
        if (!scan_on || tstep % scan_interval != 0) return;
        for (int solid = 1; solid >= 0; solid--) {
            PointSet<R> &ps = solid ? sp : fp;
            for (size_t i = 0; i < scan_pts[solid].size(); i++) {
                const int p = scan_pts[solid][i];
                for (int c = 0; c < ps.ndim; c++)
                    scan_one(scan_st[solid][i][c], &ps.displ[(size_t)ps.off[p] * ps.ndim + c], ps.ndim, ps.nu[p],
                             scan_tf, scan_rel, scan_abs, scan_peaks);
            }
        }
    }
    void scanning_nr(int32_t *out_s, int32_t *out_f) override {
        for (int solid = 1; solid >= 0; solid--) {
            int32_t *out = solid ? out_s : out_f;
            if (!out) continue;
            PointSet<R> &ps = solid ? sp : fp;
            for (int p = 0; p < ps.n; p++) out[p] = -1;
            if (!scan_on) continue;
            for (size_t i = 0; i < scan_pts[solid].size(); i++) {
                const int p = scan_pts[solid][i];
                int best = 1;
                for (int c = 0; c < ps.ndim; c++) {
                    const Scan1D &sc = scan_st[solid][i][c];
                    int r = 1;
                    if (!sc.cand.empty()) {
                        int nu = 0;
                        for (auto &kv : sc.cand) nu = std::max(nu, kv.second);
                        r = std::min(nu * 2 + 1, ps.nr[p]);
                    }
                    best = std::max(best, r);
                }
                out[p] = best;
            }
        }
    }

    void record(int tstep) override {
        scan(tstep);
        if (st.empty() || tstep % rec_interval != 0) return;
        size_t base = seis.size();
        seis.resize(base + st.size() * 3);
        for (size_t i = 0; i < st.size(); i++) {
            const SolidElem<R> &el = se[st[i].elem];
            int nu = el.nu;
            for (int c = 0; c < 3; c++) {
                double acc = 0;
                for (int a = 0; a < nu; a++) {
                    // in-plane sum over points with non-zero weight, in Real
                    Cx<R> x = 0;
                    for (int q = 0; q < N; q++) {
                        if (st[i].w[q] == 0.) continue;
                        int p = el.pts[q];
                        Cx<R> u = a < sp.nu[p] ? sp.displ[((size_t)sp.off[p] + a) * 3 + c] : Cx<R>(0);
                        x += u * (R)st[i].w[q];
                    }
                    // computeTwoExpIAlphaPhi / computeFourierAtPhiExp (eigen_tools.hpp:78-106)
                    Cx<R> e2 = a == 0 ? Cx<R>(1) : (R)2 * std::exp(Cx<R>(0, (R)a * (R)st[i].phi));
                    acc += (double)(e2 * x).real();
                }
                seis[base + i * 3 + c] = acc;
            }
        }
        nrec++;
    }

    void run(int nsteps, int nthreads) override {
        // NewmarkTimeScheme::solve loop body (NewmarkTimeScheme.cpp:41-108)
        for (int i = 0; i < nsteps; i++) {
            apply_sources(step);
            compute_stiffness(nthreads);
            bc_before();
            record(step);
            if (cfg.stability_interval > 0 && step % cfg.stability_interval == 0) {
                for (auto &x : sp.displ)
                    if (!std::isfinite((double)x.real()) || !std::isfinite((double)x.imag()))
                        throw std::runtime_error("Domain::checkStability || Non-finite displacement.");
            }
            bc_after();
            stiff_to_accel();
            newmark();
            step++;
        }
    }

    PointSet<R> &set_of(int solid) { return solid ? sp : fp; }
    std::vector<Cx<R>> &field_of(PointSet<R> &ps, int which) {
        switch (which) {
            case AXG_FIELD_STIFF: return ps.stiff;
            case AXG_FIELD_DISPL: return ps.displ;
            case AXG_FIELD_VELOC: return ps.veloc;
            default: return ps.accel;
        }
    }
    void get_field(int solid, int which, double *out) override {
        PointSet<R> &ps = set_of(solid);
        auto &f = field_of(ps, which);
        for (size_t q = 0; q < f.size(); q++) {
            out[2 * q] = (double)f[q].real();
            out[2 * q + 1] = (double)f[q].imag();
        }
    }
    void set_field(int solid, int which, const double *in) override {
        PointSet<R> &ps = set_of(solid);
        auto &f = field_of(ps, which);
        for (size_t q = 0; q < f.size(); q++) f[q] = Cx<R>((R)in[2 * q], (R)in[2 * q + 1]);
    }
    int64_t field_size(int solid) override {
        PointSet<R> &ps = set_of(solid);
        return (int64_t)(ps.total * ps.ndim);
    }
    int get_seismograms(double *out) override {
        if (out) std::memcpy(out, seis.data(), seis.size() * sizeof(double));
        return nrec;
    }
};

}  // namespace

// ============================== C interface ==================================
extern "C" {

// G matrices (row-major 25 each, G(j, i) = l_j'(x_i), rounded to 12 decimals)
// from oracle/spectral.py, so the C++ oracle and the Python pin share one source
int axo_set_spectral(const double *gll, const double *glj) {
    for (int j = 0; j < P; j++)
        for (int i = 0; i < P; i++) {
            gSpectral.G_GLL[j][i] = gll[j * P + i];
            gSpectral.G_GLJ[j][i] = glj[j * P + i];
        }
    gSpectralSet = true;
    return 0;
}
int axo_get_gmat(double *gll, double *glj) {
    for (int j = 0; j < P; j++)
        for (int i = 0; i < P; i++) {
            gll[j * P + i] = gSpectral.G_GLL[j][i];
            glj[j * P + i] = gSpectral.G_GLJ[j][i];
        }
    return 0;
}

void *axo_create(const axg_config *cfg) {
    if (!gSpectralSet) return nullptr;
    if (cfg->precision == AXG_FP32) return static_cast<OracleBase *>(new Oracle<float>(cfg));
    return static_cast<OracleBase *>(new Oracle<double>(cfg));
}
void axo_destroy(void *h) { delete static_cast<OracleBase *>(h); }

#define AXO_TRY(stmt)                                              \
    try { stmt; return 0; } catch (const std::exception &ex) {     \
        static_cast<OracleBase *>(h)->err = ex.what(); return -1; }

const char *axo_last_error(void *h) { return static_cast<OracleBase *>(h)->err.c_str(); }
int axo_set_solid_points(void *h, const axg_solid_points *p) { AXO_TRY(static_cast<OracleBase *>(h)->set_solid_points(p)) }
int axo_set_fluid_points(void *h, const axg_fluid_points *p) { AXO_TRY(static_cast<OracleBase *>(h)->set_fluid_points(p)) }
int axo_set_solid_elements(void *h, const axg_solid_elements *e) { AXO_TRY(static_cast<OracleBase *>(h)->set_solid_elements(e)) }
int axo_set_fluid_elements(void *h, const axg_fluid_elements *e) { AXO_TRY(static_cast<OracleBase *>(h)->set_fluid_elements(e)) }
int axo_set_solid_fluid(void *h, const axg_solid_fluid *c) { AXO_TRY(static_cast<OracleBase *>(h)->set_solid_fluid(c)) }
int axo_set_moment_sources(void *h, const axg_moment_sources *s) { AXO_TRY(static_cast<OracleBase *>(h)->set_moment_sources(s)) }
int axo_set_force_sources(void *h, const axg_force_sources *s) { AXO_TRY(static_cast<OracleBase *>(h)->set_force_sources(s)) }
int axo_set_pressure_sources(void *h, const axg_pressure_sources *s) { AXO_TRY(static_cast<OracleBase *>(h)->set_pressure_sources(s)) }
int axo_set_solid_fluid3d(void *h, int n, const int *sp_, const int *fp_, const int64_t *off, const double *nu3,
                          const double *na3, const double *mf) {
    AXO_TRY(static_cast<OracleBase *>(h)->set_solid_fluid3d(n, sp_, fp_, off, nu3, na3, mf))
}
int axo_set_stf_table(void *h, int kind, int index, int n, const double *t, const double *v, int padding, double left,
                      double right, int pad_first) {
    AXO_TRY(static_cast<OracleBase *>(h)->set_stf_table(kind, index, n, t, v, padding, left, right, pad_first))
}
int axo_set_stations(void *h, const axg_stations *s, int interval) { AXO_TRY(static_cast<OracleBase *>(h)->set_stations(s, interval)) }
int axo_set_clayton(void *h, int solid, const axg_clayton *c) { AXO_TRY(static_cast<OracleBase *>(h)->set_clayton(solid, c)) }
int axo_set_sponge(void *h, int solid, int n, const int32_t *pt, const double *g) { AXO_TRY(static_cast<OracleBase *>(h)->set_sponge(solid, n, pt, g)) }
int axo_set_ocean_load(void *h, int n, const int32_t *pt, const double *mo, const double *theta) { AXO_TRY(static_cast<OracleBase *>(h)->set_ocean_load(n, pt, mo, theta)) }
int axo_set_ocean_load3d(void *h, int n, const int32_t *pt, const int64_t *off, const double *mo, const double *nrm) { AXO_TRY(static_cast<OracleBase *>(h)->set_ocean_load3d(n, pt, off, mo, nrm)) }
int axo_set_prt(void *h, int n, const int32_t *e, const int64_t *off, const uint8_t *x3d, const double *x) { AXO_TRY(static_cast<OracleBase *>(h)->set_prt(n, e, off, x3d, x)) }
int axo_set_prt_fluid(void *h, int n, const int32_t *e, const int64_t *off, const uint8_t *x3d, const double *x, const double *th) { AXO_TRY(static_cast<OracleBase *>(h)->set_prt_fluid(n, e, off, x3d, x, th)) }
int axo_set_scanning(void *h, const axg_scanning *s) { AXO_TRY(static_cast<OracleBase *>(h)->set_scanning(s)) }
int axo_scanning_nr(void *h, int32_t *s, int32_t *f) { AXO_TRY(static_cast<OracleBase *>(h)->scanning_nr(s, f)) }
int axo_set_clayton3d(void *h, int solid, const axg_clayton3d *c) { AXO_TRY(static_cast<OracleBase *>(h)->set_clayton3d(solid, c)) }
int axo_set_sponge3d(void *h, int solid, int n, const int32_t *pt, const int64_t *off, const double *g) { AXO_TRY(static_cast<OracleBase *>(h)->set_sponge3d(solid, n, pt, off, g)) }
int axo_apply_sources(void *h, int tstep) { AXO_TRY(static_cast<OracleBase *>(h)->apply_sources(tstep)) }
int axo_compute_stiffness(void *h, int nthreads) { AXO_TRY(static_cast<OracleBase *>(h)->compute_stiffness(nthreads)) }
int axo_compute_stiffness_part(void *h, int nthreads, int part) {
    AXO_TRY(static_cast<OracleBase *>(h)->compute_stiffness_part(nthreads, part))
}
int axo_set_element_parts(void *h, const uint8_t *s, int ns, const uint8_t *f, int nf) {
    AXO_TRY(static_cast<OracleBase *>(h)->set_element_parts(s, ns, f, nf))
}
int axo_bc_before(void *h) { AXO_TRY(static_cast<OracleBase *>(h)->bc_before()) }
int axo_bc_after(void *h) { AXO_TRY(static_cast<OracleBase *>(h)->bc_after()) }
int axo_stiff_to_accel(void *h) { AXO_TRY(static_cast<OracleBase *>(h)->stiff_to_accel()) }
int axo_newmark(void *h) { AXO_TRY(static_cast<OracleBase *>(h)->newmark()) }
int axo_record(void *h, int tstep) { AXO_TRY(static_cast<OracleBase *>(h)->record(tstep)) }
int axo_run(void *h, int nsteps, int nthreads) { AXO_TRY(static_cast<OracleBase *>(h)->run(nsteps, nthreads)) }
int axo_get_field(void *h, int solid, int which, double *out) { AXO_TRY(static_cast<OracleBase *>(h)->get_field(solid, which, out)) }
int axo_set_field(void *h, int solid, int which, const double *in) { AXO_TRY(static_cast<OracleBase *>(h)->set_field(solid, which, in)) }
int64_t axo_field_size(void *h, int solid) { return static_cast<OracleBase *>(h)->field_size(solid); }
int axo_get_seismograms(void *h, double *out) { return static_cast<OracleBase *>(h)->get_seismograms(out); }
int axo_reset_attenuation(void *h) { AXO_TRY(static_cast<OracleBase *>(h)->reset_attenuation()) }
int axo_current_step(void *h) { return static_cast<OracleBase *>(h)->step; }

}  // extern "C"
