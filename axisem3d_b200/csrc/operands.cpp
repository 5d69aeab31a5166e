// operands.cpp -- host-side construction of the numbers the kernels consume
// (the reference's preloop): spectral tables, quad geometry, dt, attenuation
// coefficients. All in double, as in the reference.
#include "engine.hpp"

#include <algorithm>
#include <cmath>
#include <limits>

namespace axg {

namespace {

// Jacobi polynomial P_n^(a,b)(x) and its derivative (three-term recurrence)
void jacobi(int n, long double a, long double b, long double x, long double &p, long double &dp) {
    long double p0 = 1, p1 = 0.5L * (a - b + (a + b + 2) * x);
    long double d0 = 0, d1 = 0.5L * (a + b + 2);
    if (n == 0) { p = p0; dp = d0; return; }
    for (int k = 2; k <= n; k++) {
        long double k2ab = 2 * k + a + b;
        long double a1 = 2 * k * (k + a + b) * (k2ab - 2);
        long double a2 = (k2ab - 1) * (a * a - b * b);
        long double a3 = (k2ab - 2) * (k2ab - 1) * k2ab;
        long double a4 = 2 * (k + a - 1) * (k + b - 1) * k2ab;
        long double p2 = ((a2 + a3 * x) * p1 - a4 * p0) / a1;
        long double d2 = ((a2 + a3 * x) * d1 + a3 * p1 - a4 * d0) / a1;
        p0 = p1; p1 = p2; d0 = d1; d1 = d2;
    }
    p = p1; dp = d1;
}

// zeros of P_n^(a,b) by Newton iteration with deflation (ascending order)
std::vector<long double> jacobi_zeros(int n, long double a, long double b) {
    std::vector<long double> z(n);
    const long double pi = 3.14159265358979323846264338327950288L;
    for (int k = 0; k < n; k++) {
        long double r = -std::cos((2.0L * k + 1) * pi / (2.0L * n));
        if (k > 0) r = 0.5L * (r + z[k - 1]);
        for (int it = 0; it < 200; it++) {
            long double p, dp;
            jacobi(n, a, b, r, p, dp);
            long double s = 0;
            for (int i = 0; i < k; i++) s += 1.0L / (r - z[i]);
            long double delta = -p / (dp - s * p);
            r += delta;
            if (std::fabs(delta) < 1e-30L) break;
        }
        z[k] = r;
    }
    std::sort(z.begin(), z.end());
    return z;
}

double round12(long double v) {
    double r = (double)std::round(v * 1e12L) / 1e12;
    return r == 0.0 ? 0.0 : r;
}

void solve5(long double A[5][5], long double b[5], long double x[5]) {
    // Gaussian elimination with partial pivoting
    for (int c = 0; c < 5; c++) {
        int piv = c;
        for (int r = c + 1; r < 5; r++)
            if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
        for (int k = 0; k < 5; k++) std::swap(A[c][k], A[piv][k]);
        std::swap(b[c], b[piv]);
        for (int r = c + 1; r < 5; r++) {
            long double f = A[r][c] / A[c][c];
            for (int k = c; k < 5; k++) A[r][k] -= f * A[c][k];
            b[r] -= f * b[c];
        }
    }
    for (int r = 4; r >= 0; r--) {
        long double s = b[r];
        for (int k = r + 1; k < 5; k++) s -= A[r][k] * x[k];
        x[r] = s / A[r][r];
    }
}

void weights(const long double x[5], const long double mom[5], long double w[5]) {
    long double A[5][5], b[5];
    for (int k = 0; k < 5; k++) {
        for (int i = 0; i < 5; i++) A[k][i] = std::pow(x[i], (long double)k);
        b[k] = mom[k];
    }
    solve5(A, b, w);
}

long double lagrange_deriv(const long double x[5], int j, long double xi) {
    long double sum = 0;
    for (int m = 0; m < 5; m++) {
        if (m == j) continue;
        long double prod = 1.0L / (x[j] - x[m]);
        for (int k = 0; k < 5; k++) {
            if (k == j || k == m) continue;
            prod *= (xi - x[k]) / (x[j] - x[k]);
        }
        sum += prod;
    }
    return sum;
}

SpectralTables build_tables() {
    // GLL: +-1 and the zeros of P_4' (proportional to P_3^(1,1));
    // GLJ (axial direction, weight 1 + xi): +-1 and the zeros of P_3^(1,2)
    // (SOLVER/src/preloop/se_model/quad/spectrals.hpp:73-102 tabulates both)
    SpectralTables t;
    std::vector<long double> zl = jacobi_zeros(3, 1, 1), zj = jacobi_zeros(3, 1, 2);
    long double xl[5] = {-1, zl[0], zl[1], zl[2], 1}, xj[5] = {-1, zj[0], zj[1], zj[2], 1};
    long double ml[5], mj[5];
    for (int k = 0; k < 5; k++) {
        ml[k] = (k % 2 == 0) ? 2.0L / (k + 1) : 0.0L;
        mj[k] = ml[k] + ((k % 2 == 1) ? 2.0L / (k + 2) : 0.0L);
    }
    long double wl[5], wj[5];
    weights(xl, ml, wl);
    weights(xj, mj, wj);
    for (int i = 0; i < 5; i++) {
        t.xGLL[i] = round12(xl[i]); t.xGLJ[i] = round12(xj[i]);
        t.wGLL[i] = round12(wl[i]); t.wGLJ[i] = round12(wj[i]);
    }
    for (int j = 0; j < 5; j++)
        for (int i = 0; i < 5; i++) {
            t.G_GLL[j * 5 + i] = round12(lagrange_deriv(xl, j, xl[i]));
            t.G_GLJ[j * 5 + i] = round12(lagrange_deriv(xj, j, xj[i]));
        }
    return t;
}

}  // namespace

const SpectralTables &spectral_tables() {
    static const SpectralTables t = build_tables();
    return t;
}

namespace {

struct Jac { double J00, J01, J10, J11; };

// MappingLinear (mapping/MappingLinear.hpp): bilinear map of the 4 nodes
void map_linear(const double *n, double xi, double eta, double &s, double &z, Jac &J) {
    double xip = 1 + xi, xim = 1 - xi, etp = 1 + eta, etm = 1 - eta;
    double shp[4] = {xim * etm, xip * etm, xip * etp, xim * etp};
    double dxi[4] = {-etm, etm, etp, -etp};
    double deta[4] = {-xim, -xip, xip, xim};
    s = z = 0;
    J = {0, 0, 0, 0};
    for (int k = 0; k < 4; k++) {
        s += .25 * n[2 * k] * shp[k];
        z += .25 * n[2 * k + 1] * shp[k];
        J.J00 += .25 * n[2 * k] * dxi[k];
        J.J01 += .25 * n[2 * k] * deta[k];
        J.J10 += .25 * n[2 * k + 1] * dxi[k];
        J.J11 += .25 * n[2 * k + 1] * deta[k];
    }
}

// MappingSpherical (mapping/MappingSpherical.hpp): the curved outer edge is
// found from the nodal radii, the quad is rotated by Q2 so that edge lies on
// edge 2 (Mapping::rotateQ2), mapped there, and rotated back.
const double kQ2[4][4] = {{-1., 0., 0., -1.}, {0., -1., 1., 0.}, {1., 0., 0., 1.}, {0., 1., -1., 0.}};

inline int cycle4(int p) { return p > 3 ? p - 4 : (p < 0 ? p + 4 : p); }

inline void angles_close(double &a, double &b) {
    if (a - b > M_PI) b += 2. * M_PI;
    if (b - a > M_PI) a += 2. * M_PI;
}

int curved_outer(const double *n) {
    double r[4], e[4];
    for (int k = 0; k < 4; k++) r[k] = std::hypot(n[2 * k], n[2 * k + 1]);
    for (int k = 0; k < 4; k++) {
        int k1 = (k + 1) % 4;
        e[k] = std::hypot(n[2 * k] - n[2 * k1], n[2 * k + 1] - n[2 * k1 + 1]);
    }
    double tol = std::min(std::min(e[0], e[1]), std::min(e[2], e[3])) * 1e-3;
    if (std::fabs(r[0] - r[1]) < tol && std::fabs(r[2] - r[3]) < tol) return r[2] > r[0] ? 2 : 0;
    if (std::fabs(r[1] - r[2]) < tol && std::fabs(r[3] - r[0]) < tol) return r[3] > r[1] ? 3 : 1;
    return -1;
}

void map_spherical(const double *n, int co, double xi0, double eta0, double &s, double &z, Jac &J) {
    const double *Q = kQ2[co];
    double rt[2][4];
    for (int k = 0; k < 4; k++) {
        double sq = Q[0] * n[2 * k] + Q[1] * n[2 * k + 1];
        double zq = Q[2] * n[2 * k] + Q[3] * n[2 * k + 1];
        rt[0][k] = std::hypot(sq, zq);
        rt[1][k] = M_PI * .5 - std::atan2(zq, sq);   // angle from the z axis
    }
    double xi = Q[0] * xi0 + Q[1] * eta0, eta = Q[2] * xi0 + Q[3] * eta0;
    double r0 = rt[0][cycle4(co - 2)], r2 = rt[0][cycle4(co)];
    double t0 = rt[1][cycle4(co - 2)], t1 = rt[1][cycle4(co - 1)];
    double t2 = rt[1][cycle4(co)], t3 = rt[1][cycle4(co + 1)];
    angles_close(t3, t2);
    angles_close(t0, t1);
    double t01 = ((1. - xi) * t0 + (1. + xi) * t1) * .5;
    double t32 = ((1. - xi) * t3 + (1. + xi) * t2) * .5;
    double r0m = (1. - eta) * r0 * .5;
    double r2p = (1. + eta) * r2 * .5;
    double t01_xi = (t1 - t0) * .5, t32_xi = (t2 - t3) * .5;
    double r0m_eta = -r0 * .5, r2p_eta = r2 * .5;
    double sq = r0m * std::sin(t01) + r2p * std::sin(t32);
    double zq = r0m * std::cos(t01) + r2p * std::cos(t32);
    double j00 = r0m * std::cos(t01) * t01_xi + r2p * std::cos(t32) * t32_xi;
    double j10 = (r0m * std::sin(t01) * t01_xi + r2p * std::sin(t32) * t32_xi) * (-1.);
    double j01 = r0m_eta * std::sin(t01) + r2p_eta * std::sin(t32);
    double j11 = r0m_eta * std::cos(t01) + r2p_eta * std::cos(t32);
    // back: sz = Q^T sz', J = Q^T J' Q
    s = Q[0] * sq + Q[2] * zq;
    z = Q[1] * sq + Q[3] * zq;
    double a00 = Q[0] * j00 + Q[2] * j10, a01 = Q[0] * j01 + Q[2] * j11;
    double a10 = Q[1] * j00 + Q[3] * j10, a11 = Q[1] * j01 + Q[3] * j11;
    J.J00 = a00 * Q[0] + a01 * Q[2];
    J.J01 = a00 * Q[1] + a01 * Q[3];
    J.J10 = a10 * Q[0] + a11 * Q[2];
    J.J11 = a10 * Q[1] + a11 * Q[3];
}

// MappingSemiSpherical (mapping/MappingSemiSpherical.hpp): one curved outer edge (equal
// nodal radii, the larger ones), the opposite edge straight; rotated by Q2 like the spherical
// mapping, blended linearly between the straight edge and the arc.
int curved_outer_semi(const double *n) {
    double r[4], e[4];
    for (int k = 0; k < 4; k++) r[k] = std::hypot(n[2 * k], n[2 * k + 1]);
    for (int k = 0; k < 4; k++) {
        int k1 = (k + 1) % 4;
        e[k] = std::hypot(n[2 * k] - n[2 * k1], n[2 * k + 1] - n[2 * k1 + 1]);
    }
    double tol = std::min(std::min(e[0], e[1]), std::min(e[2], e[3])) * 1e-3;
    if (std::fabs(r[0] - r[1]) < tol && r[0] > r[2]) return 0;
    if (std::fabs(r[1] - r[2]) < tol && r[1] > r[3]) return 1;
    if (std::fabs(r[2] - r[3]) < tol && r[2] > r[0]) return 2;
    if (std::fabs(r[3] - r[0]) < tol && r[3] > r[1]) return 3;
    return -1;
}

void map_semi_spherical(const double *n, int co, double xi0, double eta0, double &s, double &z,
                        Jac &J) {
    const double *Q = kQ2[co];
    double sq_n[4], zq_n[4], t_n[4];
    for (int k = 0; k < 4; k++) {
        sq_n[k] = Q[0] * n[2 * k] + Q[1] * n[2 * k + 1];
        zq_n[k] = Q[2] * n[2 * k] + Q[3] * n[2 * k + 1];
        t_n[k] = M_PI * .5 - std::atan2(zq_n[k], sq_n[k]);
    }
    double xi = Q[0] * xi0 + Q[1] * eta0, eta = Q[2] * xi0 + Q[3] * eta0;
    const int i0 = cycle4(co - 2), i1 = cycle4(co - 1), i2 = cycle4(co), i3 = cycle4(co + 1);
    double s0 = sq_n[i0], z0 = zq_n[i0], s1 = sq_n[i1], z1 = zq_n[i1];
    double r2 = std::hypot(sq_n[i2], zq_n[i2]);
    double t2 = t_n[i2], t3 = t_n[i3];
    angles_close(t3, t2);
    double s01 = ((1. - xi) * s0 + (1. + xi) * s1) * .5;
    double z01 = ((1. - xi) * z0 + (1. + xi) * z1) * .5;
    double t32 = ((1. - xi) * t3 + (1. + xi) * t2) * .5;
    double etam = (1. - eta) * .5, r2p = (1. + eta) * r2 * .5;
    double s01_xi = (s1 - s0) * .5, z01_xi = (z1 - z0) * .5, t32_xi = (t2 - t3) * .5;
    double sq = etam * s01 + r2p * std::sin(t32);
    double zq = etam * z01 + r2p * std::cos(t32);
    double j00 = etam * s01_xi + r2p * std::cos(t32) * t32_xi;
    double j10 = etam * z01_xi - r2p * std::sin(t32) * t32_xi;
    double j01 = -.5 * s01 + r2 * .5 * std::sin(t32);
    double j11 = -.5 * z01 + r2 * .5 * std::cos(t32);
    s = Q[0] * sq + Q[2] * zq;
    z = Q[1] * sq + Q[3] * zq;
    double a00 = Q[0] * j00 + Q[2] * j10, a01 = Q[0] * j01 + Q[2] * j11;
    double a10 = Q[1] * j00 + Q[3] * j10, a11 = Q[1] * j01 + Q[3] * j11;
    J.J00 = a00 * Q[0] + a01 * Q[2];
    J.J01 = a00 * Q[1] + a01 * Q[3];
    J.J10 = a10 * Q[0] + a11 * Q[2];
    J.J11 = a10 * Q[1] + a11 * Q[3];
}

}  // namespace
}  // namespace axg

using namespace axg;

extern "C" {

int axg_spectral_tables(double *xgll, double *xglj, double *wgll, double *wglj, double *ggll,
                        double *gglj) {
    const SpectralTables &t = spectral_tables();
    for (int i = 0; i < 5; i++) {
        xgll[i] = t.xGLL[i]; xglj[i] = t.xGLJ[i]; wgll[i] = t.wGLL[i]; wglj[i] = t.wGLJ[i];
    }
    for (int i = 0; i < 25; i++) { ggll[i] = t.G_GLL[i]; gglj[i] = t.G_GLJ[i]; }
    return AXG_OK;
}

// Quad::createGradient + Quad::computeIntegralFactor (Quad.hpp:155-184, Quad.cpp:403-435)
int axg_quad_geometry(int32_t mapping, const double *nodal_sz, int32_t axial,
                      double *out_geometry, double *out_sz) {
    if (!nodal_sz || !out_geometry) return AXG_E_ARG;
    int co = -1;
    if (mapping == AXG_MAP_SPHERICAL) {
        co = curved_outer(nodal_sz);
        if (co < 0) return AXG_E_ARG;   // "Error identifying curved outer edge."
    } else if (mapping == AXG_MAP_SEMI_SPHERICAL) {
        co = curved_outer_semi(nodal_sz);
        if (co < 0) return AXG_E_ARG;
    } else if (mapping != AXG_MAP_LINEAR) {
        return AXG_E_ARG;
    }
    const SpectralTables &t = spectral_tables();
    const double *xi_n = axial ? t.xGLJ : t.xGLL;
    const double *w_xi = axial ? t.wGLJ : t.wGLL;
    double *dsdxii = out_geometry, *dsdeta = out_geometry + 25, *dzdxii = out_geometry + 50,
           *dzdeta = out_geometry + 75, *inv_s = out_geometry + 100, *ifact = out_geometry + 125;
    for (int ipol = 0; ipol < 5; ipol++)
        for (int jpol = 0; jpol < 5; jpol++) {
            int q = ipol * 5 + jpol;
            double xi = xi_n[ipol], eta = t.xGLL[jpol];
            double s, z;
            Jac J;
            if (mapping == AXG_MAP_LINEAR) map_linear(nodal_sz, xi, eta, s, z, J);
            else if (mapping == AXG_MAP_SPHERICAL) map_spherical(nodal_sz, co, xi, eta, s, z, J);
            else map_semi_spherical(nodal_sz, co, xi, eta, s, z, J);
            double det = J.J00 * J.J11 - J.J01 * J.J10;
            double f = w_xi[ipol] * t.wGLL[jpol] * det;
            if (axial) f *= (ipol == 0) ? J.J00 : s / (1. + xi);
            else f *= s;
            ifact[q] = f;
            dsdxii[q] = J.J00 / det;
            dsdeta[q] = -J.J01 / det;
            dzdxii[q] = -J.J10 / det;
            dzdeta[q] = J.J11 / det;
            inv_s[q] = (axial && ipol == 0) ? 0. : 1. / s;
            if (out_sz) { out_sz[q] = s; out_sz[25 + q] = z; }
        }
    return AXG_OK;
}

// Mapping::mapping and Mapping::jacobian at one (xi, eta): out = s, z, J00, J01, J10, J11
int axg_quad_map(int32_t mapping, const double *nodal_sz, double xi, double eta, double *out) {
    if (!nodal_sz || !out) return AXG_E_ARG;
    double s, z;
    Jac J;
    if (mapping == AXG_MAP_LINEAR) {
        map_linear(nodal_sz, xi, eta, s, z, J);
    } else if (mapping == AXG_MAP_SPHERICAL) {
        int co = curved_outer(nodal_sz);
        if (co < 0) return AXG_E_ARG;
        map_spherical(nodal_sz, co, xi, eta, s, z, J);
    } else if (mapping == AXG_MAP_SEMI_SPHERICAL) {
        int co = curved_outer_semi(nodal_sz);
        if (co < 0) return AXG_E_ARG;
        map_semi_spherical(nodal_sz, co, xi, eta, s, z, J);
    } else {
        return AXG_E_ARG;
    }
    out[0] = s; out[1] = z;
    out[2] = J.J00; out[3] = J.J01; out[4] = J.J10; out[5] = J.J11;
    return AXG_OK;
}

// batch form of axg_quad_geometry over n quads (nodal_sz [n*8], axial [n])
int axg_quad_geometry_batch(int32_t n, int32_t mapping, const double *nodal_sz,
                            const uint8_t *axial, double *out_geometry, double *out_sz) {
    if (n < 0 || !nodal_sz || !axial || !out_geometry) return AXG_E_ARG;
    for (int32_t e = 0; e < n; e++) {
        int rc = axg_quad_geometry(mapping, nodal_sz + (size_t)e * 8, axial[e],
                                   out_geometry + (size_t)e * 150,
                                   out_sz ? out_sz + (size_t)e * 50 : nullptr);
        if (rc != AXG_OK) return rc;
    }
    return AXG_OK;
}

// Quad::computeDt (Quad.cpp:271-349) for a 1-D element: min neighbour distance / vmax
int axg_quad_dt(const double *sz, double vmax, double *dt) {
    if (!sz || !dt || !(vmax > 0)) return AXG_E_ARG;
    double hmin = std::numeric_limits<double>::max();
    for (int p0 = 0; p0 < 24; p0++) {
        int i0 = p0 / 5, j0 = p0 % 5;
        for (int p1 = p0 + 1; p1 < 25; p1++) {
            int i1 = p1 / 5, j1 = p1 % 5;
            if (std::abs(i1 - i0) <= 1 && std::abs(j1 - j0) <= 1)
                hmin = std::min(hmin, std::hypot(sz[p1] - sz[p0], sz[25 + p1] - sz[25 + p0]));
        }
    }
    *dt = hmin / vmax;
    return AXG_OK;
}

// AttBuilder::setAlphaBetaGamma (AttBuilder.cpp:183-198)
int axg_att_alpha_beta_gamma(int32_t nsls, const double *w, const double *y, double dt,
                             double *alpha, double *beta, double *gamma) {
    if (nsls <= 0 || nsls > AXG_MAX_SLS) return AXG_E_ARG;
    double ysum = 0;
    for (int i = 0; i < nsls; i++) ysum += y[i];
    for (int i = 0; i < nsls; i++) {
        double yUn = y[i] / ysum, wDt = w[i] * dt;
        alpha[i] = std::exp(-wDt);
        beta[i] = yUn * ((1. - alpha[i]) / wDt - alpha[i]);
        gamma[i] = yUn * ((alpha[i] - 1.) / wDt + 1.);
    }
    return AXG_OK;
}

// AttBuilder::createAttenuation, FULL branch (AttBuilder.cpp:102-178): relaxed
// kappa, mu -> unrelaxed (in place) and dkappa, dmu per sample
int axg_att_moduli(int32_t nsls, const double *w, const double *y, double fmin, double fmax,
                   double fref, int32_t n, const double *qkappa, const double *qmu, double *kp,
                   double *mu, double *dkp, double *dmu) {
    if (nsls <= 0 || nsls > AXG_MAX_SLS || n < 0) return AXG_E_ARG;
    const double pi = M_PI;
    double ysum = 0;
    for (int i = 0; i < nsls; i++) ysum += y[i];
    double w0 = fref * (2 * pi);
    double w1 = std::sqrt(fmin * fmax) * (2. * pi);
    double w10f = 2. * std::log(w1 / w0) / pi;
    double fact = 0;
    for (int i = 0; i < nsls; i++) fact += y[i] * w[i] * w[i] / (w[i] * w[i] + w1 * w1);
    fact /= ysum;
    for (int k = 0; k < n; k++) {
        double kpNA = 1. + w10f / qkappa[k];
        double dk = kpNA / (qkappa[k] / ysum + (1. - fact));
        double kpAT = kpNA + dk * fact;
        double muNA = 1. + w10f / qmu[k];
        double dm = muNA / (qmu[k] / ysum + (1. - fact));
        double muAT = muNA + dm * fact;
        dkp[k] = dk * kp[k];
        dmu[k] = dm * mu[k];
        kp[k] *= kpAT;
        mu[k] *= muAT;
    }
    return AXG_OK;
}

}  // extern "C"
