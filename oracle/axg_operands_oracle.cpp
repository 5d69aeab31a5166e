// axg_operands_oracle.cpp -- TEST INFRASTRUCTURE: the oracle's own restatement of the
// preloop numbers the stiffness loop consumes, written independently of the engine's
// operand builder (axisem3d_b200/csrc/operands.cpp) so that a parity test can see an error
// in either. Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
//
// It follows the reference's classes, kept in their shape (a Mapping with mapping() and
// jacobian() over a 2 x 4 nodal matrix, a 2 x 2 Jacobian with its determinant):
//   Mapping / MappingLinear / MappingSpherical
//       SOLVER/src/preloop/se_model/quad/mapping/{Mapping,MappingLinear,MappingSpherical}.hpp
//   spectrals::getXiEtaElement / getWeightsElement    quad/spectrals.hpp:321-350
//   Quad::computeIntegralFactor                        quad/Quad.cpp:403-435
//   Quad::createGradient (Jacobian inverse, 1/s)       quad/Quad.hpp:155-184
//   Quad::computeDt (neighbour distances / vmax)       quad/Quad.cpp:271-349
//   AttBuilder::setAlphaBetaGamma                      quad/physical/AttBuilder.cpp:183-198
//   AttBuilder::createAttenuation (FULL moduli)        quad/physical/AttBuilder.cpp:102-178
// The GLL / GLJ tables come from the caller (oracle/spectral.py derives them from their
// definitions; tests pin them to the reference's 12-decimal values).
#include <cmath>
#include <limits>
#include <memory>
#include <stdexcept>

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

struct Col2 {
    double v[2];
    double &operator()(int i) { return v[i]; }
    double operator()(int i) const { return v[i]; }
};

struct Mat22 {
    double m[2][2];
    double &operator()(int i, int j) { return m[i][j]; }
    double operator()(int i, int j) const { return m[i][j]; }
    double determinant() const { return m[0][0] * m[1][1] - m[0][1] * m[1][0]; }
    Mat22 transpose() const { return {{{m[0][0], m[1][0]}, {m[0][1], m[1][1]}}}; }
};

Mat22 mul(const Mat22 &a, const Mat22 &b) {
    Mat22 c;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) c(i, j) = a(i, 0) * b(0, j) + a(i, 1) * b(1, j);
    return c;
}

Col2 mul(const Mat22 &a, const Col2 &x) {
    return {{a(0, 0) * x(0) + a(0, 1) * x(1), a(1, 0) * x(0) + a(1, 1) * x(1)}};
}

// nodal (s, z) as the reference's DMat24: column k is node k
struct Mat24 {
    double m[2][4];
};

// ---------------------------------------------------------------- Mapping ---
class Mapping {
public:
    explicit Mapping(const Mat24 &nodal) : mNodalSZ(nodal) {
        double len[4];
        for (int k = 0; k < 4; k++) {
            const int k1 = (k + 1) % 4;
            const double ds = nodal.m[0][k] - nodal.m[0][k1], dz = nodal.m[1][k] - nodal.m[1][k1];
            len[k] = std::sqrt(ds * ds + dz * dz);
        }
        mMinEdgeLength = std::fmin(std::fmin(len[0], len[1]), std::fmin(len[2], len[3]));
    }
    virtual ~Mapping() = default;
    virtual Col2 mapping(const Col2 &xieta) const = 0;
    virtual Mat22 jacobian(const Col2 &xieta) const = 0;

protected:
    static int cycle4(int p) { return p > 3 ? p - 4 : (p < 0 ? p + 4 : p); }
    static void makeAnglesClose(double &a, double &b) {
        if (a - b > kPi) b += 2. * kPi;
        if (b - a > kPi) a += 2. * kPi;
    }
    static Mat22 orthogQ2(int c) {
        static const Mat22 Q[4] = {{{{-1., 0.}, {0., -1.}}},
                                   {{{0., -1.}, {1., 0.}}},
                                   {{{1., 0.}, {0., 1.}}},
                                   {{{0., 1.}, {-1., 0.}}}};
        return Q[c];
    }
    // Mapping::rotateQ2: nodes and (xi, eta) rotated so that the curved outer edge is edge 2,
    // then (r, angle from the z axis) of every node (geodesy::xy2sphi, undefined = 0)
    void rotateQ2(const Col2 &xieta, double rt[2][4], Col2 &xietaQ2) const {
        const Mat22 Q = orthogQ2(mCurvedOuter);
        for (int k = 0; k < 4; k++) {
            const Col2 n = mul(Q, Col2{{mNodalSZ.m[0][k], mNodalSZ.m[1][k]}});
            rt[0][k] = std::sqrt(n(0) * n(0) + n(1) * n(1));
            const double eps = std::numeric_limits<double>::epsilon();
            const double phi = (std::fabs(n(0)) < eps && std::fabs(n(1)) < eps) ? 0. : std::atan2(n(1), n(0));
            rt[1][k] = kPi * .5 - phi;
        }
        xietaQ2 = mul(Q, xieta);
    }

    Mat24 mNodalSZ;
    double mMinEdgeLength = 0.;
    int mCurvedOuter = -1;
};

class MappingLinear : public Mapping {
public:
    using Mapping::Mapping;
    Col2 mapping(const Col2 &xieta) const override {
        const double xip = 1. + xieta(0), xim = 1. - xieta(0), etp = 1. + xieta(1), etm = 1. - xieta(1);
        const double shp[4] = {xim * etm, xip * etm, xip * etp, xim * etp};
        Col2 sz{{0., 0.}};
        for (int r = 0; r < 2; r++) {
            for (int k = 0; k < 4; k++) sz(r) += mNodalSZ.m[r][k] * shp[k];
            sz(r) *= .25;
        }
        return sz;
    }
    Mat22 jacobian(const Col2 &xieta) const override {
        const double xip = 1. + xieta(0), xim = 1. - xieta(0), etp = 1. + xieta(1), etm = 1. - xieta(1);
        const double dshp[2][4] = {{-etm, etm, etp, -etp}, {-xim, -xip, xip, xim}};
        Mat22 J{{{0., 0.}, {0., 0.}}};
        for (int r = 0; r < 2; r++)
            for (int c = 0; c < 2; c++) {
                for (int k = 0; k < 4; k++) J(r, c) += mNodalSZ.m[r][k] * dshp[c][k];
                J(r, c) *= .25;
            }
        return J;
    }
};

class MappingSpherical : public Mapping {
public:
    explicit MappingSpherical(const Mat24 &nodal) : Mapping(nodal) {
        double r[4];
        for (int k = 0; k < 4; k++) r[k] = std::sqrt(nodal.m[0][k] * nodal.m[0][k] + nodal.m[1][k] * nodal.m[1][k]);
        const double tol = mMinEdgeLength * 1e-3;
        if (std::fabs(r[0] - r[1]) < tol && std::fabs(r[2] - r[3]) < tol) {
            mCurvedOuter = r[2] > r[0] ? 2 : 0;
        } else if (std::fabs(r[1] - r[2]) < tol && std::fabs(r[3] - r[0]) < tol) {
            mCurvedOuter = r[3] > r[1] ? 3 : 1;
        } else {
            throw std::runtime_error("MappingSpherical::MappingSpherical || Error identifying curved outer edge.");
        }
    }
    Col2 mapping(const Col2 &xieta) const override {
        double r0, r2, t0, t1, t2, t3, xi, eta;
        coordsQ2(xieta, r0, r2, t0, t1, t2, t3, xi, eta);
        const double t01 = ((1. - xi) * t0 + (1. + xi) * t1) * .5;
        const double t32 = ((1. - xi) * t3 + (1. + xi) * t2) * .5;
        const double r0m = (1. - eta) * r0 * .5, r2p = (1. + eta) * r2 * .5;
        const Col2 sz{{r0m * std::sin(t01) + r2p * std::sin(t32), r0m * std::cos(t01) + r2p * std::cos(t32)}};
        return mul(orthogQ2(mCurvedOuter).transpose(), sz);
    }
    Mat22 jacobian(const Col2 &xieta) const override {
        double r0, r2, t0, t1, t2, t3, xi, eta;
        coordsQ2(xieta, r0, r2, t0, t1, t2, t3, xi, eta);
        const double t01 = ((1. - xi) * t0 + (1. + xi) * t1) * .5;
        const double t32 = ((1. - xi) * t3 + (1. + xi) * t2) * .5;
        const double r0m = (1. - eta) * r0 * .5, r2p = (1. + eta) * r2 * .5;
        const double t01_xi = (t1 - t0) * .5, t32_xi = (t2 - t3) * .5;
        const double r0m_eta = -r0 * .5, r2p_eta = r2 * .5;
        Mat22 J;
        J(0, 0) = r0m * std::cos(t01) * t01_xi + r2p * std::cos(t32) * t32_xi;
        J(1, 0) = (r0m * std::sin(t01) * t01_xi + r2p * std::sin(t32) * t32_xi) * (-1.);
        J(0, 1) = r0m_eta * std::sin(t01) + r2p_eta * std::sin(t32);
        J(1, 1) = r0m_eta * std::cos(t01) + r2p_eta * std::cos(t32);
        const Mat22 Q = orthogQ2(mCurvedOuter);
        return mul(mul(Q.transpose(), J), Q);
    }

private:
    void coordsQ2(const Col2 &xieta, double &r0, double &r2, double &t0, double &t1, double &t2,
                  double &t3, double &xi, double &eta) const {
        double rt[2][4];
        Col2 xq;
        rotateQ2(xieta, rt, xq);
        r0 = rt[0][cycle4(mCurvedOuter - 2)];
        r2 = rt[0][cycle4(mCurvedOuter + 0)];
        t0 = rt[1][cycle4(mCurvedOuter - 2)];
        t1 = rt[1][cycle4(mCurvedOuter - 1)];
        t2 = rt[1][cycle4(mCurvedOuter + 0)];
        t3 = rt[1][cycle4(mCurvedOuter + 1)];
        xi = xq(0);
        eta = xq(1);
        makeAnglesClose(t3, t2);
        makeAnglesClose(t0, t1);
    }
};

// ------------------------------------------------------------------- Quad ---
// tables in the reference's order: positions and weights of GLL and GLJ (5 each)
struct Tables {
    double pGLL[5], pGLJ[5], wGLL[5], wGLJ[5];
};

// Quad::computeIntegralFactor + Quad::createGradient for one quad: geometry [6][25] =
// dsdxii, dsdeta, dzdxii, dzdeta, inv_s, ifact; sz [2][25]
void quad_geometry(const Mapping &map, bool axial, const Tables &t, double *g, double *szo) {
    for (int ipol = 0; ipol < 5; ipol++)
        for (int jpol = 0; jpol < 5; jpol++) {
            const int ipnt = ipol * 5 + jpol;
            // spectrals::getXiEtaElement / getWeightsElement (row-major weight matrix)
            const Col2 xieta{{axial ? t.pGLJ[ipol] : t.pGLL[ipol], t.pGLL[jpol]}};
            const double weight = (axial ? t.wGLJ[ipol] : t.wGLL[ipol]) * t.wGLL[jpol];
            const Mat22 J = map.jacobian(xieta);
            double ifact = weight * J.determinant();
            const Col2 sz = map.mapping(xieta);
            const double s = sz(0);
            if (axial) {
                if (ipnt / 5 == 0) ifact *= J(0, 0);            // L'Hospital on the axis
                else ifact *= s / (1. + xieta(0));
            } else {
                ifact *= s;
            }
            const double detJ = J.determinant();
            g[0 * 25 + ipnt] = J(0, 0) / detJ;
            g[1 * 25 + ipnt] = -J(0, 1) / detJ;
            g[2 * 25 + ipnt] = -J(1, 0) / detJ;
            g[3 * 25 + ipnt] = J(1, 1) / detJ;
            g[4 * 25 + ipnt] = (axial && ipol == 0) ? 0. : 1. / s;
            g[5 * 25 + ipnt] = ifact;
            if (szo) {
                szo[ipnt] = sz(0);
                szo[25 + ipnt] = sz(1);
            }
        }
}

}  // namespace

extern "C" {

// Quad geometry of n quads: mapping 0 = linear, 1 = spherical; nodal [n][8] (s0 z0 ... s3 z3);
// tables = pGLL, pGLJ, wGLL, wGLJ (20 doubles). Returns 0, or -1 (bad mapping / curved
// outer edge not found, the reference's exception).
int axo_quad_geometry_batch(int n, int mapping, const double *nodal, const unsigned char *axial,
                            const double *tables, double *geometry, double *sz) {
    Tables t;
    for (int i = 0; i < 5; i++) {
        t.pGLL[i] = tables[i];
        t.pGLJ[i] = tables[5 + i];
        t.wGLL[i] = tables[10 + i];
        t.wGLJ[i] = tables[15 + i];
    }
    try {
        for (int e = 0; e < n; e++) {
            Mat24 nd;
            for (int k = 0; k < 4; k++) {
                nd.m[0][k] = nodal[(size_t)e * 8 + 2 * k];
                nd.m[1][k] = nodal[(size_t)e * 8 + 2 * k + 1];
            }
            std::unique_ptr<Mapping> map;
            if (mapping == 0) map = std::make_unique<MappingLinear>(nd);
            else if (mapping == 1) map = std::make_unique<MappingSpherical>(nd);
            else return -1;
            quad_geometry(*map, axial[e] != 0, t, geometry + (size_t)e * 150, sz ? sz + (size_t)e * 50 : nullptr);
        }
    } catch (const std::exception &) {
        return -1;
    }
    return 0;
}

// Quad::computeDt for one reference configuration (one slice): the smallest distance
// between neighbouring GLL points (|di| <= 1 and |dj| <= 1) over vmax; sz [2][25]
int axo_quad_dt(const double *sz, double vmax, double *dt) {
    double hmin = std::numeric_limits<double>::max();
    for (int ipnt0 = 0; ipnt0 < 25 - 1; ipnt0++) {
        const int ipol0 = ipnt0 / 5, jpol0 = ipnt0 % 5;
        for (int ipnt1 = ipnt0 + 1; ipnt1 < 25; ipnt1++) {
            const int ipol1 = ipnt1 / 5, jpol1 = ipnt1 % 5;
            if (std::abs(ipol1 - ipol0) <= 1 && std::abs(jpol1 - jpol0) <= 1) {
                const double ds = sz[ipnt1] - sz[ipnt0], dz = sz[25 + ipnt1] - sz[25 + ipnt0];
                hmin = std::fmin(hmin, std::sqrt(ds * ds + dz * dz));
            }
        }
    }
    *dt = hmin / vmax;
    return 0;
}

// AttBuilder::setAlphaBetaGamma: y normalised by its sum, then per SLS
// alpha = exp(-w dt), beta = y (( 1 - alpha) / (w dt) - alpha), gamma = y ((alpha - 1) / (w dt) + 1)
int axo_att_alpha_beta_gamma(int nsls, const double *w, const double *y, double dt, double *alpha,
                             double *beta, double *gamma) {
    double sumY = 0.;
    for (int i = 0; i < nsls; i++) sumY += y[i];
    for (int i = 0; i < nsls; i++) {
        const double yi = y[i] / sumY, wdt = w[i] * dt;
        alpha[i] = std::exp(-wdt);
        beta[i] = yi * ((1. - alpha[i]) / wdt - alpha[i]);
        gamma[i] = yi * ((alpha[i] - 1.) / wdt + 1.);
    }
    return 0;
}

// AttBuilder::createAttenuation, FULL: relaxed kappa, mu (in place) -> unrelaxed, with the
// SLS modulus defects dkappa, dmu of each sample
int axo_att_moduli(int nsls, const double *w, const double *y, double fmin, double fmax, double fref,
                   int n, const double *qkappa, const double *qmu, double *kappa, double *mu,
                   double *dkappa, double *dmu) {
    double sumY = 0.;
    for (int i = 0; i < nsls; i++) sumY += y[i];
    const double w0 = fref * (2. * kPi);
    const double w1 = std::sqrt(fmin * fmax) * (2. * kPi);
    const double logTerm = 2. * std::log(w1 / w0) / kPi;
    double ws = 0.;
    for (int i = 0; i < nsls; i++) ws += y[i] * w[i] * w[i] / (w[i] * w[i] + w1 * w1);
    ws /= sumY;
    for (int k = 0; k < n; k++) {
        const double fk = 1. + logTerm / qkappa[k];
        const double dk = fk / (qkappa[k] / sumY + (1. - ws));
        const double fm = 1. + logTerm / qmu[k];
        const double dm = fm / (qmu[k] / sumY + (1. - ws));
        dkappa[k] = dk * kappa[k];
        dmu[k] = dm * mu[k];
        kappa[k] *= fk + dk * ws;
        mu[k] *= fm + dm * ws;
    }
    return 0;
}

}  // extern "C"
