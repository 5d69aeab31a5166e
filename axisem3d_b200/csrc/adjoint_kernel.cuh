// adjoint_kernel.cuh -- the time-reversed adjoint of the elastic time step.
//
// The reference has no adjoint (no sensitivity kernels, no checkpointing); this is
// the discrete adjoint of the forward loop the engine runs (NewmarkTimeScheme::solve,
// SOLVER/src/core/time/NewmarkTimeScheme.cpp:41-108), for isotropic elements whose
// moduli are constant in phi (the in-Fourier path), without attenuation.
//
// Forward step n:   a_n = M^-1 P (F_n - K u_n)
//                   v_{n+1} = v_n + h/2 (a_{n-1} + a_n)
//                   u_{n+1} = u_n + h v_{n+1} + h^2/2 a_n
//                   seismograms d_n = R u_n
// with P the (symmetric) axial / Nyquist projection. With phi-constant moduli
// the modes decouple and the quadrature is the Hermitian transpose of the
// gradient with the integral factor (GradientQuadrature.hpp:294-324 vs
// 207-231), so each mode's stiffness block is Hermitian: as a real-linear map
// K^T = K, and the transpose is applied with the forward kernel itself.
// Since u_{n+1} = u_n + h v_n + h^2/2 a_{n-1} + h^2 a_n, a_n enters v_{n+1} with h/2,
// u_{n+1} with h^2, and step n+1 (as its a_{n-1}) with the cotangent abar_out.
// Reverse step n (cotangents ubar, vbar of u_{n+1}, v_{n+1}), real inner products:
//   abar_n  = abar_out + h/2 vbar + h^2 ubar           (total cotangent of a_n)
//   g       = P (M^-1 abar_n)                        (cotangent of the stiffness)
//   ubar_n  = ubar + (-K g) + R^T r_n
//   vbar_n  = vbar + h ubar
//   abar_out' = h/2 vbar + h^2/2 ubar = h/2 vbar_n     (cotangent of a_{n-1})
//   dJ/dM_p     += -<abar_n, a_n>_p / M_p
//   dJ/dlambda  += -sum_a ifact_q Re(conj(tr e(g)) tr e(u_n))
//   dJ/dmu      += -sum_a ifact_q Re(conj(e(g)) . D_mu e(u_n)),  D_mu = diag(2,2,2,1,1,1)
#pragma once

#include "common.cuh"
#include "point_kernels.cuh"
#include "solid_kernel.cuh"

namespace axg {

template <class T>
struct AdjointArgs {
    int n_elem;
    const int *nr, *pts;
    const uint8_t *axial;
    const T *geom;              // [n][10][25]
    const T *mod;               // lambda, mu pool [2][25] per element
    const int64_t *mod_off;
    const int *pt_off, *pt_nu;
    const cx_t<T> *u;           // forward displacement at step n
    const cx_t<T> *g;           // P M^-1 abar_n
    cx_t<T> *out;               // receives -K g (scatter-add)
    const T *ifact;             // [n][25] integral factor
    T *grad;                    // [n][2][25]: dJ/dlambda, dJ/dmu per element point
    const T *gmat;
    // per-slice sensitivities (NULL = off): dJ/dlambda, dJ/dmu at the slices
    // phi_k = 2 pi k / nr of every element point, [2][nr][25] per element from grad3_off
    T *grad3;
    const int64_t *grad3_off;
    const T *tw;                // twiddle pool: for each nr, nr cos then nr sin
    const int *tw_off;
    // wider rheologies (the GENERIC instantiation): per element the rheology code (RHEO_ISO,
    // RHEO_TISO, RHEO_ANISO), the RTZ flag with sin t, cos t, sin 2t, cos 2t per point
    // ([n][4][25]), and the offsets of the element's moduli [nmod][25] in mod (mod_off) and of
    // its sensitivities [nmod][25] in grad (grad_off)
    const int *rheo;
    const uint8_t *rtz;
    const T *trig;
    const int64_t *grad_off;
    // attenuating elements (GENERIC): att code per element (ATT_NONE / ATT_FULL / ATT_CG4), its
    // dlambda, dmu [2][npa] at attmod_off, and its adjoint SLS state at astate_off (complex
    // units): [nsls + 1][6][nu][npa], the cotangents of the memory variables and, last, of the
    // dstress; npa = 25 (FULL) or 4 (CG4)
    const int *att;
    const T *attmod;
    const int64_t *attmod_off;
    cx_t<T> *astate;
    const int64_t *astate_off;
    int nsls;
    T alpha[8], beta[8], gamma[8];
};

// Sensitivities of one (mode, point) of a TI or 21-Cij element: the derivative of
// Re(conj(e(g)) . C e(u)) by each modulus, with P(i, j) = Re(conj(eg_i) eu_j) over the
// engineering (Voigt) strains that stress_tiso / stress_aniso take. TI (A, C, F, L, N):
//   A: (g0 + g1)(u0 + u1)   C: g2 u2   F: (g0 + g1) u2 + g2 (u0 + u1)
//   L: g3 u3 + g4 u4        N: -2 (g0 u1 + g1 u0) + g5 u5
// 21 Cij, upper triangle row by row: P(i, i) on the diagonal, P(i, j) + P(j, i) off it.
template <class T>
__device__ __forceinline__ T pcx(const cx_t<T> &g, const cx_t<T> &u) { return g.x * u.x + g.y * u.y; }
template <class T>
__device__ __forceinline__ void add_sens_tiso(const cx_t<T> eg[6], const cx_t<T> eu[6], T *sG, int q) {
    const cx_t<T> g01 = cadd(eg[0], eg[1]), u01 = cadd(eu[0], eu[1]);
    atomicAdd(&sG[q], pcx<T>(g01, u01));
    atomicAdd(&sG[25 + q], pcx<T>(eg[2], eu[2]));
    atomicAdd(&sG[50 + q], pcx<T>(g01, eu[2]) + pcx<T>(eg[2], u01));
    atomicAdd(&sG[75 + q], pcx<T>(eg[3], eu[3]) + pcx<T>(eg[4], eu[4]));
    atomicAdd(&sG[100 + q], (T)-2 * (pcx<T>(eg[0], eu[1]) + pcx<T>(eg[1], eu[0])) + pcx<T>(eg[5], eu[5]));
}
template <class T>
__device__ __forceinline__ void add_sens_aniso(const cx_t<T> eg[6], const cx_t<T> eu[6], T *sG, int q) {
    int k = 0;
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
        for (int j = i; j < 6; j++, k++)
            atomicAdd(&sG[k * 25 + q], i == j ? pcx<T>(eg[i], eu[i]) : pcx<T>(eg[i], eu[j]) + pcx<T>(eg[j], eu[i]));
}

// The per-slice sensitivities. A 3-D element's stress at slice k is C(phi_k) e(phi_k) with the
// strain slices e(phi_k) = C2R(e) and the stress modes R2C(sigma) (SolverFFTW conventions), so
// the derivative of -<g, K u> by a modulus at (slice k, point q) is
//     -ifact_q / nr  sum_d  dsigma_d/dtheta(e_u(phi_k))  y_d(phi_k),
//     y(phi_k) = Re E_0 + sum_{0 < a < nu} w_a Re(E_a e^{i a phi_k}),  w_a = 1/2 at a = nr/2,
// E = e(g), the real adjoint of R2C at slice k: the conjugate-transpose sum with the R2C rules
// (imaginary part of mode 0 dropped, the Nyquist mode halved). At phi-constant moduli with odd
// nr a 3-D element equals the 1-D one, and these values are the gradient of the 3-D
// parameterisation of the same step; their sum over the slices is the 1-D gradient.
template <class T>
__device__ __forceinline__ void slice_sums(const cx_t<T> *E, int nu, int nr, int k, const T *cs, const T *sn,
                                           T &c2r, T &adj) {
    // c2r = C2R(E)(phi_k) = Re E_0 + 2 sum_a Re(E_a e^{i a phi_k}); adj = y(phi_k)
    T sum = 0, half = 0;
    int j = 0;
    for (int al = 1; al < nu; al++) {
        j += k;
        j = j >= nr ? j - nr : j;
        const T v = E[al * 150].x * cs[j] - E[al * 150].y * sn[j];
        if (2 * al == nr) half += v;
        else sum += v;
    }
    c2r = E[0].x + (T)2 * (sum + half);
    adj = E[0].x + sum + (T)0.5 * half;
}

// strains of one element field at (mode al, point q) from U[a][c][25] in shared memory
template <class T>
__device__ __forceinline__ void strain_at(const cx_t<T> *U, int al, int q, bool axial, const T *Gxi,
                                          const T *sGll, const T *geo, cx_t<T> eps[6]) {
    using C = cx_t<T>;
    const int ii = q / 5, jj = q - ii * 5;
    const T *dsdxii = geo, *dsdeta = geo + 25, *dzdxii = geo + 50, *dzdeta = geo + 75, *invs = geo + 100;
    C X[3], Y[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        C x = mk<T>(0, 0), y = mk<T>(0, 0);
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const T gx = Gxi[k * 5 + ii], gy = sGll[k * 5 + jj];
            const C uc = U[c * 25 + k * 5 + jj], ur = U[c * 25 + ii * 5 + k];
            x.x += gx * uc.x; x.y += gx * uc.y;
            y.x += ur.x * gy; y.y += ur.y * gy;
        }
        X[c] = x; Y[c] = y;
    }
    const T ze = dzdeta[q], zx = dzdxii[q], se = dsdeta[q], sx = dsdxii[q];
    eps[0] = cadd(cscale(X[0], ze), cscale(Y[0], zx));
    eps[4] = cadd(cscale(X[0], se), cscale(Y[0], sx));
    eps[5] = cadd(cscale(X[1], ze), cscale(Y[1], zx));
    eps[3] = cadd(cscale(X[1], se), cscale(Y[1], sx));
    const C e1t = cadd(cscale(X[2], ze), cscale(Y[2], zx));
    eps[2] = cadd(cscale(X[2], se), cscale(Y[2], sx));
    eps[4] = cadd(eps[4], e1t);
    const T alf = (T)al;
    const C A0 = csub(cia(alf, U[q]), U[25 + q]);
    const C A1 = cadd(cia(alf, U[25 + q]), U[q]);
    const C A2 = cia(alf, U[50 + q]);
    const T is = invs[q];
    eps[5] = cadd(eps[5], cscale(A0, is));
    eps[1] = cscale(A1, is);
    eps[3] = cadd(eps[3], cscale(A2, is));
    if (axial && ii == 0) {
        C ax[3], ay[3];
#pragma unroll
        for (int c = 0; c < 3; c++) { ax[c] = mk<T>(0, 0); ay[c] = mk<T>(0, 0); }
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const T gx = Gxi[k * 5 + 0], gy = sGll[k * 5 + jj];
            const C v0 = U[k * 5 + jj], v1 = U[25 + k * 5 + jj], v2 = U[50 + k * 5 + jj];
            const C w0 = U[k], w1 = U[25 + k], w2 = U[50 + k];
            C a0 = csub(cia(alf, v0), v1), a1 = cadd(cia(alf, v1), v0), a2 = cia(alf, v2);
            C b0 = csub(cia(alf, w0), w1), b1 = cadd(cia(alf, w1), w0), b2 = cia(alf, w2);
            ax[0] = cadd(ax[0], cscale(a0, gx)); ax[1] = cadd(ax[1], cscale(a1, gx));
            ax[2] = cadd(ax[2], cscale(a2, gx));
            ay[0] = cadd(ay[0], cscale(b0, gy)); ay[1] = cadd(ay[1], cscale(b1, gy));
            ay[2] = cadd(ay[2], cscale(b2, gy));
        }
        eps[5] = cadd(eps[5], cadd(cscale(ax[0], ze), cscale(ay[0], zx)));
        eps[1] = cadd(cscale(ax[1], ze), cscale(ay[1], zx));
        eps[3] = cadd(eps[3], cadd(cscale(ax[2], ze), cscale(ay[2], zx)));
    }
}

// one CTA (team of blockDim.x threads) per element: -K g scattered to `out`, and the
// lambda / mu sensitivities of this step accumulated into grad
// SLICES: the instantiation that also accumulates the per-slice sensitivities (a.grad3); the
// other holds none of that code, so it costs the plain adjoint no registers
// GENERIC: the instantiation for models holding TI or 21-Cij elements (moduli and
// sensitivities per element at mod_off / grad_off, RTZ frames); the isotropic one keeps its
// lambda / mu layout. GENERIC is not combined with SLICES.
template <class T, bool SLICES, bool GENERIC = false>
__global__ void __launch_bounds__(256) adjoint_stiffness_kernel(const AdjointArgs<T> a, const int nu_max) {
    static_assert(!(SLICES && GENERIC), "per-slice sensitivities are isotropic only");
    using C = cx_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T sGll[25], sGlj[25], sGeo[250];
    __shared__ int sOff[25], sNu[25];
    __shared__ T sGl[25], sGm[25];
    __shared__ T sGx[GENERIC ? 23 * 25 : 1];   // GENERIC: per (modulus, point) sums
    C *Ug = reinterpret_cast<C *>(smem_raw);            // [nu][3][25] g, then A terms
    C *Uu = Ug + (size_t)nu_max * 75;                    // [nu][3][25] u
    C *S = Uu + (size_t)nu_max * 75;                     // [nu][6][25] stress of g, then X/Y
    C *Eg = S + (size_t)nu_max * 150;                    // per-slice sensitivities only:
    C *Eu = Eg + (size_t)nu_max * 150;                   // [nu][6][25] strains of g and of u
    for (int i = threadIdx.x; i < 25; i += blockDim.x) {
        sGll[i] = a.gmat[i];
        sGlj[i] = a.gmat[25 + i];
    }
    for (int e = blockIdx.x; e < a.n_elem; e += gridDim.x) {
        const int nr = a.nr[e], nu = nr / 2 + 1;
        const bool axial = a.axial[e] != 0;
        __syncthreads();
        for (int i = threadIdx.x; i < 250; i += blockDim.x) sGeo[i] = a.geom[(size_t)e * 250 + i];
        for (int i = threadIdx.x; i < 25; i += blockDim.x) {
            const int p = a.pts[(size_t)e * 25 + i];
            sOff[i] = a.pt_off[p];
            sNu[i] = a.pt_nu[p];
            sGl[i] = 0;
            sGm[i] = 0;
        }
        if constexpr (GENERIC)
            for (int i = threadIdx.x; i < 23 * 25; i += blockDim.x) sGx[i] = 0;
        __syncthreads();
        const T *Gxi = axial ? sGlj : sGll;
        for (int i = threadIdx.x; i < nu * 25; i += blockDim.x) {
            const int q = i / nu, al = i - q * nu;
            C g0 = mk<T>(0, 0), g1 = g0, g2 = g0, u0 = g0, u1 = g0, u2 = g0;
            if (al < sNu[q]) {
                const size_t o = (size_t)(sOff[q] + al) * 3;
                g0 = a.g[o]; g1 = a.g[o + 1]; g2 = a.g[o + 2];
                u0 = a.u[o]; u1 = a.u[o + 1]; u2 = a.u[o + 2];
            }
            Ug[(al * 3 + 0) * 25 + q] = g0; Ug[(al * 3 + 1) * 25 + q] = g1; Ug[(al * 3 + 2) * 25 + q] = g2;
            Uu[(al * 3 + 0) * 25 + q] = u0; Uu[(al * 3 + 1) * 25 + q] = u1; Uu[(al * 3 + 2) * 25 + q] = u2;
        }
        __syncthreads();
        const T *mod = a.mod + a.mod_off[e];
        for (int i = threadIdx.x; i < nu * 25; i += blockDim.x) {
            const int al = i / 25, q = i - al * 25;
            C eg[6], eu[6], sg[6];
            strain_at<T>(Ug + al * 75, al, q, axial, Gxi, sGll, sGeo, eg);
            strain_at<T>(Uu + al * 75, al, q, axial, Gxi, sGll, sGeo, eu);
            if constexpr (GENERIC) {
                // the forward rheology (elastic_at), in the RTZ frame where the element asks:
                // sigma = R^T C R e with R = spz_to_rtz6 and R^T = rtz_to_spz6, so each mode's
                // block stays Hermitian and the sensitivities are those of the RTZ strains
                const int rh = a.rheo[e];
                const bool rtz = a.rtz[e] != 0;
                T s1 = 0, c1 = 1, s2 = 0, c2 = 1;
                if (rtz) {
                    const T *tr = a.trig + (size_t)e * 100;
                    s1 = tr[q]; c1 = tr[25 + q]; s2 = tr[50 + q]; c2 = tr[75 + q];
                    spz_to_rtz6(eg, s1, c1, s2, c2);
                    spz_to_rtz6(eu, s1, c1, s2, c2);
                }
                if (rh == RHEO_ISO) {
                    stress_iso(eg, sg, mod[q], mod[25 + q]);
                    const C tg = cadd(cadd(eg[0], eg[1]), eg[2]), tu = cadd(cadd(eu[0], eu[1]), eu[2]);
                    T pm = 0;
#pragma unroll
                    for (int d = 0; d < 6; d++) pm += (d < 3 ? (T)2 : (T)1) * pcx<T>(eg[d], eu[d]);
                    atomicAdd(&sGx[q], pcx<T>(tg, tu));
                    atomicAdd(&sGx[25 + q], pm);
                } else if (rh == RHEO_TISO) {
                    stress_tiso(eg, sg, mod[q], mod[25 + q], mod[50 + q], mod[75 + q], mod[100 + q]);
                    add_sens_tiso<T>(eg, eu, sGx, q);
                } else {
                    T cm[21];
#pragma unroll
                    for (int k = 0; k < 21; k++) cm[k] = mod[k * 25 + q];
                    stress_aniso(eg, sg, cm);
                    add_sens_aniso<T>(eg, eu, sGx, q);
                }
                const int at = a.att[e];
                const int k4 = at == ATT_CG4 ? cg4_slot(q) : q;
                if (at != ATT_NONE && k4 >= 0) {
                    // the reverse SLS recursion. Forward (AttenuationFull::apply, in the frame of
                    // the elastic stress): sigma_n = C e_n - sum_l m_l^n,
                    // m_l^{n+1} = alpha_l m_l^n + beta_l d^n + gamma_l D e_n, d^{n+1} = D e_n, with
                    // D = iso(dlambda, dmu). With the cotangents divided by the integral factor
                    // (mb_l of m_l, db of d, held per slot from step n+1): z = sum_l gamma_l mb_l
                    // + db enters the stress of g as sigma = C e(g) - D z, then db <- sum_l
                    // beta_l mb_l and mb_l <- alpha_l mb_l + e(g); dJ/d(dlambda, dmu) gains
                    // +ifact Re(conj(z) . dD e(u_n)).
                    const int npa = at == ATT_CG4 ? 4 : 25;
                    const size_t ns = (size_t)nu * npa, sl = (size_t)al * npa + k4;
                    C *st = a.astate + a.astate_off[e];
                    const T *am = a.attmod + a.attmod_off[e];
                    C z[6], dn[6], dz[6];
#pragma unroll
                    for (int d = 0; d < 6; d++) {
                        z[d] = st[((size_t)a.nsls * 6 + d) * ns + sl];
                        dn[d] = mk<T>(0, 0);
                    }
                    for (int l = 0; l < a.nsls; l++) {
                        const T al_ = a.alpha[l], be = a.beta[l], ga = a.gamma[l];
#pragma unroll
                        for (int d = 0; d < 6; d++) {
                            C &mv = st[((size_t)l * 6 + d) * ns + sl];
                            const C m = mv;
                            z[d] = cadd(z[d], cscale(m, ga));
                            dn[d] = cadd(dn[d], cscale(m, be));
                            mv = cadd(cscale(m, al_), eg[d]);
                        }
                    }
#pragma unroll
                    for (int d = 0; d < 6; d++) st[((size_t)a.nsls * 6 + d) * ns + sl] = dn[d];
                    stress_iso(z, dz, am[k4], am[npa + k4]);
#pragma unroll
                    for (int d = 0; d < 6; d++) sg[d] = csub(sg[d], dz[d]);
                    const int nm = rh == RHEO_ISO ? 2 : rh == RHEO_TISO ? 5 : 21;
                    const C tz = cadd(cadd(z[0], z[1]), z[2]), tu = cadd(cadd(eu[0], eu[1]), eu[2]);
                    T pm = 0;
#pragma unroll
                    for (int d = 0; d < 6; d++) pm += (d < 3 ? (T)2 : (T)1) * pcx<T>(z[d], eu[d]);
                    atomicAdd(&sGx[nm * 25 + q], -pcx<T>(tz, tu));
                    atomicAdd(&sGx[(nm + 1) * 25 + q], -pm);
                }
                if (rtz) rtz_to_spz6(sg, s1, c1, s2, c2);
#pragma unroll
                for (int d = 0; d < 6; d++) S[(al * 6 + d) * 25 + q] = sg[d];
            } else {
                const T lam = mod[q], mu = mod[25 + q];
                stress_iso(eg, sg, lam, mu);
#pragma unroll
                for (int d = 0; d < 6; d++) S[(al * 6 + d) * 25 + q] = sg[d];
                if constexpr (SLICES) {
#pragma unroll
                    for (int d = 0; d < 6; d++) {
                        Eg[(al * 6 + d) * 25 + q] = eg[d];
                        Eu[(al * 6 + d) * 25 + q] = eu[d];
                    }
                }
                // sensitivities Re(conj(e(g)) . de/dm e(u)), times ifact below
                const C tg = cadd(cadd(eg[0], eg[1]), eg[2]), tu = cadd(cadd(eu[0], eu[1]), eu[2]);
                const T pl = tg.x * tu.x + tg.y * tu.y;
                T pm = 0;
#pragma unroll
                for (int d = 0; d < 6; d++) pm += (d < 3 ? (T)2 : (T)1) * (eg[d].x * eu[d].x + eg[d].y * eu[d].y);
                atomicAdd(&sGl[q], pl);
                atomicAdd(&sGm[q], pm);
            }
        }
        __syncthreads();
        if constexpr (SLICES) {
            const T *cs = a.tw + a.tw_off[nr], *sn = cs + nr;
            T *g3 = a.grad3 + a.grad3_off[e];
            for (int i = threadIdx.x; i < nr * 25; i += blockDim.x) {
                const int k = i / 25, q = i - k * 25;
                T u6[6], y6[6];
#pragma unroll
                for (int d = 0; d < 6; d++) {
                    T c_u, a_u, c_g, a_g;
                    slice_sums<T>(Eu + d * 25 + q, nu, nr, k, cs, sn, c_u, a_u);
                    slice_sums<T>(Eg + d * 25 + q, nu, nr, k, cs, sn, c_g, a_g);
                    u6[d] = c_u;
                    y6[d] = a_g;
                }
                const T f = a.ifact[(size_t)e * 25 + q] / (T)nr;
                const T gl = (u6[0] + u6[1] + u6[2]) * (y6[0] + y6[1] + y6[2]);
                T gm = 0;
#pragma unroll
                for (int d = 0; d < 6; d++) gm += (d < 3 ? (T)2 : (T)1) * u6[d] * y6[d];
                g3[(size_t)k * 25 + q] -= f * gl;
                g3[(size_t)(nr + k) * 25 + q] -= f * gm;
            }
        }
        // quadrature of the stress of g (computeQuad6): pass 1, X/Y in place, A terms in Ug.
        // out == NULL: sensitivities only (models with 3-D elements take -K^T g from the
        // forward kernels)
        if (a.out) {
        const T *dsdxii_if = sGeo + 125, *dsdeta_if = sGeo + 150, *dzdxii_if = sGeo + 175,
                *dzdeta_if = sGeo + 200, *invs_if = sGeo + 225;
        for (int i = threadIdx.x; i < nu * 25; i += blockDim.x) {
            const int al = i / 25, q = i - al * 25;
            C s[6];
#pragma unroll
            for (int d = 0; d < 6; d++) s[d] = S[(al * 6 + d) * 25 + q];
            const T ze = dzdeta_if[q], zx = dzdxii_if[q], se = dsdeta_if[q], sx = dsdxii_if[q];
            C *xy = S + al * 150;
            xy[0 * 25 + q] = cadd(cscale(s[0], ze), cscale(s[4], se));
            xy[1 * 25 + q] = cadd(cscale(s[0], zx), cscale(s[4], sx));
            xy[2 * 25 + q] = cadd(cscale(s[5], ze), cscale(s[3], se));
            xy[3 * 25 + q] = cadd(cscale(s[5], zx), cscale(s[3], sx));
            xy[4 * 25 + q] = cadd(cscale(s[4], ze), cscale(s[2], se));
            xy[5 * 25 + q] = cadd(cscale(s[4], zx), cscale(s[2], sx));
            const T alf = (T)al;
            Ug[(al * 3 + 0) * 25 + q] = csub(cia(alf, s[5]), s[1]);
            Ug[(al * 3 + 1) * 25 + q] = cadd(cia(alf, s[1]), s[5]);
            Ug[(al * 3 + 2) * 25 + q] = cia(alf, s[3]);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nu * 25; i += blockDim.x) {
            const int al = i / 25, q = i - al * 25;
            const int ii = q / 5, jj = q - ii * 5;
            const C *xy = S + al * 150;
            const C *A = Ug + al * 75;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                C g1 = mk<T>(0, 0), g2 = mk<T>(0, 0);
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    const T gx = Gxi[ii * 5 + k], gt = sGll[jj * 5 + k];
                    const C xv = xy[(2 * c) * 25 + k * 5 + jj], yv = xy[(2 * c + 1) * 25 + ii * 5 + k];
                    g1.x += gx * xv.x; g1.y += gx * xv.y;
                    g2.x += yv.x * gt; g2.y += yv.y * gt;
                }
                C fc = cadd(g1, g2);
                fc = csub(fc, cscale(A[c * 25 + q], invs_if[q]));
                if (axial) {
                    fc = csub(fc, cscale(cscale(A[c * 25 + jj], dzdeta_if[jj]), Gxi[ii * 5 + 0]));
                    if (ii == 0) {
                        C b = mk<T>(0, 0);
#pragma unroll
                        for (int k = 0; k < 5; k++) {
                            const C y0 = cscale(A[c * 25 + k], dzdxii_if[k]);
                            const T gt = sGll[jj * 5 + k];
                            b.x += y0.x * gt; b.y += y0.y * gt;
                        }
                        fc = csub(fc, b);
                    }
                }
                if (al < sNu[q]) atomic_add_cx(a.out + (size_t)(sOff[q] + al) * 3 + c, mk<T>(-fc.x, -fc.y));
            }
        }
        }
        __syncthreads();
        // grad (each element belongs to one CTA per launch, so no race): -ifact * products
        if constexpr (GENERIC) {
            const int rh = a.rheo[e];
            const int nm = (rh == RHEO_ISO ? 2 : rh == RHEO_TISO ? 5 : 21) + (a.att[e] != ATT_NONE ? 2 : 0);
            T *gr = a.grad + a.grad_off[e];
            for (int i = threadIdx.x; i < nm * 25; i += blockDim.x) {
                const int q = i % 25;
                gr[i] -= a.ifact[(size_t)e * 25 + q] * sGx[i];
            }
        } else {
            for (int q = threadIdx.x; q < 25; q += blockDim.x) {
                const T f = a.ifact[(size_t)e * 25 + q];
                T *gr = a.grad + (size_t)e * 50;
                gr[q] -= f * sGl[q];
                gr[25 + q] -= f * sGm[q];
            }
        }
    }
}

// Models with 3-D (per-slice) moduli. The element's slice transforms make its stiffness
// self-adjoint in the azimuthally weighted product <a, W b> (w = 1 for mode 0, 2 for the other
// modes, 4 for the Nyquist mode of an even nr, where C2R doubles and R2C halves it), not in the
// plain one, so K^T = W K W^-1: stage 0 forms gw = W^-1 g for the forward kernels, which add
// -K gw to kt; stage 1 adds W kt to ubar and clears kt.
template <class T>
__global__ void adjoint_weight_kernel(int nvals, const int *mode_pt, const int *off, const int *nr,
                                      const cx_t<T> *g, cx_t<T> *gw, cx_t<T> *ubar, cx_t<T> *kt, int stage) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nvals) return;
    const int m = q / 3, p = mode_pt[m], al = m - off[p], n = nr[p];
    const T w = al == 0 ? (T)1 : ((n & 1) == 0 && 2 * al == n) ? (T)4 : (T)2;
    if (stage == 0) {
        gw[q] = mk<T>(g[q].x / w, g[q].y / w);
    } else {
        const cx_t<T> k = kt[q];
        ubar[q] = mk<T>(ubar[q].x + w * k.x, ubar[q].y + w * k.y);
        kt[q] = mk<T>(0, 0);
    }
}

// per point mode: abar_n, dJ/dM, g = P M^-1 abar_n, vbar_n, abar_out'
template <class T>
struct AdjPointArgs {
    int nmodes;
    const int *mode_pt, *off, *nr;
    const uint8_t *flags;
    const T *inv_mass1;
    cx_t<T> *ubar, *vbar, *abar_out;   // in: step n+1 cotangents; out: updated
    const cx_t<T> *a_n;                // forward acceleration of step n
    cx_t<T> *g;                        // out
    T *grad_mass;                      // [npoints] dJ/dM
    T h;
};

// One thread per complex value (mode m, component c), blocks of ADJ_POINT_BLOCK threads holding
// whole modes, so that the seven cotangent and field streams move in consecutive words. The
// block shares the scaled cotangents for the axial order-1 rule (which mixes components 0 and 1)
// and the mass terms, which it sums per point before one atomic add per (point, block).
constexpr int ADJ_POINT_BLOCK = 288;   // 96 modes of 3 components
template <class T>
__global__ void __launch_bounds__(ADJ_POINT_BLOCK) adjoint_point_kernel(const AdjPointArgs<T> a) {
    __shared__ cx_t<T> sab[ADJ_POINT_BLOCK];
    __shared__ T sdm[ADJ_POINT_BLOCK];
    const int t = threadIdx.x;
    const int64_t q64 = (int64_t)blockIdx.x * ADJ_POINT_BLOCK + t;
    const bool valid = q64 < (int64_t)a.nmodes * 3;
    const size_t q = valid ? (size_t)q64 : 0;
    const int m = (int)(q / 3), c = (int)(q - (size_t)m * 3);
    const int p = a.mode_pt[m];
    const int off = a.off[p], nr = a.nr[p], nu = nr / 2 + 1, al = m - off;
    const T im = a.inv_mass1[p];
    const T h = a.h;
    cx_t<T> ab = mk<T>(0, 0);
    T dm = 0;
    if (valid) {
        const cx_t<T> ub = a.ubar[q], vb = a.vbar[q], ao = a.abar_out[q];
        const cx_t<T> abn = mk<T>(ao.x + h / 2 * vb.x + h * h * ub.x, ao.y + h / 2 * vb.y + h * h * ub.y);
        const cx_t<T> an = a.a_n[q];
        dm = -(abn.x * an.x + abn.y * an.y) * im;
        ab = cscale(abn, im);
        const cx_t<T> vn = mk<T>(vb.x + h * ub.x, vb.y + h * ub.y);
        a.vbar[q] = vn;
        a.abar_out[q] = mk<T>(h / 2 * vn.x, h / 2 * vn.y);
    }
    sab[t] = ab;
    sdm[t] = dm;
    __syncthreads();
    if (!valid) return;
    // P is symmetric (axial projection and Nyquist rule), so P^T = P: point_bc on the mode,
    // this thread's component
    const int t0 = t - c;   // component 0 of this mode in the block
    cx_t<T> f[3] = {sab[t0], sab[t0 + 1], sab[t0 + 2]};
    point_bc<T>(f, 3, al, nu, nr, a.flags[p], true);
    a.g[q] = f[c];
    // the mass terms of this point's modes in the block, summed by the thread of the first
    if (c == 0 && (al == 0 || t0 == 0)) {
        T sum = 0;
        for (int u = t0; u < ADJ_POINT_BLOCK && (int64_t)blockIdx.x * ADJ_POINT_BLOCK + u < (int64_t)a.nmodes * 3;
             u += 3) {
            if (u != t0 && a.mode_pt[(int)(((int64_t)blockIdx.x * ADJ_POINT_BLOCK + u) / 3)] != p) break;
            sum += sdm[u] + sdm[u + 1] + sdm[u + 2];
        }
        atomicAdd(&a.grad_mass[p], sum);
    }
}

// per-slice mass sensitivities of step n, before adjoint_point_kernel updates the cotangents.
// The axial and Nyquist projection acts on the stiffness before the mass term, so with a 3-D
// mass a(phi_k) = f(phi_k) / M(phi_k) (Mass3D) the derivative by M at slice k of a point is
// -(1/nr) sum_c a_c(phi_k) y_c(phi_k) / M, y = the adjoint R2C sum of abar_n (see slice_sums);
// a grid-stride walk over the (point, slice) pairs, [nr_p] per point from off3
template <class T>
__global__ void adjoint_mass_slices_kernel(int npoints, const int *off, const int *nrp, const int64_t *off3,
                                           const T *inv_mass1, const cx_t<T> *ubar, const cx_t<T> *vbar,
                                           const cx_t<T> *abar_out, const cx_t<T> *a_n, T h, const T *tw,
                                           const int *tw_off, T *gmass3) {
    const int64_t total = off3[npoints];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        // the point of pair i by its slice offsets (binary search)
        int lo = 0, hi = npoints;
        while (hi - lo > 1) {
            const int mid = (lo + hi) / 2;
            if (off3[mid] <= i) lo = mid;
            else hi = mid;
        }
        const int p = lo, nr = nrp[p], nu = nr / 2 + 1, k = (int)(i - off3[p]);
        const T *cs = tw + tw_off[nr], *sn = cs + nr;
        T acc = 0;
        for (int c = 0; c < 3; c++) {
            T sa = 0, ha = 0, sy = 0, hy = 0, a0 = 0, y0 = 0;
            int j = 0;
            for (int al = 0; al < nu; al++) {
                const size_t q = (size_t)(off[p] + al) * 3 + c;
                const cx_t<T> ub = ubar[q], vb = vbar[q], ao = abar_out[q], an = a_n[q];
                const cx_t<T> abn = mk<T>(ao.x + h / 2 * vb.x + h * h * ub.x, ao.y + h / 2 * vb.y + h * h * ub.y);
                if (al == 0) { a0 = an.x; y0 = abn.x; continue; }
                j += k;
                j = j >= nr ? j - nr : j;
                const T va = an.x * cs[j] - an.y * sn[j], vy = abn.x * cs[j] - abn.y * sn[j];
                if (2 * al == nr) { ha += va; hy += vy; }
                else { sa += va; sy += vy; }
            }
            const T ak = a0 + (T)2 * (sa + ha), yk = y0 + sy + (T)0.5 * hy;
            acc += ak * yk;
        }
        gmass3[i] -= acc * inv_mass1[p] / (T)nr;
    }
}


// R^T r_n: the seismogram cotangent of step n injected into ubar
template <class T>
__global__ void adjoint_station_kernel(int nst, const int *elem, const T *w, const T *phi, const int *e_nr,
                                       const int *e_pts, const int *pt_off, const int *pt_nu,
                                       const double *r, cx_t<T> *ubar) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nst * 3) return;
    const int s = t / 3, c = t % 3;
    const int e = elem[s], nu = e_nr[e] / 2 + 1;
    const T rv = (T)r[(size_t)s * 3 + c];
    for (int al = 0; al < nu; al++) {
        // seismogram = sum_a Re(z_a x_a), z_0 = 1, z_a = 2 e^{i a phi}: cotangent conj(z_a) rv
        T zr = 1, zi = 0;
        if (al > 0) {
            T sn, cs;
            if constexpr (sizeof(T) == 4) sincosf((T)al * phi[s], &sn, &cs);
            else sincos((T)al * phi[s], &sn, &cs);
            zr = 2 * cs; zi = 2 * sn;
        }
        for (int q = 0; q < 25; q++) {
            const T wq = w[(size_t)s * 25 + q];
            if (wq == (T)0) continue;
            const int p = e_pts[(size_t)e * 25 + q];
            if (al >= pt_nu[p]) continue;
            atomic_add_cx(ubar + (size_t)(pt_off[p] + al) * 3 + c, mk<T>(rv * wq * zr, -rv * wq * zi));
        }
    }
}

}  // namespace axg
