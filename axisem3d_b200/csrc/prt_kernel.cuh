// prt_kernel.cuh -- solid elements with particle relabelling (PRT, undulated geometry).
//
// SolidElement::displToStiff, PRT branch (SOLVER/src/core/element/SolidElement.cpp:113-161):
//   gather u; 9-component gradient (GradientQuadrature::computeGrad9, GradientQuadrature.hpp:181-205);
//   [spherical] CoordTransformSpherical::transformSPZ_RTZ9 (crd/CoordTransformSpherical.hpp:102-141);
//   1-D material and PRT: per Fourier mode PRT::sphericalToUndulated6 (9 -> 6), strainToStress_FR
//     with attenuation, PRT::undulatedToSpherical6 (6 -> 9, J^-1 scaled by |J|) (PRT/PRT.hpp);
//   else: the 9 components to slices (computeC2R), the same three steps per slice with the 1-D or
//     per-slice PRT factors, back to Fourier (computeR2C);
//   transformRTZ_SPZ9; GradientQuadrature::computeQuad9 (GradientQuadrature.hpp:258-292); scatter-add.
// One team per element with every phase in shared memory; these elements are the few under
// topography, so the kernel keeps the simple shared-memory layout of the generic path.
//
// Shared memory per team: geometry 10 x 25 T, trig 4 x 25 T, point tables 3 x 25 int,
// twiddles 2 x nr T, region A 9 x nu x 25 C (gradient, then stress), region B
// max(3 x nu x 25 C, nr x 9 x qc T) (u, then slices, then quadrature A terms).
#pragma once

#include "solid_kernel.cuh"

namespace axg {

template <class T, class AT>
struct PrtArgs {
    SolidArgs<T, AT> s;
    const T *x;                  // pool: per element [8][nsl][25] = X0..X3, X0|J|..X3|J|
    const int64_t *x_off;        // [n] into the pool
    const uint8_t *x3d;          // [n] 1 = PRT factors per slice (nsl = nr), else nsl = 1
};

struct PrtLayout {
    size_t geom, trig, ipt, tw, regA, regB, total;
};

template <class T>
__host__ __device__ inline PrtLayout prt_layout(int nr_max, int qc) {
    PrtLayout L;
    const int nu_max = nr_max / 2 + 1;
    size_t o = 0;
    auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
    L.geom = o; o = al(o + 10 * 25 * sizeof(T));
    L.trig = o; o = al(o + 4 * 25 * sizeof(T));
    L.ipt = o;  o = al(o + 3 * 25 * sizeof(int));
    L.tw = o;   o = al(o + 2 * (size_t)nr_max * sizeof(T));
    L.regA = o; o = al(o + 9 * (size_t)nu_max * 25 * 2 * sizeof(T));
    size_t b1 = 3 * (size_t)nu_max * 25 * 2 * sizeof(T);
    size_t b2 = (size_t)nr_max * 9 * qc * sizeof(T);
    L.regB = o; o = al(o + (b1 > b2 ? b1 : b2));
    L.total = o;
    return L;
}

// PRT::sphericalToUndulated6 (9 -> 6 Voigt)
template <class V, class R>
__device__ __forceinline__ void prt_sph_to_und6(const V g[9], V u[6], R X0, R X1, R X2, R X3) {
    u[0] = cadd(cscale(g[0], X0), cscale(g[2], X1));
    u[1] = cadd(cscale(g[4], X0), cscale(g[5], X2));
    u[2] = cscale(g[8], X3);
    u[3] = cadd(cadd(cscale(g[7], X0), cscale(g[8], X2)), cscale(g[5], X3));
    u[4] = cadd(cadd(cscale(g[6], X0), cscale(g[8], X1)), cscale(g[2], X3));
    u[5] = cadd(cadd(cscale(cadd(g[3], g[1]), X0), cscale(g[5], X1)), cscale(g[2], X2));
}
// PRT::undulatedToSpherical6 (6 -> 9), with the factors scaled by |J|
template <class V, class R>
__device__ __forceinline__ void prt_und_to_sph6(const V u[6], V g[9], R X0, R X1, R X2, R X3) {
    g[0] = cscale(u[0], X0);
    g[1] = cscale(u[5], X0);
    g[2] = cadd(cadd(cscale(u[0], X1), cscale(u[4], X3)), cscale(u[5], X2));
    g[3] = g[1];
    g[4] = cscale(u[1], X0);
    g[5] = cadd(cadd(cscale(u[1], X2), cscale(u[3], X3)), cscale(u[5], X1));
    g[6] = cscale(u[4], X0);
    g[7] = cscale(u[3], X0);
    g[8] = cadd(cadd(cscale(u[2], X3), cscale(u[3], X2)), cscale(u[4], X1));
}
// CoordTransformSpherical::transformSPZ_RTZ9 / transformRTZ_SPZ9 (one point of one mode)
template <bool TO_RTZ, class V, class T>
__device__ __forceinline__ void rtz9(V n[9], T s1, T c1, T s2, T c2) {
    const T half = (T)0.5;
    const V s08 = cadd(n[0], n[8]), d08 = csub(n[0], n[8]);
    const V s26 = cadd(n[2], n[6]), d26 = csub(n[2], n[6]);
    if (TO_RTZ) {
        n[0] = cscale(csub(cadd(s08, cscale(d08, c2)), cscale(s26, s2)), half);
        n[2] = cscale(cadd(cadd(d26, cscale(s26, c2)), cscale(d08, s2)), half);
    } else {
        n[0] = cscale(cadd(cadd(s08, cscale(d08, c2)), cscale(s26, s2)), half);
        n[2] = cscale(csub(cadd(d26, cscale(s26, c2)), cscale(d08, s2)), half);
    }
    n[6] = csub(n[2], d26);
    n[8] = csub(s08, n[0]);
    const V t1 = n[1], t3 = n[3];
    if (TO_RTZ) {
        n[1] = csub(cscale(t1, c1), cscale(n[7], s1));
        n[7] = cadd(cscale(n[7], c1), cscale(t1, s1));
        n[3] = csub(cscale(t3, c1), cscale(n[5], s1));
        n[5] = cadd(cscale(n[5], c1), cscale(t3, s1));
    } else {
        n[1] = cadd(cscale(t1, c1), cscale(n[7], s1));
        n[7] = csub(cscale(n[7], c1), cscale(t1, s1));
        n[3] = cadd(cscale(t3, c1), cscale(n[5], s1));
        n[5] = csub(cscale(n[5], c1), cscale(t3, s1));
    }
}

template <class T, class AT, int RHEO, int ATT, bool IS3D, bool RTZ>
__global__ void __launch_bounds__(256)
solid_prt_kernel(const PrtArgs<T, AT> pa, const int nr_max, const int qc_max, const int teams_per_cta,
                 const size_t team_bytes) {
    using C = cx_t<T>;
    const SolidArgs<T, AT> &a = pa.s;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int TEAM = blockDim.x / teams_per_cta;
    const int team = threadIdx.x / TEAM;
    const int lane = threadIdx.x % TEAM;
    __shared__ T sGll[25], sGlj[25];
    for (int i = threadIdx.x; i < 25; i += blockDim.x) {
        sGll[i] = a.gmat[i];
        sGlj[i] = a.gmat[25 + i];
    }
    __syncthreads();
    if (team >= teams_per_cta) return;
    const PrtLayout L = prt_layout<T>(nr_max, qc_max);
    unsigned char *base = smem_raw + (size_t)team * team_bytes;
    T *sGeo = reinterpret_cast<T *>(base + L.geom);
    T *sTrig = reinterpret_cast<T *>(base + L.trig);
    int *sPt = reinterpret_cast<int *>(base + L.ipt);
    int *sOff = sPt + 25;
    int *sNu = sPt + 50;
    T *sTw = reinterpret_cast<T *>(base + L.tw);
    C *rA = reinterpret_cast<C *>(base + L.regA);
    C *rBc = reinterpret_cast<C *>(base + L.regB);
    T *rBr = reinterpret_cast<T *>(base + L.regB);
    const T *dsdxii = sGeo, *dsdeta = sGeo + 25, *dzdxii = sGeo + 50, *dzdeta = sGeo + 75, *invs = sGeo + 100;
    const T *dsdxii_if = sGeo + 125, *dsdeta_if = sGeo + 150, *dzdxii_if = sGeo + 175,
            *dzdeta_if = sGeo + 200, *invs_if = sGeo + 225;
    constexpr int NPA = ATT == ATT_CG4 ? 4 : 25;
    const int stride = gridDim.x * teams_per_cta;
    for (int e = blockIdx.x * teams_per_cta + team; e < a.n_elem; e += stride) {
        const int nr = a.nr[e], nu = nr / 2 + 1;
        const bool axial = a.axial[e] != 0;
        const T *Gxi = axial ? sGlj : sGll;
        const bool x3 = pa.x3d[e] != 0;
        const int xns = x3 ? nr : 1;
        const T *xp = pa.x + pa.x_off[e];   // [8][xns][25]
        for (int i = lane; i < 250; i += TEAM) sGeo[i] = a.geom[(size_t)e * 250 + i];
        if constexpr (RTZ)
            for (int i = lane; i < 100; i += TEAM) sTrig[i] = a.trig[(size_t)e * 100 + i];
        for (int i = lane; i < 25; i += TEAM) {
            const int p = a.pts[(size_t)e * 25 + i];
            sPt[i] = p;
            sOff[i] = a.pt_off[p];
            sNu[i] = a.pt_nu[p];
        }
        if constexpr (IS3D) {
            const T *tw = a.tw + a.tw_off[nr];
            for (int i = lane; i < 2 * nr; i += TEAM) sTw[i] = tw[i];
        }
        team_sync(team, TEAM);
        const int64_t moff = a.mod_off[e];
        for (int w = 0; w < a.nwave; w++) {
            const C *displw = a.displ + (size_t)w * a.fstride;
            C *stiffw = a.stiff + (size_t)w * a.fstride;
            AT *statew = a.state + (size_t)w * a.sstride;
            for (int i = lane; i < nu * 25; i += TEAM) {
                const int q = i / nu, al = i - q * nu;
                C u0 = mk<T>(0, 0), u1 = u0, u2 = u0;
                if (al < sNu[q]) {
                    const C *src = displw + (size_t)(sOff[q] + al) * 3;
                    u0 = src[0]; u1 = src[1]; u2 = src[2];
                }
                rBc[(al * 3 + 0) * 25 + q] = u0;
                rBc[(al * 3 + 1) * 25 + q] = u1;
                rBc[(al * 3 + 2) * 25 + q] = u2;
            }
            team_sync(team, TEAM);
            // ---- computeGrad9 (+ RTZ), and for Fourier-space elements the whole material step
            for (int i = lane; i < nu * 25; i += TEAM) {
                const int al = i / 25, q = i - al * 25;
                const int ii = q / 5, jj = q - ii * 5;
                const C *U = rBc + al * 75;
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
                C g[9];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    g[3 * c] = cadd(cscale(X[c], ze), cscale(Y[c], zx));       // d/ds
                    g[3 * c + 2] = cadd(cscale(X[c], se), cscale(Y[c], sx));   // d/dz
                }
                const T alf = (T)al, is = invs[q];
                const C A0 = csub(cia(alf, U[q]), U[25 + q]);
                const C A1 = cadd(cia(alf, U[25 + q]), U[q]);
                const C A2 = cia(alf, U[50 + q]);
                g[1] = cscale(A0, is);
                g[4] = cscale(A1, is);
                g[7] = cscale(A2, is);
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
                    g[1] = cadd(cscale(ax[0], ze), cscale(ay[0], zx));
                    g[4] = cadd(cscale(ax[1], ze), cscale(ay[1], zx));
                    g[7] = cadd(cscale(ax[2], ze), cscale(ay[2], zx));
                }
                if constexpr (RTZ) rtz9<true>(g, sTrig[q], sTrig[25 + q], sTrig[50 + q], sTrig[75 + q]);
                if constexpr (!IS3D) {
                    // Fourier space: 1-D material and 1-D PRT
                    C eu[6], su[6];
                    prt_sph_to_und6(g, eu, xp[q], xp[25 + q], xp[50 + q], xp[75 + q]);
                    elastic_at<RHEO>(a.mod + moff, 1, 0, q, eu, su);
                    if constexpr (ATT == ATT_FULL) {
                        AT *st = statew + a.state_off[e];
                        const int64_t ao = a.att_off[e];
                        attenuate<T, AT, true>(a, st, (size_t)nu * 25, (size_t)al * 25 + q, eu, su,
                                               a.attmod[ao + q], a.attmod[ao + 25 + q]);
                    } else if constexpr (ATT == ATT_CG4) {
                        const int k4 = cg4_slot(q);
                        if (k4 >= 0) {
                            AT *st = statew + a.state_off[e];
                            const int64_t ao = a.att_off[e];
                            attenuate<T, AT, true>(a, st, (size_t)nu * 4, (size_t)al * 4 + k4, eu, su,
                                                   a.attmod[ao + k4], a.attmod[ao + 4 + k4]);
                        }
                    }
                    prt_und_to_sph6(su, g, xp[100 + q], xp[125 + q], xp[150 + q], xp[175 + q]);
                    if constexpr (RTZ) rtz9<false>(g, sTrig[q], sTrig[25 + q], sTrig[50 + q], sTrig[75 + q]);
                }
#pragma unroll
                for (int d = 0; d < 9; d++) rA[(al * 9 + d) * 25 + q] = g[d];
            }
            team_sync(team, TEAM);
            if constexpr (IS3D) {
                const T *twc = sTw, *tws = sTw + nr;
                const T inv_nr = (T)1 / (T)nr;
                for (int q0 = 0; q0 < 25; q0 += qc_max) {
                    const int qcnt = min(qc_max, 25 - q0);
                    // slices: computeC2R of the 9 components, PRT, stress, attenuation, PRT back
                    for (int i = lane; i < nr * qcnt; i += TEAM) {
                        const int k = i / qcnt, qq = i - k * qcnt, q = q0 + qq;
                        re1<T> g[9];
#pragma unroll
                        for (int d = 0; d < 9; d++) {
                            T acc = rA[d * 25 + q].x;
                            int j = 0;
                            for (int al = 1; al < nu; al++) {
                                j += k;
                                j = j >= nr ? j - nr : j;
                                const C v = rA[(al * 9 + d) * 25 + q];
                                acc += (T)2 * (v.x * twc[j] - v.y * tws[j]);
                            }
                            g[d].x = acc;
                        }
                        const size_t xo = (size_t)(x3 ? k : 0) * 25 + q, xs = (size_t)xns * 25;
                        re1<T> eu[6], su[6];
                        prt_sph_to_und6(g, eu, xp[xo], xp[xs + xo], xp[2 * xs + xo], xp[3 * xs + xo]);
                        elastic_at<RHEO>(a.mod + moff, nr, k, q, eu, su);
                        if constexpr (ATT == ATT_FULL) {
                            AT *st = statew + a.state_off[e];
                            const int64_t ao = a.att_off[e];
                            const size_t ns = (size_t)nr * 25;
                            attenuate<T, AT, false>(a, st, ns, (size_t)k * 25 + q, eu, su,
                                                    a.attmod[ao + (size_t)k * 25 + q],
                                                    a.attmod[ao + ns + (size_t)k * 25 + q]);
                        } else if constexpr (ATT == ATT_CG4) {
                            const int k4 = cg4_slot(q);
                            if (k4 >= 0) {
                                AT *st = statew + a.state_off[e];
                                const int64_t ao = a.att_off[e];
                                const size_t ns = (size_t)nr * NPA;
                                attenuate<T, AT, false>(a, st, ns, (size_t)k * NPA + k4, eu, su,
                                                        a.attmod[ao + (size_t)k * NPA + k4],
                                                        a.attmod[ao + ns + (size_t)k * NPA + k4]);
                            }
                        }
                        prt_und_to_sph6(su, g, xp[4 * xs + xo], xp[5 * xs + xo], xp[6 * xs + xo],
                                        xp[7 * xs + xo]);
#pragma unroll
                        for (int d = 0; d < 9; d++) rBr[((size_t)k * 9 + d) * qcnt + qq] = g[d].x;
                    }
                    team_sync(team, TEAM);
                    // computeR2C of the 9 components, then RTZ -> SPZ
                    for (int i = lane; i < nu * qcnt; i += TEAM) {
                        const int al = i / qcnt, qq = i - al * qcnt, q = q0 + qq;
                        C s9[9];
                        const int step = al % nr;
#pragma unroll
                        for (int d = 0; d < 9; d++) {
                            T re = 0, im = 0;
                            int j = 0;
                            for (int k = 0; k < nr; k++) {
                                const T x = rBr[((size_t)k * 9 + d) * qcnt + qq] * inv_nr;
                                re += x * twc[j];
                                im -= x * tws[j];
                                j += step;
                                j = j >= nr ? j - nr : j;
                            }
                            if (al == 0) im = 0;
                            if ((nr & 1) == 0 && al == nr / 2) { re *= (T)0.5; im = 0; }
                            s9[d] = mk<T>(re, im);
                        }
                        if constexpr (RTZ) rtz9<false>(s9, sTrig[q], sTrig[25 + q], sTrig[50 + q], sTrig[75 + q]);
#pragma unroll
                        for (int d = 0; d < 9; d++) rA[(al * 9 + d) * 25 + q] = s9[d];
                    }
                    team_sync(team, TEAM);
                }
            }
            // ---- computeQuad9, pass 1: X / Y per component, A terms in region B
            for (int i = lane; i < nu * 25; i += TEAM) {
                const int al = i / 25, q = i - al * 25;
                C s[9];
#pragma unroll
                for (int d = 0; d < 9; d++) s[d] = rA[(al * 9 + d) * 25 + q];
                const T ze = dzdeta_if[q], zx = dzdxii_if[q], se = dsdeta_if[q], sx = dsdxii_if[q];
                // X0 Y0 X1 Y1 X2 Y2 overwrite stress slots 0..5 of this (al, q) only
                C *xy = rA + al * 225;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    xy[(2 * c) * 25 + q] = cadd(cscale(s[3 * c], ze), cscale(s[3 * c + 2], se));
                    xy[(2 * c + 1) * 25 + q] = cadd(cscale(s[3 * c], zx), cscale(s[3 * c + 2], sx));
                }
                const T alf = (T)al;
                rBc[(al * 3 + 0) * 25 + q] = csub(cia(alf, s[1]), s[4]);
                rBc[(al * 3 + 1) * 25 + q] = cadd(cia(alf, s[4]), s[1]);
                rBc[(al * 3 + 2) * 25 + q] = cia(alf, s[7]);
            }
            team_sync(team, TEAM);
            // ---- pass 2 + scatter-add
            for (int i = lane; i < nu * 25; i += TEAM) {
                const int al = i / 25, q = i - al * 25;
                const int ii = q / 5, jj = q - ii * 5;
                const C *xy = rA + al * 225;
                const C *A = rBc + al * 75;
                C f[3];
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
                        const T g0 = Gxi[ii * 5 + 0];
                        fc = csub(fc, cscale(cscale(A[c * 25 + jj], dzdeta_if[jj]), g0));
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
                    f[c] = fc;
                }
                if (al < sNu[q]) {
                    C *dst = stiffw + (size_t)(sOff[q] + al) * 3;
#pragma unroll
                    for (int c = 0; c < 3; c++) atomic_add_cx(dst + c, mk<T>(-f[c].x, -f[c].y));
                }
            }
            team_sync(team, TEAM);
        }
    }
}

}  // namespace axg
