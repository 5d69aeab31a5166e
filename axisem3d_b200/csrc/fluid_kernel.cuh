// fluid_kernel.cuh -- fused stiffness of fluid spectral elements (scalar potential).
//
//   gather chi (FluidPoint::scatterDisplToElement, SOLVER/src/core/point/FluidPoint.hpp:82-95)
//   GradientQuadrature::computeGrad3 (GradientQuadrature.hpp:163-175)
//   Acoustic::strainToStress, K = 1/rho (material/acoustic/Acoustic.hpp:85-92);
//     3-D K through the phi transform (FluidElement.cpp:135-142)
//   GradientQuadrature::computeQuad3 (GradientQuadrature.hpp:234-252)
//   scatter-add: point.stiff -= f  (FluidPoint::gatherStiffFromElement, FluidPoint.hpp:98-103)
#pragma once

#include "common.cuh"
#include "solid_kernel.cuh"

namespace axg {

template <class T>
struct FluidArgs {
    int n_elem;
    const int *nr;
    const int *pts;
    const uint8_t *axial;
    const T *geom;            // [n][10][25]
    const T *K;               // pool
    const int64_t *K_off;     // [n]
    const int *pt_off;
    const int *pt_nu;
    const cx_t<T> *displ;     // [sum nu]
    cx_t<T> *stiff;           // [sum nu]
    const T *tw;
    const int *tw_off;
    const T *gmat;
    int nwave;
    size_t fstride;
    // particle relabelling (PRT kernels only): per element [8][nsl][25] X0..X3, X0|J|..X3|J|,
    // nsl = nr where x3d, else 1; trig [n][2][25] sin, cos of theta (RTZ frame)
    const T *x;
    const int64_t *x_off;
    const uint8_t *x3d;
    const T *trig;
};

// PRT::sphericalToUndulated3 / undulatedToSpherical3 (PRT/PRT.hpp:313-371), as written there:
// the phi row of the forward map takes X1 (the solid map's takes X2)
template <class V, class R>
__device__ __forceinline__ void prt_sph_to_und3(const V g[3], V u[3], R X0, R X1, R X2, R X3) {
    (void)X2;
    u[0] = cadd(cscale(g[0], X0), cscale(g[2], X1));
    u[1] = cadd(cscale(g[1], X0), cscale(g[2], X1));
    u[2] = cscale(g[2], X3);
}
template <class V, class R>
__device__ __forceinline__ void prt_und_to_sph3(const V u[3], V g[3], R X0, R X1, R X2, R X3) {
    g[0] = cscale(u[0], X0);
    g[1] = cscale(u[1], X0);
    g[2] = cadd(cadd(cscale(u[0], X1), cscale(u[1], X2)), cscale(u[2], X3));
}
// CoordTransformSpherical::transformSPZ_RTZ3 / transformRTZ_SPZ3 (CoordTransformSpherical.hpp:54-100)
template <bool TO_RTZ, class V, class T>
__device__ __forceinline__ void rtz3(V g[3], T s1, T c1) {
    const V u0 = g[0];
    if (TO_RTZ) {
        g[0] = csub(cscale(u0, c1), cscale(g[2], s1));
        g[2] = cadd(cscale(g[2], c1), cscale(u0, s1));
    } else {
        g[0] = cadd(cscale(u0, c1), cscale(g[2], s1));
        g[2] = csub(cscale(g[2], c1), cscale(u0, s1));
    }
}

template <class T>
__host__ __device__ inline TeamLayout fluid_layout(int nr_max) {
    TeamLayout L;
    L.nr_max = nr_max;
    L.nu_max = nr_max / 2 + 1;
    L.qc = 25;
    size_t o = 0;
    auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
    L.geom = o; o = al(o + 10 * 25 * sizeof(T));
    L.trig = o; o = al(o + 2 * 25 * sizeof(T));
    L.ipt = o;  o = al(o + 3 * 25 * sizeof(int));
    L.tw = o;   o = al(o + 2 * (size_t)nr_max * sizeof(T));
    L.regA = o; o = al(o + 3 * (size_t)L.nu_max * 25 * 2 * sizeof(T));   // q[a][3][25]
    size_t b1 = (size_t)L.nu_max * 25 * 2 * sizeof(T);                     // chi, then A
    size_t b2 = (size_t)nr_max * 3 * 25 * sizeof(T);                       // slices
    L.regB = o; o = al(o + (b1 > b2 ? b1 : b2));
    L.total = o;
    return L;
}

// PRT: 0 = none, 1 = particle relabelling, 2 = particle relabelling in the RTZ frame
template <class T, bool IS3D, int PRT>
__global__ void __launch_bounds__(256)
fluid_stiffness_kernel(const FluidArgs<T> a, const int nr_max, const int teams_per_cta,
                       const size_t team_bytes) {
    using C = cx_t<T>;
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

    const TeamLayout L = fluid_layout<T>(nr_max);
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
    const T *dsdxii = sGeo, *dsdeta = sGeo + 25, *dzdxii = sGeo + 50, *dzdeta = sGeo + 75,
            *invs = sGeo + 100;
    const T *dsdxii_if = sGeo + 125, *dsdeta_if = sGeo + 150, *dzdxii_if = sGeo + 175,
            *dzdeta_if = sGeo + 200, *invs_if = sGeo + 225;

    for (int e = blockIdx.x * teams_per_cta + team; e < a.n_elem; e += gridDim.x * teams_per_cta) {
        const int nr = a.nr[e];
        const int nu = nr / 2 + 1;
        const bool axial = a.axial[e] != 0;
        const T *Gxi = axial ? sGlj : sGll;
        for (int i = lane; i < 250; i += TEAM) sGeo[i] = a.geom[(size_t)e * 250 + i];
        if constexpr (PRT == 2)
            for (int i = lane; i < 50; i += TEAM) sTrig[i] = a.trig[(size_t)e * 50 + i];
        const T *xp = nullptr;
        int xns = 1;
        if constexpr (PRT > 0) {
            xp = a.x + a.x_off[e];
            xns = a.x3d[e] ? nr : 1;
        }
        for (int i = lane; i < 25; i += TEAM) {
            int p = a.pts[(size_t)e * 25 + i];
            sPt[i] = p;
            sOff[i] = a.pt_off[p];
            sNu[i] = a.pt_nu[p];
        }
        if constexpr (IS3D) {
            const T *tw = a.tw + a.tw_off[nr];
            for (int i = lane; i < 2 * nr; i += TEAM) sTw[i] = tw[i];
        }
        team_sync(team, TEAM);
        for (int w = 0; w < a.nwave; w++) {
        const C *displw = a.displ + (size_t)w * a.fstride;
        C *stiffw = a.stiff + (size_t)w * a.fstride;
        for (int i = lane; i < nu * 25; i += TEAM) {
            const int q = i / nu, al = i - q * nu;
            rBc[al * 25 + q] = al < sNu[q] ? displw[sOff[q] + al] : mk<T>(0, 0);
        }
        team_sync(team, TEAM);
        const int64_t koff = a.K_off[e];
        // computeGrad3
        for (int i = lane; i < nu * 25; i += TEAM) {
            const int al = i / 25, q = i - al * 25;
            const int ii = q / 5, jj = q - ii * 5;
            const C *X0 = rBc + al * 25;
            C x = mk<T>(0, 0), y = mk<T>(0, 0);
#pragma unroll
            for (int k = 0; k < 5; k++) {
                const T gx = Gxi[k * 5 + ii], gy = sGll[k * 5 + jj];
                const C uc = X0[k * 5 + jj], ur = X0[ii * 5 + k];
                x.x += gx * uc.x; x.y += gx * uc.y;
                y.x += ur.x * gy; y.y += ur.y * gy;
            }
            const T ze = dzdeta[q], zx = dzdxii[q], se = dsdeta[q], sx = dsdxii[q];
            C g[3];
            g[0] = cadd(cscale(x, ze), cscale(y, zx));
            g[2] = cadd(cscale(x, se), cscale(y, sx));
            const T alf = (T)al;
            g[1] = cscale(cia(alf, X0[q]), invs[q]);
            if (axial && ii == 0) {
                C ax = mk<T>(0, 0), ay = mk<T>(0, 0);
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    ax = cadd(ax, cscale(cia(alf, X0[k * 5 + jj]), Gxi[k * 5 + 0]));
                    ay = cadd(ay, cscale(cia(alf, X0[k]), sGll[k * 5 + jj]));
                }
                g[1] = cadd(cscale(ax, ze), cscale(ay, zx));
            }
            if constexpr (PRT == 2) rtz3<true>(g, sTrig[q], sTrig[25 + q]);
            if constexpr (!IS3D) {
                // Acoustic::strainToStress_FR, through the PRT maps when relabelled
                const T K = __ldg(a.K + koff + q);
                if constexpr (PRT > 0) {
                    C u[3];
                    prt_sph_to_und3(g, u, xp[q], xp[25 + q], xp[50 + q], xp[75 + q]);
#pragma unroll
                    for (int c = 0; c < 3; c++) u[c] = cscale(u[c], K);
                    prt_und_to_sph3(u, g, xp[100 + q], xp[125 + q], xp[150 + q], xp[175 + q]);
                    if constexpr (PRT == 2) rtz3<false>(g, sTrig[q], sTrig[25 + q]);
                } else {
#pragma unroll
                    for (int c = 0; c < 3; c++) g[c] = cscale(g[c], K);
                }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) rA[(al * 3 + c) * 25 + q] = g[c];
        }
        team_sync(team, TEAM);
        if constexpr (IS3D) {
            const T *twc = sTw, *tws = sTw + nr;
            const T inv_nr = (T)1 / (T)nr;
            for (int i = lane; i < nr * 25; i += TEAM) {
                const int k = i / 25, q = i - k * 25;
                T acc[3];
#pragma unroll
                for (int c = 0; c < 3; c++) acc[c] = rA[c * 25 + q].x;
                int j = 0;
                for (int al = 1; al < nu; al++) {
                    j += k; j = j >= nr ? j - nr : j;
                    const T cs = twc[j], sn = tws[j];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const C v = rA[(al * 3 + c) * 25 + q];
                        acc[c] += (T)2 * (v.x * cs - v.y * sn);
                    }
                }
                const T K = __ldg(a.K + koff + (size_t)k * 25 + q);
                if constexpr (PRT > 0) {
                    const size_t xs = (size_t)xns * 25, xo = (size_t)(xns > 1 ? k : 0) * 25 + q;
                    re1<T> gv[3], u[3];
#pragma unroll
                    for (int c = 0; c < 3; c++) gv[c].x = acc[c];
                    prt_sph_to_und3(gv, u, xp[xo], xp[xs + xo], xp[2 * xs + xo], xp[3 * xs + xo]);
#pragma unroll
                    for (int c = 0; c < 3; c++) u[c].x = u[c].x * K;
                    prt_und_to_sph3(u, gv, xp[4 * xs + xo], xp[5 * xs + xo], xp[6 * xs + xo], xp[7 * xs + xo]);
#pragma unroll
                    for (int c = 0; c < 3; c++) rBr[((size_t)k * 3 + c) * 25 + q] = gv[c].x;
                } else {
#pragma unroll
                    for (int c = 0; c < 3; c++) rBr[((size_t)k * 3 + c) * 25 + q] = acc[c] * K;
                }
            }
            team_sync(team, TEAM);
            for (int i = lane; i < nu * 25; i += TEAM) {
                const int al = i / 25, q = i - al * 25;
                T re[3] = {0, 0, 0}, im[3] = {0, 0, 0};
                int j = 0;
                const int step = al % nr;
                for (int k = 0; k < nr; k++) {
                    const T cs = twc[j], sn = tws[j];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const T x = rBr[((size_t)k * 3 + c) * 25 + q] * inv_nr;
                        re[c] += x * cs;
                        im[c] -= x * sn;
                    }
                    j += step; j = j >= nr ? j - nr : j;
                }
                C out[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    T r = re[c], m = im[c];
                    if (al == 0) m = 0;
                    if ((nr & 1) == 0 && al == nr / 2) { r *= (T)0.5; m = 0; }
                    out[c] = mk<T>(r, m);
                }
                if constexpr (PRT == 2) rtz3<false>(out, sTrig[q], sTrig[25 + q]);
#pragma unroll
                for (int c = 0; c < 3; c++) rA[(al * 3 + c) * 25 + q] = out[c];
            }
            team_sync(team, TEAM);
        }
        // computeQuad3 pass 1: X, Y in place of q0, q2; A = i alpha q1 in region B
        for (int i = lane; i < nu * 25; i += TEAM) {
            const int al = i / 25, q = i - al * 25;
            const C q0 = rA[(al * 3 + 0) * 25 + q], q1 = rA[(al * 3 + 1) * 25 + q],
                    q2 = rA[(al * 3 + 2) * 25 + q];
            rA[(al * 3 + 0) * 25 + q] = cadd(cscale(q0, dzdeta_if[q]), cscale(q2, dsdeta_if[q]));
            rA[(al * 3 + 2) * 25 + q] = cadd(cscale(q0, dzdxii_if[q]), cscale(q2, dsdxii_if[q]));
            rBc[al * 25 + q] = cia((T)al, q1);
        }
        team_sync(team, TEAM);
        for (int i = lane; i < nu * 25; i += TEAM) {
            const int al = i / 25, q = i - al * 25;
            const int ii = q / 5, jj = q - ii * 5;
            const C *X = rA + (al * 3 + 0) * 25, *Y = rA + (al * 3 + 2) * 25, *A = rBc + al * 25;
            C g1 = mk<T>(0, 0), g2 = mk<T>(0, 0);
#pragma unroll
            for (int k = 0; k < 5; k++) {
                const T gx = Gxi[ii * 5 + k], gt = sGll[jj * 5 + k];
                const C xv = X[k * 5 + jj], yv = Y[ii * 5 + k];
                g1.x += gx * xv.x; g1.y += gx * xv.y;
                g2.x += yv.x * gt; g2.y += yv.y * gt;
            }
            C f = cadd(g1, g2);
            f = csub(f, cscale(A[q], invs_if[q]));
            if (axial) {
                f = csub(f, cscale(cscale(A[jj], dzdeta_if[jj]), Gxi[ii * 5 + 0]));
                if (ii == 0) {
                    C b = mk<T>(0, 0);
#pragma unroll
                    for (int k = 0; k < 5; k++) {
                        const C y0 = cscale(A[k], dzdxii_if[k]);
                        const T gt = sGll[jj * 5 + k];
                        b.x += y0.x * gt; b.y += y0.y * gt;
                    }
                    f = csub(f, b);
                }
            }
            if (al < sNu[q]) atomic_add_cx(stiffw + sOff[q] + al, mk<T>(-f.x, -f.y));
        }
        team_sync(team, TEAM);
        }   // wavefields
    }
}

}  // namespace axg
