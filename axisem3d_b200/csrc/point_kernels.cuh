// point_kernels.cuh -- point-wise kernels of one time step.
//
//   solid_fluid_kernel      SolidFluidCoupling::apply (boundary/solid_fluid/SolidFluidCoupling.cpp:30-36,
//                           SolidFluidCoupling1D.hpp:26-37)
//   mass3d_kernel           Nyquist + boundary conditions + Mass3D::computeAccel (point/mass/Mass3D.cpp:41-68)
//   point_update_kernel     AxialBoundary::apply (boundary/axial/AxialBoundary.cpp:21-51),
//                           FluidSurfaceBoundary::apply (surface/FluidSurfaceBoundary.cpp:20-26),
//                           Solid/FluidPoint::computeStiffToAccel (SolidPoint.cpp:28-36, FluidPoint.cpp:28-54),
//                           Mass1D::computeAccel (mass/Mass1D.hpp:25-32),
//                           NewmarkTimeScheme::update (time/NewmarkTimeScheme.hpp:47-59)
//   moment_source_kernel    SolidMoment::apply -> SolidElement::addMomentSource
//                           (source/elem_src/solid/SolidMoment.cpp:29-33, element/SolidElement.cpp:273-356)
//   force_source_kernel     SolidForce::apply -> SolidPoint::addForceSource (SolidPoint.hpp:112-119)
//   station_kernel          StationSolid::record, displacement (output/station-wise/station/StationSolid.cpp:58-66,
//                           Station.hpp:53-72, shared/eigen/eigen_tools.hpp:78-106)
#pragma once

#include "common.cuh"

namespace axg {

// point flags
constexpr uint8_t PT_AXIAL = 1, PT_SURFACE = 2, PT_MASS3D = 4, PT_OCEAN = 8;

// ------------------------------------------------------ solid-fluid coupling ---
template <class T>
struct CouplingArgs {
    int n;
    const int *sp, *fp;            // point indices
    const T *nsu, *nzu, *nsa_m, *nza_m;
    const int *s_off, *f_off, *f_nu;
    const cx_t<T> *s_displ;
    cx_t<T> *s_stiff, *f_stiff;
    int nwave;
    size_t s_stride, f_stride;     // complex values between wavefields
};

template <class T>
__global__ void solid_fluid_kernel(const CouplingArgs<T> a) {
    // one warp per pair, lanes over modes
    const int pair = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (pair >= a.n) return;
    const int s = a.sp[pair], f = a.fp[pair];
    const int nu = a.f_nu[f];
    const T nsu = a.nsu[pair], nzu = a.nzu[pair], nsa = a.nsa_m[pair], nza = a.nza_m[pair];
    for (int w = 0; w < a.nwave; w++) {
        const cx_t<T> *sd = a.s_displ + (size_t)w * a.s_stride;
        cx_t<T> *sst = a.s_stiff + (size_t)w * a.s_stride;
        cx_t<T> *fst = a.f_stiff + (size_t)w * a.f_stride;
        for (int al = lane; al < nu; al += 32) {
            const cx_t<T> us = sd[(size_t)(a.s_off[s] + al) * 3 + 0];
            const cx_t<T> uz = sd[(size_t)(a.s_off[s] + al) * 3 + 2];
            cx_t<T> fs = fst[a.f_off[f] + al];
            fs = cadd(fs, cscale(us, nsu));
            fs = cadd(fs, cscale(uz, nzu));
            fst[a.f_off[f] + al] = fs;
            cx_t<T> *ss = sst + (size_t)(a.s_off[s] + al) * 3;
            ss[0] = csub(ss[0], cscale(fs, nsa));
            ss[2] = csub(ss[2], cscale(fs, nza));
        }
    }
}

// ----------------------------------------------------- Clayton-Engquist ABC ---
// ClaytonSolid1D::apply (ABC/ClaytonSolid1D.cpp:16-29) and ClaytonFluid1D::apply
// (ABC/ClaytonFluid1D.cpp:16-24): stiff -= C veloc, one warp per point, lanes over modes.
// A point on several boundaries (a corner) carries one condition per boundary, applied in
// the order given; conditions are grouped per point (first[i] .. first[i+1]) so that one
// warp owns the point and no two warps update the same stiffness entries.
template <class T, class D>
struct ClaytonArgs {
    int n, ndim;                 // n distinct points
    const int *pt, *first;       // point index; conditions of point i: first[i] .. first[i+1]-1
    const int *off, *nu;
    const T *c;                  // per condition; solid: [4] (ss, zz, sz, pp); fluid: area / (rho vp)
    const cx_t<D> *veloc;
    cx_t<T> *stiff;
    int nwave;
    size_t fstride;
};

template <class T, class D>
__global__ void clayton_kernel(const ClaytonArgs<T, D> a) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (i >= a.n) return;
    const int p = a.pt[i];
    const int c0 = a.first[i], c1 = a.first[i + 1];
    for (int w = 0; w < a.nwave; w++) {
        const cx_t<D> *v = a.veloc + (size_t)w * a.fstride;
        cx_t<T> *f = a.stiff + (size_t)w * a.fstride;
        for (int al = lane; al < a.nu[p]; al += 32) {
            const size_t q = (size_t)(a.off[p] + al) * a.ndim;
            if (a.ndim == 3) {
                const cx_t<T> v0 = mk<T>((T)v[q].x, (T)v[q].y), v1 = mk<T>((T)v[q + 1].x, (T)v[q + 1].y),
                              v2 = mk<T>((T)v[q + 2].x, (T)v[q + 2].y);
                cx_t<T> f0 = f[q], f1 = f[q + 1], f2 = f[q + 2];
                for (int k = c0; k < c1; k++) {
                    const T css = a.c[4 * k], czz = a.c[4 * k + 1], csz = a.c[4 * k + 2], cpp = a.c[4 * k + 3];
                    f0 = csub(f0, cadd(cscale(v0, css), cscale(v2, csz)));
                    f2 = csub(f2, cadd(cscale(v0, csz), cscale(v2, czz)));
                    f1 = csub(f1, cscale(v1, cpp));
                }
                f[q] = f0; f[q + 1] = f1; f[q + 2] = f2;
            } else {
                const cx_t<T> v0 = mk<T>((T)v[q].x, (T)v[q].y);
                cx_t<T> f0 = f[q];
                for (int k = c0; k < c1; k++) f0 = csub(f0, cscale(v0, a.c[k]));
                f[q] = f0;
            }
        }
    }
}

// -------------------------------------------------------- 3-D mass points ---
template <class T>
struct Mass3DArgs {
    int n;                       // number of Mass3D points
    const int *pt;               // their indices
    const int *nr, *off;
    const uint8_t *flags;
    const T *inv_mass;           // pool
    const int64_t *im_off;       // [npoints]
    const T *tw;                 // twiddle pool (cos then sin for each nr)
    const int *tw_off;
    cx_t<T> *stiff;
    int ndim;
    int solid;
    int nr_max;                  // scratch reals per warp
    int nwave;
    size_t fstride;
    int mask;                    // 1 = boundary conditions, 2 = 1/M
};

// Boundary conditions on one mode of one point, in the reference order:
// AxialBoundary (after assembly) then the Nyquist rule of computeStiffToAccel.
template <class T>
__device__ __forceinline__ void point_bc(cx_t<T> *f, int ndim, int al, int nu, int nr,
                                         uint8_t flags, bool solid) {
    const T half = (T)0.5;
    if (flags & PT_AXIAL) {
        if (solid) {
            if (al == 0) {
                f[0] = mk<T>(0, 0); f[1] = mk<T>(0, 0);
            } else if (al == 1) {
                const cx_t<T> a0 = f[0], a1 = f[1];
                // (stiff(1,0) - i stiff(1,1)) * 0.5, then stiff(1,1) = i stiff(1,0)
                const cx_t<T> t = mk<T>((a0.x + a1.y) * half, (a0.y - a1.x) * half);
                f[0] = t;
                f[1] = mk<T>(-t.y, t.x);
                f[2] = mk<T>(0, 0);
            } else {
                f[0] = mk<T>(0, 0); f[1] = mk<T>(0, 0); f[2] = mk<T>(0, 0);
            }
        } else if (al >= 1) {
            f[0] = mk<T>(0, 0);
        }
    }
    if (!solid && (flags & PT_SURFACE)) f[0] = mk<T>(0, 0);
    if ((nr & 1) == 0 && al == nu - 1)
        for (int c = 0; c < ndim; c++) f[c].y = 0;
}

template <class T>
__global__ void mass3d_kernel(const Mass3DArgs<T> a) {
    // one warp per point: boundary conditions, then per dimension
    // C2R -> x 1/M_k -> R2C with a per-warp scratch of nr reals
    extern __shared__ __align__(16) unsigned char sm[];
    const int w = threadIdx.x / 32, lane = threadIdx.x & 31;
    const int item = blockIdx.x * (blockDim.x / 32) + w;
    if (item >= a.n * a.nwave) return;
    const int ip = item % a.n, wf = item / a.n;
    cx_t<T> *stiff = a.stiff + (size_t)wf * a.fstride;
    const int p = a.pt[ip];
    const int nr = a.nr[p], nu = nr / 2 + 1, off = a.off[p], nd = a.ndim;
    const uint8_t fl = a.flags[p];
    T *r = reinterpret_cast<T *>(sm) + (size_t)w * a.nr_max;
    const T *twc = a.tw + a.tw_off[nr], *tws = twc + nr;
    if (a.mask & 1) {
        for (int al = lane; al < nu; al += 32) {
            cx_t<T> f[3];
            for (int d = 0; d < nd; d++) f[d] = stiff[(size_t)(off + al) * nd + d];
            point_bc<T>(f, nd, al, nu, nr, fl, a.solid);
            for (int d = 0; d < nd; d++) stiff[(size_t)(off + al) * nd + d] = f[d];
        }
        __syncwarp();
    }
    if (!(a.mask & 2)) return;
    const T *im = a.inv_mass + a.im_off[p];
    const T inv_nr = (T)1 / (T)nr;
    for (int c = 0; c < nd; c++) {
        for (int k = lane; k < nr; k += 32) {
            T acc = stiff[(size_t)off * nd + c].x;
            int j = 0;
            for (int al = 1; al < nu; al++) {
                j += k; j = j >= nr ? j - nr : j;
                const cx_t<T> v = stiff[(size_t)(off + al) * nd + c];
                acc += (T)2 * (v.x * twc[j] - v.y * tws[j]);
            }
            r[k] = acc * im[k];
        }
        __syncwarp();
        for (int al = lane; al < nu; al += 32) {
            T re = 0, imv = 0;
            int j = 0;
            const int step = al % nr;
            for (int k = 0; k < nr; k++) {
                const T x = r[k] * inv_nr;
                re += x * twc[j];
                imv -= x * tws[j];
                j += step; j = j >= nr ? j - nr : j;
            }
            if (al == 0) imv = 0;
            if ((nr & 1) == 0 && al == nr / 2) { re *= (T)0.5; imv = 0; }
            stiff[(size_t)(off + al) * nd + c] = mk<T>(re, imv);
        }
        __syncwarp();
    }
}

// ------------------------------------------------ stiff -> accel + Newmark ---
// T: stiffness/acceleration type; D: displacement/velocity storage type.
// MIXED (T = float, D = double): increments formed in double, optionally
// accumulated with compensated (Kahan) summation; a float copy of d feeds the
// elements.
// ------------------------------------------------- 3-D absorbing boundaries ---
// Warp-level computeC2R / computeR2C of one component of one point (SolverFFTW.hpp:101-172
// conventions: c2r doubles every mode above 0 and ignores the imaginary parts of the DC and
// Nyquist terms; r2c scales by 1/nr and halves the Nyquist term), lanes over slices / modes.
template <class T, class V>
__device__ __forceinline__ void warp_c2r(const V *f, int stride, int nu, int nr, const T *twc, const T *tws,
                                         T *r, int lane) {
    for (int k = lane; k < nr; k += 32) {
        T acc = (T)f[0].x;
        int j = 0;
        for (int al = 1; al < nu; al++) {
            j += k;
            j = j >= nr ? j - nr : j;
            const V v = f[(size_t)al * stride];
            acc += (T)2 * ((T)v.x * twc[j] - (T)v.y * tws[j]);
        }
        r[k] = acc;
    }
}
template <class T>
__device__ __forceinline__ cx_t<T> r2c_mode(const T *r, int nr, int al, const T *twc, const T *tws) {
    const T inv_nr = (T)1 / (T)nr;
    T re = 0, im = 0;
    int j = 0;
    const int step = al % nr;
    for (int k = 0; k < nr; k++) {
        const T x = r[k] * inv_nr;
        re += x * twc[j];
        im -= x * tws[j];
        j += step;
        j = j >= nr ? j - nr : j;
    }
    if (al == 0) im = 0;
    if ((nr & 1) == 0 && al == nr / 2) { re *= (T)0.5; im = 0; }
    return mk<T>(re, im);
}

// ClaytonSolid3D::apply (ABC/ClaytonSolid3D.cpp): a = rsa v + (v . k) k in slices,
// stiff -= R2C(a); ClaytonFluid3D::apply (ABC/ClaytonFluid3D.cpp): a = (area / rho vp) v.
// One warp per point; its conditions (one per boundary) in the order given.
template <class T, class D>
struct Clayton3DArgs {
    int n, ndim;                 // distinct points
    const int *pt, *first;       // conditions of point i: first[i] .. first[i+1]-1
    const int64_t *coff;         // per condition: offset of its per-slice coefficients
    const T *c;                  // solid: [nr][4] (rsa, k_s, k_phi, k_z); fluid: [nr]
    const int *nr, *off;
    const T *tw; const int *tw_off;
    const cx_t<D> *veloc;
    cx_t<T> *stiff;
    int nr_max, nwave;
    size_t fstride;
};

template <class T, class D>
__global__ void clayton3d_kernel(const Clayton3DArgs<T, D> a) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int w = threadIdx.x / 32, lane = threadIdx.x & 31;
    const int item = blockIdx.x * (blockDim.x / 32) + w;
    if (item >= a.n * a.nwave) return;
    const int i = item % a.n, wf = item / a.n;
    const int p = a.pt[i], nr = a.nr[p], nu = nr / 2 + 1, nd = a.ndim;
    T *vr = reinterpret_cast<T *>(sm) + (size_t)w * 2 * 3 * a.nr_max;   // [nd][nr_max] velocity slices
    T *ar = vr + (size_t)3 * a.nr_max;                                  // [nd][nr_max] result slices
    const T *twc = a.tw + a.tw_off[nr], *tws = twc + nr;
    const cx_t<D> *v = a.veloc + (size_t)wf * a.fstride + (size_t)a.off[p] * nd;
    cx_t<T> *f = a.stiff + (size_t)wf * a.fstride + (size_t)a.off[p] * nd;
    for (int c = 0; c < nd; c++) warp_c2r<T, cx_t<D>>(v + c, nd, nu, nr, twc, tws, vr + (size_t)c * a.nr_max, lane);
    __syncwarp();
    for (int q = a.first[i]; q < a.first[i + 1]; q++) {
        const T *cf = a.c + a.coff[q];
        for (int k = lane; k < nr; k += 32) {
            if (nd == 3) {
                const T v0 = vr[k], v1 = vr[a.nr_max + k], v2 = vr[2 * a.nr_max + k];
                const T rsa = cf[4 * k], k0 = cf[4 * k + 1], k1 = cf[4 * k + 2], k2 = cf[4 * k + 3];
                const T dot = v0 * k0 + v1 * k1 + v2 * k2;
                ar[k] = rsa * v0 + dot * k0;
                ar[a.nr_max + k] = rsa * v1 + dot * k1;
                ar[2 * a.nr_max + k] = rsa * v2 + dot * k2;
            } else {
                ar[k] = vr[k] * cf[k];
            }
        }
        __syncwarp();
        for (int al = lane; al < nu; al += 32)
            for (int c = 0; c < nd; c++) {
                const cx_t<T> x = r2c_mode<T>(ar + (size_t)c * a.nr_max, nr, al, twc, tws);
                f[(size_t)al * nd + c] = csub(f[(size_t)al * nd + c], x);
            }
        __syncwarp();
    }
}

// SolidFluidCoupling3D (core/boundary/solid_fluid/SolidFluidCoupling3D.cpp:40-94): in the
// slices of the pair's nr, fluid stiff += R2C(n_u . C2R(solid displ)), then solid stiff -=
// R2C(C2R(fluid stiff) n_a / m_fluid), modes below nr/2 + 1. One warp per (pair, wavefield).
template <class T>
struct Coupling3DArgs {
    int n;
    const int *sp, *fp;
    const int64_t *coff;           // per pair: offset of its nr slices
    const T *nu3, *na3;            // [nr][3] unassembled normal, assembled normal / fluid mass
    const int *s_off, *s_nr, *f_off;
    const T *tw; const int *tw_off;
    const cx_t<T> *s_displ;
    cx_t<T> *s_stiff, *f_stiff;
    int nr_max, nwave;
    size_t s_stride, f_stride;
};

template <class T>
__global__ void solid_fluid3d_kernel(const Coupling3DArgs<T> a) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int w = threadIdx.x / 32, lane = threadIdx.x & 31;
    const int item = blockIdx.x * (blockDim.x / 32) + w;
    if (item >= a.n * a.nwave) return;
    const int i = item % a.n, wf = item / a.n;
    const int s = a.sp[i], f = a.fp[i], nr = a.s_nr[s], nu = nr / 2 + 1;
    T *ur = reinterpret_cast<T *>(sm) + (size_t)w * 4 * a.nr_max;        // [3][nr_max] solid slices
    T *fr = ur + (size_t)3 * a.nr_max;                                   // [nr_max] fluid slices
    const T *twc = a.tw + a.tw_off[nr], *tws = twc + nr;
    const cx_t<T> *u = a.s_displ + (size_t)wf * a.s_stride + (size_t)a.s_off[s] * 3;
    cx_t<T> *sst = a.s_stiff + (size_t)wf * a.s_stride + (size_t)a.s_off[s] * 3;
    cx_t<T> *fst = a.f_stiff + (size_t)wf * a.f_stride + a.f_off[f];
    const T *nu3 = a.nu3 + (size_t)a.coff[i] * 3, *na3 = a.na3 + (size_t)a.coff[i] * 3;
    for (int c = 0; c < 3; c++) warp_c2r<T, cx_t<T>>(u + c, 3, nu, nr, twc, tws, ur + (size_t)c * a.nr_max, lane);
    __syncwarp();
    for (int k = lane; k < nr; k += 32)
        fr[k] = nu3[3 * k] * ur[k] + nu3[3 * k + 1] * ur[a.nr_max + k] + nu3[3 * k + 2] * ur[2 * a.nr_max + k];
    __syncwarp();
    for (int al = lane; al < nu; al += 32) fst[al] = cadd(fst[al], r2c_mode<T>(fr, nr, al, twc, tws));
    __syncwarp();
    warp_c2r<T, cx_t<T>>(fst, 1, nu, nr, twc, tws, fr, lane);
    __syncwarp();
    for (int k = lane; k < nr; k += 32)
        for (int c = 0; c < 3; c++) ur[(size_t)c * a.nr_max + k] = fr[k] * na3[3 * k + c];
    __syncwarp();
    for (int al = lane; al < nu; al += 32)
        for (int c = 0; c < 3; c++)
            sst[(size_t)al * 3 + c] = csub(sst[(size_t)al * 3 + c], r2c_mode<T>(ur + (size_t)c * a.nr_max, nr, al, twc, tws));
}

// Sponge::apply, 3-D branch (ABC/Sponge.hpp:74-98): in slices, accel -= 2 gamma veloc +
// gamma^2 displ, then back to Fourier; after the mass term. One warp per point.
template <class T, class D>
struct Sponge3DArgs {
    int n, ndim;
    const int *pt;
    const int64_t *goff;         // per point: offset of its nr gammas
    const T *gamma;
    const int *nr, *off;
    const T *tw; const int *tw_off;
    const cx_t<D> *veloc, *displ;
    cx_t<T> *stiff;
    int nr_max, nwave;
    size_t fstride;
};

template <class T, class D>
__global__ void sponge3d_kernel(const Sponge3DArgs<T, D> a) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int w = threadIdx.x / 32, lane = threadIdx.x & 31;
    const int item = blockIdx.x * (blockDim.x / 32) + w;
    if (item >= a.n * a.nwave) return;
    const int i = item % a.n, wf = item / a.n;
    const int p = a.pt[i], nr = a.nr[p], nu = nr / 2 + 1, nd = a.ndim;
    T *sr = reinterpret_cast<T *>(sm) + (size_t)w * 3 * a.nr_max;      // stiff, veloc, displ slices
    T *vr = sr + a.nr_max, *ur = vr + a.nr_max;
    const T *twc = a.tw + a.tw_off[nr], *tws = twc + nr;
    const T *g = a.gamma + a.goff[i];
    const size_t o = (size_t)wf * a.fstride + (size_t)a.off[p] * nd;
    cx_t<T> *f = a.stiff + o;
    const T two = 2;
    for (int c = 0; c < nd; c++) {
        warp_c2r<T, cx_t<T>>(f + c, nd, nu, nr, twc, tws, sr, lane);
        warp_c2r<T, cx_t<D>>(a.veloc + o + c, nd, nu, nr, twc, tws, vr, lane);
        warp_c2r<T, cx_t<D>>(a.displ + o + c, nd, nu, nr, twc, tws, ur, lane);
        __syncwarp();
        for (int k = lane; k < nr; k += 32) sr[k] -= (two * g[k]) * vr[k] + (g[k] * g[k]) * ur[k];
        __syncwarp();
        for (int al = lane; al < nu; al += 32) f[(size_t)al * nd + c] = r2c_mode<T>(sr, nr, al, twc, tws);
        __syncwarp();
    }
}

// ------------------------------------------------------- wavefield scanning ---
// Scanning1D::doScanning (point/Point.hpp:106-174) on the displacement of one component of
// one point, every `interval` steps: energy peaks of the Fourier series (H2 norm) and the
// number of modes each needs; the reference's std::map of candidates (ascending H2 keys)
// is a sorted array of at most AXG_SCAN_CAP entries per component.
#ifndef AXG_SCAN_CAP
#define AXG_SCAN_CAP 32
#endif
template <class T, class D>
struct ScanArgs {
    int n, ndim;                 // scanned points; components per point
    const int *pt, *off, *nr;
    const cx_t<D> *displ;
    T tol_fourier_h2, rel_tol_h2, abs_tol_h2;
    int max_peaks, interval;
    const int *step;
    T *h2p, *h2pp;               // [n * ndim]
    int *cnt;                    // [n * ndim]
    T *key;                      // [AXG_SCAN_CAP][n * ndim]
    int *nu1;                    // [AXG_SCAN_CAP][n * ndim]
};

template <class T, class D>
__global__ void scan_kernel(const ScanArgs<T, D> a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = a.n * a.ndim;
    if (t >= m || (*a.step) % a.interval != 0) return;
    const int i = t / a.ndim, c = t - i * a.ndim;
    const int p = a.pt[i], nu = a.nr[p] / 2 + 1;
    const cx_t<D> *f = a.displ + (size_t)a.off[p] * a.ndim + c;
    // l2 and h2 norms (the series in the working precision)
    T l2 = 0;
    for (int al = 0; al < nu; al++) {
        const T x = (T)f[(size_t)al * a.ndim].x, y = (T)f[(size_t)al * a.ndim].y;
        l2 += x * x + y * y;
    }
    const T x0 = (T)f[0].x, y0 = (T)f[0].y;
    const T h2 = (T)((double)l2 - .5 * (double)(x0 * x0 + y0 * y0));
    int n = a.cnt[t];
    const T max_h2 = n > 0 ? a.key[(size_t)(n - 1) * m + t] : (T)0;
    const T hp = a.h2p[t], hpp = a.h2pp[t];
    a.h2pp[t] = hp;
    a.h2p[t] = h2;
    if (!(h2 > a.abs_tol_h2 && h2 > a.rel_tol_h2 * max_h2 && hp > h2 && hp > hpp)) return;
    // smallest number of modes whose truncation error is below tol * H2
    const T abs_fourier = h2 * a.tol_fourier_h2;
    int new_nu1 = 1;
    T head = 0;
    for (; new_nu1 < nu; new_nu1++) {
        const T x = (T)f[(size_t)(new_nu1 - 1) * a.ndim].x, y = (T)f[(size_t)(new_nu1 - 1) * a.ndim].y;
        head += x * x + y * y;
        if (l2 - head < abs_fourier) break;
    }
    T *key = a.key + t;
    int *nv = a.nu1 + t;
    int hit = -1;
    for (int k = 0; k < n; k++)
        if (key[(size_t)k * m] == h2) { hit = k; break; }
    if (hit >= 0) {
        nv[(size_t)hit * m] = max(nv[(size_t)hit * m], new_nu1);
    } else {
        if (max_h2 < h2) {
            // drop the keys below rel_tol * H2 (map::erase(begin, lower_bound(rel_tol * H2)))
            const T cut = a.rel_tol_h2 * h2;
            int drop = 0;
            while (drop < n && key[(size_t)drop * m] < cut) drop++;
            for (int k = drop; k < n; k++) {
                key[(size_t)(k - drop) * m] = key[(size_t)k * m];
                nv[(size_t)(k - drop) * m] = nv[(size_t)k * m];
            }
            n -= drop;
        }
        // insert in ascending order; at capacity, inserting and then erasing the smallest key
        // (the map's steps) keeps the set as it is when the new key is the smallest
        if (n == AXG_SCAN_CAP) {
            if (h2 < key[0]) { a.cnt[t] = n; return; }
            for (int k = 1; k < n; k++) {
                key[(size_t)(k - 1) * m] = key[(size_t)k * m];
                nv[(size_t)(k - 1) * m] = nv[(size_t)k * m];
            }
            n--;
        }
        int pos = n;
        while (pos > 0 && key[(size_t)(pos - 1) * m] > h2) {
            key[(size_t)pos * m] = key[(size_t)(pos - 1) * m];
            nv[(size_t)pos * m] = nv[(size_t)(pos - 1) * m];
            pos--;
        }
        key[(size_t)pos * m] = h2;
        nv[(size_t)pos * m] = new_nu1;
        n++;
    }
    if (n > a.max_peaks) {
        for (int k = 1; k < n; k++) {
            key[(size_t)(k - 1) * m] = key[(size_t)k * m];
            nv[(size_t)(k - 1) * m] = nv[(size_t)k * m];
        }
        n--;
    }
    a.cnt[t] = n;
}

// ------------------------------------------------------------- ocean load ---
// MassOceanLoad1D::computeAccel (point/mass/MassOceanLoad1D.hpp): the point's own mass acts
// along the surface, mass + ocean mass across it; one warp per point, lanes over modes,
// after the boundary conditions of the point (as for Mass3D points)
template <class T>
struct OceanArgs {
    int n;
    const int *pt;               // ocean points
    const T *c;                  // [n][4]: (ss, zz, sz, pp) inverse-mass coefficients
    const int *nr, *off;
    const uint8_t *flags;
    cx_t<T> *stiff;
    int nwave;
    size_t fstride;
    int mask;                    // 1 = boundary conditions, 2 = ocean-loaded 1/M
};

template <class T>
__global__ void ocean_mass_kernel(const OceanArgs<T> a) {
    const int item = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (item >= a.n * a.nwave) return;
    const int i = item % a.n, wf = item / a.n;
    const int p = a.pt[i];
    const int nr = a.nr[p], nu = nr / 2 + 1, off = a.off[p];
    const uint8_t fl = a.flags[p];
    const T css = a.c[4 * i], czz = a.c[4 * i + 1], csz = a.c[4 * i + 2], cpp = a.c[4 * i + 3];
    cx_t<T> *stiff = a.stiff + (size_t)wf * a.fstride;
    for (int al = lane; al < nu; al += 32) {
        cx_t<T> *f = stiff + (size_t)(off + al) * 3;
        cx_t<T> v[3] = {f[0], f[1], f[2]};
        if (a.mask & 1) point_bc<T>(v, 3, al, nu, nr, fl, true);
        if (a.mask & 2) {
            const cx_t<T> s0 = v[0];
            v[0] = cadd(cscale(s0, css), cscale(v[2], csz));
            v[2] = cadd(cscale(s0, csz), cscale(v[2], czz));
            v[1] = cscale(v[1], cpp);
        }
        f[0] = v[0]; f[1] = v[1]; f[2] = v[2];
    }
}

// MassOceanLoad3D::computeAccel (point/mass/MassOceanLoad3D.cpp): in slices,
// a = F / m - (F . k) k; one warp per point, after its boundary conditions
template <class T>
struct Ocean3DArgs {
    int n;
    const int *pt;
    const int64_t *coff;         // per point: offset of its [nr][4] (1/m, k_s, k_phi, k_z)
    const T *c;
    const int *nr, *off;
    const uint8_t *flags;
    const T *tw; const int *tw_off;
    cx_t<T> *stiff;
    int nr_max, nwave;
    size_t fstride;
    int mask;
};

template <class T>
__global__ void ocean3d_kernel(const Ocean3DArgs<T> a) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int w = threadIdx.x / 32, lane = threadIdx.x & 31;
    const int item = blockIdx.x * (blockDim.x / 32) + w;
    if (item >= a.n * a.nwave) return;
    const int i = item % a.n, wf = item / a.n;
    const int p = a.pt[i], nr = a.nr[p], nu = nr / 2 + 1;
    cx_t<T> *f = a.stiff + (size_t)wf * a.fstride + (size_t)a.off[p] * 3;
    if (a.mask & 1) {
        for (int al = lane; al < nu; al += 32) {
            cx_t<T> v[3] = {f[al * 3], f[al * 3 + 1], f[al * 3 + 2]};
            point_bc<T>(v, 3, al, nu, nr, a.flags[p], true);
            f[al * 3] = v[0]; f[al * 3 + 1] = v[1]; f[al * 3 + 2] = v[2];
        }
        __syncwarp();
    }
    if (!(a.mask & 2)) return;
    T *fr = reinterpret_cast<T *>(sm) + (size_t)w * 3 * a.nr_max;   // [3][nr_max] slices
    const T *twc = a.tw + a.tw_off[nr], *tws = twc + nr;
    const T *cf = a.c + a.coff[i];
    for (int c = 0; c < 3; c++) warp_c2r<T, cx_t<T>>(f + c, 3, nu, nr, twc, tws, fr + (size_t)c * a.nr_max, lane);
    __syncwarp();
    for (int k = lane; k < nr; k += 32) {
        const T f0 = fr[k], f1 = fr[a.nr_max + k], f2 = fr[2 * a.nr_max + k];
        const T im = cf[4 * k], k0 = cf[4 * k + 1], k1 = cf[4 * k + 2], k2 = cf[4 * k + 3];
        const T dot = f0 * k0 + f1 * k1 + f2 * k2;
        fr[k] = im * f0 - dot * k0;
        fr[a.nr_max + k] = im * f1 - dot * k1;
        fr[2 * a.nr_max + k] = im * f2 - dot * k2;
    }
    __syncwarp();
    for (int al = lane; al < nu; al += 32)
        for (int c = 0; c < 3; c++) f[al * 3 + c] = r2c_mode<T>(fr + (size_t)c * a.nr_max, nr, al, twc, tws);
}

template <class T, class D>
struct PointArgs {
    int nmodes;                  // sum nu
    int ndim;
    int solid;
    const int *mode_pt;          // [nmodes] owning point
    const int *off, *nr;         // per point
    const uint8_t *flags;
    const T *inv_mass1;          // per point (1-D mass)
    cx_t<T> *stiff;
    cx_t<T> *accel;
    cx_t<D> *displ, *veloc;
    cx_t<float> *cd, *cv;        // compensation terms (MIXED + compensated)
    cx_t<T> *displ_elem;         // float copy of d for elements (MIXED) or null
    D dt, half_dt, half_dt_dt;
    int *nonfinite;
    int mask;                    // 1 = BC after assembly, 2 = 1/M, 4 = Newmark
    int nwave;                   // wavefields; fields are [nwave][nmodes][ndim]
    const T *sponge;             // [npoints] Kosloff gamma (0 = none) or null
};

// One thread per complex value of the point fields ([nwave][nmodes][ndim]), so that every field
// is read and written in consecutive 8- / 16-byte words. The only condition that mixes the
// components of a mode (the axial order-1 rule) reads the other component before the block's
// barrier and every thread writes after it; blocks of POINT_BLOCK threads hold whole modes.
constexpr int POINT_BLOCK = 288;   // 96 modes of 3 components, 9 warps
template <class T, class D, bool COMP>
__global__ void __launch_bounds__(POINT_BLOCK) point_update_kernel(const PointArgs<T, D> a) {
    const int nd = a.ndim;
    const int64_t q64 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = q64 < (int64_t)a.nmodes * a.nwave * nd;
    const size_t q = valid ? (size_t)q64 : 0;
    const size_t m = nd == 3 ? q / 3 : q;              // mode of the batched fields
    const int d = (int)(q - m * nd);
    const int mm = a.nwave == 1 ? (int)m : (int)(m % (size_t)a.nmodes);
    const int p = a.mode_pt[mm];
    const int off = a.off[p], nr = a.nr[p], nu = nr / 2 + 1, al = mm - off;
    const uint8_t fl = a.flags[p];
    cx_t<T> f = valid ? a.stiff[q] : mk<T>(0, 0);
    // the axial rule of order 1 (solid): both horizontal components of the mode
    const bool mix = valid && (a.mask & 1) && a.solid && (fl & PT_AXIAL) && al == 1 && d < 2 &&
                     !(fl & (PT_MASS3D | PT_OCEAN));
    cx_t<T> g0 = f, g1 = f;
    if (mix) {
        g0 = a.stiff[m * 3];
        g1 = a.stiff[m * 3 + 1];
    }
    __syncthreads();
    if (!valid) return;
    if (!(fl & (PT_MASS3D | PT_OCEAN))) {
        if (a.mask & 1) {
            // point_bc for one component (AxialBoundary::apply, the fluid surface, the Nyquist
            // imaginary parts)
            const T half = (T)0.5;
            if (fl & PT_AXIAL) {
                if (a.solid) {
                    if (al == 0) {
                        if (d < 2) f = mk<T>(0, 0);
                    } else if (al == 1) {
                        const cx_t<T> t = mk<T>((g0.x + g1.y) * half, (g0.y - g1.x) * half);
                        f = d == 0 ? t : d == 1 ? mk<T>(-t.y, t.x) : mk<T>(0, 0);
                    } else {
                        f = mk<T>(0, 0);
                    }
                } else if (al >= 1) {
                    f = mk<T>(0, 0);
                }
            }
            if (!a.solid && (fl & PT_SURFACE)) f = mk<T>(0, 0);
            if ((nr & 1) == 0 && al == nu - 1) f.y = 0;
        }
        if (a.mask & 2) f = cscale(f, a.inv_mass1[p]);
    }
    if ((a.mask & 2) && a.sponge) {
        // Sponge::apply (ABC/Sponge.hpp:74-98), 1-D gamma, on the acceleration
        const T g = a.sponge[p];
        if (g != (T)0) {
            const T two = 2;
            const cx_t<T> v = mk<T>((T)a.veloc[q].x, (T)a.veloc[q].y);
            const cx_t<T> u = mk<T>((T)a.displ[q].x, (T)a.displ[q].y);
            f = csub(f, cadd(cscale(v, two * g), cscale(u, g * g)));
        }
    }
    if (!(a.mask & 4)) {
        // stages without the update: the result stays in the stiffness field, as
        // computeStiffToAccel works in place on mStiff
        a.stiff[q] = f;
        return;
    }
    const cx_t<T> acc = a.accel[q];
    cx_t<D> v = a.veloc[q], u = a.displ[q];
    if constexpr (sizeof(D) == sizeof(T)) {
        // NewmarkTimeScheme::update in the working precision
        v.x += a.half_dt * (acc.x + f.x);
        v.y += a.half_dt * (acc.y + f.y);
        u.x += a.dt * v.x + a.half_dt_dt * f.x;
        u.y += a.dt * v.y + a.half_dt_dt * f.y;
    } else {
        const D dvx = a.half_dt * ((D)acc.x + (D)f.x);
        const D dvy = a.half_dt * ((D)acc.y + (D)f.y);
        if constexpr (COMP) {
            cx_t<float> cv = a.cv[q], cd = a.cd[q];
            D y = dvx - (D)cv.x, t = v.x + y; cv.x = (float)((t - v.x) - y); v.x = t;
            y = dvy - (D)cv.y; t = v.y + y; cv.y = (float)((t - v.y) - y); v.y = t;
            const D dux = a.dt * v.x + a.half_dt_dt * (D)f.x;
            const D duy = a.dt * v.y + a.half_dt_dt * (D)f.y;
            y = dux - (D)cd.x; t = u.x + y; cd.x = (float)((t - u.x) - y); u.x = t;
            y = duy - (D)cd.y; t = u.y + y; cd.y = (float)((t - u.y) - y); u.y = t;
            a.cv[q] = cv;
            a.cd[q] = cd;
        } else {
            v.x += dvx; v.y += dvy;
            u.x += a.dt * v.x + a.half_dt_dt * (D)f.x;
            u.y += a.dt * v.y + a.half_dt_dt * (D)f.y;
        }
        a.displ_elem[q] = mk<T>((T)u.x, (T)u.y);
    }
    a.veloc[q] = v;
    a.displ[q] = u;
    a.accel[q] = f;
    a.stiff[q] = mk<T>(0, 0);
    if (!(isfinite(u.x) && isfinite(u.y))) atomicOr(a.nonfinite, 1);
}

// ------------------------------------------------------------------ sources ---
template <class T>
struct MomentArgs {
    int nsrc;
    const int *elem, *nu;              // per source; nu = pattern rows
    const int64_t *pat_off;            // complex offset
    const cx_t<T> *pattern;            // [nu][6][25]
    const T *stf;                      // [nsteps][nsrc]
    int stf_steps;
    const int *step;                   // device step counter
    const int *e_nr, *e_pts;           // solid elements
    const uint8_t *e_axial;
    const T *e_geom;                   // [ne][10][25]
    const int *pt_off, *pt_nu;
    cx_t<T> *stiff;
    const T *gmat;
    const int *wave;                   // wavefield of each source
    size_t fstride;
};

template <class T>
__global__ void moment_source_kernel(const MomentArgs<T> a) {
    using C = cx_t<T>;
    const int s = blockIdx.x;
    if (s >= a.nsrc) return;
    __shared__ T sGll[25], sGlj[25], sGeo[125];
    __shared__ C sS[3][6][25];     // at most 3 modes on the axis; loop for more
    __shared__ C sA[3][3][25];
    __shared__ int sOff[25], sNu[25];
    if (a.stf_steps <= 0 || a.stf == nullptr) return;
    const int e = a.elem[s];
    const int enu = a.e_nr[e] / 2 + 1;
    const int nuco = min(enu, a.nu[s]);
    const bool axial = a.e_axial[e] != 0;
    const int st = max(0, min(*a.step, a.stf_steps - 1));
    const T v = a.stf[(size_t)st * a.nsrc + s];
    for (int i = threadIdx.x; i < 25; i += blockDim.x) {
        sGll[i] = a.gmat[i]; sGlj[i] = a.gmat[25 + i];
        const int p = a.e_pts[(size_t)e * 25 + i];
        sOff[i] = a.pt_off[p]; sNu[i] = a.pt_nu[p];
    }
    for (int i = threadIdx.x; i < 125; i += blockDim.x) sGeo[i] = a.e_geom[(size_t)e * 250 + i];
    __syncthreads();
    const T *Gxi = axial ? sGlj : sGll;
    const T *dsdxii = sGeo, *dsdeta = sGeo + 25, *dzdxii = sGeo + 50, *dzdeta = sGeo + 75,
            *invs = sGeo + 100;
    for (int a0 = 0; a0 < nuco; a0 += 3) {
        const int na = min(3, nuco - a0);
        // stress = -pattern * stf; X/Y/A terms (computeQuad6_NoIntegration, plain operators)
        for (int i = threadIdx.x; i < na * 25; i += blockDim.x) {
            const int aa = i / 25, q = i % 25, al = a0 + aa;
            C sg[6];
            for (int d = 0; d < 6; d++) {
                const C pv = a.pattern[a.pat_off[s] + ((size_t)al * 6 + d) * 25 + q];
                sg[d] = mk<T>(-(pv.x * v), -(pv.y * v));
            }
            const T ze = dzdeta[q], zx = dzdxii[q], se = dsdeta[q], sx = dsdxii[q];
            sS[aa][0][q] = cadd(cscale(sg[0], ze), cscale(sg[4], se));
            sS[aa][1][q] = cadd(cscale(sg[0], zx), cscale(sg[4], sx));
            sS[aa][2][q] = cadd(cscale(sg[5], ze), cscale(sg[3], se));
            sS[aa][3][q] = cadd(cscale(sg[5], zx), cscale(sg[3], sx));
            sS[aa][4][q] = cadd(cscale(sg[4], ze), cscale(sg[2], se));
            sS[aa][5][q] = cadd(cscale(sg[4], zx), cscale(sg[2], sx));
            const T alf = (T)al;
            sA[aa][0][q] = csub(cia(alf, sg[5]), sg[1]);
            sA[aa][1][q] = cadd(cia(alf, sg[1]), sg[5]);
            sA[aa][2][q] = cia(alf, sg[3]);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < na * 25; i += blockDim.x) {
            const int aa = i / 25, q = i % 25, al = a0 + aa;
            const int ii = q / 5, jj = q % 5;
            for (int c = 0; c < 3; c++) {
                C g1 = mk<T>(0, 0), g2 = mk<T>(0, 0);
                for (int k = 0; k < 5; k++) {
                    const C xv = sS[aa][2 * c][k * 5 + jj], yv = sS[aa][2 * c + 1][ii * 5 + k];
                    const T gx = Gxi[ii * 5 + k], gt = sGll[jj * 5 + k];
                    g1.x += gx * xv.x; g1.y += gx * xv.y;
                    g2.x += yv.x * gt; g2.y += yv.y * gt;
                }
                C f = cadd(g1, g2);
                f = csub(f, cscale(sA[aa][c][q], invs[q]));
                if (axial) {
                    f = csub(f, cscale(cscale(sA[aa][c][jj], dzdeta[jj]), Gxi[ii * 5 + 0]));
                    if (ii == 0) {
                        C b = mk<T>(0, 0);
                        for (int k = 0; k < 5; k++) {
                            const C y0 = cscale(sA[aa][c][k], dzdxii[k]);
                            const T gt = sGll[jj * 5 + k];
                            b.x += y0.x * gt; b.y += y0.y * gt;
                        }
                        f = csub(f, b);
                    }
                }
                if (al < sNu[q])
                    atomic_add_cx(a.stiff + (size_t)a.wave[s] * a.fstride + (size_t)(sOff[q] + al) * 3 + c,
                                  mk<T>(-f.x, -f.y));
            }
        }
        __syncthreads();
    }
}

template <class T>
struct ForceArgs {
    int nsrc;
    const int *elem, *nu;
    const int64_t *pat_off;
    const cx_t<T> *pattern;            // [nu][3][25]
    const T *stf;
    int stf_steps;
    const int *step;
    const int *e_pts;
    const int *pt_off, *pt_nu;
    cx_t<T> *stiff;
    const int *wave;
    size_t fstride;
};

template <class T>
__global__ void force_source_kernel(const ForceArgs<T> a) {
    const int s = blockIdx.x;
    if (s >= a.nsrc || a.stf_steps <= 0 || a.stf == nullptr) return;
    const int e = a.elem[s];
    const int st = max(0, min(*a.step, a.stf_steps - 1));
    const T v = a.stf[(size_t)st * a.nsrc + s];
    for (int i = threadIdx.x; i < a.nu[s] * 25; i += blockDim.x) {
        const int al = i / 25, q = i % 25;
        const int p = a.e_pts[(size_t)e * 25 + q];
        if (al >= a.pt_nu[p]) continue;
        for (int c = 0; c < 3; c++) {
            const cx_t<T> pv = a.pattern[a.pat_off[s] + ((size_t)al * 3 + c) * 25 + q];
            atomic_add_cx(a.stiff + (size_t)a.wave[s] * a.fstride + (size_t)(a.pt_off[p] + al) * 3 + c,
                          mk<T>(pv.x * v, pv.y * v));
        }
    }
}

// FluidPressure::apply (core/source/elem_src/fluid/FluidPressure.cpp) -> FluidPoint::
// addPressureSource (FluidPoint.hpp:113-119): pattern [nu][25] x STF(t) added to the fluid
// points' acceleration after the mass term (FluidPoint::computeStiffToAccel, FluidPoint.cpp:
// 42-48), modes below the point's nu; same arguments as the force sources, one component
template <class T>
__global__ void pressure_source_kernel(const ForceArgs<T> a) {
    const int s = blockIdx.x;
    if (s >= a.nsrc || a.stf_steps <= 0 || a.stf == nullptr) return;
    const int e = a.elem[s];
    const int st = max(0, min(*a.step, a.stf_steps - 1));
    const T v = a.stf[(size_t)st * a.nsrc + s];
    for (int i = threadIdx.x; i < a.nu[s] * 25; i += blockDim.x) {
        const int al = i / 25, q = i % 25;
        const int p = a.e_pts[(size_t)e * 25 + q];
        if (al >= a.pt_nu[p]) continue;
        const cx_t<T> pv = a.pattern[a.pat_off[s] + (size_t)al * 25 + q];
        atomic_add_cx(a.stiff + (size_t)a.wave[s] * a.fstride + (size_t)(a.pt_off[p] + al),
                      mk<T>(pv.x * v, pv.y * v));
    }
}

// ----------------------------------------------------------------- stations ---
template <class T>
struct StationArgs {
    int nst;
    const int *elem;
    const T *w;               // [nst][25]
    const T *phi;             // [nst]
    const int *e_nr, *e_pts;
    const int *pt_off, *pt_nu;
    const cx_t<T> *displ;
    double *out;              // [nrec][nst][3]
    int interval;
    int max_rec;
    const int *step;
    int nwave;
    size_t fstride;
};

// one warp per (station, wavefield): the lanes take the (point, mode) pairs of the element,
// modes fastest (consecutive modes of a point are consecutive in memory, so the loads
// coalesce, and small nr still fills the warp); each lane adds the weighted terms of its
// pairs to the synthesis at phi, and a warp sum gives the three components
template <class T>
__global__ void station_kernel(const StationArgs<T> a) {
    const int warp = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= a.nst * a.nwave) return;              // whole warps leave together
    const int step = *a.step;
    if (step < 0 || a.out == nullptr || step % a.interval != 0) return;
    const int rec = step / a.interval;
    if (rec >= a.max_rec) return;
    const int wf = warp / a.nst, s = warp - wf * a.nst;
    const cx_t<T> *displ = a.displ + (size_t)wf * a.fstride;
    const int e = a.elem[s];
    const int nu = a.e_nr[e] / 2 + 1;
    const T phi = a.phi[s];
    T acc[3] = {0, 0, 0};
    for (int i = lane; i < nu * 25; i += 32) {
        const int q = i / nu, al = i - q * nu;
        const T w = a.w[(size_t)s * 25 + q];
        if (w == (T)0) continue;
        const int p = a.e_pts[(size_t)e * 25 + q];
        if (al >= a.pt_nu[p]) continue;
        const cx_t<T> *src = displ + (size_t)(a.pt_off[p] + al) * 3;
        if (al == 0) {
#pragma unroll
            for (int c = 0; c < 3; c++) acc[c] += w * src[c].x;
        } else {
            T sn, cs;
            if constexpr (sizeof(T) == 4) sincosf((T)al * phi, &sn, &cs);
            else sincos((T)al * phi, &sn, &cs);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const cx_t<T> x = src[c];
                acc[c] += (T)2 * w * (cs * x.x - sn * x.y);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], off);
    if (lane == 0) {
        double *o = a.out + (((size_t)rec * a.nwave + wf) * a.nst + s) * 3;
#pragma unroll
        for (int c = 0; c < 3; c++) o[c] = (double)acc[c];
    }
}

// displacement gradient at the stations (SolidElement::getNablaField without PRT, then
// Station::interpolate): one warp per (station, wavefield), lanes over the (point, mode)
// pairs; each lane forms d_j u_i (computeGrad9: index 3 i + j, s / phi / z) at its point
// from the element's 5 x 5 operators, with the L'Hopital row on the axis, and adds its
// weighted terms of the synthesis at phi; a warp sum gives the nine components
template <class T>
struct StationGradArgs {
    int nst;
    const int *elem;
    const T *w, *phi;
    const int *e_nr, *e_pts;
    const uint8_t *e_axial;
    const T *e_geom;          // [ne][250]: dsdxii, dsdeta, dzdxii, dzdeta, 1/s, ... (25 each)
    const T *gmat;            // [2][25]: G_GLL, G_GLJ
    const int *pt_off, *pt_nu;
    const cx_t<T> *displ;
    double *out;              // [nrec][nwave][nst][9]
    int interval, max_rec;
    const int *step;
    int nwave;
    size_t fstride;
};

// computeGrad9 (GradientQuadrature.hpp:177-202) of Fourier order al at GLL point q of one
// element, with the L'Hopital rows on the axis (:421-459): g[c * 3 + d] = d_d u_c, d = (s, phi, z)
template <class T>
__device__ __forceinline__ void grad9_point(const cx_t<T> *displ, const int *pts, const int *pt_off,
                                            const int *pt_nu, const T *geo, const T *Gxi, const T *Gll,
                                            bool axial, int q, int al, cx_t<T> g[9]) {
    using C = cx_t<T>;
    const int ii = q / 5, jj = q - ii * 5;
    auto U = [&](int pq, int c) -> C {
        const int p = pts[pq];
        return al < pt_nu[p] ? displ[(size_t)(pt_off[p] + al) * 3 + c] : mk<T>(0, 0);
    };
    const T alf = (T)al;
    // A_c = (i alpha u0 - u1, i alpha u1 + u0, i alpha u2) at point pq
    auto A = [&](int pq, int c) -> C {
        const C u0 = U(pq, 0), u1 = U(pq, 1), u2 = U(pq, 2);
        return c == 0 ? csub(cia(alf, u0), u1) : c == 1 ? cadd(cia(alf, u1), u0) : cia(alf, u2);
    };
    const T sx = geo[q], se = geo[25 + q], zx = geo[50 + q], ze = geo[75 + q], is = geo[100 + q];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        C x = mk<T>(0, 0), y = mk<T>(0, 0);
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const C uc = U(k * 5 + jj, c), ur = U(ii * 5 + k, c);
            const T gx = Gxi[k * 5 + ii], gy = Gll[k * 5 + jj];
            x.x += gx * uc.x; x.y += gx * uc.y;
            y.x += ur.x * gy; y.y += ur.y * gy;
        }
        g[c * 3 + 0] = cadd(cscale(x, ze), cscale(y, zx));        // d/ds
        g[c * 3 + 2] = cadd(cscale(x, se), cscale(y, sx));        // d/dz
        g[c * 3 + 1] = cscale(A(q, c), is);                       // (1/s) d/dphi terms
    }
    if (axial && ii == 0) {
        // L'Hopital on the axis: A / s replaced by dA/ds
#pragma unroll
        for (int c = 0; c < 3; c++) {
            C ax = mk<T>(0, 0), ay = mk<T>(0, 0);
#pragma unroll
            for (int k = 0; k < 5; k++) {
                ax = cadd(ax, cscale(A(k * 5 + jj, c), Gxi[k * 5 + 0]));
                ay = cadd(ay, cscale(A(k, c), Gll[k * 5 + jj]));
            }
            g[c * 3 + 1] = cadd(g[c * 3 + 1], cadd(cscale(ax, ze), cscale(ay, zx)));
        }
    }
}

template <class T>
__global__ void station_grad_kernel(const StationGradArgs<T> a) {
    using C = cx_t<T>;
    const int warp = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= a.nst * a.nwave) return;              // whole warps leave together
    const int step = *a.step;
    if (step < 0 || a.out == nullptr || step % a.interval != 0) return;
    const int rec = step / a.interval;
    if (rec >= a.max_rec) return;
    const int wf = warp / a.nst, s = warp - wf * a.nst;
    const C *displ = a.displ + (size_t)wf * a.fstride;
    const int e = a.elem[s];
    const int nu = a.e_nr[e] / 2 + 1;
    const bool axial = a.e_axial[e] != 0;
    const T *Gxi = axial ? a.gmat + 25 : a.gmat, *Gll = a.gmat;
    const T *geo = a.e_geom + (size_t)e * 250;
    const int *pts = a.e_pts + (size_t)e * 25;
    const T phi = a.phi[s];
    T acc[9];
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = 0;
    for (int i = lane; i < nu * 25; i += 32) {
        const int q = i / nu, al = i - q * nu;
        const T w = a.w[(size_t)s * 25 + q];
        if (w == (T)0) continue;
        C g[9];
        grad9_point<T>(displ, pts, a.pt_off, a.pt_nu, geo, Gxi, Gll, axial, q, al, g);
        if (al == 0) {
#pragma unroll
            for (int k = 0; k < 9; k++) acc[k] += w * g[k].x;
        } else {
            const T alf = (T)al;
            T sn, cs;
            if constexpr (sizeof(T) == 4) sincosf(alf * phi, &sn, &cs);
            else sincos(alf * phi, &sn, &cs);
#pragma unroll
            for (int k = 0; k < 9; k++) acc[k] += (T)2 * w * (cs * g[k].x - sn * g[k].y);
        }
    }
#pragma unroll
    for (int k = 0; k < 9; k++)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], off);
    if (lane == 0) {
        double *o = a.out + (((size_t)rec * a.nwave + wf) * a.nst + s) * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) o[k] = (double)acc[k];
    }
}

// Element-wise output (ElementOpSolid::record, core/output/element-wise/element/ElementOpSolid.cpp:
// 48-80, before its RTZ transform and channel forming): at every step that is a multiple of the
// interval, the Fourier coefficients of orders alpha < nr/2 + 1 of the element (the element's
// nu_1, collectDisplFromPoints) of the displacement (kind 0: 3 components) or of its gradient
// (kind 1: 9 components, computeGrad9) at one GLL point of one solid element, into slot
// (step / interval) % ring of a device ring of records, [ring][nwave][words], the entry's
// words at off[entry] with orders slowest and components fastest.
template <class T>
struct ElemRecordArgs {
    int n;
    const int *elem, *gll, *kind;
    const int64_t *off;
    int64_t words;
    const int *e_nr, *e_pts;
    const uint8_t *e_axial;
    const T *e_geom;
    const T *gmat;
    const int *pt_off, *pt_nu;
    const cx_t<T> *displ;
    cx_t<T> *out;
    int interval, ring;
    const int *step;
    int nwave;
    size_t fstride;
};

// one warp per (entry, wavefield); displacement entries: the lanes take consecutive
// (order, component) words, which are consecutive in the point's field and in the record
// (coalesced copy); gradient entries: one order per lane, all nine components
template <class T>
__global__ void element_record_kernel(const ElemRecordArgs<T> a) {
    using C = cx_t<T>;
    const int warp = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= a.n * a.nwave) return;                // whole warps leave together
    const int step = *a.step;
    if (step < 0 || step % a.interval != 0) return;
    const int slot = (step / a.interval) % a.ring;
    const int wf = warp / a.n, k = warp - wf * a.n;
    const C *displ = a.displ + (size_t)wf * a.fstride;
    C *out = a.out + ((size_t)slot * a.nwave + wf) * (size_t)a.words + (size_t)a.off[k];
    const int e = a.elem[k], q = a.gll[k];
    const int nu = a.e_nr[e] / 2 + 1;
    const int *pts = a.e_pts + (size_t)e * 25;
    if (a.kind[k] == 0) {
        const int p = pts[q];
        const int pnu = a.pt_nu[p];
        const C *src = displ + (size_t)a.pt_off[p] * 3;
        for (int i = lane; i < nu * 3; i += 32)
            out[i] = i / 3 < pnu ? src[i] : mk<T>(0, 0);
    } else {
        const bool axial = a.e_axial[e] != 0;
        const T *Gxi = axial ? a.gmat + 25 : a.gmat, *Gll = a.gmat;
        const T *geo = a.e_geom + (size_t)e * 250;
        for (int al = lane; al < nu; al += 32) {
            C g[9];
            grad9_point<T>(displ, pts, a.pt_off, a.pt_nu, geo, Gxi, Gll, axial, q, al, g);
#pragma unroll
            for (int c = 0; c < 9; c++) out[(size_t)al * 9 + c] = g[c];
        }
    }
}

// element-facing float copy of a double displacement (mixed precision)
template <class T, class D>
__global__ void narrow_kernel(const cx_t<D> *src, cx_t<T> *dst, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = mk<T>((T)src[i].x, (T)src[i].y);
}

template <class T>
__global__ void advance_step_kernel(int *step) { *step += 1; }


// ------------------------------------------------- boundary-stiffness exchange ---
// MessageRank::gatherFromPoints / scatterToPoints (MessageRank.cpp:40-63) with
// SolidPoint::feedComm / extractComm (SolidPoint.hpp:55-67): the point stiffness of the points a
// rank shares with a neighbour, as a list of complex slots of the field, copied into a
// contiguous buffer and, after the exchange, the neighbour's buffer added back.
template <class C>
__global__ void gather_slots_kernel(const C *__restrict__ field, const int64_t *__restrict__ slots, int64_t n,
                                    C *__restrict__ buf) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        buf[i] = field[slots[i]];
}
template <class C>
__global__ void scatter_add_slots_kernel(C *__restrict__ field, const int64_t *__restrict__ slots, int64_t n,
                                         const C *__restrict__ buf) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        C v = field[slots[i]];
        const C b = buf[i];
        v.x += b.x;
        v.y += b.y;
        field[slots[i]] = v;
    }
}

}  // namespace axg
