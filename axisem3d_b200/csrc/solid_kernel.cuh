// solid_kernel.cuh -- fused stiffness of solid spectral elements (nPol = 4).
//
// One team of threads evaluates one element at a time, entirely on chip:
//   gather u from the points (zero-padded above each point's nu)
//     SolidPoint::scatterDisplToElement   (SOLVER/src/core/point/SolidPoint.hpp:82-98)
//   GLL gradient + analytic d/dphi, axial L'Hopital rows
//     GradientQuadrature::computeGrad6    (SOLVER/src/core/element/grad/GradientQuadrature.hpp:207-231)
//   [RTZ] CoordTransformSpherical::transformSPZ_RTZ6 (crd/CoordTransformSpherical.hpp:186-216)
//   1-D material: strainToStress_FR per Fourier mode
//   3-D material: Fourier -> phi slices (direct DFT in shared memory, FFTW conventions,
//     SOLVER/src/core/fft/SolverFFTW.hpp:101-172), strainToStress_CD per slice,
//     slices -> Fourier
//   Isotropic / TransverselyIsotropic / Anisotropic::strainToStress
//     (material/elastic/anisotropy/*.hpp)
//   AttenuationFull / AttenuationCG4::apply (material/elastic/attenuation/*.hpp)
//   [RTZ] transformRTZ_SPZ6
//   GradientQuadrature::computeQuad6 (GradientQuadrature.hpp:294-324)
//   scatter-add: point.stiff -= f   SolidPoint::gatherStiffFromElement (SolidPoint.hpp:101-109)
//
// Shared memory per team (T = float or double, C = complex T):
//   geometry 10 x 25 T, trig 4 x 25 T, point tables 3 x 25 int, twiddles 2 x nr T,
//   region A: 6 x nu x 25 C  (strain E, then stress S, then quadrature X/Y)
//   region B: max(3 x mt x 25 C, nr x 6 x qc T)  (u, then stress slices, then A terms)
// The gather + gradient and the two quadrature passes run over tiles of mt modes (each
// Fourier mode is independent there), so region B holds one tile of u and of the A terms;
// mt = nu unless the element's nr is too large for that (one tile, the common case).
#pragma once

#include "common.cuh"

namespace axg {

constexpr int RHEO_ISO = 0, RHEO_TISO = 1, RHEO_ANISO = 2;
constexpr int ATT_NONE = 0, ATT_FULL = 1, ATT_CG4 = 2;
// register blocking of the two phi transforms and the occupancy target of the
// solid kernel (build-time tuning knobs)
#ifndef AXG_KB
#define AXG_KB 2
#endif
#ifndef AXG_AB
#define AXG_AB 2
#endif
#ifndef AXG_SOLID_MIN_BLOCKS
#define AXG_SOLID_MIN_BLOCKS 2
#endif
#ifndef AXG_PREFETCH_NEXT
#define AXG_PREFETCH_NEXT 0
#endif
// 1 = the register-resident slice path sums slices k and nr - k together (a pass of its
// own); 0 = one Fourier -> slice sum per (slice, point) inside the stress pass
#ifndef AXG_SLICE_PAIRS
#define AXG_SLICE_PAIRS 1
#endif
#ifndef AXG_KP
#define AXG_KP 2
#endif
// the same two blockings for elements without attenuation, whose slice pass holds no SLS
// state in registers and can afford wider blocks
#ifndef AXG_KP_ELASTIC
#define AXG_KP_ELASTIC 4
#endif
#ifndef AXG_AB_ELASTIC
#define AXG_AB_ELASTIC 4
#endif
// 1 = the stress pass of 3-D elements streams the SLS state of a (slice, point) in two
// groups of three stress components (the recursion acts on each component alone), so that
// 12 state words are live at a time instead of 24; 0 = the whole state loaded at once
#ifndef AXG_SLS_SPLIT
#define AXG_SLS_SPLIT 0
#endif
// > 0: each team prefetches into L2 the operands of the element AXG_PREFETCH_AHEAD waves of
// resident CTAs ahead (the distance in SolidArgs::prefetch_ahead)
#ifndef AXG_PREFETCH_AHEAD
#define AXG_PREFETCH_AHEAD 0
#endif
// 1 = attenuating 3-D elements on the direct sums run the Fourier -> slice sums and the stress
// pass as one pass: a thread per (slice pair, point) loads the operands of slice k, forms slices
// k and nr - k, and applies stress and SLS recursion to both (one barrier less, no strain slices
// through shared memory, the first slice's loads under the sums)
#ifndef AXG_FUSED_SLICE
#define AXG_FUSED_SLICE 0
#endif
// 1 = the stress pass's first (slice, point) of each thread has its SLS state loaded before the
// Fourier -> slice pass (its latency hidden under that pass)
#ifndef AXG_STATE_EARLY
#define AXG_STATE_EARLY 0
#endif
// 1 = L2 prefetch of an element's slice operands (moduli, attenuation moduli, SLS state)
// at the start of its slice phase
#ifndef AXG_PREFETCH_SLICES
#define AXG_PREFETCH_SLICES 1
#endif
// 1 = when a chunk holds all 25 points (and, for the slice -> Fourier pass, outside RTZ
// elements), the two direct-sum passes give each thread 6 consecutive columns of the
// (component, point) block instead of the 6 components of one point, read and written as
// 16- / 8-byte vectors, and order the threads 5 column groups by pair (or mode) groups, so
// that a warp touches few distinct words of region A, region B and the twiddle table per step
#ifndef AXG_COLUMN_TILES
#define AXG_COLUMN_TILES 1
#endif
// 1 = in FP32 arithmetic (the FP32 and mixed modes) the two direct-sum passes of a chunk of all
// 25 points run on the tensor cores as small matrix products, (columns x modes) x (modes x
// slice pairs) and (columns x slice pairs) x (slice pairs x modes), each operand split into a
// TF32 head and tail and three products accumulated in FP32 (head x head + head x tail +
// tail x head: the FP32 accuracy of the direct sums); the slice -> Fourier pass only outside
// RTZ elements. Warp-level mma.sync tiles: parity holds, but measured slower than the column-
// tiled FP32 sums on B200, so off
#ifndef AXG_TC_DFT
#define AXG_TC_DFT 0
#endif
// unrolling of the mode loop (Fourier -> slice) and of the slice loop (slice -> Fourier) of
// the column-tiled passes
#ifndef AXG_DFT_UNROLL
#define AXG_DFT_UNROLL 1
#endif
constexpr int KP = AXG_KP;   // slice pairs per thread in the paired Fourier -> slice pass
constexpr int KB = AXG_KB;   // slices per thread in the Fourier -> slice transform
constexpr int AB = AXG_AB;   // modes per thread in the slice -> Fourier transform
constexpr int DFT_UNROLL = AXG_DFT_UNROLL;

// The SLS state is read once and written once per step: with AXG_STREAM_STATE its loads and
// stores carry the streaming cache hint (evict first), so that it does not push the moduli and
// the point fields out of L2.
#ifndef AXG_STREAM_STATE
#define AXG_STREAM_STATE 0
#endif
template <class AT>
__device__ __forceinline__ AT state_ld(const AT *p) {
#if AXG_STREAM_STATE
    return __ldcs(p);
#else
    return *p;
#endif
}
template <class AT>
__device__ __forceinline__ void state_st(AT *p, AT v) {
#if AXG_STREAM_STATE
    __stcs(p, v);
#else
    *p = v;
#endif
}

template <class T, class AT>
struct SolidArgs {
    int n_elem;
    const int *nr;             // [n]
    const int *pts;            // [n*25]
    const uint8_t *axial;      // [n]
    const T *geom;             // [n][10][25]
    const T *trig;             // [n][4][25] sin t, cos t, sin 2t, cos 2t (RTZ only)
    const T *mod;              // moduli pool
    const int64_t *mod_off;    // [n]
    const T *attmod;           // dlambda, dmu pool
    const int64_t *att_off;    // [n]
    AT *state;                 // attenuation state pool
    const int64_t *state_off;  // [n] in AT units
    const int *pt_off;         // [npoints] first mode of each point
    const int *pt_nu;          // [npoints]
    const cx_t<T> *displ;      // [sum nu][3]
    cx_t<T> *stiff;            // [sum nu][3]
    const T *tw;               // twiddle pool: for each nr, nr cos then nr sin
    const int *tw_off;         // [nr_max + 1]
    int nsls;
    AT alpha[8], beta[8], gamma[8];
    const T *gmat;             // [2][25]: G_GLL, G_GLJ (row-major, G(j,i) = l_j'(x_i))
    int nwave;                 // wavefields sharing the mesh (independent sources)
    size_t fstride;            // complex values between wavefields in displ / stiff
    size_t sstride;            // AT values between wavefields in the state pool
    int fft_min_nr;            // 3-D elements with nr >= this (and 13-smooth nr) take the FFT; 0 = never
    int prefetch_ahead;        // > 0: each team prefetches into L2 the operands of the element this
                               // many places ahead (about one wave of resident CTAs); 0 = off
};

// shared memory layout of one team
struct TeamLayout {
    int nr_max, nu_max, qc;
    size_t geom, trig, ipt, tw, tws, regA, regB, total;
};

template <class T>
__host__ __device__ inline TeamLayout team_layout(int nr_max, int qc, int mt) {
    TeamLayout L;
    L.nr_max = nr_max;
    L.nu_max = nr_max / 2 + 1;
    L.qc = qc;
    mt = mt < L.nu_max ? mt : L.nu_max;
    size_t o = 0;
    auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
    L.geom = o; o = al(o + 10 * 25 * sizeof(T));
    L.trig = o; o = al(o + 4 * 25 * sizeof(T));
    L.ipt = o;  o = al(o + 3 * 25 * sizeof(int));
    L.tw = o;   o = al(o + 2 * (size_t)nr_max * sizeof(T));
    // the twiddles split for the tensor-core sums: (cos head, cos tail, sin head, sin tail)
    L.tws = o;  o = al(o + (AXG_TC_DFT && sizeof(T) == 4 ? 4 * (size_t)nr_max * sizeof(T) : 0));
    L.regA = o; o = al(o + 6 * (size_t)L.nu_max * 25 * 2 * sizeof(T));
    size_t b1 = 3 * (size_t)mt * 25 * 2 * sizeof(T);
    size_t b2 = (size_t)nr_max * 6 * qc * sizeof(T);
    L.regB = o; o = al(o + (b1 > b2 ? b1 : b2));
    L.total = o;
    return L;
}

// six consecutive complex / real values of a team's shared buffers as 16- or 8-byte vectors;
// complex groups start on 16 bytes, real groups on 2 T (the callers' column groups start at
// even offsets of 16-byte aligned regions)
template <class T>
__device__ __forceinline__ void ld6c(const cx_t<T> *p, cx_t<T> (&v)[6]) {
    if constexpr (sizeof(T) == 4) {
        const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float4 t = q[i];
            v[2 * i] = mk<T>(t.x, t.y);
            v[2 * i + 1] = mk<T>(t.z, t.w);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 6; i++) v[i] = p[i];
    }
}
template <class T>
__device__ __forceinline__ void st6c(cx_t<T> *p, const cx_t<T> (&v)[6]) {
    if constexpr (sizeof(T) == 4) {
        float4 *q = reinterpret_cast<float4 *>(p);
#pragma unroll
        for (int i = 0; i < 3; i++) q[i] = make_float4(v[2 * i].x, v[2 * i].y, v[2 * i + 1].x, v[2 * i + 1].y);
    } else {
#pragma unroll
        for (int i = 0; i < 6; i++) p[i] = v[i];
    }
}
template <class T>
__device__ __forceinline__ void ld6r(const T *p, T (&v)[6]) {
    const cx_t<T> *q = reinterpret_cast<const cx_t<T> *>(p);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const cx_t<T> t = q[i];
        v[2 * i] = t.x;
        v[2 * i + 1] = t.y;
    }
}
template <class T>
__device__ __forceinline__ void st6r(T *p, const T (&v)[6]) {
    cx_t<T> *q = reinterpret_cast<cx_t<T> *>(p);
#pragma unroll
    for (int i = 0; i < 3; i++) q[i] = mk<T>(v[2 * i], v[2 * i + 1]);
}

// ------------------------------------------------- tensor-core direct sums ---
// TF32 head of x (round to nearest, ties away: exact in TF32, whatever the tensor core does with
// the low 13 bits of an operand) and the tail x - head (exact in FP32; its own rounding to TF32
// costs at most 2^-22 |x|)
__device__ __forceinline__ uint32_t tf32_head(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void tf32_split(float x, uint32_t &h, uint32_t &t) {
    h = tf32_head(x);
    t = tf32_head(x - __uint_as_float(h));
}
// d += a b for one m16n8k8 tile: a (16 x 8, row-major fragment: a0 (g, c), a1 (g + 8, c),
// a2 (g, c + 4), a3 (g + 8, c + 4)), b (8 x 8: b0 (c, g), b1 (c + 4, g)), d (16 x 8: d0 (g, 2c),
// d1 (g, 2c + 1), d2 (g + 8, 2c), d3 (g + 8, 2c + 1)); g = lane / 4, c = lane % 4
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// (ah + at) (bh + bt) without the tail x tail product, into three accumulators (head x head,
// and the two cross terms) so that the three products do not wait on one another
__device__ __forceinline__ void mma_tf32x3(float (&d)[3][4], const uint32_t (&ah)[4], const uint32_t (&at)[4],
                                           uint32_t bh0, uint32_t bh1, uint32_t bt0, uint32_t bt1) {
    mma_tf32(d[0], ah, bh0, bh1);
    mma_tf32(d[1], at, bh0, bh1);
    mma_tf32(d[2], ah, bt0, bt1);
}
// x mod n for 0 <= x < 2^22 with rn = 1 / n (a float quotient off by at most one, corrected)
__device__ __forceinline__ int mod_n(int x, int n, float rn) {
    int r = x - (int)((float)x * rn) * n;
    r += r < 0 ? n : 0;
    return r >= n ? r - n : r;
}

// Fourier -> slices of a chunk holding all 25 points, on the tensor cores. Rows n = d * 25 + q of
// the (component, point) block (10 tiles of 16), columns k = slice pairs 0 .. nr/2 (tiles of 8),
// modes a = 1 .. nu - 1 in steps of 8: A[n][k] = sum_a Re c_a[n] cos(a k 2pi/nr) and
// B[n][k] = sum_a Im c_a[n] sin(a k 2pi/nr), then x_k = c0 + 2 (A - B), x_{nr-k} = c0 + 2 (A + B)
// (the paired direct sums, each product in three TF32 parts)
template <class T>
__device__ __forceinline__ void tc_fourier_to_slices(const cx_t<T> *rA, T *rBr, const float4 *tws, int nr,
                                                     int lane, int TEAM) {
    if constexpr (sizeof(T) == 4) {
        const int nu = nr / 2 + 1;
        const int wi = lane >> 5, nw = TEAM >> 5, g = (lane & 31) >> 2, c = lane & 3;
        const int NT = (nu + 7) >> 3, KS = (nu - 1 + 7) >> 3;
        const float rnr = 1.f / (float)nr;
        for (int t = wi; t < 10 * NT; t += nw) {
            const int mt = t % 10, nt = t / 10;
            const int n0 = mt * 16 + g, n1 = n0 + 8, kp = nt * 8 + g;
            float dA[3][4] = {}, dB[3][4] = {};
            // twiddle indices (a k) mod nr of this thread's two B rows, modes 1 + c and 5 + c
            int j0 = mod_n((1 + c) * kp, nr, rnr), j1 = mod_n((5 + c) * kp, nr, rnr);
            const int s8 = mod_n(8 * kp, nr, rnr);
            for (int ks = 0; ks < KS; ks++) {
                const int a0 = 1 + 8 * ks + c, a1 = a0 + 4;
                const float2 z = make_float2(0.f, 0.f);
                float2 v[4];
                v[0] = (a0 < nu && n0 < 150) ? rA[a0 * 150 + n0] : z;
                v[1] = (a0 < nu && n1 < 150) ? rA[a0 * 150 + n1] : z;
                v[2] = (a1 < nu && n0 < 150) ? rA[a1 * 150 + n0] : z;
                v[3] = (a1 < nu && n1 < 150) ? rA[a1 * 150 + n1] : z;
                uint32_t rh[4], rt[4], ih[4], it[4];
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    tf32_split(v[r].x, rh[r], rt[r]);
                    tf32_split(v[r].y, ih[r], it[r]);
                }
                const float4 w0 = tws[j0], w1 = tws[j1];
                mma_tf32x3(dA, rh, rt, __float_as_uint(w0.x), __float_as_uint(w1.x), __float_as_uint(w0.y),
                           __float_as_uint(w1.y));
                mma_tf32x3(dB, ih, it, __float_as_uint(w0.z), __float_as_uint(w1.z), __float_as_uint(w0.w),
                           __float_as_uint(w1.w));
                j0 += s8;
                j0 = j0 >= nr ? j0 - nr : j0;
                j1 += s8;
                j1 = j1 >= nr ? j1 - nr : j1;
            }
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int n = r < 2 ? n0 : n1, k = nt * 8 + 2 * c + (r & 1);
                if (n < 150 && k < nu) {
                    const float c0 = rA[n].x;
                    const float A = dA[0][r] + (dA[1][r] + dA[2][r]), B = dB[0][r] + (dB[1][r] + dB[2][r]);
                    rBr[k * 150 + n] = c0 + 2.f * (A - B);
                    if (k != 0 && 2 * k != nr) rBr[(nr - k) * 150 + n] = c0 + 2.f * (A + B);
                }
            }
        }
    }
}

// slices -> Fourier of a chunk holding all 25 points, on the tensor cores: rows n of the block,
// columns a = 0 .. nu - 1 (tiles of 8), slice pairs k = 0 .. nr/2 in steps of 8:
// Re S_a[n] = sum_k xs_k[n] cos(a k 2pi/nr) / nr, Im S_a[n] = -sum_k xd_k[n] sin(a k 2pi/nr) / nr
// with xs_k = x_k + x_{nr-k}, xd_k = x_k - x_{nr-k} (x_k alone at k = 0 and nr/2), the Nyquist
// mode halved and the imaginary parts of modes 0 and nr/2 dropped
template <class T>
__device__ __forceinline__ void tc_slices_to_fourier(cx_t<T> *rA, const T *rBr, const float4 *tws, int nr,
                                                     T inv_nr, int lane, int TEAM) {
    if constexpr (sizeof(T) == 4) {
        const int nu = nr / 2 + 1;
        const int wi = lane >> 5, nw = TEAM >> 5, g = (lane & 31) >> 2, c = lane & 3;
        const int NT = (nu + 7) >> 3, KS = (nu + 7) >> 3;
        const float rnr = 1.f / (float)nr;
        auto sd = [&](int k, int n, float &xs, float &xd) {
            xs = 0.f;
            xd = 0.f;
            if (k < nu && n < 150) {
                const float x1 = rBr[k * 150 + n];
                xs = x1;
                if (k != 0 && 2 * k != nr) {
                    const float x2 = rBr[(nr - k) * 150 + n];
                    xs = x1 + x2;
                    xd = x1 - x2;
                }
            }
        };
        for (int t = wi; t < 10 * NT; t += nw) {
            const int mt = t % 10, nt = t / 10;
            const int n0 = mt * 16 + g, n1 = n0 + 8, am = nt * 8 + g;
            float dC[3][4] = {}, dS[3][4] = {};
            // twiddle indices (k a) mod nr of this thread's two B rows, slices c and c + 4
            int j0 = mod_n(c * am, nr, rnr), j1 = mod_n((c + 4) * am, nr, rnr);
            const int s8 = mod_n(8 * am, nr, rnr);
            for (int ks = 0; ks < KS; ks++) {
                const int k0 = 8 * ks + c, k1 = k0 + 4;
                float xs[4], xd[4];
                sd(k0, n0, xs[0], xd[0]);
                sd(k0, n1, xs[1], xd[1]);
                sd(k1, n0, xs[2], xd[2]);
                sd(k1, n1, xs[3], xd[3]);
                uint32_t sh[4], st[4], dh[4], dt[4];
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    tf32_split(xs[r], sh[r], st[r]);
                    tf32_split(xd[r], dh[r], dt[r]);
                }
                const float4 w0 = tws[j0], w1 = tws[j1];
                mma_tf32x3(dC, sh, st, __float_as_uint(w0.x), __float_as_uint(w1.x), __float_as_uint(w0.y),
                           __float_as_uint(w1.y));
                mma_tf32x3(dS, dh, dt, __float_as_uint(w0.z), __float_as_uint(w1.z), __float_as_uint(w0.w),
                           __float_as_uint(w1.w));
                j0 += s8;
                j0 = j0 >= nr ? j0 - nr : j0;
                j1 += s8;
                j1 = j1 >= nr ? j1 - nr : j1;
            }
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int n = r < 2 ? n0 : n1, al = nt * 8 + 2 * c + (r & 1);
                if (n < 150 && al < nu) {
                    const bool nyq = (nr & 1) == 0 && al == nr / 2;
                    const float re = (dC[0][r] + (dC[1][r] + dC[2][r])) * (nyq ? 0.5f * inv_nr : inv_nr);
                    const float im = (al == 0 || nyq) ? 0.f : -(dS[0][r] + (dS[1][r] + dS[2][r])) * inv_nr;
                    rA[al * 150 + n] = make_float2(re, im);
                }
            }
        }
    }
}

// ------------------------------------------------------------ rheology ---
// Isotropic::strainToStress (Isotropic.hpp:154-170); 2 mu is exact as mu + mu
template <class V, class R>
__device__ __forceinline__ void stress_iso(const V e[6], V s[6], R lam, R mu) {
    R mu2 = mu + mu;
    V sii = cscale(cadd(cadd(e[0], e[1]), e[2]), lam);
    s[0] = cadd(sii, cscale(e[0], mu2));
    s[1] = cadd(sii, cscale(e[1], mu2));
    s[2] = cadd(sii, cscale(e[2], mu2));
    s[3] = cscale(e[3], mu);
    s[4] = cscale(e[4], mu);
    s[5] = cscale(e[5], mu);
}
// TransverselyIsotropic::strainToStress (TransverselyIsotropic.hpp:160-180)
template <class V, class R>
__device__ __forceinline__ void stress_tiso(const V e[6], V s[6], R A, R C, R F, R L, R Nn) {
    R mN2 = -(Nn + Nn);
    V t3 = cadd(e[0], e[1]);
    V t4 = cadd(cscale(t3, A), cscale(e[2], F));
    s[0] = cadd(t4, cscale(e[1], mN2));
    s[1] = cadd(t4, cscale(e[0], mN2));
    s[2] = cadd(cscale(t3, F), cscale(e[2], C));
    s[3] = cscale(e[3], L);
    s[4] = cscale(e[4], L);
    s[5] = cscale(e[5], Nn);
}
// Anisotropic::strainToStress (Anisotropic.hpp:202-274); c = upper triangle row-major
template <class V, class R>
__device__ __forceinline__ void stress_aniso(const V e[6], V s[6], const R c[21]) {
    const int idx[6][6] = {{0, 1, 2, 3, 4, 5},      {1, 6, 7, 8, 9, 10},
                           {2, 7, 11, 12, 13, 14},  {3, 8, 12, 15, 16, 17},
                           {4, 9, 13, 16, 18, 19},  {5, 10, 14, 17, 19, 20}};
#pragma unroll
    for (int i = 0; i < 6; i++) {
        V acc = cscale(e[0], c[idx[i][0]]);
#pragma unroll
        for (int j = 1; j < 6; j++) acc = cadd(acc, cscale(e[j], c[idx[i][j]]));
        s[i] = acc;
    }
}

// scalar "complex" wrapper so that the rheology templates serve real slices too
template <class T> struct re1 { T x; };
template <class T> __device__ __forceinline__ re1<T> cadd(re1<T> a, re1<T> b) { return {a.x + b.x}; }
template <class T> __device__ __forceinline__ re1<T> csub(re1<T> a, re1<T> b) { return {a.x - b.x}; }
template <class T, class R> __device__ __forceinline__ re1<T> cscale(re1<T> a, R s) { return {a.x * (T)s}; }

template <int RHEO, class T, class V>
__device__ __forceinline__ void elastic_at(const T *mod, int nslice, int slice, int q,
                                           const V e[6], V s[6]) {
    const size_t ns = (size_t)nslice * 25, o = (size_t)slice * 25 + q;
    if constexpr (RHEO == RHEO_ISO) {
        stress_iso(e, s, __ldg(mod + o), __ldg(mod + ns + o));
    } else if constexpr (RHEO == RHEO_TISO) {
        stress_tiso(e, s, __ldg(mod + o), __ldg(mod + ns + o), __ldg(mod + 2 * ns + o),
                    __ldg(mod + 3 * ns + o), __ldg(mod + 4 * ns + o));
    } else {
        T c[21];
#pragma unroll
        for (int k = 0; k < 21; k++) c[k] = __ldg(mod + k * ns + o);
        stress_aniso(e, s, c);
    }
}

// CoordTransformSpherical::transformSPZ_RTZ6 / transformRTZ_SPZ6 (one point of one mode)
template <class V, class T>
__device__ __forceinline__ void spz_to_rtz6(V e[6], T s1, T c1, T s2, T c2) {
    const T half = (T)0.5;
    V s02 = cadd(e[0], e[2]), d02 = csub(e[0], e[2]);
    e[0] = cscale(csub(cadd(s02, cscale(d02, c2)), cscale(e[4], s2)), half);
    e[2] = csub(s02, e[0]);
    e[4] = cadd(cscale(e[4], c2), cscale(d02, s2));
    V t3 = e[3];
    e[3] = cadd(cscale(t3, c1), cscale(e[5], s1));
    e[5] = csub(cscale(e[5], c1), cscale(t3, s1));
}
template <class V, class T>
__device__ __forceinline__ void rtz_to_spz6(V s[6], T s1, T c1, T s2, T c2) {
    const T half = (T)0.5;
    V s02 = cadd(s[0], s[2]), d02 = csub(s[0], s[2]);
    s[0] = cadd(cscale(cadd(s02, cscale(d02, c2)), half), cscale(s[4], s2));
    s[2] = csub(s02, s[0]);
    s[4] = csub(cscale(s[4], c2), cscale(cscale(d02, s2), half));
    V t3 = s[3];
    s[3] = csub(cscale(t3, c1), cscale(s[5], s1));
    s[5] = cadd(cscale(s[5], c1), cscale(t3, s1));
}

// ----------------------------------------------------------- attenuation ---
// One point of one mode (complex) or slice (real):
//   stress -= sum_l mem_l; mem_l = alpha_l mem_l + beta_l dstress;
//   dstress = iso(dlambda, dmu)(strain); mem_l += gamma_l dstress
// (AttenuationFull.hpp:189-207, Attenuation.hpp:92-134). The state (dstress,
// mem) lives in AT (double in the mixed-precision mode) and is streamed from
// and to HBM once per step.
template <bool CPLX, class AT, class V>
__device__ __forceinline__ AT part(const V &v, int w) {
    if constexpr (CPLX) return (AT)(w ? v.y : v.x);
    else return (AT)v.x;
}

template <class T, class AT, bool CPLX, class V>
__device__ __forceinline__ void attenuate(const SolidArgs<T, AT> &a, AT *state, size_t nslot,
                                          size_t slot, const V e[6], V s[6], T dl, T dm) {
    constexpr int W = CPLX ? 2 : 1;
    AT *dst = state;                             // [6][nslot] (x W)
    AT *mem = state + 6 * nslot * W;             // [nsls][6][nslot] (x W)
    const size_t sls = 6 * nslot * W;
    AT ds[6][W], sv[6][W];
#pragma unroll
    for (int d = 0; d < 6; d++)
#pragma unroll
        for (int w = 0; w < W; w++) {
            ds[d][w] = dst[(d * nslot + slot) * W + w];
            sv[d][w] = part<CPLX, AT>(s[d], w);
        }
    for (int l = 0; l < a.nsls; l++) {
        AT *m = mem + l * sls;
        const AT al = a.alpha[l], be = a.beta[l];
#pragma unroll
        for (int d = 0; d < 6; d++)
#pragma unroll
            for (int w = 0; w < W; w++) {
                AT mv = m[(d * nslot + slot) * W + w];
                sv[d][w] -= mv;
                m[(d * nslot + slot) * W + w] = al * mv + be * ds[d][w];
            }
    }
    // new dstress from the strain (Isotropic::strainToStress with dlambda, dmu)
    const AT lam = (AT)dl, mu = (AT)dm, mu2 = mu + mu;
#pragma unroll
    for (int w = 0; w < W; w++) {
        const AT e0 = part<CPLX, AT>(e[0], w), e1 = part<CPLX, AT>(e[1], w),
                 e2 = part<CPLX, AT>(e[2], w);
        const AT sii = (e0 + e1 + e2) * lam;
        ds[0][w] = sii + e0 * mu2;
        ds[1][w] = sii + e1 * mu2;
        ds[2][w] = sii + e2 * mu2;
        ds[3][w] = part<CPLX, AT>(e[3], w) * mu;
        ds[4][w] = part<CPLX, AT>(e[4], w) * mu;
        ds[5][w] = part<CPLX, AT>(e[5], w) * mu;
    }
#pragma unroll
    for (int d = 0; d < 6; d++)
#pragma unroll
        for (int w = 0; w < W; w++) dst[(d * nslot + slot) * W + w] = ds[d][w];
    for (int l = 0; l < a.nsls; l++) {
        AT *m = mem + l * sls;
        const AT ga = a.gamma[l];
#pragma unroll
        for (int d = 0; d < 6; d++)
#pragma unroll
            for (int w = 0; w < W; w++) m[(d * nslot + slot) * W + w] += ga * ds[d][w];
    }
#pragma unroll
    for (int d = 0; d < 6; d++) {
        if constexpr (CPLX) { s[d].x = (T)sv[d][0]; s[d].y = (T)sv[d][1]; }
        else s[d].x = (T)sv[d][0];
    }
}

// L2 prefetch of [p, p + bytes), 128-byte lines spread over the team; every
// address issued lies inside the region (lines are aligned down only at the start,
// and pools are 256-byte aligned allocations)
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes, int lane, int team) {
    const uintptr_t a1 = (uintptr_t)p + bytes;
    uintptr_t a = ((uintptr_t)p & ~(uintptr_t)127) + (uintptr_t)lane * 128;
    for (; a < a1; a += (uintptr_t)team * 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
}

// bytes of the per-element streams (geometry, moduli, attenuation moduli, state)
template <class T, class AT, int RHEO, int ATT, bool IS3D>
__device__ __forceinline__ void prefetch_element(const SolidArgs<T, AT> &a, int e, int lane, int team) {
    const int nr = a.nr[e], nu = nr / 2 + 1, ns = IS3D ? nr : 1;
    constexpr int nmod = RHEO == RHEO_ISO ? 2 : RHEO == RHEO_TISO ? 5 : 21;
    prefetch_l2(a.geom + (size_t)e * 250, 250 * sizeof(T), lane, team);
    prefetch_l2(a.mod + a.mod_off[e], (size_t)nmod * ns * 25 * sizeof(T), lane, team);
    if constexpr (ATT != ATT_NONE) {
        constexpr int npa = ATT == ATT_CG4 ? 4 : 25;
        prefetch_l2(a.attmod + a.att_off[e], (size_t)2 * ns * npa * sizeof(T), lane, team);
        const size_t slots = IS3D ? (size_t)nr * npa : (size_t)nu * npa * 2;
        prefetch_l2(a.state + a.state_off[e], (size_t)(a.nsls + 1) * 6 * slots * sizeof(AT), lane, team);
    }
}

// SLS recursion on one real slice point with the state already in registers
// (same steps and order as attenuate<>; NS = number of SLS, a compile-time size)
template <int NS, class T, class AT>
__device__ __forceinline__ void attenuate_regs(const AT *alpha, const AT *beta, const AT *gamma, AT ds[6],
                                               AT mem[NS][6], const T e[6], T s[6], T dl, T dm) {
    AT sv[6];
#pragma unroll
    for (int d = 0; d < 6; d++) sv[d] = (AT)s[d];
#pragma unroll
    for (int l = 0; l < NS; l++)
#pragma unroll
        for (int d = 0; d < 6; d++) {
            sv[d] -= mem[l][d];
            mem[l][d] = alpha[l] * mem[l][d] + beta[l] * ds[d];
        }
    const AT lam = (AT)dl, mu = (AT)dm, mu2 = mu + mu;
    const AT e0 = (AT)e[0], e1 = (AT)e[1], e2 = (AT)e[2];
    const AT sii = (e0 + e1 + e2) * lam;
    ds[0] = sii + e0 * mu2;
    ds[1] = sii + e1 * mu2;
    ds[2] = sii + e2 * mu2;
    ds[3] = (AT)e[3] * mu;
    ds[4] = (AT)e[4] * mu;
    ds[5] = (AT)e[5] * mu;
#pragma unroll
    for (int l = 0; l < NS; l++)
#pragma unroll
        for (int d = 0; d < 6; d++) mem[l][d] += gamma[l] * ds[d];
#pragma unroll
    for (int d = 0; d < 6; d++) s[d] = (T)sv[d];
}

// SLS recursion on one real slice point with the state streamed from memory in two groups of
// three stress components, (0, 1, 2) then (3, 4, 5): each group loads its 3 + 3 NS words at once,
// updates them with the steps and order of attenuate_regs (per component the same operations,
// so the same results) and stores them back. State word j of the slot is at j * nslot + slot.
template <int NS, class T, class AT>
__device__ __forceinline__ void attenuate_slice_split(const AT *alpha, const AT *beta, const AT *gamma, AT *st,
                                                      size_t nslot, size_t slot, const T e[6], T s[6], T dl,
                                                      T dm) {
    const AT lam = (AT)dl, mu = (AT)dm, mu2 = mu + mu;
#pragma unroll
    for (int g = 0; g < 2; g++) {
        const int d0 = 3 * g;
        AT ds[3], mem[NS][3];
#pragma unroll
        for (int c = 0; c < 3; c++) ds[c] = state_ld(st + (d0 + c) * nslot + slot);
#pragma unroll
        for (int l = 0; l < NS; l++)
#pragma unroll
            for (int c = 0; c < 3; c++) mem[l][c] = state_ld(st + (6 + l * 6 + d0 + c) * nslot + slot);
        AT dn[3];
        if (g == 0) {
            const AT e0 = (AT)e[0], e1 = (AT)e[1], e2 = (AT)e[2];
            const AT sii = (e0 + e1 + e2) * lam;
            dn[0] = sii + e0 * mu2;
            dn[1] = sii + e1 * mu2;
            dn[2] = sii + e2 * mu2;
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) dn[c] = (AT)e[3 + c] * mu;
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            AT sv = (AT)s[d0 + c];
#pragma unroll
            for (int l = 0; l < NS; l++) {
                sv -= mem[l][c];
                mem[l][c] = alpha[l] * mem[l][c] + beta[l] * ds[c];
            }
#pragma unroll
            for (int l = 0; l < NS; l++) mem[l][c] += gamma[l] * dn[c];
            s[d0 + c] = (T)sv;
            state_st(st + (d0 + c) * nslot + slot, dn[c]);
        }
#pragma unroll
        for (int l = 0; l < NS; l++)
#pragma unroll
            for (int c = 0; c < 3; c++) state_st(st + (6 + l * 6 + d0 + c) * nslot + slot, mem[l][c]);
    }
}

// SLS recursion on one complex Fourier-space slot of a 1-D element, state in registers. The
// recursion is linear and acts on each stress component separately, on the real and the
// imaginary parts alike, so the slot runs in four passes: (real, imaginary) x (components
// 0-2, which share the trace of the strain, and 3-5). Each pass loads its 3 + 3 NS state
// words at once (independent loads whose latencies overlap), updates them in registers with
// the steps and order of attenuate_regs, and stores them back. Same layout and results as
// attenuate<T, AT, true>: part w of state word j of the slot is at (j * nslot + slot) * 2 + w.
template <int NS, class T, class AT>
__device__ __forceinline__ void attenuate_cplx_regs(const SolidArgs<T, AT> &a, AT *state, size_t nslot,
                                                    size_t slot, const cx_t<T> e[6], cx_t<T> s[6], T dl,
                                                    T dm) {
    const AT lam = (AT)dl, mu = (AT)dm, mu2 = mu + mu;
#pragma unroll 1
    for (int pass = 0; pass < 4; pass++) {
        const int w = pass & 1, d0 = (pass >> 1) * 3;
        AT *base = state + w;
        AT ds[3], mem[NS][3];
#pragma unroll
        for (int c = 0; c < 3; c++) ds[c] = base[((d0 + c) * nslot + slot) * 2];
#pragma unroll
        for (int l = 0; l < NS; l++)
#pragma unroll
            for (int c = 0; c < 3; c++) mem[l][c] = base[((6 + l * 6 + d0 + c) * nslot + slot) * 2];
        // new dstress of these components (Isotropic::strainToStress with dlambda, dmu)
        AT dn[3];
        if (d0 == 0) {
            const AT e0 = (AT)(w ? e[0].y : e[0].x), e1 = (AT)(w ? e[1].y : e[1].x),
                     e2 = (AT)(w ? e[2].y : e[2].x);
            const AT sii = (e0 + e1 + e2) * lam;
            dn[0] = sii + e0 * mu2;
            dn[1] = sii + e1 * mu2;
            dn[2] = sii + e2 * mu2;
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) dn[c] = (AT)(w ? e[3 + c].y : e[3 + c].x) * mu;
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            AT sv = (AT)(w ? s[d0 + c].y : s[d0 + c].x);
#pragma unroll
            for (int l = 0; l < NS; l++) {
                sv -= mem[l][c];
                mem[l][c] = a.alpha[l] * mem[l][c] + a.beta[l] * ds[c];
            }
#pragma unroll
            for (int l = 0; l < NS; l++) mem[l][c] += a.gamma[l] * dn[c];
            if (w) s[d0 + c].y = (T)sv;
            else s[d0 + c].x = (T)sv;
            base[((d0 + c) * nslot + slot) * 2] = dn[c];
        }
#pragma unroll
        for (int l = 0; l < NS; l++)
#pragma unroll
            for (int c = 0; c < 3; c++) base[((6 + l * 6 + d0 + c) * nslot + slot) * 2] = mem[l][c];
    }
}

// 1-D elements: the register-resident recursion for 3 and 5 SLS, the generic one otherwise
template <int NS, class T, class AT>
__device__ __forceinline__ void attenuate_1d(const SolidArgs<T, AT> &a, AT *state, size_t nslot, size_t slot,
                                             const cx_t<T> e[6], cx_t<T> s[6], T dl, T dm) {
    if constexpr (NS > 0) attenuate_cplx_regs<NS, T, AT>(a, state, nslot, slot, e, s, dl, dm);
    else attenuate<T, AT, true>(a, state, nslot, slot, e, s, dl, dm);
}

__device__ __forceinline__ int cg4_slot(int q) {
    // (1,1) (1,3) (3,1) (3,3) -> 0..3, else -1
    return q == 6 ? 0 : q == 8 ? 1 : q == 16 ? 2 : q == 18 ? 3 : -1;
}

// ------------------------------------------------------------- slice FFT ---
// The phi transforms of a 3-D element (SolverFFTW::computeC2R / computeR2C, SolverFFTW.hpp:
// 101-172: R2C scaled by 1/nr, the Nyquist mode halved, imaginary parts of modes 0 and nr/2
// dropped; C2R with the Nyquist mode doubled) as complex FFTs of length nr over a batch of
// S = 3 qc signals: the six strain / stress components of a point go in pairs, x_2p + i x_2p+1,
// one complex signal per pair. The FFT is a mixed-radix Stockham transform in shared memory
// (radices 4, 2, 3, 5, 7, 11, 13: every nr the reference's lucky-number rule admits), one pass
// per radix between two buffers. Signal s = pair pp of
// point qq of the chunk (s = pp qc + qq), sample n. The two buffers are views of shared memory
// the element holds anyway: region B as [n][pp][qq] (row n of 3 qc values), and the columns of
// the chunk's points in region A, whose strain the spectra were formed from and whose stress
// the last pass's unpacking writes, as rows 3 n + pp of 25 values. Twiddles come from the
// element's table of exp(2 pi i j / nr).

// radices of n, powers of 4 first, then 2, 3, 5, 7, 11, 13, packed 3 bits per pass (codes
// 1..7 for 4, 2, 3, 5, 7, 11, 13) into the returned plan; 0 if n has another prime factor
// (those transforms take the direct sums)
__device__ __forceinline__ unsigned fft_plan(int n) {
    unsigned plan = 0;
    int c = 0;
    while (n % 4 == 0) { plan |= 1u << (3 * c++); n /= 4; }
    while (n % 2 == 0) { plan |= 2u << (3 * c++); n /= 2; }
    while (n % 3 == 0) { plan |= 3u << (3 * c++); n /= 3; }
    while (n % 5 == 0) { plan |= 4u << (3 * c++); n /= 5; }
    while (n % 7 == 0) { plan |= 5u << (3 * c++); n /= 7; }
    while (n % 11 == 0) { plan |= 6u << (3 * c++); n /= 11; }
    while (n % 13 == 0) { plan |= 7u << (3 * c++); n /= 13; }
    return (n == 1 && c <= 10) ? plan : 0u;
}

// twiddle exp(sign 2 pi i m / N) from the interleaved (cos, sin) table
template <class T>
__device__ __forceinline__ cx_t<T> fft_tw(const cx_t<T> *tw2, int m, int sign) {
    const cx_t<T> w = tw2[m];
    return mk<T>(w.x, sign > 0 ? w.y : -w.y);
}
template <class T>
__device__ __forceinline__ cx_t<T> cmul(cx_t<T> a, cx_t<T> b) {
    return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// in-register DFT of R points with sign: V_t = sum_r v_r exp(sign 2 pi i r t / R)
template <int R, class T>
__device__ __forceinline__ void fft_radix(cx_t<T> v[R], int sign, const cx_t<T> *tw2, int N) {
    using C = cx_t<T>;
    if constexpr (R == 2) {
        const C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        const C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        const C s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
        // j d13 with j = sign i
        const C jd = sign > 0 ? mk<T>(-d13.y, d13.x) : mk<T>(d13.y, -d13.x);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cadd(d02, jd);
        v[3] = csub(d02, jd);
    } else {
        C V[R];
        const int step = N / R;
#pragma unroll
        for (int t = 0; t < R; t++) {
            C acc = v[0];
#pragma unroll
            for (int r = 1; r < R; r++) acc = cadd(acc, cmul<T>(v[r], fft_tw<T>(tw2, ((r * t) % R) * step, sign)));
            V[t] = acc;
        }
#pragma unroll
        for (int t = 0; t < R; t++) v[t] = V[t];
    }
}

// a batch of signals in shared memory: sample n of signal (pp, qq) at p[n rs + pp ps + qq]
template <class T>
struct FftView {
    cx_t<T> *p;
    int rs, ps;
    __device__ __forceinline__ cx_t<T> &at(int n, int pp, int qq) const { return p[n * rs + pp * ps + qq]; }
};

// quotient of 0 <= x < 2^22 by d > 0, rd = 1 / d (the float quotient is off by at most one and
// corrected): the index splits of the FFT passes without integer division
__device__ __forceinline__ int div_n(int x, int d, float rd) {
    int q = (int)((float)x * rd);
    const int r = x - q * d;
    q -= r < 0 ? 1 : 0;
    q += r >= d ? 1 : 0;
    return q;
}

// one Stockham pass of radix R over 3 qc signals: Ns = product of the earlier radices
template <int R, class T>
__device__ __forceinline__ void fft_pass_r(const FftView<T> in, const FftView<T> out, int N, int qc, int Ns,
                                           int sign, const cx_t<T> *tw2, int lane, int TEAM) {
    using C = cx_t<T>;
    const int S = 3 * qc;
    const int NR = N / R, span = N / (Ns * R);
    const float rS = 1.f / (float)S, rNs = 1.f / (float)Ns;
    for (int i = lane; i < NR * S; i += TEAM) {
        const int j = div_n(i, S, rS), s = i - j * S;
        const int pp = (s >= qc) + (s >= 2 * qc), qq = s - pp * qc;
        const int jn = div_n(j, Ns, rNs), k = j - jn * Ns;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = in.at(j + r * NR, pp, qq);
        const int step = k * span;
        int m = 0;
#pragma unroll
        for (int r = 1; r < R; r++) {
            m += step;
            m = m >= N ? m - N : m;
            if (step) v[r] = cmul<T>(v[r], fft_tw<T>(tw2, m, sign));
        }
        const int d = jn * Ns * R + k;
        if constexpr (R >= 11) {
            // the larger primes: each output summed and stored in turn (fewer live registers)
            const int stepR = N / R;
#pragma unroll 1
            for (int t = 0; t < R; t++) {
                C acc = v[0];
                int m2 = 0;
#pragma unroll
                for (int r = 1; r < R; r++) {
                    m2 += t;
                    m2 = m2 >= R ? m2 - R : m2;
                    acc = cadd(acc, cmul<T>(v[r], fft_tw<T>(tw2, m2 * stepR, sign)));
                }
                out.at(d + t * Ns, pp, qq) = acc;
            }
        } else {
            fft_radix<R, T>(v, sign, tw2, N);
#pragma unroll
            for (int r = 0; r < R; r++) out.at(d + r * Ns, pp, qq) = v[r];
        }
    }
}

// the whole transform of the 3 qc signals of length N from view b0 by the packed plan, passes
// alternating between b0 and b1; returns the view that holds the result (natural order); the
// team synchronises after every pass
template <class T>
__device__ __forceinline__ FftView<T> fft_run(FftView<T> b0, FftView<T> b1, int N, int qc, unsigned plan,
                                              int sign, const cx_t<T> *tw2, int team, int lane, int TEAM) {
    FftView<T> in = b0, out = b1;
    int Ns = 1;
    for (; plan; plan >>= 3) {
        int R;
        switch (plan & 7u) {
            case 1: fft_pass_r<4, T>(in, out, N, qc, Ns, sign, tw2, lane, TEAM); R = 4; break;
            case 2: fft_pass_r<2, T>(in, out, N, qc, Ns, sign, tw2, lane, TEAM); R = 2; break;
            case 3: fft_pass_r<3, T>(in, out, N, qc, Ns, sign, tw2, lane, TEAM); R = 3; break;
            case 4: fft_pass_r<5, T>(in, out, N, qc, Ns, sign, tw2, lane, TEAM); R = 5; break;
            case 5: fft_pass_r<7, T>(in, out, N, qc, Ns, sign, tw2, lane, TEAM); R = 7; break;
            case 6: fft_pass_r<11, T>(in, out, N, qc, Ns, sign, tw2, lane, TEAM); R = 11; break;
            default: fft_pass_r<13, T>(in, out, N, qc, Ns, sign, tw2, lane, TEAM); R = 13; break;
        }
        team_sync(team, TEAM);
        Ns *= R;
        const FftView<T> t = in; in = out; out = t;
    }
    return in;
}

// ----------------------------------------------------------------- kernel ---
// NS: compile-time number of SLS for the register-resident recursions (the slice path of 3-D
// elements, the Fourier-space path of 1-D elements); 0 = the generic path with the count
// read at run time
// FFT: the instantiation that holds the slice FFTs (3-D buckets with large nr); the others
// keep only the direct sums, so the FFT code costs them no registers
template <class T, class AT, int RHEO, int ATT, bool IS3D, bool RTZ, int NS, bool FFT = false>
__global__ void __launch_bounds__(256, AXG_SOLID_MIN_BLOCKS)
solid_stiffness_kernel(const SolidArgs<T, AT> a, const int nr_max, const int qc_max, const int mt_max,
                       const int teams_per_cta, const size_t team_bytes) {
    using C = cx_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // register blocking of the paired Fourier -> slice pass and of the slice -> Fourier pass
    constexpr int KPc = ATT == ATT_NONE ? AXG_KP_ELASTIC : KP;
    constexpr int ABc = ATT == ATT_NONE ? AXG_AB_ELASTIC : AB;
    const int TEAM = blockDim.x / teams_per_cta;
    const int team = threadIdx.x / TEAM;
    const int lane = threadIdx.x % TEAM;
    // G tables, once per CTA
    __shared__ T sGll[25], sGlj[25];
    for (int i = threadIdx.x; i < 25; i += blockDim.x) {
        sGll[i] = a.gmat[i];
        sGlj[i] = a.gmat[25 + i];
    }
    __syncthreads();
    if (team >= teams_per_cta) return;

    const TeamLayout L = team_layout<T>(nr_max, qc_max, mt_max);
    unsigned char *base = smem_raw + (size_t)team * team_bytes;
    T *sGeo = reinterpret_cast<T *>(base + L.geom);
    T *sTrig = reinterpret_cast<T *>(base + L.trig);
    int *sPt = reinterpret_cast<int *>(base + L.ipt);
    int *sOff = sPt + 25;
    int *sNu = sPt + 50;
    T *sTw = reinterpret_cast<T *>(base + L.tw);
    float4 *sTws = reinterpret_cast<float4 *>(base + L.tws);
    C *rA = reinterpret_cast<C *>(base + L.regA);
    C *rBc = reinterpret_cast<C *>(base + L.regB);
    T *rBr = reinterpret_cast<T *>(base + L.regB);

    // geometry aliases
    const T *dsdxii = sGeo, *dsdeta = sGeo + 25, *dzdxii = sGeo + 50, *dzdeta = sGeo + 75,
            *invs = sGeo + 100;
    const T *dsdxii_if = sGeo + 125, *dsdeta_if = sGeo + 150, *dzdxii_if = sGeo + 175,
            *dzdeta_if = sGeo + 200, *invs_if = sGeo + 225;

    const int stride = gridDim.x * teams_per_cta;
    if (AXG_PREFETCH_NEXT && blockIdx.x * teams_per_cta + team < a.n_elem)
        prefetch_element<T, AT, RHEO, ATT, IS3D>(a, blockIdx.x * teams_per_cta + team, lane, TEAM);
    for (int e = blockIdx.x * teams_per_cta + team; e < a.n_elem; e += stride) {
        const int nr = a.nr[e];
        const int nu = nr / 2 + 1;
        const bool axial = a.axial[e] != 0;
        const T *Gxi = axial ? sGlj : sGll;
        // the next element of this team streams into L2 while this one computes
        if (AXG_PREFETCH_NEXT && e + stride < a.n_elem)
            prefetch_element<T, AT, RHEO, ATT, IS3D>(a, e + stride, lane, TEAM);
        // the element about one wave of resident CTAs ahead streams into L2 while this one computes
        if (AXG_PREFETCH_AHEAD > 0 && a.prefetch_ahead > 0 && e + a.prefetch_ahead < a.n_elem)
            prefetch_element<T, AT, RHEO, ATT, IS3D>(a, e + a.prefetch_ahead, lane, TEAM);

        // ---------------- element header -> shared memory ----------------
        for (int i = lane; i < 250; i += TEAM) sGeo[i] = a.geom[(size_t)e * 250 + i];
        if constexpr (RTZ)
            for (int i = lane; i < 100; i += TEAM) sTrig[i] = a.trig[(size_t)e * 100 + i];
        for (int i = lane; i < 25; i += TEAM) {
            int p = a.pts[(size_t)e * 25 + i];
            sPt[i] = p;
            sOff[i] = a.pt_off[p];
            sNu[i] = a.pt_nu[p];
        }
        if constexpr (IS3D) {
            const T *tw = a.tw + a.tw_off[nr];
            // interleaved (cos, sin) pairs: one 2-word shared load per twiddle
            for (int i = lane; i < 2 * nr; i += TEAM) sTw[i] = (i & 1) ? tw[nr + (i >> 1)] : tw[i >> 1];
            if constexpr (AXG_TC_DFT && sizeof(T) == 4) {
                for (int i = lane; i < nr; i += TEAM) {
                    uint32_t ch, ct, sh, st;
                    tf32_split((float)tw[i], ch, ct);
                    tf32_split((float)tw[nr + i], sh, st);
                    sTws[i] = make_float4(__uint_as_float(ch), __uint_as_float(ct), __uint_as_float(sh),
                                          __uint_as_float(st));
                }
            }
        }
        team_sync(team, TEAM);

        // every wavefield of the batch reuses the element header loaded above
        for (int w = 0; w < a.nwave; w++) {
        const C *displw = a.displ + (size_t)w * a.fstride;
        C *stiffw = a.stiff + (size_t)w * a.fstride;
        AT *statew = a.state + (size_t)w * a.sstride;
#if AXG_PREFETCH_SLICES
        if constexpr (!IS3D && ATT != ATT_NONE && NS > 0) {
            // the SLS state of this 1-D element starts moving into L2 now, so that the stress
            // pass after the gather and the gradient finds it there
            constexpr int NPA_ = ATT == ATT_CG4 ? 4 : 25;
            prefetch_l2(statew + a.state_off[e], (size_t)(6 + 6 * NS) * nu * NPA_ * 2 * sizeof(AT), lane, TEAM);
        }
#endif
        const int64_t moff = a.mod_off[e];
        const int nslice = IS3D ? nr : 1;
        for (int t0 = 0; t0 < nu; t0 += mt_max) {
        const int mt = min(mt_max, nu - t0);
        // ---------------- gather displacement: U[a - t0][c][q] in region B ----------------
        for (int i = lane; i < mt * 25; i += TEAM) {
            const int q = i / mt, la = i - q * mt, al = t0 + la;
            C u0 = mk<T>(0, 0), u1 = u0, u2 = u0;
            if (al < sNu[q]) {
                const C *src = displw + (size_t)(sOff[q] + al) * 3;
                u0 = src[0]; u1 = src[1]; u2 = src[2];
            }
            rBc[(la * 3 + 0) * 25 + q] = u0;
            rBc[(la * 3 + 1) * 25 + q] = u1;
            rBc[(la * 3 + 2) * 25 + q] = u2;
        }
        team_sync(team, TEAM);

        // ---------------- gradient (computeGrad6) ----------------
        for (int i = lane; i < mt * 25; i += TEAM) {
            const int la = i / 25, q = i - la * 25, al = t0 + la;
            const int ii = q / 5, jj = q - ii * 5;
            const C *U = rBc + la * 75;
            C X[3], Y[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                C x = mk<T>(0, 0), y = mk<T>(0, 0);
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    const T gx = Gxi[k * 5 + ii];        // GT_xi(ii, k)
                    const T gy = sGll[k * 5 + jj];       // G_GLL(k, jj)
                    const C uc = U[c * 25 + k * 5 + jj];
                    const C ur = U[c * 25 + ii * 5 + k];
                    x.x += gx * uc.x; x.y += gx * uc.y;
                    y.x += ur.x * gy; y.y += ur.y * gy;
                }
                X[c] = x; Y[c] = y;
            }
            const T ze = dzdeta[q], zx = dzdxii[q], se = dsdeta[q], sx = dsdxii[q];
            C eps[6];
            // dS/dZ of u0 -> e0, e4 ; u1 -> e5, e3 ; u2 -> e1, e2
            eps[0] = cadd(cscale(X[0], ze), cscale(Y[0], zx));
            eps[4] = cadd(cscale(X[0], se), cscale(Y[0], sx));
            eps[5] = cadd(cscale(X[1], ze), cscale(Y[1], zx));
            eps[3] = cadd(cscale(X[1], se), cscale(Y[1], sx));
            C e1t = cadd(cscale(X[2], ze), cscale(Y[2], zx));
            eps[2] = cadd(cscale(X[2], se), cscale(Y[2], sx));
            eps[4] = cadd(eps[4], e1t);
            // lower-order terms A/s
            const T alf = (T)al;
            const C u0 = U[q], u1 = U[25 + q], u2 = U[50 + q];
            const C A0 = csub(cia(alf, u0), u1);
            const C A1 = cadd(cia(alf, u1), u0);
            const C A2 = cia(alf, u2);
            const T is = invs[q];
            eps[5] = cadd(eps[5], cscale(A0, is));
            eps[1] = cscale(A1, is);
            eps[3] = cadd(eps[3], cscale(A2, is));
            if (axial && ii == 0) {
                // L'Hopital on the axis: row 0 of A/s replaced by dA/ds
                C ax[3], ay[3];
#pragma unroll
                for (int c = 0; c < 3; c++) { ax[c] = mk<T>(0, 0); ay[c] = mk<T>(0, 0); }
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    const T gx = Gxi[k * 5 + 0];
                    const T gy = sGll[k * 5 + jj];
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
            if constexpr (RTZ) {
                spz_to_rtz6(eps, sTrig[q], sTrig[25 + q], sTrig[50 + q], sTrig[75 + q]);
            }
            if constexpr (!IS3D && !(ATT != ATT_NONE && NS > 0)) {
                // strainToStress_FR with 1-D moduli
                C sig[6];
                elastic_at<RHEO>(a.mod + moff, 1, 0, q, eps, sig);
                if constexpr (ATT == ATT_FULL) {
                    const int64_t ao = a.att_off[e];
                    AT *st = statew + a.state_off[e];
                    attenuate_1d<NS, T, AT>(a, st, (size_t)nu * 25, (size_t)al * 25 + q, eps, sig,
                                           a.attmod[ao + q], a.attmod[ao + 25 + q]);
                } else if constexpr (ATT == ATT_CG4) {
                    const int k4 = cg4_slot(q);
                    if (k4 >= 0) {
                        const int64_t ao = a.att_off[e];
                        AT *st = statew + a.state_off[e];
                        attenuate_1d<NS, T, AT>(a, st, (size_t)nu * 4, (size_t)al * 4 + k4, eps, sig,
                                               a.attmod[ao + k4], a.attmod[ao + 4 + k4]);
                    }
                }
                if constexpr (RTZ) {
                    rtz_to_spz6(sig, sTrig[q], sTrig[25 + q], sTrig[50 + q], sTrig[75 + q]);
                }
#pragma unroll
                for (int d = 0; d < 6; d++) rA[(al * 6 + d) * 25 + q] = sig[d];
            } else {
#pragma unroll
                for (int d = 0; d < 6; d++) rA[(al * 6 + d) * 25 + q] = eps[d];
            }
        }
        team_sync(team, TEAM);
        }   // mode tiles of the gather + gradient

        // ---------------- 1-D attenuation: stress pass, SLS state in registers ----------------
        // strainToStress_FR on the strain left in region A, then the SLS recursion of each
        // attenuating slot with its whole state loaded at once; with CG4 the recursion runs on
        // threads mapped to the 4 CG4 points of each mode only
        if constexpr (!IS3D && ATT != ATT_NONE && NS > 0) {
            const int64_t ao = a.att_off[e];
            AT *st = statew + a.state_off[e];
            auto stress_slot = [&](int al, int q, bool att, size_t nslot, size_t slot, T dl, T dm) {
                C ev[6], sig[6];
#pragma unroll
                for (int d = 0; d < 6; d++) ev[d] = rA[(al * 6 + d) * 25 + q];
                elastic_at<RHEO>(a.mod + moff, 1, 0, q, ev, sig);
                if (att) attenuate_cplx_regs<NS, T, AT>(a, st, nslot, slot, ev, sig, dl, dm);
                if constexpr (RTZ) {
                    rtz_to_spz6(sig, sTrig[q], sTrig[25 + q], sTrig[50 + q], sTrig[75 + q]);
                }
#pragma unroll
                for (int d = 0; d < 6; d++) rA[(al * 6 + d) * 25 + q] = sig[d];
            };
            if constexpr (ATT == ATT_FULL) {
                for (int i = lane; i < nu * 25; i += TEAM) {
                    const int al = i / 25, q = i - al * 25;
                    stress_slot(al, q, true, (size_t)nu * 25, (size_t)i, a.attmod[ao + q], a.attmod[ao + 25 + q]);
                }
            } else {
                // CG4 points (1,1) (1,3) (3,1) (3,3) = 6, 8, 16, 18 of each mode
                for (int i = lane; i < nu * 4; i += TEAM) {
                    const int al = i >> 2, k4 = i & 3;
                    const int q = 6 + 2 * (k4 & 1) + 10 * (k4 >> 1);
                    stress_slot(al, q, true, (size_t)nu * 4, (size_t)i, a.attmod[ao + k4], a.attmod[ao + 4 + k4]);
                }
                // the other 21 points of each mode: elastic only
                for (int i = lane; i < nu * 21; i += TEAM) {
                    const int al = i / 21, j = i - al * 21;
                    const int q = j + (j >= 6) + (j >= 7) + (j >= 14) + (j >= 15);
                    stress_slot(al, q, false, 0, 0, (T)0, (T)0);
                }
            }
            team_sync(team, TEAM);
        }

        // ---------------- 3-D material: slices ----------------
        if constexpr (IS3D) {
            using T2 = cx_t<T>;
            const T2 *tw2 = reinterpret_cast<const T2 *>(sTw);
            const T inv_nr = (T)1 / (T)nr;
            const int nkb = (nr + KB - 1) / KB;
            const int nab = (nu + ABc - 1) / ABc;
#if AXG_PREFETCH_SLICES
            if constexpr (NS > 0 || ATT == ATT_NONE) {
                // the slice operands of this element start moving into L2 now, so that the
                // stress pass finds them there after the Fourier -> slice pass
                constexpr int NM_ = RHEO == RHEO_ISO ? 2 : RHEO == RHEO_TISO ? 5 : 21;
                prefetch_l2(a.mod + moff, (size_t)NM_ * nr * 25 * sizeof(T), lane, TEAM);
                if constexpr (ATT != ATT_NONE) {
                    constexpr int NPA_ = ATT == ATT_CG4 ? 4 : 25;
                    const size_t slots = (size_t)nr * NPA_;
                    prefetch_l2(a.attmod + a.att_off[e], 2 * slots * sizeof(T), lane, TEAM);
                    prefetch_l2(statew + a.state_off[e], (size_t)(6 + 6 * NS) * slots * sizeof(AT), lane, TEAM);
                }
            }
#endif
            // the FFT path (register-resident slice path only): an nr the plan covers
            unsigned plan = 0;
            if constexpr (FFT && (NS > 0 || ATT == ATT_NONE)) {
                if (a.fft_min_nr > 0 && nr >= a.fft_min_nr) plan = fft_plan(nr);
            }
            const bool use_fft = FFT && plan != 0;
            for (int q0 = 0; q0 < 25; q0 += qc_max) {
                const int qcnt = min(qc_max, 25 - q0);
                // slices of this chunk: [k][d][qq] reals in region B (direct sums) or, on the
                // FFT path, x_2p + i x_2p+1 of sample k in whichever view the C2R left them
                const FftView<T> vB{rBc, 3 * qcnt, qcnt}, vA{rA + q0, 75, 25};
                FftView<T> vs = vB;
                // component d of slice k at point qq: base(k, qq) + (d >> 1) sp + (d & 1) sq
                auto sl_base = [&](int k, int qq) -> T * {
                    return use_fft ? reinterpret_cast<T *>(&vs.at(k, 0, qq)) : rBr + (size_t)k * 6 * qcnt + qq;
                };
                if constexpr (NS > 0 || ATT == ATT_NONE) {
                constexpr int NM = RHEO == RHEO_ISO ? 2 : RHEO == RHEO_TISO ? 5 : 21;
                constexpr int NSR = NS > 0 ? NS : 1;
                constexpr int NPA = ATT == ATT_CG4 ? 4 : 25;
                const T *modp = a.mod + moff;
                const size_t nsl = (size_t)nslice * 25;
#if AXG_STATE_EARLY
                // the SLS state of this thread's first (slice, point) of the stress pass is
                // loaded now, so that its latency runs under the Fourier -> slice pass
                AT ds0[6], mem0[NSR][6];
                bool pre = false;
                if constexpr (ATT != ATT_NONE && NS > 0) {
                    if (lane < nr * qcnt) {
                        const int k = lane / qcnt, q = q0 + lane - k * qcnt;
                        const int k4 = ATT == ATT_CG4 ? cg4_slot(q) : q;
                        if (k4 >= 0) {
                            const size_t nslot = (size_t)nr * NPA, slot = (size_t)k * NPA + k4;
                            const AT *st = statew + a.state_off[e];
#pragma unroll
                            for (int d = 0; d < 6; d++) ds0[d] = state_ld(st + d * nslot + slot);
#pragma unroll
                            for (int l = 0; l < NSR; l++)
#pragma unroll
                                for (int d = 0; d < 6; d++) mem0[l][d] = state_ld(st + (6 + l * 6 + d) * nslot + slot);
                            pre = true;
                        }
                    }
                }
#endif
                bool fused_done = false;
                if (FFT && use_fft) {
                    // Hermitian spectra of the component pairs, Z = Y_2p + i Y_2p+1 over all nr
                    // orders: Y_0 = Re c_0, Y_a = c_a, Y_nr-a = conj c_a, Y_nr/2 = 2 Re c_nr/2
                    for (int i = lane; i < (nr / 2 + 1) * qcnt; i += TEAM) {
                        const int al = i / qcnt, qq = i - al * qcnt, q = q0 + qq;
#pragma unroll
                        for (int pp = 0; pp < 3; pp++) {
                            const C c1 = rA[(al * 6 + 2 * pp) * 25 + q], c2 = rA[(al * 6 + 2 * pp + 1) * 25 + q];
                            if (al == 0) {
                                vB.at(0, pp, qq) = mk<T>(c1.x, c2.x);
                            } else if (2 * al == nr) {
                                vB.at(al, pp, qq) = mk<T>((T)2 * c1.x, (T)2 * c2.x);
                            } else {
                                vB.at(al, pp, qq) = mk<T>(c1.x - c2.y, c1.y + c2.x);
                                vB.at(nr - al, pp, qq) = mk<T>(c1.x + c2.y, c2.x - c1.y);
                            }
                        }
                    }
                    team_sync(team, TEAM);
                    // from here on the chunk's columns of region A are free until the unpacking
                    vs = fft_run<T>(vB, vA, nr, qcnt, plan, +1, tw2, team, lane, TEAM);
                } else {
#if AXG_FUSED_SLICE
                if constexpr (ATT != ATT_NONE && NS > 0) {
                    fused_done = true;
                    const int npair = nr / 2 + 1;
                    const size_t nslot = (size_t)nr * NPA;
                    AT *st = statew + a.state_off[e];
                    const T *am = a.attmod + a.att_off[e];
                    // the operands of (slice k, point q): moduli, attenuation moduli, SLS state
                    auto load_ops = [&](int k, int q, int k4, T (&md)[NM], T &dl, T &dmu, AT (&ds)[6],
                                        AT (&mem)[NSR][6]) {
#pragma unroll
                        for (int mm = 0; mm < NM; mm++) md[mm] = __ldg(modp + mm * nsl + (size_t)k * 25 + q);
                        if (k4 >= 0) {
                            const size_t slot = (size_t)k * NPA + k4;
                            dl = __ldg(am + slot);
                            dmu = __ldg(am + nslot + slot);
#pragma unroll
                            for (int d = 0; d < 6; d++) ds[d] = state_ld(st + d * nslot + slot);
#pragma unroll
                            for (int l = 0; l < NSR; l++)
#pragma unroll
                                for (int d = 0; d < 6; d++) mem[l][d] = state_ld(st + (6 + l * 6 + d) * nslot + slot);
                        }
                    };
                    // stress and SLS recursion of one slice; the stress to region B
                    auto stress_slice = [&](int k, int qq, int k4, const T (&x)[6], const T (&md)[NM], T dl, T dmu,
                                            AT (&ds)[6], AT (&mem)[NSR][6]) {
                        re1<T> ev[6], sg[6];
#pragma unroll
                        for (int d = 0; d < 6; d++) ev[d].x = x[d];
                        if constexpr (RHEO == RHEO_ISO) stress_iso(ev, sg, md[0], md[1]);
                        else if constexpr (RHEO == RHEO_TISO) stress_tiso(ev, sg, md[0], md[1], md[2], md[3], md[4]);
                        else stress_aniso(ev, sg, md);
                        if (k4 >= 0) {
                            const size_t slot = (size_t)k * NPA + k4;
                            T e6[6], s6[6];
#pragma unroll
                            for (int d = 0; d < 6; d++) { e6[d] = ev[d].x; s6[d] = sg[d].x; }
                            attenuate_regs<NSR, T, AT>(a.alpha, a.beta, a.gamma, ds, mem, e6, s6, dl, dmu);
#pragma unroll
                            for (int d = 0; d < 6; d++) sg[d].x = s6[d];
#pragma unroll
                            for (int d = 0; d < 6; d++) state_st(st + d * nslot + slot, ds[d]);
#pragma unroll
                            for (int l = 0; l < NSR; l++)
#pragma unroll
                                for (int d = 0; d < 6; d++) state_st(st + (6 + l * 6 + d) * nslot + slot, mem[l][d]);
                        }
#pragma unroll
                        for (int d = 0; d < 6; d++) rBr[((size_t)k * 6 + d) * qcnt + qq] = sg[d].x;
                    };
                    for (int i = lane; i < npair * qcnt; i += TEAM) {
                        const int k = i / qcnt, qq = i - k * qcnt, q = q0 + qq;
                        const int k4 = ATT == ATT_CG4 ? cg4_slot(q) : q;
                        T md[NM], dl = 0, dmu = 0;
                        AT ds[6], mem[NSR][6];
                        load_ops(k, q, k4, md, dl, dmu, ds, mem);
                        // slices k and nr - k from one pass over the modes
                        T Ac[6], Bc[6];
#pragma unroll
                        for (int d = 0; d < 6; d++) { Ac[d] = 0; Bc[d] = 0; }
                        int j = 0;
                        for (int al = 1; al < nu; al++) {
                            j += k;
                            j = j >= nr ? j - nr : j;
                            const T2 w2 = tw2[j];
#pragma unroll
                            for (int d = 0; d < 6; d++) {
                                const C ev = rA[(al * 6 + d) * 25 + q];
                                Ac[d] += ev.x * w2.x;
                                Bc[d] += ev.y * w2.y;
                            }
                        }
                        T x1[6], x2[6];
#pragma unroll
                        for (int d = 0; d < 6; d++) {
                            const T c0 = rA[d * 25 + q].x;
                            x1[d] = c0 + (T)2 * (Ac[d] - Bc[d]);
                            x2[d] = c0 + (T)2 * (Ac[d] + Bc[d]);
                        }
                        stress_slice(k, qq, k4, x1, md, dl, dmu, ds, mem);
                        if (k != 0 && 2 * k != nr) {
                            load_ops(nr - k, q, k4, md, dl, dmu, ds, mem);
                            stress_slice(nr - k, qq, k4, x2, md, dl, dmu, ds, mem);
                        }
                    }
                    team_sync(team, TEAM);
                } else
#endif
                {
                // Register-resident slice path. Two passes:
                //  1. computeC2R, one thread per (slice pair, point): slices k and nr - k
                //     share their twiddles (cos equal, sin opposite), so one pass over the
                //     modes gives both, x_k = c0 + 2 (A - B) and x_{nr-k} = c0 + 2 (A + B)
                //     with A = sum Re(c) cos, B = sum Im(c) sin; the slice strains go to the
                //     slots of region B that the slice stresses later overwrite;
                //  2. one thread per (slice, point): the global operands of the point-slice
                //     (moduli, attenuation moduli, SLS state) are loaded into registers,
                //     stress and attenuation applied, the state stored back.
#if AXG_SLICE_PAIRS
                // KPc slice pairs per thread: each mode value read from shared memory feeds
                // 2 KPc products
                const int npair = nr / 2 + 1;
                const int npb = (npair + KPc - 1) / KPc;
#if AXG_TC_DFT
                if (sizeof(T) == 4 && qcnt == 25) {
                    tc_fourier_to_slices<T>(rA, rBr, sTws, nr, lane, TEAM);
                } else
#endif
#if AXG_COLUMN_TILES
                if (qcnt == 25) {
                    // column n = d * 25 + q of the block: mode a at rA[a * 150 + n], slice k
                    // at rBr[k * 150 + n]; a thread takes KPc pairs x 6 columns
                    for (int i = lane; i < 25 * npb; i += TEAM) {
                        const int pb = (i / 5) % npb, n0 = 6 * ((i / (5 * npb)) * 5 + i % 5);
                        const int k0 = pb * KPc;
                        T A[KPc][6], B[KPc][6];
                        int j[KPc], kst[KPc];
#pragma unroll
                        for (int kk = 0; kk < KPc; kk++) {
                            j[kk] = 0;
                            kst[kk] = k0 + kk < npair ? k0 + kk : 0;
#pragma unroll
                            for (int c = 0; c < 6; c++) { A[kk][c] = 0; B[kk][c] = 0; }
                        }
#pragma unroll DFT_UNROLL
                        for (int al = 1; al < nu; al++) {
                            C ev[6];
                            ld6c<T>(rA + al * 150 + n0, ev);
#pragma unroll
                            for (int kk = 0; kk < KPc; kk++) {
                                j[kk] += kst[kk];
                                j[kk] = j[kk] >= nr ? j[kk] - nr : j[kk];
                                const T2 w2 = tw2[j[kk]];
#pragma unroll
                                for (int c = 0; c < 6; c++) {
                                    A[kk][c] += ev[c].x * w2.x;
                                    B[kk][c] += ev[c].y * w2.y;
                                }
                            }
                        }
                        C c0[6];
                        ld6c<T>(rA + n0, c0);
#pragma unroll
                        for (int kk = 0; kk < KPc; kk++) {
                            const int k = k0 + kk;
                            if (k >= npair) break;
                            T x[6];
#pragma unroll
                            for (int c = 0; c < 6; c++) x[c] = c0[c].x + (T)2 * (A[kk][c] - B[kk][c]);
                            st6r<T>(rBr + (size_t)k * 150 + n0, x);
                            if (k != 0 && 2 * k != nr) {
#pragma unroll
                                for (int c = 0; c < 6; c++) x[c] = c0[c].x + (T)2 * (A[kk][c] + B[kk][c]);
                                st6r<T>(rBr + (size_t)(nr - k) * 150 + n0, x);
                            }
                        }
                    }
                } else
#endif
                for (int i = lane; i < npb * qcnt; i += TEAM) {
                    const int pb = i / qcnt, qq = i - pb * qcnt, q = q0 + qq;
                    const int k0 = pb * KPc;
                    T A[KPc][6], B[KPc][6];
                    int j[KPc], kst[KPc];
#pragma unroll
                    for (int kk = 0; kk < KPc; kk++) {
                        j[kk] = 0;
                        kst[kk] = k0 + kk < npair ? k0 + kk : 0;
#pragma unroll
                        for (int d = 0; d < 6; d++) { A[kk][d] = 0; B[kk][d] = 0; }
                    }
                    for (int al = 1; al < nu; al++) {
                        C ev[6];
#pragma unroll
                        for (int d = 0; d < 6; d++) ev[d] = rA[(al * 6 + d) * 25 + q];
#pragma unroll
                        for (int kk = 0; kk < KPc; kk++) {
                            j[kk] += kst[kk];
                            j[kk] = j[kk] >= nr ? j[kk] - nr : j[kk];
                            const T2 w2 = tw2[j[kk]];
                            const T c = w2.x, sn = w2.y;
#pragma unroll
                            for (int d = 0; d < 6; d++) {
                                A[kk][d] += ev[d].x * c;
                                B[kk][d] += ev[d].y * sn;
                            }
                        }
                    }
#pragma unroll
                    for (int kk = 0; kk < KPc; kk++) {
                        const int k = k0 + kk;
                        if (k >= npair) break;
                        const bool two = k != 0 && 2 * k != nr;
#pragma unroll
                        for (int d = 0; d < 6; d++) {
                            const T c0 = rA[d * 25 + q].x;
                            rBr[((size_t)k * 6 + d) * qcnt + qq] = c0 + (T)2 * (A[kk][d] - B[kk][d]);
                            if (two) rBr[((size_t)(nr - k) * 6 + d) * qcnt + qq] = c0 + (T)2 * (A[kk][d] + B[kk][d]);
                        }
                    }
                }
                team_sync(team, TEAM);
#endif
                }
                }   // direct Fourier -> slice sums
                const int sp = use_fft ? 2 * vs.ps : 2 * qcnt, sq = use_fft ? 1 : qcnt;
                for (int i = lane; i < (fused_done ? 0 : nr * qcnt); i += TEAM) {
                    const int k = i / qcnt, qq = i - k * qcnt, q = q0 + qq;
                    T *slb = sl_base(k, qq);
                    T md[NM];
#pragma unroll
                    for (int mm = 0; mm < NM; mm++) md[mm] = __ldg(modp + mm * nsl + (size_t)k * 25 + q);
                    AT ds[6], mem[NSR][6];
                    T dl = 0, dmu = 0;
                    AT *st = nullptr;
                    size_t slot = 0, nslot = 0;
                    bool att_here = false;
                    if constexpr (ATT != ATT_NONE) {
                        const int k4 = ATT == ATT_CG4 ? cg4_slot(q) : q;
                        att_here = k4 >= 0;
                        if (att_here) {
                            nslot = (size_t)nr * NPA;
                            slot = (size_t)k * NPA + k4;
                            st = statew + a.state_off[e];
                            const T *am = a.attmod + a.att_off[e];
                            dl = __ldg(am + slot);
                            dmu = __ldg(am + nslot + slot);
#if !AXG_SLS_SPLIT
#if AXG_STATE_EARLY
                            if (pre && i == lane) {
#pragma unroll
                                for (int d = 0; d < 6; d++) ds[d] = ds0[d];
#pragma unroll
                                for (int l = 0; l < NSR; l++)
#pragma unroll
                                    for (int d = 0; d < 6; d++) mem[l][d] = mem0[l][d];
                            } else
#endif
                            {
#pragma unroll
                            for (int d = 0; d < 6; d++) ds[d] = state_ld(st + d * nslot + slot);
#pragma unroll
                            for (int l = 0; l < NSR; l++)
#pragma unroll
                                for (int d = 0; d < 6; d++) mem[l][d] = state_ld(st + (6 + l * 6 + d) * nslot + slot);
                            }
#endif
                        }
                    }
                    T acc[6];
#if AXG_SLICE_PAIRS
#pragma unroll
                    for (int d = 0; d < 6; d++) acc[d] = slb[(d >> 1) * sp + (d & 1) * sq];
#else
                    // computeC2R at slice k: r = Re c0 + 2 sum Re(c_a e^{i a phi_k})
#pragma unroll
                    for (int d = 0; d < 6; d++) acc[d] = rA[d * 25 + q].x;
                    int j = 0;
                    for (int al = 1; al < nu; al++) {
                        j += k;
                        j = j >= nr ? j - nr : j;
                        const T2 w2 = tw2[j];
                        const T c = w2.x, sn = w2.y;
#pragma unroll
                        for (int d = 0; d < 6; d++) {
                            const C ev = rA[(al * 6 + d) * 25 + q];
                            acc[d] += (T)2 * (ev.x * c - ev.y * sn);
                        }
                    }
#endif
                    re1<T> ev[6], sg[6];
#pragma unroll
                    for (int d = 0; d < 6; d++) ev[d].x = acc[d];
                    if constexpr (RHEO == RHEO_ISO) {
                        stress_iso(ev, sg, md[0], md[1]);
                    } else if constexpr (RHEO == RHEO_TISO) {
                        stress_tiso(ev, sg, md[0], md[1], md[2], md[3], md[4]);
                    } else {
                        stress_aniso(ev, sg, md);
                    }
                    if constexpr (ATT != ATT_NONE) {
                        if (att_here) {
                            T e6[6], s6[6];
#pragma unroll
                            for (int d = 0; d < 6; d++) { e6[d] = ev[d].x; s6[d] = sg[d].x; }
#if AXG_SLS_SPLIT
                            attenuate_slice_split<NSR, T, AT>(a.alpha, a.beta, a.gamma, st, nslot, slot, e6, s6, dl,
                                                              dmu);
#pragma unroll
                            for (int d = 0; d < 6; d++) sg[d].x = s6[d];
#else
                            attenuate_regs<NSR, T, AT>(a.alpha, a.beta, a.gamma, ds, mem, e6, s6, dl, dmu);
#pragma unroll
                            for (int d = 0; d < 6; d++) sg[d].x = s6[d];
#pragma unroll
                            for (int d = 0; d < 6; d++) state_st(st + d * nslot + slot, ds[d]);
#pragma unroll
                            for (int l = 0; l < NSR; l++)
#pragma unroll
                                for (int d = 0; d < 6; d++) state_st(st + (6 + l * 6 + d) * nslot + slot, mem[l][d]);
#endif
                        }
                    }
#pragma unroll
                    for (int d = 0; d < 6; d++) slb[(d >> 1) * sp + (d & 1) * sq] = sg[d].x;
                }
                } else
                // Fourier -> slices (computeC2R), stress, attenuation -> rBr[k][d][qq]
                for (int i = lane; i < nkb * qcnt; i += TEAM) {
                    const int kb = i / qcnt, qq = i - kb * qcnt, q = q0 + qq;
                    const int k0 = kb * KB;
                    T acc[KB][6];
                    int j[KB];
#pragma unroll
                    for (int d = 0; d < 6; d++) {
                        const T r0 = rA[d * 25 + q].x;
#pragma unroll
                        for (int kk = 0; kk < KB; kk++) acc[kk][d] = r0;
                    }
                    int kstep[KB];
#pragma unroll
                    for (int kk = 0; kk < KB; kk++) {
                        j[kk] = 0;
                        kstep[kk] = (k0 + kk < nr) ? k0 + kk : 0;
                    }
                    for (int al = 1; al < nu; al++) {
                        C ev[6];
#pragma unroll
                        for (int d = 0; d < 6; d++) ev[d] = rA[(al * 6 + d) * 25 + q];
#pragma unroll
                        for (int kk = 0; kk < KB; kk++) {
                            j[kk] += kstep[kk];
                            j[kk] = j[kk] >= nr ? j[kk] - nr : j[kk];
                            const T2 w2 = tw2[j[kk]];
                            const T c = w2.x, s = w2.y;
#pragma unroll
                            for (int d = 0; d < 6; d++)
                                acc[kk][d] += (T)2 * (ev[d].x * c - ev[d].y * s);
                        }
                    }
#pragma unroll
                    for (int kk = 0; kk < KB; kk++) {
                        const int k = k0 + kk;
                        if (k >= nr) break;
                        re1<T> ev[6], sg[6];
#pragma unroll
                        for (int d = 0; d < 6; d++) ev[d].x = acc[kk][d];
                        elastic_at<RHEO>(a.mod + moff, nslice, k, q, ev, sg);
                        if constexpr (ATT == ATT_FULL) {
                            const int64_t ao = a.att_off[e];
                            AT *st = statew + a.state_off[e];
                            const size_t ns = (size_t)nr * 25;
                            attenuate<T, AT, false>(a, st, ns, (size_t)k * 25 + q, ev, sg,
                                                    a.attmod[ao + (size_t)k * 25 + q],
                                                    a.attmod[ao + ns + (size_t)k * 25 + q]);
                        } else if constexpr (ATT == ATT_CG4) {
                            const int k4 = cg4_slot(q);
                            if (k4 >= 0) {
                                const int64_t ao = a.att_off[e];
                                AT *st = statew + a.state_off[e];
                                const size_t ns = (size_t)nr * 4;
                                attenuate<T, AT, false>(a, st, ns, (size_t)k * 4 + k4, ev, sg,
                                                        a.attmod[ao + (size_t)k * 4 + k4],
                                                        a.attmod[ao + ns + (size_t)k * 4 + k4]);
                            }
                        }
#pragma unroll
                        for (int d = 0; d < 6; d++) rBr[((size_t)k * 6 + d) * qcnt + qq] = sg[d].x;
                    }
                }
                team_sync(team, TEAM);
                if (FFT && use_fft) {
                    // forward FFT of the stress pairs, then each pair's two spectra:
                    // S_2p = (Z_a + conj Z_nr-a) / 2, S_2p+1 = (Z_a - conj Z_nr-a) / 2i, scaled by 1/nr
                    // an even number of passes in all: the spectra end in region B, and the
                    // unpacking below writes the chunk's columns of region A without a race
                    const FftView<T> Z = fft_run<T>(vs, vs.p == rBc ? vA : vB, nr, qcnt, plan, -1, tw2, team, lane, TEAM);
                    const T h = (T)0.5 * inv_nr;
                    for (int i = lane; i < nu * qcnt; i += TEAM) {
                        const int al = i / qcnt, qq = i - al * qcnt, q = q0 + qq;
                        const int bl = al == 0 ? 0 : nr - al;
                        C sg[6];
#pragma unroll
                        for (int pp = 0; pp < 3; pp++) {
                            const C za = Z.at(al, pp, qq), zb = Z.at(bl, pp, qq);
                            T r1 = (za.x + zb.x) * h, m1 = (za.y - zb.y) * h;
                            T r2 = (za.y + zb.y) * h, m2 = (zb.x - za.x) * h;
                            if (al == 0) { m1 = 0; m2 = 0; }
                            if ((nr & 1) == 0 && 2 * al == nr) { r1 *= (T)0.5; r2 *= (T)0.5; m1 = 0; m2 = 0; }
                            sg[2 * pp] = mk<T>(r1, m1);
                            sg[2 * pp + 1] = mk<T>(r2, m2);
                        }
                        if constexpr (RTZ) {
                            rtz_to_spz6(sg, sTrig[q], sTrig[25 + q], sTrig[50 + q], sTrig[75 + q]);
                        }
#pragma unroll
                        for (int d = 0; d < 6; d++) rA[(al * 6 + d) * 25 + q] = sg[d];
                    }
                    team_sync(team, TEAM);
                    continue;
                }
                // slices -> Fourier (computeR2C) into region A for these points
#if AXG_TC_DFT
                if (!RTZ && sizeof(T) == 4 && qcnt == 25) {
                    tc_slices_to_fourier<T>(rA, rBr, sTws, nr, inv_nr, lane, TEAM);
                } else
#endif
#if AXG_COLUMN_TILES
                if (!RTZ && qcnt == 25) {
                    // ABc modes x 6 columns per thread (the column layout of the Fourier ->
                    // slice pass); the 1/nr scaling applied once to the sums
                    for (int i = lane; i < 25 * nab; i += TEAM) {
                        const int ab = (i / 5) % nab, n0 = 6 * ((i / (5 * nab)) * 5 + i % 5);
                        const int a0 = ab * ABc;
                        T re[ABc][6], im[ABc][6];
                        int j[ABc], astep[ABc];
#pragma unroll
                        for (int aa = 0; aa < ABc; aa++) {
                            j[aa] = 0;
                            astep[aa] = (a0 + aa) % nr;
#pragma unroll
                            for (int c = 0; c < 6; c++) { re[aa][c] = 0; im[aa][c] = 0; }
                        }
#pragma unroll DFT_UNROLL
                        for (int k = 0; k <= nr / 2; k++) {
                            T xs[6], xd[6];
                            ld6r<T>(rBr + (size_t)k * 150 + n0, xs);
                            if (k != 0 && 2 * k != nr) {
                                T x2[6];
                                ld6r<T>(rBr + (size_t)(nr - k) * 150 + n0, x2);
#pragma unroll
                                for (int c = 0; c < 6; c++) {
                                    xd[c] = xs[c] - x2[c];
                                    xs[c] += x2[c];
                                }
                            } else {
#pragma unroll
                                for (int c = 0; c < 6; c++) xd[c] = xs[c];
                            }
#pragma unroll
                            for (int aa = 0; aa < ABc; aa++) {
                                const T2 w2 = tw2[j[aa]];
#pragma unroll
                                for (int c = 0; c < 6; c++) {
                                    re[aa][c] += xs[c] * w2.x;
                                    im[aa][c] -= xd[c] * w2.y;
                                }
                                j[aa] += astep[aa];
                                j[aa] = j[aa] >= nr ? j[aa] - nr : j[aa];
                            }
                        }
#pragma unroll
                        for (int aa = 0; aa < ABc; aa++) {
                            const int al = a0 + aa;
                            if (al >= nu) break;
                            const bool nyq = (nr & 1) == 0 && al == nr / 2;
                            const T sr = nyq ? (T)0.5 * inv_nr : inv_nr;
                            const bool noim = al == 0 || nyq;
                            C sg[6];
#pragma unroll
                            for (int c = 0; c < 6; c++) sg[c] = mk<T>(re[aa][c] * sr, noim ? (T)0 : im[aa][c] * inv_nr);
                            st6c<T>(rA + al * 150 + n0, sg);
                        }
                    }
                } else
#endif
                for (int i = lane; i < nab * qcnt; i += TEAM) {
                    const int ab = i / qcnt, qq = i - ab * qcnt, q = q0 + qq;
                    const int a0 = ab * ABc;
                    T re[ABc][6], im[ABc][6];
                    int j[ABc], astep[ABc];
#pragma unroll
                    for (int aa = 0; aa < ABc; aa++) {
                        j[aa] = 0;
                        astep[aa] = (a0 + aa) % nr;
#pragma unroll
                        for (int d = 0; d < 6; d++) { re[aa][d] = 0; im[aa][d] = 0; }
                    }
                    // slices k and nr - k in one pass: cos(a phi) is even and sin(a phi) odd
                    // in k, so they enter as x_k + x_{nr-k} and x_k - x_{nr-k}
                    for (int k = 0; k <= nr / 2; k++) {
                        const bool two = k != 0 && 2 * k != nr;
                        T xs[6], xd[6];
#pragma unroll
                        for (int d = 0; d < 6; d++) {
                            const T x1 = rBr[((size_t)k * 6 + d) * qcnt + qq];
                            const T x2 = two ? rBr[((size_t)(nr - k) * 6 + d) * qcnt + qq] : (T)0;
                            xs[d] = (x1 + x2) * inv_nr;
                            xd[d] = (x1 - x2) * inv_nr;
                        }
#pragma unroll
                        for (int aa = 0; aa < ABc; aa++) {
                            const T2 w2 = tw2[j[aa]];
                            const T c = w2.x, s = w2.y;
#pragma unroll
                            for (int d = 0; d < 6; d++) {
                                re[aa][d] += xs[d] * c;
                                im[aa][d] -= xd[d] * s;
                            }
                            j[aa] += astep[aa];
                            j[aa] = j[aa] >= nr ? j[aa] - nr : j[aa];
                        }
                    }
#pragma unroll
                    for (int aa = 0; aa < ABc; aa++) {
                        const int al = a0 + aa;
                        if (al >= nu) break;
                        C sg[6];
#pragma unroll
                        for (int d = 0; d < 6; d++) {
                            T r = re[aa][d], m = im[aa][d];
                            if (al == 0) m = 0;
                            if ((nr & 1) == 0 && al == nr / 2) { r *= (T)0.5; m = 0; }
                            sg[d] = mk<T>(r, m);
                        }
                        if constexpr (RTZ) {
                            rtz_to_spz6(sg, sTrig[q], sTrig[25 + q], sTrig[50 + q], sTrig[75 + q]);
                        }
#pragma unroll
                        for (int d = 0; d < 6; d++) rA[(al * 6 + d) * 25 + q] = sg[d];
                    }
                }
                team_sync(team, TEAM);
            }
        }

        for (int t0 = 0; t0 < nu; t0 += mt_max) {
        const int mt = min(mt_max, nu - t0);
        // ---------------- quadrature (computeQuad6), pass 1: X, Y, A ----------------
        for (int i = lane; i < mt * 25; i += TEAM) {
            const int la = i / 25, q = i - la * 25, al = t0 + la;
            C s[6];
#pragma unroll
            for (int d = 0; d < 6; d++) s[d] = rA[(al * 6 + d) * 25 + q];
            const T ze = dzdeta_if[q], zx = dzdxii_if[q], se = dsdeta_if[q], sx = dsdxii_if[q];
            C *xy = rA + al * 150;
            xy[0 * 25 + q] = cadd(cscale(s[0], ze), cscale(s[4], se));
            xy[1 * 25 + q] = cadd(cscale(s[0], zx), cscale(s[4], sx));
            xy[2 * 25 + q] = cadd(cscale(s[5], ze), cscale(s[3], se));
            xy[3 * 25 + q] = cadd(cscale(s[5], zx), cscale(s[3], sx));
            xy[4 * 25 + q] = cadd(cscale(s[4], ze), cscale(s[2], se));
            xy[5 * 25 + q] = cadd(cscale(s[4], zx), cscale(s[2], sx));
            const T alf = (T)al;
            rBc[(la * 3 + 0) * 25 + q] = csub(cia(alf, s[5]), s[1]);
            rBc[(la * 3 + 1) * 25 + q] = cadd(cia(alf, s[1]), s[5]);
            rBc[(la * 3 + 2) * 25 + q] = cia(alf, s[3]);
        }
        team_sync(team, TEAM);

        // ---------------- quadrature pass 2 + scatter-add ----------------
        for (int i = lane; i < mt * 25; i += TEAM) {
            const int la = i / 25, q = i - la * 25, al = t0 + la;
            const int ii = q / 5, jj = q - ii * 5;
            const C *xy = rA + al * 150;
            const C *A = rBc + la * 75;
            C f[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                C g1 = mk<T>(0, 0), g2 = mk<T>(0, 0);
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    const T gx = Gxi[ii * 5 + k];      // G_xi(ii, k)
                    const T gt = sGll[jj * 5 + k];     // GT_GLL(k, jj) = G_GLL(jj, k)
                    const C xv = xy[(2 * c) * 25 + k * 5 + jj];
                    const C yv = xy[(2 * c + 1) * 25 + ii * 5 + k];
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
        }   // mode tiles of the quadrature
        }   // wavefields
    }
}

}  // namespace axg
