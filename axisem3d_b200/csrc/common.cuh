// common.cuh -- device-side helpers shared by the engine's kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define AXG_NPED 5
#define AXG_NPEM 25

namespace axg {

constexpr int P = 5;
constexpr int N = 25;

// ----------------------------------------------------------------- complex ---
template <class T> struct cx;
template <> struct cx<float> { using type = float2; };
template <> struct cx<double> { using type = double2; };
template <class T> using cx_t = typename cx<T>::type;

template <class T> __host__ __device__ __forceinline__ cx_t<T> mk(T a, T b) {
    cx_t<T> r; r.x = a; r.y = b; return r;
}
template <class V> __host__ __device__ __forceinline__ V cadd(V a, V b) { a.x += b.x; a.y += b.y; return a; }
template <class V> __host__ __device__ __forceinline__ V csub(V a, V b) { a.x -= b.x; a.y -= b.y; return a; }
template <class V, class T> __host__ __device__ __forceinline__ V cscale(V a, T s) { a.x *= s; a.y *= s; return a; }
// (0 + i alpha) * a, in the operation order of std::complex multiplication
template <class V, class T> __host__ __device__ __forceinline__ V cia(T alpha, V a) {
    V r; r.x = (T)0 * a.x - alpha * a.y; r.y = (T)0 * a.y + alpha * a.x; return r;
}
// ------------------------------------------------------- team synchronisation ---
// A "team" is the set of threads that works on one element: a warp (TEAM = 32)
// or a group of warps synchronised through a named barrier (id 1..15).
__device__ __forceinline__ void team_sync(int team_id, int team_size) {
    if (team_size == 32) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(team_id + 1), "r"(team_size) : "memory");
    }
}

// ------------------------------------------------------------ atomics ---
__device__ __forceinline__ void atomic_add_cx(float2 *p, float2 v) {
    atomicAdd(p, v);   // vector atomic, global memory, sm_90+
}
__device__ __forceinline__ void atomic_add_cx(double2 *p, double2 v) {
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
}

}  // namespace axg
