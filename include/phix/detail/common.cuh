// common.cuh -- shared device/host helpers of libphix_b200 (sm_100a).
//
// Field layout: the reference's ghost-padded stored array (ScalarField.h:15-27),
// x fastest; flat(i,j,k) = origin + i + sx*(j + sy*k) for physical indices
// i,j,k (negative / >= n for ghosts).  FP32 state copies use the same shape.
//
// Rounding is pinned: every multiply-add that the reference's nvcc build
// contracts is an explicit fma here, every other product or sum an explicit
// _rn intrinsic, so the compiler cannot re-associate or contract differently
// and the CPU oracle can reproduce each value bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "phix_b200.h"

namespace phix {

// ---------------------------------------------------------------------------
// status plumbing (host)
// ---------------------------------------------------------------------------
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* where);
void count_launch(int n = 1);
// While alive on this thread, launches are not counted (kernels recorded into
// a graph under stream capture; the graph's replay counts them instead).
struct LaunchCountPause {
    LaunchCountPause();
    ~LaunchCountPause();
};

#define PHIX_TRY_CUDA(call)                                  \
    do {                                                     \
        cudaError_t _e = (call);                             \
        if (_e != cudaSuccess) return phix::cuda_status(_e, #call); \
    } while (0)

#define PHIX_LAUNCH_CHECK(what)                                      \
    do {                                                             \
        phix::count_launch();                                        \
        cudaError_t _e = cudaGetLastError();                         \
        if (_e != cudaSuccess) return phix::cuda_status(_e, what);   \
    } while (0)

// ---------------------------------------------------------------------------
// pinned arithmetic
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Second-difference sum of the 5/7-point Laplacian (Equation.cu:65-76):
//   t_a = (f[+a] - 2 f) + f[-a];  v = t_x*i2x;  v = fma(t_y, i2y, v);  v = fma(t_z, i2z, v)
template <typename T>
__device__ __forceinline__ T second_diff(T fp, T fc2, T fm) {
    return radd(rsub(fp, fc2), fm);
}
template <typename T, int DIM>
__device__ __forceinline__ T lap_combine(T tx, T ty, T tz, T i2x, T i2y, T i2z) {
    T v = rmul(tx, i2x);
    if (DIM >= 2) v = rfma(ty, i2y, v);
    if (DIM >= 3) v = rfma(tz, i2z, v);
    return v;
}

// (h, l) += d for a state kept as the unevaluated sum h + l: error-free
// two-sum of h and d, the error folded into l, then renormalised so that
// h = fl(h + l).  Used by the FP32 kernels so the state is not rounded to
// FP32 every step.
template <typename T>
__device__ __forceinline__ void twosum_update(T h, T l, T d, T* oh, T* ol) {
    const T s = radd(h, d);
    const T bp = rsub(s, h);
    const T e = radd(rsub(h, rsub(s, bp)), rsub(d, bp));
    const T l2 = radd(l, e);
    const T h2 = radd(s, l2);
    *ol = rsub(l2, rsub(h2, s));
    *oh = h2;
}

// Pointwise functors, same operation order as the reference drivers' lambdas.
template <typename T>
__device__ __forceinline__ T f_ac(T p) {  // tutorials/quickstart/main.cu:66  p - p*p*p
    T pp = rmul(p, p);
    return rfma(-pp, p, p);
}
template <typename T>  // Cahn-Hillard_double-well.cu:86-92
__device__ __forceinline__ T f_dw(T c, T two_rho, T ca, T cb) {
    T a = rmul(rmul(two_rho, rsub(c, ca)), rsub(c, cb));
    return rmul(a, rsub(rsub(rmul((T)2, c), ca), cb));
}
template <typename T>  // coupled CH+AC: df/dc of c^2(1-c)^2 + e^2(1-e)^2 + lam c^2 e^2
__device__ __forceinline__ T f_chac_c(T c, T e, T two_lam) {
    T a = rmul(rmul(rmul((T)2, c), rsub((T)1, c)), rsub((T)1, rmul((T)2, c)));
    T b = rmul(rmul(two_lam, c), e);
    return rfma(b, e, a);
}
template <typename T>  // df/deta
__device__ __forceinline__ T f_chac_e(T e, T c, T two_lam) {
    T a = rmul(rmul(rmul((T)2, e), rsub((T)1, e)), rsub((T)1, rmul((T)2, e)));
    T b = rmul(rmul(two_lam, c), c);
    return rfma(b, e, a);
}

// ---------------------------------------------------------------------------
// layout + boundary mapping
// ---------------------------------------------------------------------------
struct Layout {
    int n[3];       // physical cells per axis
    int s[3];       // element strides (1, sx, sx*sy)
    int origin;     // flat index of physical (0,0,0)
    int ghost;      // stored ghost layers
    int bc[6];      // PHIX_BC_* per [2*axis + side]
    double bcv[6];  // fixed values
};

enum : int { MAP_IN = 0, MAP_CONST = 1 };

// Map coordinate p along an axis of length n to a stored coordinate the way
// the ghost fill of that axis would have filled it.  Returns MAP_CONST with
// *cval set for Dirichlet sides and for cells past the stored ghost layers of
// sides without a BC.
__device__ __forceinline__ int map_axis(int p, int n, int bc_lo, int bc_hi, double v_lo, double v_hi, int ghost,
                                        int* q, double* cval) {
    if (p >= 0 && p < n) { *q = p; return MAP_IN; }
    int bc = p < 0 ? bc_lo : bc_hi;
    if (bc == PHIX_BC_PERIODIC) {
        int r = p % n;
        *q = r < 0 ? r + n : r;
        return MAP_IN;
    }
    if (bc == PHIX_BC_NOFLUX) { *q = p < 0 ? 0 : n - 1; return MAP_IN; }
    if (bc == PHIX_BC_FIXED) { *cval = p < 0 ? v_lo : v_hi; return MAP_CONST; }
    // no BC on this side: the stored ghost value (never rewritten), 0 beyond
    int over = p < 0 ? -p : p - n + 1;
    if (over <= ghost) { *q = p; return MAP_IN; }
    *cval = 0.0;
    return MAP_CONST;
}

}  // namespace phix
