// peak.cu -- the FMA throughput of this GPU, measured: the denominator of the
// arithmetic-pipe roofline the stencil kernels are reported against (the
// 1024^2 Cahn-Hilliard step stays in L2 and is bound by the FP64 / FP32 pipes,
// not by DRAM).  No reference counterpart.
#include <cuda_runtime.h>

#include "phix/detail/common.cuh"

namespace phix {
namespace {

constexpr int PK_NT = 256, PK_CHAINS = 8;

// Every thread runs PK_CHAINS independent multiply-add chains; the sum is
// stored only under a condition the values never meet, so no chain is dead.
template <typename T>
__global__ void __launch_bounds__(PK_NT) fma_probe(T* out, int iters, T a, T b) {
    T x[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int c = 0; c < PK_CHAINS; ++c) x[c] = rfma(x[c], a, b);
    T s = 0;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) s += x[c];
    if (s == (T)-12345.0) out[blockIdx.x] = s;
}

// The packed FP32 form (fma.rn.f32x2: two lanes per instruction) the pair
// kernels use.
__global__ void __launch_bounds__(PK_NT) fma2_probe(float* out, int iters, float a, float b) {
    float2 x[PK_CHAINS];
    const float2 av = make_float2(a, a), bv = make_float2(b, b);
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) x[c] = make_float2((threadIdx.x + c) * 1e-3f, (threadIdx.x - c) * 1e-3f);
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int c = 0; c < PK_CHAINS; ++c) x[c] = __ffma2_rn(x[c], av, bv);
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) s += x[c].x + x[c].y;
    if (s == -12345.0f) out[blockIdx.x] = s;
}

}  // namespace
}  // namespace phix

using namespace phix;

extern "C" {

// Measured multiply-add throughput of device `current`: *tflops = 2 x fused
// multiply-adds per second / 1e12, the best of three timed launches of a
// probe that keeps every SM busy with independent FMA chains.  precision:
// PHIX_F64, or PHIX_F32 (packed != 0: the two-lane f32x2 instruction).
// Synchronous; allocates and frees a small device buffer.
int phix_measure_fma_peak(int precision, int packed, double* tflops) {
    if (!tflops || (precision != PHIX_F64 && precision != PHIX_F32) || (packed && precision != PHIX_F32)) {
        set_error("measure_fma_peak: bad argument");
        return PHIX_ERR_ARG;
    }
    int dev = 0, nsm = 0;
    PHIX_TRY_CUDA(cudaGetDevice(&dev));
    PHIX_TRY_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = nsm * 8, iters = 1 << 14;
    void* out = nullptr;
    PHIX_TRY_CUDA(cudaMalloc(&out, (size_t)blocks * 8));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int rc = PHIX_OK;
    for (int rep = 0; rep < 4 && rc == PHIX_OK; ++rep) {  // the first launch warms up
        cudaEventRecord(e0);
        if (precision == PHIX_F64)
            fma_probe<double><<<blocks, PK_NT>>>((double*)out, iters, 1.0000001, 1e-7);
        else if (packed)
            fma2_probe<<<blocks, PK_NT>>>((float*)out, iters, 1.0000001f, 1e-7f);
        else
            fma_probe<float><<<blocks, PK_NT>>>((float*)out, iters, 1.0000001f, 1e-7f);
        cudaEventRecord(e1);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_status(e, "fma_probe"); break; }
        count_launch();
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (rc) return rc;
    const double fmas = (double)blocks * PK_NT * PK_CHAINS * iters * (packed ? 2.0 : 1.0);
    *tflops = 2.0 * fmas / (best * 1e-3) / 1e12;
    return PHIX_OK;
}

}  // extern "C"
