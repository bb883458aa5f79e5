// convert.cu -- moving the stepper state in and out (phix_stepper_load/store,
// phix_stepper_run_host) and FP64 <-> FP32 conversion of stored arrays.
#include <cstdint>
#include <cstring>

#include "phix/detail/common.cuh"
#include "stepper.h"

namespace phix {

// dst[i] = (float)src[i] over n stored elements, 16-byte vectorised.
// `vec` = both pointers 16-byte aligned (else scalar).
__global__ void __launch_bounds__(256) f64_to_f32(float* __restrict__ dst, const double* __restrict__ src, size_t n,
                                                  int vec) {
    size_t i = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) * 2;
    const size_t stride = (size_t)gridDim.x * blockDim.x * 2;
    if (!vec) {
        for (size_t j = i / 2; j < n; j += stride / 2) dst[j] = (float)src[j];
        return;
    }
    for (; i + 1 < n; i += stride) {
        double2 v = *reinterpret_cast<const double2*>(src + i);
        *reinterpret_cast<float2*>(dst + i) = make_float2((float)v.x, (float)v.y);
    }
    if (i < n) dst[i] = (float)src[i];
}
__global__ void __launch_bounds__(256) f32_to_f64(double* __restrict__ dst, const float* __restrict__ src, size_t n,
                                                  int vec) {
    size_t i = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) * 2;
    const size_t stride = (size_t)gridDim.x * blockDim.x * 2;
    if (!vec) {
        for (size_t j = i / 2; j < n; j += stride / 2) dst[j] = (double)src[j];
        return;
    }
    for (; i + 1 < n; i += stride) {
        float2 v = *reinterpret_cast<const float2*>(src + i);
        *reinterpret_cast<double2*>(dst + i) = make_double2((double)v.x, (double)v.y);
    }
    if (i < n) dst[i] = (double)src[i];
}

// hi[i] = (float)x[i], lo[i] = (float)(x[i] - hi[i]): x split into an
// unevaluated float pair (the compensated FP32 state).
__global__ void __launch_bounds__(256) f64_split_f32(float* __restrict__ hi, float* __restrict__ lo,
                                                     const double* __restrict__ x, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double v = x[i];
        const float h = (float)v;
        hi[i] = h;
        lo[i] = (float)(v - (double)h);
    }
}
__global__ void __launch_bounds__(256) f32_pair_to_f64(double* __restrict__ x, const float* __restrict__ hi,
                                                       const float* __restrict__ lo, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        x[i] = (double)hi[i] + (double)lo[i];
}

// The same conversions between a caller array (row pitch sx, S elements) and
// a stepper array whose rows are padded to pitch pk (>= sx).
__global__ void __launch_bounds__(256) f64_split_f32_rows(float* __restrict__ hi, float* __restrict__ lo,
                                                          const double* __restrict__ x, size_t n, int sx, int pk) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / (size_t)sx, d = r * pk + (i - r * sx);
        const double v = x[i];
        const float h = (float)v;
        hi[d] = h;
        if (lo) lo[d] = (float)(v - (double)h);
    }
}
__global__ void __launch_bounds__(256) f32_rows_to_f64(double* __restrict__ x, const float* __restrict__ hi,
                                                       const float* __restrict__ lo, size_t n, int sx, int pk) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / (size_t)sx, d = r * pk + (i - r * sx);
        x[i] = lo ? (double)hi[d] + (double)lo[d] : (double)hi[d];
    }
}

// FP64 copies between the callers' layout (pitch sx) and a row-padded one (pk).
__global__ void __launch_bounds__(256) f64_rows_to_padded(double* __restrict__ dst, const double* __restrict__ src,
                                                          size_t n, int sx, int pk) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / (size_t)sx;
        dst[r * pk + (i - r * sx)] = src[i];
    }
}
__global__ void __launch_bounds__(256) f64_rows_from_padded(double* __restrict__ dst, const double* __restrict__ src,
                                                            size_t n, int sx, int pk) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / (size_t)sx;
        dst[i] = src[r * pk + (i - r * sx)];
    }
}

static int aligned16(const void* a, const void* b) {
    return ((uintptr_t)a % 16 == 0) && ((uintptr_t)b % 16 == 0);
}

static int conv_grid(size_t n) {
    size_t b = (n / 2 + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b ? b : 1);
}

int convert_f64_to_f32(float* dst, const double* src, size_t n, cudaStream_t s) {
    f64_to_f32<<<conv_grid(n), 256, 0, s>>>(dst, src, n, aligned16(dst, src));
    PHIX_LAUNCH_CHECK("f64_to_f32");
    return PHIX_OK;
}

int convert_f32_to_f64(double* dst, const float* src, size_t n, cudaStream_t s) {
    f32_to_f64<<<conv_grid(n), 256, 0, s>>>(dst, src, n, aligned16(dst, src));
    PHIX_LAUNCH_CHECK("f32_to_f64");
    return PHIX_OK;
}

int convert_f64_split(float* hi, float* lo, const double* src, size_t n, cudaStream_t s) {
    f64_split_f32<<<conv_grid(n), 256, 0, s>>>(hi, lo, src, n);
    PHIX_LAUNCH_CHECK("f64_split_f32");
    return PHIX_OK;
}

int convert_pair_to_f64(double* dst, const float* hi, const float* lo, size_t n, cudaStream_t s) {
    f32_pair_to_f64<<<conv_grid(n), 256, 0, s>>>(dst, hi, lo, n);
    PHIX_LAUNCH_CHECK("f32_pair_to_f64");
    return PHIX_OK;
}

int stepper_copy_in(phix_stepper* h, const double* const* fields, cudaStream_t s) {
    const size_t S = stepper_stored(h);
    for (int f = 0; f < stepper_nf(h); ++f) {
        if (!fields[f]) { set_error("load: field %d is NULL", f); return PHIX_ERR_ARG; }
        // both ping-pong buffers get the full stored array, so ghost layers
        // that no BC rewrites stay identical whichever buffer is current
        // (the multi-step mu has one buffer)
        const int nb = (stepper_scheme(h) == PHIX_MULTISTEP && f == 1) ? 1 : 2;
        const int sx = stepper_grid_layout(h).s[1], pk = stepper_layout(h).s[1];
        for (int b = 0; b < nb; ++b) {
            void* dst = stepper_state_buf(h, b, f);
            if (pk != sx && stepper_prec(h) == PHIX_F64) {  // row-padded FP64 state
                f64_rows_to_padded<<<conv_grid(S), 256, 0, s>>>((double*)dst, fields[f], S, sx, pk);
                PHIX_LAUNCH_CHECK("f64_rows_to_padded");
            } else if (pk != sx) {  // row-padded FP32 state
                f64_split_f32_rows<<<conv_grid(S), 256, 0, s>>>((float*)dst, (float*)stepper_lo_buf(h, b, f), fields[f],
                                                                S, sx, pk);
                PHIX_LAUNCH_CHECK("f64_split_f32_rows");
            } else if (stepper_prec(h) == PHIX_F64) {
                if (dst == (const void*)fields[f]) continue;
                PHIX_TRY_CUDA(cudaMemcpyAsync(dst, fields[f], S * sizeof(double), cudaMemcpyDeviceToDevice, s));
            } else if (stepper_lo_buf(h, b, f)) {
                f64_split_f32<<<conv_grid(S), 256, 0, s>>>((float*)dst, (float*)stepper_lo_buf(h, b, f), fields[f], S);
                PHIX_LAUNCH_CHECK("f64_split_f32");
            } else {
                f64_to_f32<<<conv_grid(S), 256, 0, s>>>((float*)dst, fields[f], S, aligned16(dst, fields[f]));
                PHIX_LAUNCH_CHECK("f64_to_f32");
            }
        }
    }
    stepper_mark_loaded(h);
    return PHIX_OK;
}

int stepper_copy_out(phix_stepper* h, double* const* fields, cudaStream_t s) {
    const size_t S = stepper_stored(h);
    for (int f = 0; f < stepper_nf(h); ++f) {
        if (!fields[f]) { set_error("store: field %d is NULL", f); return PHIX_ERR_ARG; }
        const void* src = stepper_state(h, f);
        const int sx = stepper_grid_layout(h).s[1], pk = stepper_layout(h).s[1];
        if (pk != sx && stepper_prec(h) == PHIX_F64) {  // row-padded FP64 state
            f64_rows_from_padded<<<conv_grid(S), 256, 0, s>>>(fields[f], (const double*)src, S, sx, pk);
            PHIX_LAUNCH_CHECK("f64_rows_from_padded");
        } else if (pk != sx) {  // row-padded FP32 state
            const bool multi_mu = stepper_scheme(h) == PHIX_MULTISTEP && f == 1;
            const void* lo = multi_mu ? nullptr : stepper_lo_buf(h, stepper_cur(h), f);
            f32_rows_to_f64<<<conv_grid(S), 256, 0, s>>>(fields[f], (const float*)src, (const float*)lo, S, sx, pk);
            PHIX_LAUNCH_CHECK("f32_rows_to_f64");
        } else if (stepper_prec(h) == PHIX_F64) {
            if (src == (const void*)fields[f]) continue;
            PHIX_TRY_CUDA(cudaMemcpyAsync(fields[f], src, S * sizeof(double), cudaMemcpyDeviceToDevice, s));
        } else {
            const bool multi_mu = stepper_scheme(h) == PHIX_MULTISTEP && f == 1;
            const void* lo = multi_mu ? nullptr : stepper_lo_buf(h, stepper_cur(h), f);
            if (lo) {
                f32_pair_to_f64<<<conv_grid(S), 256, 0, s>>>(fields[f], (const float*)src, (const float*)lo, S);
                PHIX_LAUNCH_CHECK("f32_pair_to_f64");
            } else {
                f32_to_f64<<<conv_grid(S), 256, 0, s>>>(fields[f], (const float*)src, S, aligned16(src, fields[f]));
                PHIX_LAUNCH_CHECK("f32_to_f64");
            }
        }
    }
    return PHIX_OK;
}

int stepper_diag(phix_stepper* h, double* out) {
    const int nf = physics_nfields(stepper_phys(h));
    const int np = reduce_partials_needed(stepper_grid(h));
    double* part = stepper_partials(h, np);
    if (!part) { set_error("diagnostics: cudaMalloc failed"); return PHIX_ERR_CUDA; }
    if (stepper_prec(h) == PHIX_F32 || stepper_layout(h).s[1] != stepper_grid_layout(h).s[1]) {
        // FP64 value of the compensated state (hi + lo), or of a row-padded
        // FP64 state, in the grid's layout in the staging buffer
        double* stage = stepper_staging(h);
        if (!stage) { set_error("diagnostics: cudaMalloc(staging) failed"); return PHIX_ERR_CUDA; }
        const size_t S = stepper_stored(h);
        double* outs[2] = {stage, stage + S};
        int rc = stepper_copy_out(h, outs, 0);
        if (rc) return rc;
        const double* f[2] = {stage, nf > 1 ? stage + S : nullptr};
        return reduce_mass_energy<double>(f, nf, stepper_phys(h), stepper_prm(h), stepper_grid(h), part, np, out, 0);
    }
    const double* f[2] = {(const double*)stepper_state(h, 0), nf > 1 ? (const double*)stepper_state(h, 1) : nullptr};
    return reduce_mass_energy<double>(f, nf, stepper_phys(h), stepper_prm(h), stepper_grid(h), part, np, out, 0);
}

}  // namespace phix

using namespace phix;

extern "C" {

int phix_stepper_load(phix_stepper_t* h, const double* const* fields, void* stream) {
    if (!h || !fields) { set_error("load: NULL argument"); return PHIX_ERR_ARG; }
    return stepper_copy_in(h, fields, (cudaStream_t)stream);
}

int phix_stepper_store(phix_stepper_t* h, double* const* fields, void* stream) {
    if (!h || !fields) { set_error("store: NULL argument"); return PHIX_ERR_ARG; }
    return stepper_copy_out(h, fields, (cudaStream_t)stream);
}

int phix_stepper_run_host(phix_stepper_t* h, const double* const* host_in, double* const* host_out, int nsteps) {
    if (!h || !host_in || !host_out || nsteps < 0) { set_error("run_host: bad argument"); return PHIX_ERR_ARG; }
    const int nf = stepper_nf(h);
    const size_t S = stepper_stored(h);
    double* stage = stepper_staging(h);
    if (!stage) { set_error("run_host: cudaMalloc(staging) failed"); return PHIX_ERR_CUDA; }
    const double* din[2] = {stage, stage + S};
    double* dout[2] = {stage, stage + S};
    for (int f = 0; f < nf; ++f)
        PHIX_TRY_CUDA(cudaMemcpyAsync(stage + f * S, host_in[f], S * sizeof(double), cudaMemcpyHostToDevice, 0));
    int rc = stepper_copy_in(h, din, 0);
    if (rc) return rc;
    if ((rc = phix_stepper_advance(h, nsteps, 0))) return rc;
    if ((rc = stepper_copy_out(h, dout, 0))) return rc;
    for (int f = 0; f < nf; ++f)
        PHIX_TRY_CUDA(cudaMemcpyAsync(host_out[f], stage + f * S, S * sizeof(double), cudaMemcpyDeviceToHost, 0));
    PHIX_TRY_CUDA(cudaStreamSynchronize(0));
    return PHIX_OK;
}

int phix_stepper_diagnostics(phix_stepper_t* h, double* out) {
    if (!h || !out) { set_error("diagnostics: NULL argument"); return PHIX_ERR_ARG; }
    return stepper_diag(h, out);
}

}  // extern "C"
