// stepper.h -- internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "phix_b200.h"
#include "phix/detail/common.cuh"

namespace phix {

template <typename T> struct StageArgs;

int validate_grid(const phix_grid_t* g, Layout* L, size_t* stored);
int physics_nfields(int phys);
template <typename T> void make_coeffs(int phys, const double* prm, T* p);
int prepare_stage(int phys, int dim, int prec);
template <typename T> int launch_stage(int phys, int dim, int mode, const StageArgs<T>& A, cudaStream_t s, int tile = -1);

// accessors into the opaque stepper (stepper.cu)
void* stepper_state(phix_stepper* h, int f);
void* stepper_state_buf(phix_stepper* h, int b, int f);
void* stepper_lo_buf(phix_stepper* h, int b, int f);
int stepper_cur(const phix_stepper* h);
size_t stepper_stored(const phix_stepper* h);
// Layout of the stepper's own arrays: the grid's, except that 3-D FP32
// steppers pad each stored row to a multiple of 16 bytes (TMA row strides).
const Layout& stepper_layout(const phix_stepper* h);
const Layout& stepper_grid_layout(const phix_stepper* h);
int stepper_prec(const phix_stepper* h);
int stepper_nf(const phix_stepper* h);
int stepper_phys(const phix_stepper* h);
int stepper_scheme(const phix_stepper* h);
void stepper_mark_loaded(phix_stepper* h);
const phix_grid_t* stepper_grid(const phix_stepper* h);
const double* stepper_prm(const phix_stepper* h);
double* stepper_staging(phix_stepper* h);
double* stepper_partials(phix_stepper* h, int n);

// All BCs of g applied to a stored array (ops.cu); low_part: the array is the
// low part of a compensated state.
template <typename T> int bc_fill(T* field, const phix_grid_t* g, bool low_part, cudaStream_t s);
template <typename T> int bc_fill_layout(T* field, const phix_grid_t* g, const Layout& L, bool low_part, cudaStream_t s);

// FP64 <-> FP32 copies of n stored elements (convert.cu)
int convert_f64_to_f32(float* dst, const double* src, size_t n, cudaStream_t s);
int convert_f32_to_f64(double* dst, const float* src, size_t n, cudaStream_t s);
// x <-> compensated float pair (hi + lo)
int convert_f64_split(float* hi, float* lo, const double* src, size_t n, cudaStream_t s);
int convert_pair_to_f64(double* dst, const float* hi, const float* lo, size_t n, cudaStream_t s);

// diagnostics core (reduce.cu): fields in precision T, FP64 accumulation.
template <typename T>
int reduce_mass_energy(const T* const* fields, int nf, int phys, const double* prm, const phix_grid_t* g,
                       double* partials, int partials_n, double* out, cudaStream_t s);
int reduce_partials_needed(const phix_grid_t* g);

}  // namespace phix
