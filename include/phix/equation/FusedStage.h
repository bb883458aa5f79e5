#pragma once
// One fused stage of a single-field right-hand side built from lap / pw terms
// of the unknown, as handed by Solver to a term's fuse::PwKernels:
//   pattern FLAT     : rhs = sum_i c_i * op_i(y)
//   pattern COMPOSITE: rhs = M * lap( sum_i c_i * op_i(y), bcs )
// op_i is the Laplacian of y or the term's functor of y; y is the stage state.

#include "phix/detail/stage.cuh"
#include "phix/detail/step2d_pair.cuh"

namespace PhiX {
namespace fuse {

enum : int { OP_LAP = 0, OP_PW = 1 };
enum : int { PATTERN_FLAT = 0, PATTERN_COMPOSITE = 1 };
constexpr int MAX_OPS = 8;

struct StageSpec {
    int pattern = PATTERN_FLAT;
    int nops = 0;
    int op[MAX_OPS] = {0};
    double c[MAX_OPS] = {0};
    double M = 0.0;
    int dim = 2;
    int mode = phix::MODE_K;             // phix::MODE_*
    phix::StageArgs<double> A{};         // layout, pointers, a, dtf, i2
    double dt_half = 0.0, dt_full = 0.0;  // MODE_RK4_STEP: the stage-state factors dt/2 and dt
};

// Stage policy evaluating the term program with the user's functor F.
template <class F, int PATTERN>
struct PolUser {
    static constexpr int NF = 1, H = PATTERN == PATTERN_FLAT ? 1 : 2;
    static constexpr bool MU = PATTERN == PATTERN_COMPOSITE, LAP_Y0 = PATTERN == PATTERN_FLAT, LAP_Y1 = false;
    F f;
    int nops;
    int op[MAX_OPS];
    double c[MAX_OPS];
    double M;

    // rhs = 0; rhs += c_i * op_i  (Equation::computeRHS order)
    __device__ __forceinline__ double program(double y, double lapy) const {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < MAX_OPS; ++i) {  // unrolled: no run-time trip count
            if (i >= nops) break;
            const double v = op[i] == OP_LAP ? lapy : (double)f(y);
            acc = __fma_rn(c[i], v, acc);
        }
        return acc;
    }
    template <typename T>
    __device__ __forceinline__ T mu(const phix::StageArgs<T>&, T y, T lapy, T) const { return program(y, lapy); }
    template <typename T>
    __device__ __forceinline__ void rhs(const phix::StageArgs<T>&, T lapmu, T y0, T lapy0, T, T, T* k) const {
        if (PATTERN == PATTERN_FLAT) k[0] = program(y0, lapy0);
        else k[0] = __fma_rn(M, lapmu, 0.0);
    }
};

// The two-term composite program of the Cahn-Hilliard form,
// mu = c0 * f(y) + c1 * lap(y) (PW_FIRST) or c0 * lap(y) + c1 * f(y), with the
// term order compiled in: the same multiply-adds as PolUser's walk over its
// term list (acc = fma(c0, v0, 0); acc = fma(c1, v1, acc)), without the walk.
template <class F, bool PW_FIRST>
struct PolUserCH2 {
    static constexpr int NF = 1, H = 2;
    static constexpr bool MU = true, LAP_Y0 = false, LAP_Y1 = false;
    F f;
    double c0, c1, M;
    template <typename T>
    __device__ __forceinline__ T mu(const phix::StageArgs<T>&, T y, T lapy, T) const {
        const double v0 = PW_FIRST ? (double)f(y) : lapy, v1 = PW_FIRST ? lapy : (double)f(y);
        return __fma_rn(c1, v1, __fma_rn(c0, v0, 0.0));
    }
    template <typename T>
    __device__ __forceinline__ void rhs(const phix::StageArgs<T>&, T lapmu, T, T, T, T, T* k) const {
        k[0] = __fma_rn(M, lapmu, 0.0);
    }
};

}  // namespace fuse
}  // namespace PhiX
