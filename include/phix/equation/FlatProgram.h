#pragma once
// One SolverStep of a multi-step Solver as one kernel: the step's right-hand
// side, compiled from its terms into a short per-cell program, evaluated in
// the operation order of the reference's term-by-term accumulation, with the
// step's write fused in.
//
// Terms a program holds (at most one pw functor, of 1-3 fields):
//   lap(f)            acc = fma(c, lap f, acc)                       Equation.cu:40-80
//   grad(f, a)        acc = fma(c * (f[+a] - f[-a]), 1/(2 d_a), acc) Equation.cu:89-124
//   pw(f1[,f2,f3], F) acc = fma(c, F(f1[,f2,f3]), acc)              TermPW.inl:18-37
//   expr * f          s = expr materialised from 0; acc = fma(c * s, f, acc)
//   expr1 * expr2     s1, s2 materialised from 0; acc = fma(c * s1, s2, acc)
//                     (termTimesField / termTimesTerm, Equation.cu:386-404)
// The program is postfix over a small value stack: ZERO pushes a fresh
// accumulator, every term op folds into the top, MULF / MUL2 pop their
// materialised operands.
//
// The write covers every stored cell, as the reference's does:
//   STEADY     (computeRHS into the unknown): physical cells = acc, ghosts 0;
//   TRANSIENT  (rhs into scratch, then u += dt rhs over the stored array):
//              physical cells = fma(dt, acc, u), ghosts fma(dt, 0, u); written to the
//              other time-level buffer, which the Solver then swaps in.

#include <cuda_runtime.h>

#include "phix/detail/common.cuh"
#include "phix_b200.h"

namespace PhiX {
namespace fuse {

enum : int { FL_ZERO = 0, FL_LAP = 1, FL_GRAD = 2, FL_PW = 3, FL_MULF = 4, FL_MUL2 = 5 };
constexpr int FLAT_MAX_OPS = 32, FLAT_MAX_FIELDS = 8, FLAT_MAX_DEPTH = 4;

struct FlatOp {
    int kind;
    int field;  // field slot (LAP, GRAD, MULF)
    int axis;   // GRAD
    double c;   // the term's coefficient
};

struct FlatSpec {
    int nops = 0;
    FlatOp op[FLAT_MAX_OPS];
    const double* f[FLAT_MAX_FIELDS] = {};  // field slots, resolved at launch
    int pw_slot[3] = {0, 0, 0};             // argument slots of the pw functor
    phix::Layout L{};                       // shared stored layout of every field
    int dim = 2;
    int sdims[3] = {1, 1, 1};               // stored extents
    double i2[3] = {0, 0, 0};               // 1/d^2 per active axis
    double inv2d[3] = {0, 0, 0};            // 0.5/d per axis
    int transient = 0;
    double dt = 0.0;
    const double* u = nullptr;  // TRANSIENT: the unknown's current level
    double* out = nullptr;      // STEADY: the unknown; TRANSIENT: its other level
};

// Launches the step kernel of a program whose pw term (if any) is this
// launcher's functor; implemented per functor and arity where the term is
// made (TermPW.inl).
struct FlatKernels {
    virtual ~FlatKernels() = default;
    virtual int launch(const FlatSpec& spec, void* stream) const = 0;
};

// F is called with NA arguments (NA = 0: the program has no pw term).  The
// value stack (at most FLAT_MAX_DEPTH = 4 deep, which the program builder
// enforces) lives in four registers: t is the top, s1..s3 the values below;
// a push or pop shifts them, so no stack slot is indexed at run time.
template <class F, int NA>
__device__ __forceinline__ double flat_eval(const FlatSpec& S, const F& func, int c) {
    static_assert(FLAT_MAX_DEPTH == 4, "the register stack holds four values");
    double t = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int q = 0; q < S.nops; ++q) {
        const FlatOp o = S.op[q];
        switch (o.kind) {
            case FL_ZERO:
                s3 = s2;
                s2 = s1;
                s1 = t;
                t = 0.0;
                break;
            case FL_LAP: {
                const double* f = S.f[o.field];
                const double f2 = phix::rmul(2.0, f[c]);
                const double tx = phix::second_diff(f[c + 1], f2, f[c - 1]);
                double v;
                if (S.dim == 1) {
                    v = phix::lap_combine<double, 1>(tx, 0.0, 0.0, S.i2[0], 0.0, 0.0);
                } else {
                    const double ty = phix::second_diff(f[c + S.L.s[1]], f2, f[c - S.L.s[1]]);
                    if (S.dim == 2) {
                        v = phix::lap_combine<double, 2>(tx, ty, 0.0, S.i2[0], S.i2[1], 0.0);
                    } else {
                        const double tz = phix::second_diff(f[c + S.L.s[2]], f2, f[c - S.L.s[2]]);
                        v = phix::lap_combine<double, 3>(tx, ty, tz, S.i2[0], S.i2[1], S.i2[2]);
                    }
                }
                t = phix::rfma(o.c, v, t);
                break;
            }
            case FL_GRAD: {
                const double* f = S.f[o.field];
                const int off = S.L.s[o.axis];
                t = phix::rfma(phix::rmul(o.c, phix::rsub(f[c + off], f[c - off])), S.inv2d[o.axis], t);
                break;
            }
            case FL_PW: {
                double v = 0.0;
                if constexpr (NA == 1) v = func(S.f[S.pw_slot[0]][c]);
                else if constexpr (NA == 2) v = func(S.f[S.pw_slot[0]][c], S.f[S.pw_slot[1]][c]);
                else if constexpr (NA == 3) v = func(S.f[S.pw_slot[0]][c], S.f[S.pw_slot[1]][c], S.f[S.pw_slot[2]][c]);
                t = __fma_rn(o.c, v, t);
                break;
            }
            case FL_MULF: {  // pop the materialised operand, fold into the value below
                const double m = t;
                t = s1;
                s1 = s2;
                s2 = s3;
                t = phix::rfma(phix::rmul(o.c, m), S.f[o.field][c], t);
                break;
            }
            default: {  // FL_MUL2: pop two materialised operands
                const double m2 = t, m1 = s1;
                t = s2;
                s1 = s3;
                s2 = 0.0;
                t = phix::rfma(phix::rmul(o.c, m1), m2, t);
                break;
            }
        }
    }
    return t;
}

// One thread per stored cell: x along the stored row, y over the stored rows
// of a z plane, z by the grid.
template <class F, int NA>
__global__ void __launch_bounds__(256) flat_step(const FlatSpec S, const F func) {
    const int sx = blockIdx.x * 32 + threadIdx.x, sy = blockIdx.y * 8 + threadIdx.y, sz = blockIdx.z;
    if (sx >= S.sdims[0] || sy >= S.sdims[1]) return;
    const int c = sx + S.L.s[1] * sy + S.L.s[2] * sz;
    const int g = S.L.ghost;
    const int i = sx - g, j = S.dim >= 2 ? sy - g : 0, k = S.dim >= 3 ? sz - g : 0;
    bool phys = i >= 0 && i < S.L.n[0];
    phys = phys && (S.dim >= 2 ? (j >= 0 && j < S.L.n[1]) : sy == g);
    phys = phys && (S.dim >= 3 ? (k >= 0 && k < S.L.n[2]) : sz == g);
    if (!phys) {
        // the reference's memset (STEADY) or u + dt * 0 over the stored array
        S.out[c] = S.transient ? phix::rfma(S.dt, 0.0, S.u[c]) : 0.0;
        return;
    }
    const double acc = flat_eval<F, NA>(S, func, c);
    S.out[c] = S.transient ? phix::rfma(S.dt, acc, S.u[c]) : acc;
}

template <class F, int NA>
struct FlatKernelsImpl final : FlatKernels {
    F func;
    explicit FlatKernelsImpl(const F& f) : func(f) {}
    int launch(const FlatSpec& s, void* stream) const override {
        dim3 grid((s.sdims[0] + 31) / 32, (s.sdims[1] + 7) / 8, s.sdims[2]);
        flat_step<F, NA><<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(s, func);
        return cudaGetLastError() == cudaSuccess ? PHIX_OK : PHIX_ERR_CUDA;
    }
};

}  // namespace fuse
}  // namespace PhiX
