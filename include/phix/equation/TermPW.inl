// TermPW.inl -- pw(...) factories for user functors (included by Term.h).
// The unfused launcher runs one accumulate kernel per term, like the
// reference (include/equation/TermPW.inl:18-90); single-field pw terms also
// carry fused stage kernels instantiated here for the functor.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "equation/FlatProgram.h"
#include "equation/FusedStage.h"
#include "phix/detail/step2d_pair_ms.cuh"
#include "phix_b200.h"

namespace PhiX {
namespace detail {

// host-side geometry of a field for the accumulate kernels
struct PwGeom {
    int n0, n1, n2, sx, sy, g;
};
inline PwGeom pw_geom(const ScalarField& f) {
    return {f.mesh.n[0], f.mesh.n[1], f.mesh.n[2], f.storedDims[0], f.storedDims[1], f.ghost};
}
inline dim3 pw_grid(const PwGeom& G) { return dim3((G.n0 + 31) / 32, (G.n1 + 7) / 8, G.n2); }

// rhs += coeff * F(a[, b[, c]]) on physical cells (2-D launch, z by grid)
template <typename F, int NA>
__global__ void __launch_bounds__(256) pw_accumulate_kernel(double* __restrict__ rhs, const double* __restrict__ a,
                                                            const double* __restrict__ b, const double* __restrict__ c,
                                                            F func, double coeff, PwGeom G) {
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
    if (i >= G.n0 || j >= G.n1) return;
    const int idx = (i + G.g) + G.sx * ((j + G.g) + G.sy * (k + G.g));
    double v;
    if constexpr (NA == 1) v = func(a[idx]);
    else if constexpr (NA == 2) v = func(a[idx], b[idx]);
    else v = func(a[idx], b[idx], c[idx]);
    rhs[idx] = __fma_rn(coeff, v, rhs[idx]);
}

void count_user_launch();
void throw_cuda(cudaError_t e, const char* what);

template <typename F, int NA>
void launch_pw(double* rhs, const double* a, const double* b, const double* c, const F& func, double coeff,
               const PwGeom& G) {
    pw_accumulate_kernel<F, NA><<<pw_grid(G), dim3(32, 8)>>>(rhs, a, b, c, func, coeff, G);
    count_user_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw_cuda(e, "pw kernel");
}

// Fused stage kernels for functor F (see FusedStage.h).
template <typename F>
struct PwKernelsImpl final : fuse::PwKernels {
    F func;
    explicit PwKernelsImpl(const F& f) : func(f) {}

    template <int PAT, int DIM, int MODE>
    int run(const fuse::StageSpec& s, cudaStream_t st) const {
        using Pol = fuse::PolUser<F, PAT>;
        Pol pol{func, s.nops, {}, {}, s.M};
        for (int i = 0; i < fuse::MAX_OPS; ++i) {
            pol.op[i] = s.op[i];
            pol.c[i] = s.c[i];
        }
        const phix::StageArgs<double>& A = s.A;
        if constexpr (MODE == phix::MODE_RK4_STEP) {
            // the whole RK4 step as one launch of the pair kernel (64x28 tiles,
            // 8 row blocks: the FP64 shape the C ABI picks at 1024^2)
            if constexpr (DIM == 2 && PAT == fuse::PATTERN_COMPOSITE) {
                if (!phix::step_pair_supported(A.L, 2)) return PHIX_ERR_UNSUPPORTED;
                using G = phix::StepPair<double, 64, 28, 8>;
                phix::StepArgs<double> B;
                B.S = A;
                B.dt2 = s.dt_half;
                B.dt = s.dt_full;
                dim3 grid((A.L.n[0] + 63) / 64, (A.L.n[1] + 27) / 28, 1);
                // one launch per Solver::advance: each step is a programmatic
                // dependent of the previous one, so its CTAs are resident and
                // waiting (griddepcontrol.wait in step_pair) when that one ends
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = grid;
                cfg.blockDim = dim3(G::NT);
                cfg.dynamicSmemBytes = G::smem_bytes();
                cfg.stream = st;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                at[0].val.programmaticStreamSerializationAllowed = 1;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                auto go = [&]() -> cudaError_t {
                    if (s.nops == 2 && s.op[0] != s.op[1]) {
                        // the two-term CH program (pw and lap, either order) compiled in
                        if (s.op[0] == fuse::OP_PW) {
                            fuse::PolUserCH2<F, true> p2{func, s.c[0], s.c[1], s.M};
                            return cudaLaunchKernelEx(&cfg, phix::step_pair<double, fuse::PolUserCH2<F, true>, 64, 28, 8>,
                                                      B, p2);
                        }
                        fuse::PolUserCH2<F, false> p2{func, s.c[0], s.c[1], s.M};
                        return cudaLaunchKernelEx(&cfg, phix::step_pair<double, fuse::PolUserCH2<F, false>, 64, 28, 8>,
                                                  B, p2);
                    }
                    return cudaLaunchKernelEx(&cfg, phix::step_pair<double, Pol, 64, 28, 8>, B, pol);
                };
                cudaError_t e = go();
                if (e == cudaErrorNotSupported || e == cudaErrorInvalidValue) {
                    // a stream or device without dependent launches: an ordinary launch
                    (void)cudaGetLastError();
                    cfg.numAttrs = 0;
                    e = go();
                }
                count_user_launch();
                return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? PHIX_OK : PHIX_ERR_CUDA;
            } else {
                return PHIX_ERR_UNSUPPORTED;
            }
        } else {
            return run_stage<PAT, DIM, MODE>(pol, s, st);
        }
    }
    template <int PAT, int DIM, int MODE, class Pol>
    int run_stage(const Pol& pol, const fuse::StageSpec& s, cudaStream_t st) const {
        const phix::StageArgs<double>& A = s.A;
        if constexpr (DIM == 2 && MODE == phix::MODE_MULTISTEP && PAT == fuse::PATTERN_COMPOSITE) {
            if (phix::step_pair_supported(A.L, 2)) {
                // the multi-step form on four periodic sides: the pair kernel
                // (64x16 tiles, 4 row blocks: 22 KB of shared memory, no opt-in)
                using G = phix::MsPair<double, 64, 16, 4>;
                dim3 grid((A.L.n[0] + 63) / 64, (A.L.n[1] + 15) / 16, 1);
                phix::step_pair_ms<double, Pol, 64, 16, 4><<<grid, G::NT, G::smem_bytes(), st>>>(A, pol);
                count_user_launch();
                return cudaGetLastError() == cudaSuccess ? PHIX_OK : PHIX_ERR_CUDA;
            }
        }
        if (DIM == 3) {
            using G = phix::March3D<double, Pol, 32, 8>;
            dim3 grid((A.L.n[0] + 31) / 32, (A.L.n[1] + 7) / 8, (A.L.n[2] + 15) / 16);
            phix::stage_march3d<double, Pol, MODE, 32, 8, 16, 256><<<grid, 256, G::smem_bytes(), st>>>(A, pol);
        } else if (DIM == 2) {
            dim3 grid((A.L.n[0] + 63) / 64, (A.L.n[1] + 15) / 16, 1);
            phix::stage_box<double, Pol, 2, MODE, 64, 16, 256><<<grid, 256, 0, st>>>(A, pol);
        } else {
            dim3 grid((A.L.n[0] + 255) / 256, 1, 1);
            phix::stage_box<double, Pol, 1, MODE, 256, 1, 256><<<grid, 256, 0, st>>>(A, pol);
        }
        count_user_launch();
        return cudaGetLastError() == cudaSuccess ? PHIX_OK : PHIX_ERR_CUDA;
    }
    template <int PAT, int DIM>
    int by_mode(const fuse::StageSpec& s, cudaStream_t st) const {
        switch (s.mode) {
            case phix::MODE_K: return run<PAT, DIM, phix::MODE_K>(s, st);
            case phix::MODE_RK4_FINAL: return run<PAT, DIM, phix::MODE_RK4_FINAL>(s, st);
            case phix::MODE_EULER_FINAL: return run<PAT, DIM, phix::MODE_EULER_FINAL>(s, st);
            case phix::MODE_MULTISTEP:
                if (PAT == fuse::PATTERN_COMPOSITE && DIM < 3) return run<PAT, DIM, phix::MODE_MULTISTEP>(s, st);
                return PHIX_ERR_UNSUPPORTED;
            case phix::MODE_RK4_STEP:
                if (PAT == fuse::PATTERN_COMPOSITE && DIM == 2) return run<PAT, DIM, phix::MODE_RK4_STEP>(s, st);
                return PHIX_ERR_UNSUPPORTED;
        }
        return PHIX_ERR_ARG;
    }
    template <int PAT>
    int by_dim(const fuse::StageSpec& s, cudaStream_t st) const {
        switch (s.dim) {
            case 1: return by_mode<PAT, 1>(s, st);
            case 2: return by_mode<PAT, 2>(s, st);
            case 3: return by_mode<PAT, 3>(s, st);
        }
        return PHIX_ERR_ARG;
    }
    template <int PAT, int MODE>
    static int prepare_march() {
        using Pol = fuse::PolUser<F, PAT>;
        using G = phix::March3D<double, Pol, 32, 8>;
        cudaError_t e = cudaFuncSetAttribute(phix::stage_march3d<double, Pol, MODE, 32, 8, 16, 256>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes());
        return e == cudaSuccess ? PHIX_OK : PHIX_ERR_CUDA;
    }
    int prepare(int dim) const override {
        if (dim == 2) {  // the one-launch RK4 step's shared memory (99 KB)
            using Pol = fuse::PolUser<F, fuse::PATTERN_COMPOSITE>;
            using G = phix::StepPair<double, 64, 28, 8>;
            const int b = (int)G::smem_bytes();
            cudaError_t e = cudaFuncSetAttribute(phix::step_pair<double, Pol, 64, 28, 8>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, b);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(phix::step_pair<double, fuse::PolUserCH2<F, true>, 64, 28, 8>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, b);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(phix::step_pair<double, fuse::PolUserCH2<F, false>, 64, 28, 8>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, b);
            return e == cudaSuccess ? PHIX_OK : PHIX_ERR_CUDA;
        }
        if (dim != 3) return PHIX_OK;
        int rc = PHIX_OK;
        if (!rc) rc = prepare_march<fuse::PATTERN_FLAT, phix::MODE_K>();
        if (!rc) rc = prepare_march<fuse::PATTERN_FLAT, phix::MODE_RK4_FINAL>();
        if (!rc) rc = prepare_march<fuse::PATTERN_FLAT, phix::MODE_EULER_FINAL>();
        if (!rc) rc = prepare_march<fuse::PATTERN_COMPOSITE, phix::MODE_K>();
        if (!rc) rc = prepare_march<fuse::PATTERN_COMPOSITE, phix::MODE_RK4_FINAL>();
        if (!rc) rc = prepare_march<fuse::PATTERN_COMPOSITE, phix::MODE_EULER_FINAL>();
        return rc;
    }
    int launch(const fuse::StageSpec& s, void* stream) const override {
        cudaStream_t st = (cudaStream_t)stream;
        return s.pattern == fuse::PATTERN_FLAT ? by_dim<fuse::PATTERN_FLAT>(s, st) : by_dim<fuse::PATTERN_COMPOSITE>(s, st);
    }
};

inline void check_same_layout(const ScalarField& a, const ScalarField& b, const char* what) {
    if (a.mesh.n[0] != b.mesh.n[0] || a.mesh.n[1] != b.mesh.n[1] || a.mesh.n[2] != b.mesh.n[2] ||
        a.ghost != b.ghost)
        throw std::invalid_argument(std::string(what) + ": fields must share the same mesh dimensions and ghost width");
}

}  // namespace detail

template <typename Functor>
Term pw(const ScalarField& f, Functor func, double coeff) {
    Term t;
    t.type = TermType::POINTWISE;
    t.field = &f;
    t.coeff = coeff;
    const detail::PwGeom G = detail::pw_geom(f);
    const ScalarField* pf = &f;  // d_curr is read at launch (late binding)
    t.gpu_launcher = [func, pf, G](double* d_rhs, double c, ScratchPool&) {
        if (!pf->d_curr) throw std::runtime_error("pw GPU: source field not on device");
        detail::launch_pw<Functor, 1>(d_rhs, pf->d_curr, nullptr, nullptr, func, c, G);
    };
    t.cpu_kernel = [func, pf, G](double* rhs, double c, ScratchPool&) {
        const double* src = pf->curr.data();
        for (int k = 0; k < G.n2; ++k)
            for (int j = 0; j < G.n1; ++j)
                for (int i = 0; i < G.n0; ++i) {
                    const int idx = (i + G.g) + G.sx * ((j + G.g) + G.sy * (k + G.g));
                    rhs[idx] += c * func(src[idx]);
                }
    };
    auto info = std::make_shared<fuse::Info>();
    info->kind = fuse::Info::PW1;
    info->field = pf;
    info->pw = std::make_shared<detail::PwKernelsImpl<Functor>>(func);
    info->nargs = 1;
    info->args[0] = pf;
    info->flat = std::make_shared<fuse::FlatKernelsImpl<Functor, 1>>(func);
    t.fusion = info;
    return t;
}

template <typename Functor>
Term pw(const ScalarField& f1, const ScalarField& f2, Functor func, double coeff) {
    detail::check_same_layout(f1, f2, "pw(f1, f2)");
    Term t;
    t.type = TermType::POINTWISE;
    t.field = &f1;
    t.coeff = coeff;
    const detail::PwGeom G = detail::pw_geom(f1);
    const ScalarField *p1 = &f1, *p2 = &f2;
    t.gpu_launcher = [func, p1, p2, G](double* d_rhs, double c, ScratchPool&) {
        if (!p1->d_curr || !p2->d_curr) throw std::runtime_error("pw(f1,f2) GPU: a field not on device");
        detail::launch_pw<Functor, 2>(d_rhs, p1->d_curr, p2->d_curr, nullptr, func, c, G);
    };
    t.cpu_kernel = [func, p1, p2, G](double* rhs, double c, ScratchPool&) {
        const double *a = p1->curr.data(), *b = p2->curr.data();
        for (int k = 0; k < G.n2; ++k)
            for (int j = 0; j < G.n1; ++j)
                for (int i = 0; i < G.n0; ++i) {
                    const int idx = (i + G.g) + G.sx * ((j + G.g) + G.sy * (k + G.g));
                    rhs[idx] += c * func(a[idx], b[idx]);
                }
    };
    auto info = std::make_shared<fuse::Info>();
    info->kind = fuse::Info::PWN;
    info->nargs = 2;
    info->args[0] = p1;
    info->args[1] = p2;
    info->flat = std::make_shared<fuse::FlatKernelsImpl<Functor, 2>>(func);
    t.fusion = info;
    return t;
}

template <typename Functor>
Term pw(const ScalarField& f1, const ScalarField& f2, const ScalarField& f3, Functor func, double coeff) {
    detail::check_same_layout(f1, f2, "pw(f1,f2,f3)");
    detail::check_same_layout(f1, f3, "pw(f1,f2,f3)");
    Term t;
    t.type = TermType::POINTWISE;
    t.field = &f1;
    t.coeff = coeff;
    const detail::PwGeom G = detail::pw_geom(f1);
    const ScalarField *p1 = &f1, *p2 = &f2, *p3 = &f3;
    t.gpu_launcher = [func, p1, p2, p3, G](double* d_rhs, double c, ScratchPool&) {
        if (!p1->d_curr || !p2->d_curr || !p3->d_curr) throw std::runtime_error("pw(f1,f2,f3) GPU: a field not on device");
        detail::launch_pw<Functor, 3>(d_rhs, p1->d_curr, p2->d_curr, p3->d_curr, func, c, G);
    };
    t.cpu_kernel = [func, p1, p2, p3, G](double* rhs, double c, ScratchPool&) {
        const double *a = p1->curr.data(), *b = p2->curr.data(), *d = p3->curr.data();
        for (int k = 0; k < G.n2; ++k)
            for (int j = 0; j < G.n1; ++j)
                for (int i = 0; i < G.n0; ++i) {
                    const int idx = (i + G.g) + G.sx * ((j + G.g) + G.sy * (k + G.g));
                    rhs[idx] += c * func(a[idx], b[idx], d[idx]);
                }
    };
    auto info = std::make_shared<fuse::Info>();
    info->kind = fuse::Info::PWN;
    info->nargs = 3;
    info->args[0] = p1;
    info->args[1] = p2;
    info->args[2] = p3;
    info->flat = std::make_shared<fuse::FlatKernelsImpl<Functor, 3>>(func);
    t.fusion = info;
    return t;
}

template <typename Functor>
VectorRHSExpr pw(const VectorField& vf, Functor func, double coeff) {
    VectorRHSExpr e(vf.nComponents());
    for (int c = 0; c < vf.nComponents(); ++c) e[c] = RHSExpr(pw(vf[c], func, coeff));
    return e;
}
template <typename Functor>
VectorRHSExpr pw(const VectorField& vf, const ScalarField& sf, Functor func, double coeff) {
    VectorRHSExpr e(vf.nComponents());
    for (int c = 0; c < vf.nComponents(); ++c) e[c] = RHSExpr(pw(vf[c], sf, func, coeff));
    return e;
}
template <typename Functor>
VectorRHSExpr pw(const VectorField& vf1, const VectorField& vf2, Functor func, double coeff) {
    if (vf1.nComponents() != vf2.nComponents())
        throw std::invalid_argument("pw(vf1, vf2): VectorFields must have the same number of components");
    VectorRHSExpr e(vf1.nComponents());
    for (int c = 0; c < vf1.nComponents(); ++c) e[c] = RHSExpr(pw(vf1[c], vf2[c], func, coeff));
    return e;
}

}  // namespace PhiX

#include "equation/FieldOps.inl"
