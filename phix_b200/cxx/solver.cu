// solver.cu -- Solver and VectorSolver of the drop-in C++ API.
//
// Solver::advance compiles the equation once (FusedPlan) when its right-hand
// side is a sum of lap / pw terms of the unknown (one pw functor), or
// M*lap(such a sum, bcs) with the solver's own BCs, and every BC is a
// PeriodicBC / NoFluxBC / FixedBC: each RK stage is then one fused kernel
// (phix/detail/stage.cuh with the term program of the equation), the
// multi-step Cahn-Hilliard form one kernel per step.  Other multi-step
// systems, and Euler steps of other right-hand sides, compile each step into
// a flat program (equation/FlatProgram.h: lap, grad, pw of up to three
// fields, products) run as one kernel, with the BC fills in the reference's
// order.  Anything else runs the reference's sequence (Solver.cu:162-259,
// :317-340) on this library's kernels: BC fills, one accumulate kernel per
// term, rk4 combination kernels.
#include <cuda_runtime.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>

#include "boundary/BoundaryCondition.h"
#include "equation/FlatProgram.h"
#include "equation/FusedStage.h"
#include "phix_b200.h"
#include "solver/Solver.h"
#include "solver/VectorSolver.h"

namespace PhiX {

namespace {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// combination kernels of the unfused path (Solver.cu:30-71)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_rk4_tmp(double* __restrict__ tmp, const double* __restrict__ phi,
                                                 const double* __restrict__ k, double c, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        tmp[i] = __fma_rn(c, k[i], phi[i]);
}
__global__ void __launch_bounds__(256) k_rk4_update(double* __restrict__ phi, const double* __restrict__ k1,
                                                    const double* __restrict__ k2, const double* __restrict__ k3,
                                                    const double* __restrict__ k4, double dt6, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double s = __dadd_rn(k1[i], __dmul_rn(2.0, k2[i]));
        s = __dadd_rn(s, __dmul_rn(2.0, k3[i]));
        s = __dadd_rn(s, k4[i]);
        phi[i] = __fma_rn(dt6, s, phi[i]);
    }
}
int grid_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}
void rk4_tmp(double* tmp, const double* phi, const double* k, double c, size_t n) {
    if (k && c != 0.0) k_rk4_tmp<<<grid_for(n), 256>>>(tmp, phi, k, c, n);
    else cuda_check(cudaMemcpyAsync(tmp, phi, n * sizeof(double), cudaMemcpyDeviceToDevice, 0), "rk4 copy");
    phix::count_launch(1);
    cuda_check(cudaGetLastError(), "rk4_tmp");
}
void rk4_update(double* phi, const double* k1, const double* k2, const double* k3, const double* k4, double dt6,
                size_t n) {
    k_rk4_update<<<grid_for(n), 256>>>(phi, k1, k2, k3, k4, dt6, n);
    phix::count_launch(1);
    cuda_check(cudaGetLastError(), "rk4_update");
}
void axpy(double* dst, const double* src, double c, size_t n) {
    if (phix_axpy(dst, src, c, n, nullptr) != PHIX_OK) throw std::runtime_error(phix_last_error());
}

// Identity functor: the fused kernels of right-hand sides without a pw term.
struct IdentityFn {
    __host__ __device__ double operator()(double v) const { return v; }
};

// ---------------------------------------------------------------------------
// plan analysis
// ---------------------------------------------------------------------------
bool bc_layout(const std::vector<BoundaryCondition*>& bcs, int dim, phix::Layout& L) {
    bool set[6] = {false, false, false, false, false, false};
    for (int i = 0; i < 6; ++i) {
        L.bc[i] = PHIX_BC_NONE;
        L.bcv[i] = 0.0;
    }
    for (const auto* bc : bcs) {
        const int k = bc->fusedKind();
        const int a = static_cast<int>(bc->axis);
        if (k < 0 || a >= dim) return false;
        const bool lo = bc->side == Side::LOW || bc->side == Side::BOTH || k == PHIX_BC_PERIODIC;
        const bool hi = bc->side == Side::HIGH || bc->side == Side::BOTH || k == PHIX_BC_PERIODIC;
        for (int s = 0; s < 2; ++s) {
            if (!(s == 0 ? lo : hi)) continue;
            if (set[2 * a + s]) return false;  // two BCs on one side: order-dependent, not fused
            set[2 * a + s] = true;
            L.bc[2 * a + s] = k;
            L.bcv[2 * a + s] = bc->fusedValue();
        }
    }
    return true;
}

bool same_bcs(const phix::Layout& a, const phix::Layout& b) {
    for (int i = 0; i < 6; ++i)
        if (a.bc[i] != b.bc[i] || (a.bc[i] == PHIX_BC_FIXED && a.bcv[i] != b.bcv[i])) return false;
    return true;
}

// sum of c_i * {lap(u) | f(u)} with at most one pw functor
bool flat_program(const RHSExpr& e, const ScalarField* u, fuse::StageSpec& spec,
                  std::shared_ptr<const fuse::PwKernels>& kern) {
    if (e.terms.empty() || e.terms.size() > (size_t)fuse::MAX_OPS) return false;
    spec.nops = 0;
    for (const auto& t : e.terms) {
        if (!t.fusion) return false;
        const fuse::Info& I = *t.fusion;
        if (I.kind == fuse::Info::LAP && I.field == u) {
            spec.op[spec.nops] = fuse::OP_LAP;
        } else if (I.kind == fuse::Info::PW1 && I.field == u) {
            if (kern && kern != I.pw) return false;
            kern = I.pw;
            spec.op[spec.nops] = fuse::OP_PW;
        } else {
            return false;
        }
        spec.c[spec.nops++] = t.coeff;
    }
    return true;
}

phix::Layout field_layout(const ScalarField& f) {
    phix::Layout L{};
    for (int a = 0; a < 3; ++a) L.n[a] = f.mesh.n[a];
    L.s[0] = 1;
    L.s[1] = f.storedDims[0];
    L.s[2] = f.storedDims[0] * f.storedDims[1];
    L.ghost = f.ghost;
    L.origin = f.ghost + L.s[1] * f.ghost + L.s[2] * f.ghost;
    return L;
}

}  // namespace

// The compiled fused path.
// One SolverStep of a general multi-step Solver compiled into one flat_step
// launch (equation/FlatProgram.h), or left to the reference's sequence.
struct FlatStepPlan {
    bool fused = false;
    fuse::FlatSpec spec;  // program and layout; field pointers are set at launch
    const ScalarField* slots[fuse::FLAT_MAX_FIELDS] = {};
    int nslots = 0;
    std::shared_ptr<const fuse::FlatKernels> kern;
};

struct FusedPlan {
    std::shared_ptr<const fuse::PwKernels> kern;
    fuse::StageSpec spec;  // program, pattern, dim, layout; per-stage fields set at launch
    bool multistep = false;
    ScalarField* c = nullptr;   // multi-step: the TRANSIENT unknown
    ScalarField* mu = nullptr;  // multi-step: the STEADY unknown
    bool filled = false;        // the first step's full BC fill (padding ghosts) is done
    std::vector<FlatStepPlan> flat;  // general multi-step: one entry per SolverStep
};

static std::shared_ptr<const fuse::PwKernels> identity_kernels() {
    static auto k = std::make_shared<detail::PwKernelsImpl<IdentityFn>>(IdentityFn{});
    return k;
}

// The flat program of a right-hand side (equation/FlatProgram.h): the terms
// in order, products as nested sub-programs; false when a term is not one the
// program holds, a second pw functor appears, or the fields differ in layout.
class FlatBuilder {
public:
    FlatBuilder(FlatStepPlan& P, const ScalarField& layout) : P_(P), u_(layout) {}
    bool expr(const RHSExpr& e, int sp) {
        for (const auto& t : e.terms) {
            if (!t.fusion) return false;
            const fuse::Info& I = *t.fusion;
            switch (I.kind) {
                case fuse::Info::LAP:
                case fuse::Info::GRAD: {
                    const int k = slot(I.field);
                    if (k < 0 || !push(I.kind == fuse::Info::LAP ? fuse::FL_LAP : fuse::FL_GRAD, k, I.axis, t.coeff))
                        return false;
                    break;
                }
                case fuse::Info::PW1:
                case fuse::Info::PWN: {
                    if (P_.kern || !I.flat || I.nargs < 1 || I.nargs > 3) return false;  // one functor per program
                    P_.kern = I.flat;
                    for (int a = 0; a < I.nargs; ++a)
                        if ((P_.spec.pw_slot[a] = slot(I.args[a])) < 0) return false;
                    if (!push(fuse::FL_PW, 0, 0, t.coeff)) return false;
                    break;
                }
                case fuse::Info::TIMES_FIELD: {
                    if (sp + 1 > fuse::FLAT_MAX_DEPTH || !push(fuse::FL_ZERO, 0, 0, 0.0) || !expr(*I.inner, sp + 1))
                        return false;
                    const int k = slot(I.field);
                    if (k < 0 || !push(fuse::FL_MULF, k, 0, t.coeff)) return false;
                    break;
                }
                case fuse::Info::TIMES_EXPR:
                    if (sp + 2 > fuse::FLAT_MAX_DEPTH || !push(fuse::FL_ZERO, 0, 0, 0.0) || !expr(*I.inner, sp + 1) ||
                        !push(fuse::FL_ZERO, 0, 0, 0.0) || !expr(*I.inner2, sp + 2) || !push(fuse::FL_MUL2, 0, 0, t.coeff))
                        return false;
                    break;
                default:
                    return false;
            }
        }
        return true;
    }
    bool reads(const ScalarField* f) const {
        for (int k = 0; k < P_.nslots; ++k)
            if (P_.slots[k] == f) return true;
        return false;
    }

private:
    FlatStepPlan& P_;
    const ScalarField& u_;
    bool push(int kind, int field, int axis, double c) {
        if (P_.spec.nops >= fuse::FLAT_MAX_OPS) return false;
        P_.spec.op[P_.spec.nops++] = fuse::FlatOp{kind, field, axis, c};
        return true;
    }
    int slot(const ScalarField* f) {
        if (!f) return -1;
        for (int k = 0; k < P_.nslots; ++k)
            if (P_.slots[k] == f) return k;
        if (P_.nslots >= fuse::FLAT_MAX_FIELDS || f->ghost != u_.ghost) return -1;
        for (int a = 0; a < 3; ++a)
            if (f->mesh.n[a] != u_.mesh.n[a] || f->mesh.d[a] != u_.mesh.d[a] || f->storedDims[a] != u_.storedDims[a])
                return -1;
        P_.slots[P_.nslots] = f;
        return P_.nslots++;
    }
};

static std::shared_ptr<const fuse::FlatKernels> identity_flat() {
    static auto k = std::make_shared<fuse::FlatKernelsImpl<IdentityFn, 0>>(IdentityFn{});
    return k;
}

// A SolverStep as one flat_step launch, where its right-hand side compiles.
static void plan_flat_step(const SolverStep& s, FlatStepPlan& P) {
    P = FlatStepPlan{};
    const ScalarField& u = s.equation->unknown;
    if (!s.equation->hasRHS() || u.mesh.dim < 1 || u.mesh.dim > 3) return;
    FlatBuilder b(P, u);
    P.spec.op[P.spec.nops++] = fuse::FlatOp{fuse::FL_ZERO, 0, 0, 0.0};
    if (!b.expr(s.equation->rhsExpr(), 1)) return;
    const bool transient = s.type == EquationType::TRANSIENT;
    // a STEADY unknown is zeroed before its own right-hand side runs
    if (!transient && b.reads(&u)) return;
    if (transient && !u.d_prev) return;
    fuse::FlatSpec& S = P.spec;
    S.L = field_layout(u);
    S.dim = u.mesh.dim;
    for (int a = 0; a < 3; ++a) {
        S.sdims[a] = u.storedDims[a];
        S.i2[a] = a < S.dim ? 1.0 / (u.mesh.d[a] * u.mesh.d[a]) : 0.0;
        S.inv2d[a] = a < S.dim ? 0.5 / u.mesh.d[a] : 0.0;
    }
    S.transient = transient ? 1 : 0;
    if (!P.kern) P.kern = identity_flat();
    P.fused = true;
}

// Single-equation plan, or null.
static std::unique_ptr<FusedPlan> plan_single(const Equation& eq, const std::vector<BoundaryCondition*>& bcs) {
    const ScalarField& u = eq.unknown;
    auto P = std::make_unique<FusedPlan>();
    fuse::StageSpec& S = P->spec;
    S.dim = u.mesh.dim;
    S.A.L = field_layout(u);
    if (!bc_layout(bcs, S.dim, S.A.L)) return nullptr;
    const auto& terms = eq.rhsExpr().terms;
    if (terms.size() == 1 && terms[0].fusion && terms[0].fusion->kind == fuse::Info::LAP_EXPR) {
        const fuse::Info& I = *terms[0].fusion;
        phix::Layout Lc = S.A.L;
        if (!bc_layout(I.bcs, S.dim, Lc) || !same_bcs(Lc, S.A.L)) return nullptr;
        if (!flat_program(*I.inner, &u, S, P->kern)) return nullptr;
        S.pattern = fuse::PATTERN_COMPOSITE;
        S.M = terms[0].coeff;
    } else {
        if (!flat_program(eq.rhsExpr(), &u, S, P->kern)) return nullptr;
        S.pattern = fuse::PATTERN_FLAT;
    }
    if (!P->kern) P->kern = identity_kernels();
    for (int a = 0; a < 3; ++a) S.A.i2[a] = a < S.dim ? 1.0 / (u.mesh.d[a] * u.mesh.d[a]) : 0.0;
    if (P->kern->prepare(S.dim) != PHIX_OK) return nullptr;
    return P;
}

// General multi-step plan: every step that compiles runs as one flat_step
// launch; null when none does.
static std::unique_ptr<FusedPlan> plan_multistep_flat(const std::vector<SolverStep>& steps, double dt) {
    auto P = std::make_unique<FusedPlan>();
    P->flat.resize(steps.size());
    bool any = false;
    for (std::size_t i = 0; i < steps.size(); ++i) {
        plan_flat_step(steps[i], P->flat[i]);
        P->flat[i].spec.dt = dt;
        any = any || P->flat[i].fused;
    }
    if (!any) return nullptr;
    return P;
}

// Multi-step Cahn-Hilliard plan: [mu STEADY <- program(c); c TRANSIENT <- M lap(mu)].
static std::unique_ptr<FusedPlan> plan_multistep_ch(const std::vector<SolverStep>& steps) {
    if (steps.size() != 2 || steps[0].type != EquationType::STEADY || steps[1].type != EquationType::TRANSIENT)
        return nullptr;
    ScalarField& mu = steps[0].equation->unknown;
    ScalarField& c = steps[1].equation->unknown;
    if (steps[0].sourceField != &c || steps[1].sourceField != &mu || c.mesh.dim > 2 || c.ghost != 1) return nullptr;
    const auto& t1 = steps[1].equation->rhsExpr().terms;
    if (t1.size() != 1 || !t1[0].fusion || t1[0].fusion->kind != fuse::Info::LAP || t1[0].fusion->field != &mu)
        return nullptr;
    auto P = std::make_unique<FusedPlan>();
    fuse::StageSpec& S = P->spec;
    S.dim = c.mesh.dim;
    S.A.L = field_layout(c);
    phix::Layout L1 = S.A.L;
    if (!bc_layout(steps[0].bcs, S.dim, S.A.L) || !bc_layout(steps[1].bcs, S.dim, L1) || !same_bcs(S.A.L, L1))
        return nullptr;
    if (!flat_program(steps[0].equation->rhsExpr(), &c, S, P->kern)) return nullptr;
    if (!P->kern) P->kern = identity_kernels();
    S.pattern = fuse::PATTERN_COMPOSITE;
    S.M = t1[0].coeff;
    for (int a = 0; a < 3; ++a) S.A.i2[a] = a < S.dim ? 1.0 / (c.mesh.d[a] * c.mesh.d[a]) : 0.0;
    P->multistep = true;
    P->c = &c;
    P->mu = &mu;
    return P;
}

// ---------------------------------------------------------------------------
// Solver
// ---------------------------------------------------------------------------
static ScalarField scratch_like(const ScalarField& ref, const std::string& tag) {
    ScalarField f(ref.mesh, tag, ref.ghost);
    f.allocDevice();
    return f;
}

Solver::Solver(Equation& equation, std::vector<BoundaryCondition*> bcs, double dt_, TimeScheme scheme_)
    : dt(dt_),
      scheme(scheme_),
      equation_(equation),
      bcs_(std::move(bcs)),
      rhs_(scratch_like(equation.unknown, equation.unknown.name + "_rhs")),
      k1_(scratch_like(equation.unknown, "_k1")),
      k2_(scratch_like(equation.unknown, "_k2")),
      k3_(scratch_like(equation.unknown, "_k3")),
      k4_(scratch_like(equation.unknown, "_k4")),
      phi_tmp_(scratch_like(equation.unknown, "_phi_tmp")),
      use_rk4_(scheme_ == TimeScheme::RK4) {
    if (!equation_.unknown.deviceAllocated())
        throw std::runtime_error("Solver: equation.unknown must have device memory allocated before constructing the Solver.");
    if (equation_.hasRHS()) plan_ = plan_single(equation_, bcs_);
    if (!plan_ && !use_rk4_ && equation_.hasRHS()) {
        // an Euler step whose terms the stage kernels do not take (grad, div,
        // products, pw of several fields): the step {BCs on the unknown; rhs;
        // u += dt rhs} as one flat_step launch where the terms compile
        std::vector<SolverStep> one = {{&equation_.unknown, bcs_, &equation_, EquationType::TRANSIENT}};
        auto P = plan_multistep_flat(one, dt);
        if (P && P->flat[0].fused) {
            steps_ = std::move(one);
            stepScratch_.push_back(nullptr);
            plan_ = std::move(P);
        }
    }
}

Solver::Solver(std::vector<SolverStep> steps, double dt_, TimeScheme scheme_)
    : dt(dt_),
      scheme(scheme_),
      equation_(*steps.at(0).equation),
      bcs_({}),
      rhs_(scratch_like(steps[0].equation->unknown, "_ms_rhs")),
      k1_(scratch_like(steps[0].equation->unknown, "_k1")),
      k2_(scratch_like(steps[0].equation->unknown, "_k2")),
      k3_(scratch_like(steps[0].equation->unknown, "_k3")),
      k4_(scratch_like(steps[0].equation->unknown, "_k4")),
      phi_tmp_(scratch_like(steps[0].equation->unknown, "_phi_tmp")),
      use_rk4_(false),
      multiStep_(true),
      steps_(std::move(steps)) {
    for (auto& s : steps_) {
        if (!s.equation->unknown.deviceAllocated())
            throw std::runtime_error("Solver (multi-step): all equation unknowns must have device memory allocated "
                                     "before constructing the Solver.");
        if (s.type == EquationType::TRANSIENT)
            stepScratch_.push_back(std::make_unique<ScalarField>(scratch_like(s.equation->unknown, s.equation->name + "_rhs")));
        else
            stepScratch_.push_back(nullptr);
    }
    bool all_rhs = true;
    for (auto& s : steps_) all_rhs = all_rhs && s.equation->hasRHS();
    if (all_rhs) {
        plan_ = plan_multistep_ch(steps_);
        if (!plan_) plan_ = plan_multistep_flat(steps_, dt);
    }
}

Solver::~Solver() = default;

void Solver::disableFusion() { plan_.reset(); }

void Solver::applyBCsGPU() {
    for (auto* bc : bcs_) bc->applyOnGPU(equation_.unknown);
}
void Solver::applyBCsCPU() {
    for (auto* bc : bcs_) bc->applyOnCPU(equation_.unknown);
}

void Solver::eulerUpdateGPU() { axpy(equation_.unknown.d_curr, rhs_.d_curr, dt, equation_.unknown.storedSize); }
void Solver::eulerUpdateCPU() {
    auto& phi = equation_.unknown.curr;
    for (std::size_t i = 0; i < phi.size(); ++i) {
        volatile double d = dt * rhs_.curr[i];
        phi[i] += d;
    }
}

// BC fill of phi_tmp (Solver.cu prepTmpGPU): the BCs act on a shell of it.
static void apply_bcs_to(const std::vector<BoundaryCondition*>& bcs, ScalarField& like, double* buf) {
    ScalarField shell = ScalarField::makeShell(like.mesh, like.ghost, buf);
    for (auto* bc : bcs) bc->applyOnGPU(shell);
}

void Solver::rk4AdvanceGPU() {
    ScalarField& phi = equation_.unknown;
    const size_t n = phi.storedSize;
    const double dt2 = dt * 0.5, dt6 = dt / 6.0;
    applyBCsGPU();
    equation_.computeRHS(k1_);
    ScalarField* ks[3] = {&k1_, &k2_, &k3_};
    ScalarField* kn[3] = {&k2_, &k3_, &k4_};
    const double as[3] = {dt2, dt2, dt};
    for (int s = 0; s < 3; ++s) {
        rk4_tmp(phi_tmp_.d_curr, phi.d_curr, ks[s]->d_curr, as[s], n);
        apply_bcs_to(bcs_, phi, phi_tmp_.d_curr);
        double* orig = phi.d_curr;  // terms read d_curr at launch
        phi.d_curr = phi_tmp_.d_curr;
        try {
            equation_.computeRHS(*kn[s]);
        } catch (...) {
            phi.d_curr = orig;
            throw;
        }
        phi.d_curr = orig;
    }
    rk4_update(phi.d_curr, k1_.d_curr, k2_.d_curr, k3_.d_curr, k4_.d_curr, dt6, n);
    cuda_check(cudaDeviceSynchronize(), "Solver::rk4AdvanceGPU");
}

// The reference's host RK4 (Solver.cu:267-300), including where it applies BCs.
void Solver::rk4AdvanceCPU() {
    auto& phi = equation_.unknown.curr;
    auto& tmp = phi_tmp_.curr;
    const std::size_t N = phi.size();
    const double dt2 = dt * 0.5, dt6 = dt / 6.0;
    auto stage = [&](const std::vector<double>& k, double a, std::vector<double>& kout) {
        for (std::size_t i = 0; i < N; ++i) {
            volatile double d = a * k[i];
            tmp[i] = phi[i] + d;
        }
        std::swap(phi, tmp);
        equation_.computeRHSCPU(rhs_);
        std::copy(rhs_.curr.begin(), rhs_.curr.end(), kout.begin());
        std::swap(phi, tmp);
    };
    applyBCsCPU();
    equation_.computeRHSCPU(rhs_);
    std::copy(rhs_.curr.begin(), rhs_.curr.end(), k1_.curr.begin());
    // the reference refreshes the BCs of phi (not of the stage state) here
    for (std::size_t i = 0; i < N; ++i) {
        volatile double d = dt2 * k1_.curr[i];
        tmp[i] = phi[i] + d;
    }
    applyBCsCPU();
    std::swap(phi, tmp);
    equation_.computeRHSCPU(rhs_);
    std::copy(rhs_.curr.begin(), rhs_.curr.end(), k2_.curr.begin());
    std::swap(phi, tmp);
    stage(k2_.curr, dt2, k3_.curr);
    stage(k3_.curr, dt, k4_.curr);
    for (std::size_t i = 0; i < N; ++i) {
        volatile double a = 2.0 * k2_.curr[i];
        volatile double b = 2.0 * k3_.curr[i];
        volatile double s = k1_.curr[i] + a;
        s = s + b;
        s = s + k4_.curr[i];
        volatile double d = dt6 * s;
        phi[i] += d;
    }
}

void Solver::multiStepAdvanceGPU() {
    for (std::size_t i = 0; i < steps_.size(); ++i) {
        auto& s = steps_[i];
        for (auto* bc : s.bcs) bc->applyOnGPU(*s.sourceField);
        if (s.type == EquationType::STEADY) {
            s.equation->computeRHS(s.equation->unknown);
        } else {
            s.equation->computeRHS(*stepScratch_[i]);
            axpy(s.equation->unknown.d_curr, stepScratch_[i]->d_curr, dt, s.equation->unknown.storedSize);
            cuda_check(cudaDeviceSynchronize(), "Solver::multiStepAdvanceGPU");
        }
    }
    for (auto& s : steps_)
        if (s.type == EquationType::TRANSIENT) s.equation->unknown.advanceTimeLevelGPU();
}

void Solver::multiStepAdvanceCPU() {
    for (std::size_t i = 0; i < steps_.size(); ++i) {
        auto& s = steps_[i];
        for (auto* bc : s.bcs) bc->applyOnCPU(*s.sourceField);
        if (s.type == EquationType::STEADY) {
            s.equation->computeRHSCPU(s.equation->unknown);
        } else {
            s.equation->computeRHSCPU(*stepScratch_[i]);
            auto& phi = s.equation->unknown.curr;
            auto& rhs = stepScratch_[i]->curr;
            for (std::size_t j = 0; j < phi.size(); ++j) {
                volatile double d = dt * rhs[j];
                phi[j] += d;
            }
        }
    }
    for (auto& s : steps_)
        if (s.type == EquationType::TRANSIENT) s.equation->unknown.advanceTimeLevelCPU();
}

// One fused step: stage kernels write the new state into d_prev, then d_curr
// and d_prev swap (d_prev keeps the previous time level).
void Solver::fusedAdvance() {
    FusedPlan& P = *plan_;
    if (!P.flat.empty()) {
        // general multi-step: the reference's step order (Solver.cu:317-340),
        // each compiled step one flat_step launch; a TRANSIENT step writes the
        // unknown's other level and swaps it in (d_prev keeps the old level)
        for (std::size_t i = 0; i < steps_.size(); ++i) {
            auto& s = steps_[i];
            for (auto* bc : s.bcs) bc->applyOnGPU(*s.sourceField);
            FlatStepPlan& F = P.flat[i];
            ScalarField& u = s.equation->unknown;
            if (!F.fused) {
                if (s.type == EquationType::STEADY) {
                    s.equation->computeRHS(u);
                } else {
                    s.equation->computeRHS(*stepScratch_[i]);
                    axpy(u.d_curr, stepScratch_[i]->d_curr, dt, u.storedSize);
                    cuda_check(cudaDeviceSynchronize(), "Solver::multiStepAdvanceGPU");
                }
                continue;
            }
            fuse::FlatSpec S = F.spec;
            for (int k = 0; k < F.nslots; ++k) {
                S.f[k] = F.slots[k]->d_curr;
                if (!S.f[k]) throw std::runtime_error("Solver: a field of step " + std::to_string(i) + " is not on device");
            }
            if (S.transient) {
                S.u = u.d_curr;
                S.out = u.d_prev;
            } else {
                S.out = u.d_curr;
            }
            if (F.kern->launch(S, nullptr) != PHIX_OK)
                throw std::runtime_error(std::string("Solver: fused step launch failed: ") +
                                         cudaGetErrorString(cudaGetLastError()));
            phix::count_launch(1);
            if (S.transient) std::swap(u.d_curr, u.d_prev);
        }
        for (std::size_t i = 0; i < steps_.size(); ++i)
            if (steps_[i].type == EquationType::TRANSIENT && !P.flat[i].fused)
                steps_[i].equation->unknown.advanceTimeLevelGPU();
        return;
    }
    fuse::StageSpec S = P.spec;
    phix::StageArgs<double>& A = S.A;
    ScalarField& u = P.multistep ? *P.c : equation_.unknown;
    if (!u.d_curr || !u.d_prev) throw std::runtime_error("Solver: unknown not on device");
    if (!P.filled) {
        // the reference fills every ghost of the stored array at each step;
        // padding-plane ghosts never change afterwards, so one fill of both
        // time levels covers them (the kernels keep the physical plane's)
        if (P.multistep) {
            cuda_check(cudaMemset(P.mu->d_curr, 0, P.mu->storedSize * sizeof(double)), "Solver: mu");
            for (auto* bc : steps_[1].bcs) bc->applyOnGPU(*P.mu);
            for (auto* bc : steps_[0].bcs) bc->applyOnGPU(u);
            apply_bcs_to(steps_[0].bcs, u, u.d_prev);
        } else {
            applyBCsGPU();
            apply_bcs_to(bcs_, u, u.d_prev);
        }
        P.filled = true;
    }
    A.u[0] = u.d_curr;
    int rc;
    if (P.multistep) {
        S.mode = phix::MODE_MULTISTEP;
        A.out[0] = u.d_prev;
        A.mu_out = P.mu->d_curr;
        A.dtf = dt;
        if ((rc = P.kern->launch(S, nullptr)) != PHIX_OK) throw std::runtime_error("Solver: fused multi-step launch failed");
    } else if (!use_rk4_) {
        S.mode = phix::MODE_EULER_FINAL;
        A.out[0] = u.d_prev;
        A.dtf = dt;
        if ((rc = P.kern->launch(S, nullptr)) != PHIX_OK) throw std::runtime_error("Solver: fused Euler launch failed");
    } else if (S.pattern == fuse::PATTERN_COMPOSITE && S.dim == 2 && phix::step_pair_supported(A.L, 2)) {
        // the whole RK4 step in one launch (the pair kernel, four periodic
        // sides): the same operations per cell as the four stage launches
        S.mode = phix::MODE_RK4_STEP;
        A.out[0] = u.d_prev;
        A.dtf = dt / 6.0;
        S.dt_half = dt * 0.5;
        S.dt_full = dt;
        if ((rc = P.kern->launch(S, nullptr)) != PHIX_OK) throw std::runtime_error("Solver: fused RK4 step launch failed");
    } else {
        double* ks[3] = {k1_.d_curr, k2_.d_curr, k3_.d_curr};
        S.mode = phix::MODE_K;
        for (int st = 0; st < 3; ++st) {
            A.kin[0] = st == 0 ? nullptr : ks[st - 1];
            A.a = dt * 0.5;
            A.out[0] = ks[st];
            if ((rc = P.kern->launch(S, nullptr)) != PHIX_OK) throw std::runtime_error("Solver: fused stage launch failed");
        }
        S.mode = phix::MODE_RK4_FINAL;
        A.kin[0] = ks[2];
        A.k1[0] = ks[0];
        A.k2[0] = ks[1];
        A.a = dt;
        A.dtf = dt / 6.0;
        A.out[0] = u.d_prev;
        if ((rc = P.kern->launch(S, nullptr)) != PHIX_OK) throw std::runtime_error("Solver: fused stage launch failed");
    }
    cuda_check(cudaGetLastError(), "Solver::advance");
    std::swap(u.d_curr, u.d_prev);
}

void Solver::advance() {
    if (plan_) {
        fusedAdvance();
    } else if (multiStep_) {
        multiStepAdvanceGPU();
    } else {
        if (use_rk4_) {
            rk4AdvanceGPU();
        } else {
            applyBCsGPU();
            equation_.computeRHS(rhs_);
            eulerUpdateGPU();
            cuda_check(cudaDeviceSynchronize(), "Solver::advance");
        }
        equation_.unknown.advanceTimeLevelGPU();
    }
    ++step;
    time += dt;
}

void Solver::advanceCPU() {
    if (multiStep_) {
        multiStepAdvanceCPU();
    } else {
        if (use_rk4_) {
            rk4AdvanceCPU();
        } else {
            applyBCsCPU();
            equation_.computeRHSCPU(rhs_);
            eulerUpdateCPU();
        }
        equation_.unknown.advanceTimeLevelCPU();
    }
    ++step;
    time += dt;
}

void Solver::run(int nSteps, int callbackEvery, std::function<void(const Solver&)> callback) {
    for (int s = 0; s < nSteps; ++s) {
        advance();
        if (callback && callbackEvery > 0 && step % callbackEvery == 0) {
            cuda_check(cudaDeviceSynchronize(), "Solver::run");
            callback(*this);
        }
    }
    cuda_check(cudaDeviceSynchronize(), "Solver::run");
}

// ---------------------------------------------------------------------------
// VectorSolver (VectorSolver.cu:77-228): every component advanced from one
// consistent stage state.
// ---------------------------------------------------------------------------
static VectorField vector_scratch(const VectorField& ref, const std::string& tag) {
    VectorField vf(ref.mesh, tag, ref.nComponents(), ref.ghost);
    vf.allocDevice();
    return vf;
}

VectorSolver::VectorSolver(VectorEquation& equation, std::vector<BoundaryCondition*> bcs, double dt_,
                           TimeScheme scheme_)
    : dt(dt_),
      scheme(scheme_),
      equation_(equation),
      bcs_(std::move(bcs)),
      use_rk4_(scheme_ == TimeScheme::RK4),
      rhs_(vector_scratch(equation.unknown, equation.unknown.name + "_rhs")),
      k1_(vector_scratch(equation.unknown, equation.unknown.name + "_k1")),
      k2_(vector_scratch(equation.unknown, equation.unknown.name + "_k2")),
      k3_(vector_scratch(equation.unknown, equation.unknown.name + "_k3")),
      k4_(vector_scratch(equation.unknown, equation.unknown.name + "_k4")),
      phi_tmp_(vector_scratch(equation.unknown, equation.unknown.name + "_tmp")) {
    for (int c = 0; c < equation.unknown.nComponents(); ++c)
        if (!equation_.unknown[c].deviceAllocated())
            throw std::runtime_error("VectorSolver: all components of equation.unknown must have device memory "
                                     "allocated before constructing VectorSolver.");
}

void VectorSolver::applyBCsGPU() {
    for (auto* bc : bcs_) bc->applyOnGPU(equation_.unknown);
}
void VectorSolver::applyBCsCPU() {
    for (auto* bc : bcs_) bc->applyOnCPU(equation_.unknown);
}

void VectorSolver::rk4AdvanceGPU() {
    VectorField& phi = equation_.unknown;
    const int N = phi.nComponents();
    const double dt2 = dt * 0.5, dt6 = dt / 6.0;
    applyBCsGPU();
    equation_.computeRHS(k1_);
    VectorField* ks[3] = {&k1_, &k2_, &k3_};
    VectorField* kn[3] = {&k2_, &k3_, &k4_};
    const double as[3] = {dt2, dt2, dt};
    std::vector<double*> orig(N);
    for (int s = 0; s < 3; ++s) {
        for (int c = 0; c < N; ++c) rk4_tmp(phi_tmp_[c].d_curr, phi[c].d_curr, (*ks[s])[c].d_curr, as[s], phi[c].storedSize);
        for (int c = 0; c < N; ++c) {
            orig[c] = phi[c].d_curr;
            phi[c].d_curr = phi_tmp_[c].d_curr;
        }
        try {
            for (auto* bc : bcs_) bc->applyOnGPU(phi);
            equation_.computeRHS(*kn[s]);
        } catch (...) {
            for (int c = 0; c < N; ++c) phi[c].d_curr = orig[c];
            throw;
        }
        for (int c = 0; c < N; ++c) phi[c].d_curr = orig[c];
    }
    for (int c = 0; c < N; ++c)
        rk4_update(phi[c].d_curr, k1_[c].d_curr, k2_[c].d_curr, k3_[c].d_curr, k4_[c].d_curr, dt6, phi[c].storedSize);
    cuda_check(cudaDeviceSynchronize(), "VectorSolver::rk4AdvanceGPU");
}

void VectorSolver::rk4AdvanceCPU() {
    const int N = equation_.unknown.nComponents();
    const double dt2 = dt * 0.5, dt6 = dt / 6.0;
    auto eval = [&](VectorField& off, double coeff, VectorField& ki) {
        for (int c = 0; c < N; ++c) {
            auto& phi = equation_.unknown[c].curr;
            auto& tmp = phi_tmp_[c].curr;
            for (std::size_t i = 0; i < phi.size(); ++i) {
                volatile double d = coeff * off[c].curr[i];
                tmp[i] = phi[i] + d;
            }
        }
        for (int c = 0; c < N; ++c) std::swap(equation_.unknown[c].curr, phi_tmp_[c].curr);
        applyBCsCPU();
        equation_.computeRHSCPU(rhs_);
        for (int c = 0; c < N; ++c) std::copy(rhs_[c].curr.begin(), rhs_[c].curr.end(), ki[c].curr.begin());
        for (int c = 0; c < N; ++c) std::swap(equation_.unknown[c].curr, phi_tmp_[c].curr);
    };
    applyBCsCPU();
    equation_.computeRHSCPU(rhs_);
    for (int c = 0; c < N; ++c) std::copy(rhs_[c].curr.begin(), rhs_[c].curr.end(), k1_[c].curr.begin());
    eval(k1_, dt2, k2_);
    eval(k2_, dt2, k3_);
    eval(k3_, dt, k4_);
    for (int c = 0; c < N; ++c) {
        auto& phi = equation_.unknown[c].curr;
        for (std::size_t i = 0; i < phi.size(); ++i) {
            volatile double a = 2.0 * k2_[c].curr[i];
            volatile double b = 2.0 * k3_[c].curr[i];
            volatile double s = k1_[c].curr[i] + a;
            s = s + b;
            s = s + k4_[c].curr[i];
            volatile double d = dt6 * s;
            phi[i] += d;
        }
    }
}

void VectorSolver::advance() {
    if (use_rk4_) {
        rk4AdvanceGPU();
    } else {
        applyBCsGPU();
        equation_.computeRHS(rhs_);
        for (int c = 0; c < equation_.unknown.nComponents(); ++c)
            axpy(equation_.unknown[c].d_curr, rhs_[c].d_curr, dt, equation_.unknown[c].storedSize);
        cuda_check(cudaDeviceSynchronize(), "VectorSolver::advance");
    }
    for (int c = 0; c < equation_.unknown.nComponents(); ++c) equation_.unknown[c].advanceTimeLevelGPU();
    ++step;
    time += dt;
}

void VectorSolver::advanceCPU() {
    if (use_rk4_) {
        rk4AdvanceCPU();
    } else {
        applyBCsCPU();
        equation_.computeRHSCPU(rhs_);
        for (int c = 0; c < equation_.unknown.nComponents(); ++c) {
            auto& phi = equation_.unknown[c].curr;
            for (std::size_t i = 0; i < phi.size(); ++i) {
                volatile double d = dt * rhs_[c].curr[i];
                phi[i] += d;
            }
        }
    }
    for (int c = 0; c < equation_.unknown.nComponents(); ++c) equation_.unknown[c].advanceTimeLevelCPU();
    ++step;
    time += dt;
}

void VectorSolver::run(int nSteps, int callbackEvery, std::function<void(const VectorSolver&)> callback) {
    for (int s = 0; s < nSteps; ++s) {
        advance();
        if (callback && callbackEvery > 0 && step % callbackEvery == 0) callback(*this);
    }
}

}  // namespace PhiX
