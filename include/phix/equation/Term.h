#pragma once
// Term / RHSExpr -- the right-hand-side DSL (API of the reference's
// include/equation/Term.h): lap, grad, pw, div, curl, composites
// lap(expr, bcs) / grad(expr, axis, bcs), coefficient arithmetic.
//
// Every Term keeps the reference's type-erased launchers (gpu_launcher,
// cpu_kernel: one accumulate per term).  In addition it carries a fusion
// descriptor: lap / pw / lap(expr, bcs) terms record what they compute, and
// a pw term records a launcher of fused stage kernels instantiated for its
// functor in the caller's translation unit.  Solver uses the descriptors to
// compile a whole right-hand side into one fused kernel per RK stage.

#include <cstddef>
#include <functional>
#include <memory>
#include <vector>

#include "field/ScalarField.h"
#include "field/VectorField.h"

#define PHIX_FN [=] __host__ __device__

namespace PhiX {

class BoundaryCondition;

// Recyclable scratch buffers of composite terms, reset per computeRHS.
class ScratchPool {
public:
    ScratchPool() = default;
    ~ScratchPool();
    ScratchPool(const ScratchPool&) = delete;
    ScratchPool& operator=(const ScratchPool&) = delete;
    double* acquireDevice(std::size_t size);
    double* acquireHost(std::size_t size);
    void reset() { next_dev_ = 0; next_host_ = 0; }

private:
    std::vector<double*> dev_bufs_;
    std::vector<std::size_t> dev_sizes_;
    std::size_t next_dev_ = 0;
    std::vector<std::vector<double>> host_bufs_;
    std::size_t next_host_ = 0;
};

using TermLauncher = std::function<void(double* /*rhs*/, double /*coeff*/, ScratchPool& /*pool*/)>;

enum class TermType { LAPLACIAN, GRADIENT, POINTWISE, COMPOSITE };

struct Term;
struct RHSExpr;

namespace fuse {
struct StageSpec;  // phix/equation/FusedStage.h

// Launches fused stage kernels whose pointwise term is one user functor.
// Implemented per functor type in the caller's translation unit (TermPW.inl).
struct PwKernels {
    virtual ~PwKernels() = default;
    virtual int launch(const StageSpec& spec, void* stream) const = 0;
    // One-time launch setup (shared-memory opt-in) for grids of `dim`;
    // called outside any stream capture.
    virtual int prepare(int dim) const = 0;
};

struct FlatKernels;  // phix/equation/FlatProgram.h

// What a term computes, for the fused path.
struct Info {
    enum Kind { LAP, PW1, LAP_EXPR, GRAD, PWN, TIMES_FIELD, TIMES_EXPR, OTHER } kind = OTHER;
    const ScalarField* field = nullptr;         // LAP, PW1, GRAD, TIMES_FIELD (the field factor)
    std::shared_ptr<const PwKernels> pw;        // PW1
    std::shared_ptr<const RHSExpr> inner;       // LAP_EXPR, TIMES_FIELD, TIMES_EXPR (first factor)
    std::shared_ptr<const RHSExpr> inner2;      // TIMES_EXPR (second factor)
    std::vector<BoundaryCondition*> bcs;        // LAP_EXPR
    int axis = 0;                               // GRAD
    int nargs = 0;                              // PW1, PWN: the functor's fields
    const ScalarField* args[3] = {nullptr, nullptr, nullptr};
    std::shared_ptr<const FlatKernels> flat;    // PW1, PWN: step kernels with this functor
};
}  // namespace fuse

struct Term {
    TermType type = TermType::LAPLACIAN;
    double coeff = 1.0;
    const ScalarField* field = nullptr;
    int axis = 0;
    TermLauncher gpu_launcher;
    TermLauncher cpu_kernel;
    std::shared_ptr<const fuse::Info> fusion;  // null: not fusable

    Term operator*(double s) const { Term t = *this; t.coeff *= s; return t; }
    Term operator/(double s) const { return *this * (1.0 / s); }
    Term operator-() const { return *this * (-1.0); }
};

inline Term operator*(double s, const Term& t) { return t * s; }
inline Term operator/(const Term& t, double s) { return t * (1.0 / s); }

struct RHSExpr {
    std::vector<Term> terms;
    RHSExpr() = default;
    explicit RHSExpr(const Term& t) { terms.push_back(t); }
    RHSExpr& operator+=(const Term& t) { terms.push_back(t); return *this; }
    RHSExpr& operator-=(const Term& t) { terms.push_back(-t); return *this; }
    RHSExpr& operator+=(const RHSExpr& e) { terms.insert(terms.end(), e.terms.begin(), e.terms.end()); return *this; }
    RHSExpr& operator-=(const RHSExpr& e) { for (const auto& t : e.terms) terms.push_back(-t); return *this; }
    RHSExpr operator+(const Term& t) const { RHSExpr r = *this; r += t; return r; }
    RHSExpr operator-(const Term& t) const { RHSExpr r = *this; r -= t; return r; }
    RHSExpr operator+(const RHSExpr& e) const { RHSExpr r = *this; r += e; return r; }
    RHSExpr operator-(const RHSExpr& e) const { RHSExpr r = *this; r -= e; return r; }
    RHSExpr operator*(double s) const { RHSExpr r; for (const auto& t : terms) r.terms.push_back(t * s); return r; }
};

inline RHSExpr operator+(const Term& a, const Term& b) { RHSExpr e(a); e += b; return e; }
inline RHSExpr operator-(const Term& a, const Term& b) { RHSExpr e(a); e -= b; return e; }
inline RHSExpr operator+(const Term& t, const RHSExpr& e) { RHSExpr r(t); r += e; return r; }
inline RHSExpr operator-(const Term& t, const RHSExpr& e) { RHSExpr r(t); r -= e; return r; }
inline RHSExpr operator*(double s, const RHSExpr& e) { return e * s; }

// coeff * lap(f): 3/5/7-point Laplacian over the active axes
Term lap(const ScalarField& f, double coeff = 1.0);
// coeff * d f / d x_axis: central difference
Term grad(const ScalarField& f, int axis, double coeff = 1.0);

// operators on materialised expressions (BCs applied to the scratch field)
Term lap(const Term& t, const std::vector<BoundaryCondition*>& bcs, double coeff = 1.0);
Term lap(const RHSExpr& expr, const std::vector<BoundaryCondition*>& bcs, double coeff = 1.0);
Term grad(const Term& t, int axis, const std::vector<BoundaryCondition*>& bcs, double coeff = 1.0);
Term grad(const RHSExpr& expr, int axis, const std::vector<BoundaryCondition*>& bcs, double coeff = 1.0);

struct VectorRHSExpr;
VectorRHSExpr grad(const Term& t, const std::vector<BoundaryCondition*>& bcs, double coeff = 1.0);
VectorRHSExpr grad(const RHSExpr& expr, const std::vector<BoundaryCondition*>& bcs, double coeff = 1.0);

template <typename Functor>
Term pw(const ScalarField& f, Functor func, double coeff = 1.0);
template <typename Functor>
Term pw(const ScalarField& f1, const ScalarField& f2, Functor func, double coeff = 1.0);
template <typename Functor>
Term pw(const ScalarField& f1, const ScalarField& f2, const ScalarField& f3, Functor func, double coeff = 1.0);

struct VectorRHSExpr {
    std::vector<RHSExpr> components;
    VectorRHSExpr() = default;
    explicit VectorRHSExpr(int n) : components(n) {}
    int nComponents() const { return static_cast<int>(components.size()); }
    RHSExpr& operator[](int c) { return components[c]; }
    const RHSExpr& operator[](int c) const { return components[c]; }
    VectorRHSExpr& operator+=(const VectorRHSExpr& o) { for (int c = 0; c < nComponents(); ++c) components[c] += o.components[c]; return *this; }
    VectorRHSExpr& operator-=(const VectorRHSExpr& o) { for (int c = 0; c < nComponents(); ++c) components[c] -= o.components[c]; return *this; }
    VectorRHSExpr operator+(const VectorRHSExpr& o) const { VectorRHSExpr r = *this; r += o; return r; }
    VectorRHSExpr operator-(const VectorRHSExpr& o) const { VectorRHSExpr r = *this; r -= o; return r; }
    VectorRHSExpr operator*(double s) const {
        VectorRHSExpr r(nComponents());
        for (int c = 0; c < nComponents(); ++c) r[c] = components[c] * s;
        return r;
    }
    VectorRHSExpr operator-() const { return (*this) * (-1.0); }
};
inline VectorRHSExpr operator*(double s, const VectorRHSExpr& e) { return e * s; }

VectorRHSExpr lap(const VectorField& vf, double coeff = 1.0);
VectorRHSExpr grad(const ScalarField& f, double coeff = 1.0);
RHSExpr div(const VectorField& vf, double coeff = 1.0);
RHSExpr div(const VectorRHSExpr& v, const std::vector<BoundaryCondition*>& bcs, double coeff = 1.0);
VectorRHSExpr curl(const VectorField& vf, double coeff = 1.0);

template <typename Functor>
VectorRHSExpr pw(const VectorField& vf, Functor func, double coeff = 1.0);
template <typename Functor>
VectorRHSExpr pw(const VectorField& vf, const ScalarField& sf, Functor func, double coeff = 1.0);
template <typename Functor>
VectorRHSExpr pw(const VectorField& vf1, const VectorField& vf2, Functor func, double coeff = 1.0);

}  // namespace PhiX

#include "equation/TermPW.inl"
