// equation.cu -- Term factories, composite terms, ScratchPool, Equation and
// VectorEquation of the drop-in C++ API.  Every GPU term runs on this
// library's kernels through the C ABI (phix_lap_accumulate, ...), whose
// arithmetic matches the reference's kernels (Equation.cu:40-124, :386-404).
// The CPU launchers follow the reference's host loops (plain a*b+c, no
// contraction, like an x86 host build).
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>

#include "boundary/BoundaryCondition.h"
#include "equation/Equation.h"
#include "equation/Term.h"
#include "equation/VectorEquation.h"
#include "phix_b200.h"

namespace phix {
void count_launch(int n);
}

namespace PhiX {

namespace {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

// C-ABI status -> the reference's exception types.
void check_rc(int rc, const char* what) {
    if (rc == PHIX_OK) return;
    const std::string msg = std::string(what) + ": " + phix_last_error();
    if (rc == PHIX_ERR_ARG) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// The C-ABI grid of a field's layout (no BCs: the ops read stored ghosts).
phix_grid_t grid_of(const ScalarField& f) {
    phix_grid_t g{};
    g.dim = f.mesh.dim;
    for (int a = 0; a < 3; ++a) {
        g.n[a] = f.mesh.n[a];
        g.d[a] = a < f.mesh.dim ? f.mesh.d[a] : 1.0;
    }
    g.ghost = f.ghost;
    return g;
}

struct HostGeom {
    int nx, ny, nz, sx, sy, g, dim;
    double i2[3];
    double d[3];
};
HostGeom host_geom(const ScalarField& f) {
    HostGeom h{f.mesh.n[0], f.mesh.n[1], f.mesh.n[2], f.storedDims[0], f.storedDims[1], f.ghost, f.mesh.dim, {}, {}};
    for (int a = 0; a < 3; ++a) {
        h.i2[a] = a < f.mesh.dim ? 1.0 / (f.mesh.d[a] * f.mesh.d[a]) : 0.0;
        h.d[a] = f.mesh.d[a];
    }
    return h;
}

// rhs += c * lap(src) on physical cells, host (reference host loop order).
void lap_host(double* rhs, const double* src, double c, const HostGeom& G) {
    const long sxy = (long)G.sx * G.sy;
    for (int k = 0; k < G.nz; ++k)
        for (int j = 0; j < G.ny; ++j)
            for (int i = 0; i < G.nx; ++i) {
                const long ctr = (i + G.g) + G.sx * ((long)(j + G.g) + (long)G.sy * (k + G.g));
                volatile double two_c = 2.0 * src[ctr];
                double v = (src[ctr + 1] - two_c + src[ctr - 1]) * G.i2[0];
                if (G.dim >= 2) v += (src[ctr + G.sx] - two_c + src[ctr - G.sx]) * G.i2[1];
                if (G.dim >= 3) v += (src[ctr + sxy] - two_c + src[ctr - sxy]) * G.i2[2];
                volatile double cv = c * v;
                rhs[ctr] += cv;
            }
}

void grad_host(double* rhs, const double* src, double c, int axis, const HostGeom& G) {
    const long off = axis == 0 ? 1 : axis == 1 ? G.sx : (long)G.sx * G.sy;
    const double inv_2d = 0.5 / G.d[axis];
    for (int k = 0; k < G.nz; ++k)
        for (int j = 0; j < G.ny; ++j)
            for (int i = 0; i < G.nx; ++i) {
                const long ctr = (i + G.g) + G.sx * ((long)(j + G.g) + (long)G.sy * (k + G.g));
                volatile double cd = c * (src[ctr + off] - src[ctr - off]);
                volatile double t = cd * inv_2d;
                rhs[ctr] += t;
            }
}

void mul_host(double* rhs, const double* s1, const double* s2, double c, const HostGeom& G) {
    for (int k = 0; k < G.nz; ++k)
        for (int j = 0; j < G.ny; ++j)
            for (int i = 0; i < G.nx; ++i) {
                const long idx = (i + G.g) + G.sx * ((long)(j + G.g) + (long)G.sy * (k + G.g));
                volatile double a = c * s1[idx];
                volatile double b = a * s2[idx];
                rhs[idx] += b;
            }
}

// Term applying a stencil `op` to the materialised `src` (lap(expr, bcs) /
// grad(expr, axis, bcs)): scratch = 0; scratch += src terms; BCs on the
// scratch; rhs += c * op(scratch)  (makeStencilOnExprTerm, Equation.cu:537-594).
template <typename SrcExpr>
Term stencil_on_expr(const SrcExpr& src, const ScalarField& layout, const std::vector<BoundaryCondition*>& bcs,
                     bool is_lap, int axis, double coeff) {
    Term out;
    out.type = TermType::COMPOSITE;
    out.axis = axis;
    out.coeff = coeff;
    out.field = &layout;
    const Mesh* pmesh = &layout.mesh;
    const int ghost = layout.ghost;
    const std::size_t S = layout.storedSize;
    const phix_grid_t grid = grid_of(layout);
    const HostGeom G = host_geom(layout);
    out.gpu_launcher = [src, pmesh, ghost, S, bcs, grid, is_lap, axis](double* d_rhs, double c, ScratchPool& pool) {
        double* d_scratch = pool.acquireDevice(S);
        detail::materialiseGPU(src, d_scratch, S, pool);
        ScalarField shell = ScalarField::makeShell(*pmesh, ghost, d_scratch);
        for (auto* bc : bcs) bc->applyOnGPU(shell);
        if (is_lap) check_rc(phix_lap_accumulate(d_rhs, d_scratch, c, &grid, nullptr), "lap(expr)");
        else check_rc(phix_grad_accumulate(d_rhs, d_scratch, c, axis, &grid, nullptr), "grad(expr)");
    };
    out.cpu_kernel = [src, pmesh, ghost, S, bcs, G, is_lap, axis](double* rhs, double c, ScratchPool& pool) {
        double* h_scratch = pool.acquireHost(S);
        detail::materialiseCPU(src, h_scratch, S, pool);
        ScalarField tmp(*pmesh, "shell_cpu", ghost);
        std::copy(h_scratch, h_scratch + S, tmp.curr.begin());
        for (auto* bc : bcs) bc->applyOnCPU(tmp);
        std::copy(tmp.curr.begin(), tmp.curr.end(), h_scratch);
        if (is_lap) lap_host(rhs, h_scratch, c, G);
        else grad_host(rhs, h_scratch, c, axis, G);
    };
    if (is_lap) {
        auto info = std::make_shared<fuse::Info>();
        info->kind = fuse::Info::LAP_EXPR;
        info->inner = std::make_shared<RHSExpr>(src);
        info->bcs = bcs;
        out.fusion = info;
    }
    return out;
}

}  // namespace

// ---------------------------------------------------------------------------
// detail helpers used by the inline headers
// ---------------------------------------------------------------------------
namespace detail {

void count_user_launch() { phix::count_launch(1); }

void throw_cuda(cudaError_t e, const char* what) {
    throw std::runtime_error(std::string(what) + " error: " + cudaGetErrorString(e));
}

const ScalarField* repField(const Term& t) {
    if (!t.field) throw std::runtime_error("Composite Term: no representative source field captured");
    return t.field;
}
const ScalarField* repField(const RHSExpr& e) {
    for (const auto& t : e.terms)
        if (t.field) return t.field;
    throw std::runtime_error("Composite RHSExpr: no representative source field captured");
}

void materialiseGPU(const RHSExpr& e, double* d_buf, std::size_t S, ScratchPool& pool) {
    cuda_check(cudaMemset(d_buf, 0, S * sizeof(double)), "materialise");
    for (const auto& t : e.terms) {
        if (!t.gpu_launcher) throw std::runtime_error("Composite GPU: a Term has no GPU launcher");
        t.gpu_launcher(d_buf, t.coeff, pool);
    }
}
void materialiseGPU(const Term& t, double* d_buf, std::size_t S, ScratchPool& pool) {
    cuda_check(cudaMemset(d_buf, 0, S * sizeof(double)), "materialise");
    if (!t.gpu_launcher) throw std::runtime_error("Composite GPU: Term has no GPU launcher");
    t.gpu_launcher(d_buf, t.coeff, pool);
}
void materialiseCPU(const RHSExpr& e, double* h_buf, std::size_t S, ScratchPool& pool) {
    std::fill(h_buf, h_buf + S, 0.0);
    for (const auto& t : e.terms) {
        if (!t.cpu_kernel) throw std::runtime_error("Composite CPU: a Term has no CPU kernel");
        t.cpu_kernel(h_buf, t.coeff, pool);
    }
}
void materialiseCPU(const Term& t, double* h_buf, std::size_t S, ScratchPool& pool) {
    std::fill(h_buf, h_buf + S, 0.0);
    if (!t.cpu_kernel) throw std::runtime_error("Composite CPU: Term has no CPU kernel");
    t.cpu_kernel(h_buf, t.coeff, pool);
}

// rhs += c * materialise(lhs) * field  (FieldOps.inl termTimesField)
Term timesField(const RHSExpr& lhs, const ScalarField& f, const ScalarField& layout) {
    Term out;
    out.type = TermType::COMPOSITE;
    out.coeff = 1.0;
    out.field = &layout;
    const std::size_t S = layout.storedSize;
    const phix_grid_t grid = grid_of(layout);
    const HostGeom G = host_geom(layout);
    const ScalarField* pf = &f;
    out.gpu_launcher = [lhs, pf, S, grid](double* d_rhs, double c, ScratchPool& pool) {
        double* s = pool.acquireDevice(S);
        materialiseGPU(lhs, s, S, pool);
        if (!pf->d_curr) throw std::runtime_error("Term*Field GPU: field not on device");
        check_rc(phix_mul_accumulate(d_rhs, s, pf->d_curr, c, &grid, nullptr), "Term*Field");
    };
    out.cpu_kernel = [lhs, pf, S, G](double* rhs, double c, ScratchPool& pool) {
        double* s = pool.acquireHost(S);
        materialiseCPU(lhs, s, S, pool);
        mul_host(rhs, s, pf->curr.data(), c, G);
    };
    auto info = std::make_shared<fuse::Info>();
    info->kind = fuse::Info::TIMES_FIELD;
    info->inner = std::make_shared<RHSExpr>(lhs);
    info->field = pf;
    out.fusion = info;
    return out;
}

// rhs += c * materialise(a) * materialise(b)  (FieldOps.inl termTimesTerm)
Term timesExpr(const RHSExpr& a, const RHSExpr& b, const ScalarField& layout) {
    Term out;
    out.type = TermType::COMPOSITE;
    out.coeff = 1.0;
    out.field = &layout;
    const std::size_t S = layout.storedSize;
    const phix_grid_t grid = grid_of(layout);
    const HostGeom G = host_geom(layout);
    out.gpu_launcher = [a, b, S, grid](double* d_rhs, double c, ScratchPool& pool) {
        double* s1 = pool.acquireDevice(S);
        materialiseGPU(a, s1, S, pool);
        double* s2 = pool.acquireDevice(S);
        materialiseGPU(b, s2, S, pool);
        check_rc(phix_mul_accumulate(d_rhs, s1, s2, c, &grid, nullptr), "Term*Term");
    };
    out.cpu_kernel = [a, b, S, G](double* rhs, double c, ScratchPool& pool) {
        double* s1 = pool.acquireHost(S);
        materialiseCPU(a, s1, S, pool);
        double* s2 = pool.acquireHost(S);
        materialiseCPU(b, s2, S, pool);
        mul_host(rhs, s1, s2, c, G);
    };
    auto info = std::make_shared<fuse::Info>();
    info->kind = fuse::Info::TIMES_EXPR;
    info->inner = std::make_shared<RHSExpr>(a);
    info->inner2 = std::make_shared<RHSExpr>(b);
    out.fusion = info;
    return out;
}

}  // namespace detail

// ---------------------------------------------------------------------------
// ScratchPool (Term.h:45-65 semantics: bump allocator, grows, reset per RHS)
// ---------------------------------------------------------------------------
ScratchPool::~ScratchPool() {
    for (double* p : dev_bufs_)
        if (p) cudaFree(p);
}

double* ScratchPool::acquireDevice(std::size_t size) {
    if (next_dev_ < dev_bufs_.size()) {
        if (dev_sizes_[next_dev_] < size) {
            cudaFree(dev_bufs_[next_dev_]);
            dev_bufs_[next_dev_] = nullptr;
            cuda_check(cudaMalloc(&dev_bufs_[next_dev_], size * sizeof(double)), "ScratchPool");
            dev_sizes_[next_dev_] = size;
        }
        return dev_bufs_[next_dev_++];
    }
    double* p = nullptr;
    cuda_check(cudaMalloc(&p, size * sizeof(double)), "ScratchPool");
    dev_bufs_.push_back(p);
    dev_sizes_.push_back(size);
    ++next_dev_;
    return p;
}

double* ScratchPool::acquireHost(std::size_t size) {
    if (next_host_ < host_bufs_.size()) {
        if (host_bufs_[next_host_].size() < size) host_bufs_[next_host_].assign(size, 0.0);
        return host_bufs_[next_host_++].data();
    }
    host_bufs_.emplace_back(size, 0.0);
    ++next_host_;
    return host_bufs_.back().data();
}

// ---------------------------------------------------------------------------
// Term factories
// ---------------------------------------------------------------------------
Term lap(const ScalarField& f, double coeff) {
    Term t;
    t.type = TermType::LAPLACIAN;
    t.field = &f;
    t.coeff = coeff;
    const ScalarField* pf = &f;  // d_curr is read at launch (the RK4 pointer swap relies on it)
    const phix_grid_t grid = grid_of(f);
    const HostGeom G = host_geom(f);
    t.gpu_launcher = [pf, grid](double* d_rhs, double c, ScratchPool&) {
        if (!pf->d_curr) throw std::runtime_error("lap GPU: source field not on device");
        check_rc(phix_lap_accumulate(d_rhs, pf->d_curr, c, &grid, nullptr), "lap GPU kernel");
    };
    t.cpu_kernel = [pf, G](double* rhs, double c, ScratchPool&) { lap_host(rhs, pf->curr.data(), c, G); };
    auto info = std::make_shared<fuse::Info>();
    info->kind = fuse::Info::LAP;
    info->field = pf;
    t.fusion = info;
    return t;
}

Term grad(const ScalarField& f, int axis, double coeff) {
    if (axis < 0 || axis >= f.mesh.dim) throw std::invalid_argument("grad: axis out of range for this mesh dimension");
    Term t;
    t.type = TermType::GRADIENT;
    t.field = &f;
    t.coeff = coeff;
    t.axis = axis;
    const ScalarField* pf = &f;
    const phix_grid_t grid = grid_of(f);
    const HostGeom G = host_geom(f);
    t.gpu_launcher = [pf, grid, axis](double* d_rhs, double c, ScratchPool&) {
        if (!pf->d_curr) throw std::runtime_error("grad GPU: source field not on device");
        check_rc(phix_grad_accumulate(d_rhs, pf->d_curr, c, axis, &grid, nullptr), "grad GPU kernel");
    };
    t.cpu_kernel = [pf, G, axis](double* rhs, double c, ScratchPool&) { grad_host(rhs, pf->curr.data(), c, axis, G); };
    auto info = std::make_shared<fuse::Info>();
    info->kind = fuse::Info::GRAD;
    info->field = pf;
    info->axis = axis;
    t.fusion = info;
    return t;
}

Term lap(const Term& t, const std::vector<BoundaryCondition*>& bcs, double coeff) {
    return stencil_on_expr(RHSExpr(t), *detail::repField(t), bcs, true, 0, coeff);
}
Term lap(const RHSExpr& e, const std::vector<BoundaryCondition*>& bcs, double coeff) {
    return stencil_on_expr(e, *detail::repField(e), bcs, true, 0, coeff);
}
Term grad(const Term& t, int axis, const std::vector<BoundaryCondition*>& bcs, double coeff) {
    const ScalarField& L = *detail::repField(t);
    if (axis < 0 || axis >= L.mesh.dim) throw std::invalid_argument("grad(expr): axis out of range");
    return stencil_on_expr(t, L, bcs, false, axis, coeff);
}
Term grad(const RHSExpr& e, int axis, const std::vector<BoundaryCondition*>& bcs, double coeff) {
    const ScalarField& L = *detail::repField(e);
    if (axis < 0 || axis >= L.mesh.dim) throw std::invalid_argument("grad(expr): axis out of range");
    return stencil_on_expr(e, L, bcs, false, axis, coeff);
}

VectorRHSExpr grad(const Term& t, const std::vector<BoundaryCondition*>& bcs, double coeff) {
    const int dim = detail::repField(t)->mesh.dim;
    VectorRHSExpr v(dim);
    for (int a = 0; a < dim; ++a) v[a] = RHSExpr(grad(t, a, bcs, coeff));
    return v;
}
VectorRHSExpr grad(const RHSExpr& e, const std::vector<BoundaryCondition*>& bcs, double coeff) {
    const int dim = detail::repField(e)->mesh.dim;
    VectorRHSExpr v(dim);
    for (int a = 0; a < dim; ++a) v[a] = RHSExpr(grad(e, a, bcs, coeff));
    return v;
}

VectorRHSExpr lap(const VectorField& vf, double coeff) {
    VectorRHSExpr v(vf.nComponents());
    for (int c = 0; c < vf.nComponents(); ++c) v[c] = RHSExpr(lap(vf[c], coeff));
    return v;
}
VectorRHSExpr grad(const ScalarField& f, double coeff) {
    VectorRHSExpr v(f.mesh.dim);
    for (int a = 0; a < f.mesh.dim; ++a) v[a] = RHSExpr(grad(f, a, coeff));
    return v;
}
RHSExpr div(const VectorField& vf, double coeff) {
    if (vf.nComponents() < vf.mesh.dim) throw std::invalid_argument("div: VectorField must have at least mesh.dim components");
    RHSExpr e;
    for (int a = 0; a < vf.mesh.dim; ++a) e += grad(vf[a], a, coeff);
    return e;
}
RHSExpr div(const VectorRHSExpr& v, const std::vector<BoundaryCondition*>& bcs, double coeff) {
    RHSExpr e;
    for (int a = 0; a < v.nComponents(); ++a) e += grad(v[a], a, bcs, coeff);
    return e;
}
VectorRHSExpr curl(const VectorField& vf, double coeff) {
    if (vf.mesh.dim != 3 || vf.nComponents() != 3)
        throw std::invalid_argument("curl: VectorField must be 3-component on a 3D mesh");
    VectorRHSExpr e(3);
    e[0] += grad(vf[2], 1, coeff);
    e[0] += grad(vf[1], 2, -coeff);
    e[1] += grad(vf[0], 2, coeff);
    e[1] += grad(vf[2], 0, -coeff);
    e[2] += grad(vf[1], 0, coeff);
    e[2] += grad(vf[0], 1, -coeff);
    return e;
}

// ---------------------------------------------------------------------------
// Equation
// ---------------------------------------------------------------------------
Equation::Equation(ScalarField& u, const std::string& n) : name(n), unknown(u) {}

void Equation::setRHS(const RHSExpr& expr) { rhs_expr_ = expr; }
void Equation::setRHS(const Term& t) { rhs_expr_ = RHSExpr(t); }

void Equation::computeRHS(ScalarField& rhs) const {
    if (!rhs.deviceAllocated()) throw std::runtime_error("Equation::computeRHS: rhs device memory not allocated");
    if (rhs_expr_.terms.empty()) throw std::runtime_error("Equation::computeRHS: RHS not set (call setRHS first)");
    cuda_check(cudaMemset(rhs.d_curr, 0, rhs.storedSize * sizeof(double)), "Equation::computeRHS");
    scratch_pool_.reset();
    for (const auto& t : rhs_expr_.terms) {
        if (!t.gpu_launcher) throw std::runtime_error("Equation::computeRHS: a Term has no GPU launcher");
        t.gpu_launcher(rhs.d_curr, t.coeff, scratch_pool_);
    }
    cuda_check(cudaDeviceSynchronize(), "Equation::computeRHS");
}

void Equation::computeRHSCPU(ScalarField& rhs) const {
    if (rhs_expr_.terms.empty()) throw std::runtime_error("Equation::computeRHSCPU: RHS not set");
    std::fill(rhs.curr.begin(), rhs.curr.end(), 0.0);
    scratch_pool_.reset();
    for (const auto& t : rhs_expr_.terms) {
        if (!t.cpu_kernel) throw std::runtime_error("Equation::computeRHSCPU: a Term has no CPU kernel.");
        t.cpu_kernel(rhs.curr.data(), t.coeff, scratch_pool_);
    }
}

// ---------------------------------------------------------------------------
// VectorEquation (VectorEquation.cu:15-60 semantics)
// ---------------------------------------------------------------------------
VectorEquation::VectorEquation(VectorField& u, const std::string& n) : name(n), unknown(u) {
    for (int c = 0; c < u.nComponents(); ++c)
        equations_.push_back(std::make_unique<Equation>(u[c], n + "_" + std::to_string(c)));
}

void VectorEquation::setRHS(const VectorRHSExpr& expr) {
    if (expr.nComponents() != unknown.nComponents())
        throw std::invalid_argument("VectorEquation::setRHS: component count mismatch");
    for (int c = 0; c < expr.nComponents(); ++c) equations_[c]->setRHS(expr[c]);
}

void VectorEquation::computeRHS(VectorField& rhs) const {
    for (int c = 0; c < unknown.nComponents(); ++c) equations_[c]->computeRHS(rhs[c]);
}
void VectorEquation::computeRHSCPU(VectorField& rhs) const {
    for (int c = 0; c < unknown.nComponents(); ++c) equations_[c]->computeRHSCPU(rhs[c]);
}

Equation& VectorEquation::componentEquation(int c) {
    if (c < 0 || c >= (int)equations_.size()) throw std::out_of_range("VectorEquation: component index out of range");
    return *equations_[c];
}
const Equation& VectorEquation::componentEquation(int c) const {
    if (c < 0 || c >= (int)equations_.size()) throw std::out_of_range("VectorEquation: component index out of range");
    return *equations_[c];
}
bool VectorEquation::hasRHS() const {
    for (const auto& e : equations_)
        if (!e->hasRHS()) return false;
    return !equations_.empty();
}

}  // namespace PhiX
