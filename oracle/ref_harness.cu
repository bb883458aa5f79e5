// ref_harness.cu -- drives the UNMODIFIED reference library through its own
// public C++ API and exposes the runs as extern "C" functions for the tests.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's own sources (src/mesh, src/field, src/boundary,
// src/equation, src/solver, src/IO/FieldIO.cpp) into oracle/_ref/libphix_ref.so.
// Nothing of the reference is copied; the sources are compiled where they lie.
//
// Two paths per case:
//   use_gpu = 1 : the reference's own Solver / VectorSolver GPU path
//                 (Solver::advance, Solver.cu:366-382; VectorSolver::advance).
//   use_gpu = 0 : the reference's CPU kernels (Equation::computeRHSCPU,
//                 BoundaryCondition::applyOnCPU) driven by a host loop that
//                 follows the GPU solver's stage semantics (Solver.cu:193-259,
//                 VectorSolver.cu:149-228).  The reference's own
//                 Solver::advanceCPU cannot be used without a GPU (its
//                 constructor allocates device scratch, Solver.cu:76-80) and
//                 its scalar RK4 applies BCs to the wrong array
//                 (Solver.cu:280-300).
// Fields are passed as ghost-padded stored arrays (ScalarField layout,
// ScalarField.h:15-27).  Returns 0 on success, a negative code on error.

#include "mesh/Mesh.h"
#include "field/ScalarField.h"
#include "field/VectorField.h"
#include "boundary/PeriodicBC.h"
#include "boundary/NoFluxBC.h"
#include "boundary/FixedBC.h"
#include "equation/Equation.h"
#include "equation/Term.h"
#include "equation/VectorEquation.h"
#include "solver/Solver.h"
#include "solver/VectorSolver.h"

#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

using namespace PhiX;

extern "C" {
typedef struct {
    int32_t dim;
    int32_t n[3];
    int32_t ghost;
    int32_t bc_type[6];
    int32_t fma_mode;  // unused here; keeps the oracle's struct layout
    double d[3];
    double bc_val[6];
} ref_grid_t;
}

namespace {

enum { BC_NONE = 0, BC_PERIODIC = 1, BC_NOFLUX = 2, BC_FIXED = 3 };
enum { PHYS_AC = 0, PHYS_CH = 1, PHYS_CHAC = 2 };

struct Setup {
    Mesh mesh;
    std::vector<std::unique_ptr<BoundaryCondition>> own;
    std::vector<BoundaryCondition*> bcs;
};

std::unique_ptr<Setup> makeSetup(const ref_grid_t* g) {
    auto s = std::make_unique<Setup>();
    if (g->dim == 1) s->mesh = Mesh::makeUniform1D(CoordSys::CARTESIAN, g->n[0], g->d[0], 0.0);
    else if (g->dim == 2)
        s->mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, g->n[0], g->d[0], 0.0, g->n[1], g->d[1], 0.0);
    else
        s->mesh = Mesh::makeUniform3D(CoordSys::CARTESIAN, g->n[0], g->d[0], 0.0, g->n[1], g->d[1], 0.0,
                                      g->n[2], g->d[2], 0.0);
    // Same ordering as buildBCs (BCFactory.cpp:50-74).
    for (int ax = 0; ax < g->dim; ++ax) {
        Axis a = static_cast<Axis>(ax);
        int tl = g->bc_type[2 * ax], th = g->bc_type[2 * ax + 1];
        if (tl == BC_PERIODIC && th == BC_PERIODIC) {
            s->own.push_back(std::make_unique<PeriodicBC>(a));
        } else {
            if (tl == BC_NOFLUX) s->own.push_back(std::make_unique<NoFluxBC>(a, Side::LOW));
            if (tl == BC_FIXED) s->own.push_back(std::make_unique<FixedBC>(a, Side::LOW, g->bc_val[2 * ax]));
            if (th == BC_NOFLUX) s->own.push_back(std::make_unique<NoFluxBC>(a, Side::HIGH));
            if (th == BC_FIXED) s->own.push_back(std::make_unique<FixedBC>(a, Side::HIGH, g->bc_val[2 * ax + 1]));
        }
    }
    for (auto& b : s->own) s->bcs.push_back(b.get());
    return s;
}

void setRHS_AC(Equation& eq, ScalarField& phi, const double* prm) {
    const double L = prm[0], kap = prm[1];
    // tutorials/quickstart/main.cu:64-67 with the mobility split into L and kappa.
    eq.setRHS(L * kap * lap(phi) + L * pw(phi, [] __host__ __device__(double p) { return p - p * p * p; }));
}

void setRHS_CH(Equation& eq, ScalarField& c, const double* prm, const std::vector<BoundaryCondition*>& bcs) {
    const double M = prm[0], kappa = prm[1], rho = prm[2], ca = prm[3], cb = prm[4];
    // Single-equation (RK4-capable) Cahn-Hilliard: M*lap(f'(c) - kappa*lap(c), bcs).
    eq.setRHS(M * lap(pw(c, PHIX_FN(double cv) { return 2.0 * rho * (cv - ca) * (cv - cb) * (2.0 * cv - ca - cb); }) -
                          kappa * lap(c),
                      bcs));
}

void setRHS_CHAC(VectorEquation& veq, VectorField& u, const double* prm,
                 const std::vector<BoundaryCondition*>& bcs) {
    const double M = prm[0], L = prm[1], kc = prm[2], ke = prm[3], lam = prm[4];
    ScalarField& c = u[0];
    ScalarField& e = u[1];
    // f = c^2(1-c)^2 + e^2(1-e)^2 + lam c^2 e^2; explicit fma so host and
    // device builds of the functor round identically.
    auto fc = PHIX_FN(double cv, double ev) {
        double a = 2.0 * cv * (1.0 - cv) * (1.0 - 2.0 * cv);
        double b = 2.0 * lam * cv * ev;
        return fma(b, ev, a);
    };
    auto fe = PHIX_FN(double ev, double cv) {
        double a = 2.0 * ev * (1.0 - ev) * (1.0 - 2.0 * ev);
        double b = 2.0 * lam * cv * cv;
        return fma(b, ev, a);
    };
    VectorRHSExpr ex(2);
    ex[0] = RHSExpr(M * lap(pw(c, e, fc) - kc * lap(c), bcs));
    ex[1] = (-L) * pw(e, c, fe) + (L * ke) * lap(e);
    veq.setRHS(ex);
}

void loadStored(ScalarField& f, const double* src) { std::memcpy(f.curr.data(), src, f.storedSize * sizeof(double)); }
void saveStored(const ScalarField& f, double* dst) { std::memcpy(dst, f.curr.data(), f.storedSize * sizeof(double)); }

void applyCPU(const std::vector<BoundaryCondition*>& bcs, ScalarField& f) {
    for (auto* b : bcs) b->applyOnCPU(f);
}

// Host loop with the GPU solver's semantics for one scalar equation.
void cpuAdvanceScalar(Equation& eq, ScalarField& phi, const std::vector<BoundaryCondition*>& bcs, int scheme,
                      double dt, int nsteps) {
    const Mesh& m = phi.mesh;
    ScalarField k1(m, "k1", phi.ghost), k2(m, "k2", phi.ghost), k3(m, "k3", phi.ghost), k4(m, "k4", phi.ghost);
    ScalarField tmp(m, "tmp", phi.ghost);
    const std::size_t S = phi.storedSize;
    const double dt2 = dt * 0.5, dt6 = dt / 6.0;
    for (int s = 0; s < nsteps; ++s) {
        applyCPU(bcs, phi);
        eq.computeRHSCPU(k1);
        if (scheme == 0) {
            for (std::size_t i = 0; i < S; ++i) phi.curr[i] += dt * k1.curr[i];
            continue;
        }
        ScalarField* ks[3] = {&k1, &k2, &k3};
        ScalarField* kn[3] = {&k2, &k3, &k4};
        double as[3] = {dt2, dt2, dt};
        for (int st = 0; st < 3; ++st) {
            for (std::size_t i = 0; i < S; ++i) tmp.curr[i] = phi.curr[i] + as[st] * ks[st]->curr[i];
            applyCPU(bcs, tmp);
            std::swap(phi.curr, tmp.curr);
            eq.computeRHSCPU(*kn[st]);
            std::swap(phi.curr, tmp.curr);
        }
        for (std::size_t i = 0; i < S; ++i)
            phi.curr[i] += dt6 * (k1.curr[i] + 2.0 * k2.curr[i] + 2.0 * k3.curr[i] + k4.curr[i]);
    }
}

// Host loop with VectorSolver's GPU semantics (all components swapped together).
void cpuAdvanceVector(VectorEquation& veq, VectorField& u, const std::vector<BoundaryCondition*>& bcs, int scheme,
                      double dt, int nsteps) {
    const Mesh& m = u.mesh;
    const int N = u.nComponents();
    VectorField k1(m, "k1", N, u.ghost), k2(m, "k2", N, u.ghost), k3(m, "k3", N, u.ghost), k4(m, "k4", N, u.ghost);
    VectorField tmp(m, "tmp", N, u.ghost);
    const std::size_t S = u[0].storedSize;
    const double dt2 = dt * 0.5, dt6 = dt / 6.0;
    for (int s = 0; s < nsteps; ++s) {
        for (int c = 0; c < N; ++c) applyCPU(bcs, u[c]);
        veq.computeRHSCPU(k1);
        if (scheme == 0) {
            for (int c = 0; c < N; ++c)
                for (std::size_t i = 0; i < S; ++i) u[c].curr[i] += dt * k1[c].curr[i];
            continue;
        }
        VectorField* ks[3] = {&k1, &k2, &k3};
        VectorField* kn[3] = {&k2, &k3, &k4};
        double as[3] = {dt2, dt2, dt};
        for (int st = 0; st < 3; ++st) {
            for (int c = 0; c < N; ++c)
                for (std::size_t i = 0; i < S; ++i) tmp[c].curr[i] = u[c].curr[i] + as[st] * (*ks[st])[c].curr[i];
            for (int c = 0; c < N; ++c) std::swap(u[c].curr, tmp[c].curr);
            for (int c = 0; c < N; ++c) applyCPU(bcs, u[c]);
            veq.computeRHSCPU(*kn[st]);
            for (int c = 0; c < N; ++c) std::swap(u[c].curr, tmp[c].curr);
        }
        for (int c = 0; c < N; ++c)
            for (std::size_t i = 0; i < S; ++i)
                u[c].curr[i] += dt6 * (k1[c].curr[i] + 2.0 * k2[c].curr[i] + 2.0 * k3[c].curr[i] + k4[c].curr[i]);
    }
}

}  // namespace

extern "C" {

int ref_abi_version(void) { return 1; }

int ref_has_gpu(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n > 0;
}

// Advance `nsteps` time steps of one physics (0 AC, 1 CH single-equation,
// 2 coupled CH+AC) with scheme 0 Euler / 1 RK4.  `fields` holds 1 (AC, CH) or
// 2 (c, eta) stored arrays, updated in place.  `elapsed_ms` (may be null)
// receives the wall time of the step loop only; on the GPU path it is bracketed
// by cudaDeviceSynchronize.
int ref_advance(int phys, int scheme, const double* prm, double dt, int nsteps, const ref_grid_t* g,
                double** fields, int use_gpu, double* elapsed_ms) {
    try {
        auto s = makeSetup(g);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (phys == PHYS_AC || phys == PHYS_CH) {
            ScalarField u(s->mesh, "u", g->ghost);
            loadStored(u, fields[0]);
            Equation eq(u, "eq");
            if (phys == PHYS_AC) setRHS_AC(eq, u, prm);
            else setRHS_CH(eq, u, prm, s->bcs);
            if (use_gpu) {
                u.allocDevice();
                u.uploadAllToDevice();
                Solver solver(eq, s->bcs, dt, scheme ? TimeScheme::RK4 : TimeScheme::EULER);
                cudaDeviceSynchronize();
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                cudaEventRecord(e0);
                for (int i = 0; i < nsteps; ++i) solver.advance();
                cudaEventRecord(e1);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (elapsed_ms) *elapsed_ms = ms;
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                u.downloadCurrFromDevice();
            } else {
                cpuAdvanceScalar(eq, u, s->bcs, scheme, dt, nsteps);
            }
            saveStored(u, fields[0]);
        } else if (phys == PHYS_CHAC) {
            VectorField u(s->mesh, "u", 2, g->ghost);
            loadStored(u[0], fields[0]);
            loadStored(u[1], fields[1]);
            VectorEquation veq(u, "chac");
            setRHS_CHAC(veq, u, prm, s->bcs);
            if (use_gpu) {
                for (int c = 0; c < 2; ++c) {
                    u[c].allocDevice();
                    u[c].uploadAllToDevice();
                }
                VectorSolver solver(veq, s->bcs, dt, scheme ? TimeScheme::RK4 : TimeScheme::EULER);
                cudaDeviceSynchronize();
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                cudaEventRecord(e0);
                for (int i = 0; i < nsteps; ++i) solver.advance();
                cudaEventRecord(e1);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (elapsed_ms) *elapsed_ms = ms;
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                for (int c = 0; c < 2; ++c) u[c].downloadCurrFromDevice();
            } else {
                cpuAdvanceVector(veq, u, s->bcs, scheme, dt, nsteps);
            }
            saveStored(u[0], fields[0]);
            saveStored(u[1], fields[1]);
        } else {
            return -2;
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_advance: %s\n", e.what());
        return -1;
    }
}

// The shipped Cahn-Hilliard app's multi-step Euler form
// (Cahn-Hillard_double-well.cu:84-106): STEADY mu then TRANSIENT c.
int ref_advance_ch_multistep(const double* prm, double dt, int nsteps, const ref_grid_t* g, double* c_stored,
                             double* mu_stored, int use_gpu) {
    try {
        auto s = makeSetup(g);
        const double M = prm[0], kappa = prm[1], rho = prm[2], ca = prm[3], cb = prm[4];
        ScalarField c(s->mesh, "c", g->ghost), mu(s->mesh, "mu", g->ghost);
        loadStored(c, c_stored);
        loadStored(mu, mu_stored);
        Equation eqMu(mu, "CH_mu");
        eqMu.setRHS(pw(c, PHIX_FN(double cv) { return 2.0 * rho * (cv - ca) * (cv - cb) * (2.0 * cv - ca - cb); }) -
                    kappa * lap(c));
        Equation eqC(c, "CH_c");
        eqC.setRHS(M * lap(mu));
        if (use_gpu) {
            c.allocDevice();
            c.uploadAllToDevice();
            mu.allocDevice();
            mu.uploadAllToDevice();
            Solver solver({{&c, s->bcs, &eqMu, EquationType::STEADY}, {&mu, s->bcs, &eqC, EquationType::TRANSIENT}},
                          dt, TimeScheme::EULER);
            for (int i = 0; i < nsteps; ++i) solver.advance();
            c.downloadCurrFromDevice();
            mu.downloadCurrFromDevice();
        } else {
            ScalarField rhs(s->mesh, "rhs", g->ghost);
            for (int i = 0; i < nsteps; ++i) {
                applyCPU(s->bcs, c);
                eqMu.computeRHSCPU(mu);
                applyCPU(s->bcs, mu);
                eqC.computeRHSCPU(rhs);
                for (std::size_t q = 0; q < c.storedSize; ++q) c.curr[q] += dt * rhs.curr[q];
            }
        }
        saveStored(c, c_stored);
        saveStored(mu, mu_stored);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_advance_ch_multistep: %s\n", e.what());
        return -1;
    }
}

// One ghost refresh with the reference BC classes (applyOnCPU / applyOnGPU).
int ref_bc_apply(double* stored, const ref_grid_t* g, int use_gpu) {
    try {
        auto s = makeSetup(g);
        ScalarField f(s->mesh, "f", g->ghost);
        loadStored(f, stored);
        if (use_gpu) {
            f.allocDevice();
            f.uploadCurrToDevice();
            for (auto* b : s->bcs) b->applyOnGPU(f);
            cudaDeviceSynchronize();
            f.downloadCurrFromDevice();
        } else {
            applyCPU(s->bcs, f);
        }
        saveStored(f, stored);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_bc_apply: %s\n", e.what());
        return -1;
    }
}

// rhs = coeff * lap(src), through Equation::computeRHS / computeRHSCPU.
int ref_lap(double* rhs_stored, const double* src_stored, double coeff, const ref_grid_t* g, int use_gpu) {
    try {
        auto s = makeSetup(g);
        ScalarField src(s->mesh, "src", g->ghost), rhs(s->mesh, "rhs", g->ghost);
        loadStored(src, src_stored);
        Equation eq(src, "lap");
        eq.setRHS(coeff * lap(src));
        if (use_gpu) {
            src.allocDevice();
            src.uploadCurrToDevice();
            rhs.allocDevice();
            eq.computeRHS(rhs);
            rhs.downloadCurrFromDevice();
        } else {
            eq.computeRHSCPU(rhs);
        }
        saveStored(rhs, rhs_stored);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_lap: %s\n", e.what());
        return -1;
    }
}

}  // extern "C"
