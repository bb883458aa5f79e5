// api_checks.cu -- GPU checks of the drop-in C++ API (include/phix): for each
// case the fused Solver path and the unfused path (Solver::disableFusion: the
// reference's sequence of one kernel per term and BC on this library's
// kernels) advance the same fields, and the physical cells must agree bit for
// bit.  The last cases check the asynchronous OutputWriter against the
// synchronous IO::writeField, byte for byte, and time both.  Prints one
// PASS/FAIL line per case; exit code 0 when all pass.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <iterator>
#include <random>
#include <string>
#include <vector>

#include "boundary/FixedBC.h"
#include "boundary/NoFluxBC.h"
#include "boundary/PeriodicBC.h"
#include "IO/FieldIO.h"
#include "IO/OutputWriter.h"
#include "equation/Equation.h"
#include "equation/VectorEquation.h"
#include "field/ScalarField.h"
#include "field/VectorField.h"
#include "mesh/Mesh.h"
#include "solver/Solver.h"
#include "solver/VectorSolver.h"

using namespace PhiX;

static int g_fail = 0;

static void report(const std::string& name, bool ok, const std::string& detail) {
    std::printf("  [%s]  %s  %s\n", ok ? "PASS" : "FAIL", name.c_str(), detail.c_str());
    if (!ok) ++g_fail;
}

static std::string slurp(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    return std::string(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
}

static void fill_random(ScalarField& f, double lo, double hi, unsigned seed) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(lo, hi);
    for (int k = 0; k < f.mesh.n[2]; ++k)
        for (int j = 0; j < f.mesh.n[1]; ++j)
            for (int i = 0; i < f.mesh.n[0]; ++i) f.curr[f.index(i, j, k)] = u(rng);
}

// max |a - b| over physical cells (host copies)
static double max_diff(const ScalarField& a, const ScalarField& b) {
    double m = 0.0;
    for (int k = 0; k < a.mesh.n[2]; ++k)
        for (int j = 0; j < a.mesh.n[1]; ++j)
            for (int i = 0; i < a.mesh.n[0]; ++i) {
                const double d = std::fabs(a.curr[a.index(i, j, k)] - b.curr[b.index(i, j, k)]);
                if (!(d <= m)) m = d;  // NaN propagates as a failure
            }
    return m;
}

// Runs `build` twice (fused, unfused) on fresh fields and compares.
static void fused_vs_unfused(const std::string& name, const Mesh& mesh, double lo, double hi, int nsteps,
                             const std::function<void(ScalarField&, bool, int)>& run) {
    ScalarField a(mesh, "a"), b(mesh, "b");
    fill_random(a, lo, hi, 7);
    fill_random(b, lo, hi, 7);
    a.allocDevice();
    b.allocDevice();
    a.uploadAllToDevice();
    b.uploadAllToDevice();
    run(a, true, nsteps);
    run(b, false, nsteps);
    a.downloadCurrFromDevice();
    b.downloadCurrFromDevice();
    const double d = max_diff(a, b);
    char buf[128];
    std::snprintf(buf, sizeof buf, "max-abs fused vs unfused %.3e after %d steps", d, nsteps);
    report(name, d == 0.0, buf);
}

int main() {
    std::printf("drop-in C++ API checks\n");
    const double M = 1.0, kappa = 0.5;
    auto fprime = [] __host__ __device__(double c) { return 2.0 * c * (c - 1.0) * (2.0 * c - 1.0); };

    // 1. Allen-Cahn, lap + pw, RK4, periodic (quickstart form)
    {
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, 130, 0.7, 0.0, 67, 1.1, 0.0);
        fused_vs_unfused("AC 2-D RK4 periodic, lap + pw", mesh, -0.3, 0.3, 40, [&](ScalarField& f, bool fused, int n) {
            PeriodicBC bx(Axis::X), by(Axis::Y);
            Equation eq(f, "ac");
            eq.setRHS(0.8 * lap(f) + 1.3 * pw(f, [] __host__ __device__(double p) { return p - p * p * p; }));
            Solver s(eq, {&bx, &by}, 0.02, TimeScheme::RK4);
            if (!fused) s.disableFusion();
            if (fused && !s.fused()) report("AC fused plan", false, "the solver did not fuse");
            s.run(n);
        });
    }
    // 2. Cahn-Hilliard single equation M*lap(pw(c, f') - kappa*lap(c), bcs), zero-flux x, periodic y
    {
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, 150, 1.0, 0.0, 70, 1.0, 0.0);
        fused_vs_unfused("CH 2-D RK4 composite, zero-flux x", mesh, 0.3, 0.7, 25, [&](ScalarField& c, bool fused, int n) {
            NoFluxBC xl(Axis::X, Side::LOW), xh(Axis::X, Side::HIGH);
            PeriodicBC by(Axis::Y);
            std::vector<BoundaryCondition*> bcs = {&xl, &xh, &by};
            Equation eq(c, "ch");
            eq.setRHS(M * lap(pw(c, fprime) - kappa * lap(c), bcs));
            Solver s(eq, bcs, 0.004, TimeScheme::RK4);
            if (!fused) s.disableFusion();
            if (fused && !s.fused()) report("CH fused plan", false, "the solver did not fuse");
            s.run(n);
        });
    }
    // 2b. The same on four periodic sides: the one-launch RK4 step (pair
    //     kernel through the user-functor policy) against the unfused path
    {
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, 200, 1.0, 0.0, 96, 0.9, 0.0);
        fused_vs_unfused("CH 2-D RK4 composite, periodic (one launch per step)", mesh, 0.3, 0.7, 25,
                         [&](ScalarField& c, bool fused, int n) {
                             PeriodicBC bx(Axis::X), by(Axis::Y);
                             std::vector<BoundaryCondition*> bcs = {&bx, &by};
                             Equation eq(c, "ch");
                             eq.setRHS(M * lap(pw(c, fprime) - kappa * lap(c), bcs));
                             Solver s(eq, bcs, 0.004, TimeScheme::RK4);
                             if (!fused) s.disableFusion();
                             s.run(n);
                         });
    }
    // 2c. Time of the C++ Solver::advance on CH 1024^2 RK4 (four periodic
    //     sides, FP64): one launch per step
    {
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, 1024, 1.0, 0.0, 1024, 1.0, 0.0);
        ScalarField c(mesh, "c");
        fill_random(c, 0.49, 0.51, 3);
        c.allocDevice();
        c.uploadAllToDevice();
        PeriodicBC bx(Axis::X), by(Axis::Y);
        std::vector<BoundaryCondition*> bcs = {&bx, &by};
        Equation eq(c, "ch");
        eq.setRHS(M * lap(pw(c, fprime) - kappa * lap(c), bcs));
        Solver s(eq, bcs, 0.005, TimeScheme::RK4);
        s.run(20);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        const int nrun = 400;
        cudaEventRecord(e0);
        for (int i = 0; i < nrun; ++i) s.advance();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        char buf[160];
        std::snprintf(buf, sizeof buf, "CH 1024^2 RK4 FP64 through Solver::advance: %.2f us per step (%d steps)",
                      1e3 * ms / nrun, nrun);
        report("C++ Solver one-launch RK4 timing", s.fused() && ms > 0.f, buf);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    // 3. Multi-step Cahn-Hilliard (mu STEADY, c TRANSIENT), Euler, periodic
    {
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, 100, 1.0, 0.0, 61, 1.0, 0.0);
        ScalarField mu_a(mesh, "mu"), mu_b(mesh, "mu");
        mu_a.allocDevice();
        mu_b.allocDevice();
        fused_vs_unfused("CH multi-step (mu STEADY, c TRANSIENT)", mesh, 0.3, 0.7, 30,
                         [&](ScalarField& c, bool fused, int n) {
                             ScalarField& mu = fused ? mu_a : mu_b;
                             PeriodicBC bx(Axis::X), by(Axis::Y);
                             std::vector<BoundaryCondition*> bcs = {&bx, &by};
                             Equation eqMu(mu, "mu"), eqC(c, "c");
                             eqMu.setRHS(pw(c, fprime) - kappa * lap(c));
                             eqC.setRHS(M * lap(mu));
                             Solver s({{&c, bcs, &eqMu, EquationType::STEADY},
                                       {&mu, bcs, &eqC, EquationType::TRANSIENT}},
                                      0.002, TimeScheme::EULER);
                             if (!fused) s.disableFusion();
                             if (fused && !s.fused()) report("multi-step fused plan", false, "the solver did not fuse");
                             s.run(n);
                         });
        mu_a.downloadCurrFromDevice();
        mu_b.downloadCurrFromDevice();
        char buf[96];
        const double d = max_diff(mu_a, mu_b);
        std::snprintf(buf, sizeof buf, "max-abs of mu %.3e", d);
        report("CH multi-step mu field", d == 0.0, buf);
    }
    // 4. Euler with Dirichlet x sides
    {
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, 90, 1.0, 0.0, 40, 0.8, 0.0);
        fused_vs_unfused("AC 2-D Euler, Dirichlet x / periodic y", mesh, -0.5, 0.5, 60,
                         [&](ScalarField& f, bool fused, int n) {
                             FixedBC xl(Axis::X, Side::LOW, 0.25), xh(Axis::X, Side::HIGH, -0.4);
                             PeriodicBC by(Axis::Y);
                             Equation eq(f, "ac");
                             eq.setRHS(lap(f) + pw(f, [] __host__ __device__(double p) { return p - p * p * p; }));
                             Solver s(eq, {&xl, &xh, &by}, 0.05, TimeScheme::EULER);
                             if (!fused) s.disableFusion();
                             s.run(n);
                         });
    }
    // 5. 3-D Cahn-Hilliard (marching kernel through the user-functor policy)
    {
        Mesh mesh = Mesh::makeUniform3D(CoordSys::CARTESIAN, 40, 1.0, 0.0, 21, 1.0, 0.0, 35, 1.0, 0.0);
        fused_vs_unfused("CH 3-D RK4 composite, periodic", mesh, 0.3, 0.7, 6, [&](ScalarField& c, bool fused, int n) {
            PeriodicBC bx(Axis::X), by(Axis::Y), bz(Axis::Z);
            std::vector<BoundaryCondition*> bcs = {&bx, &by, &bz};
            Equation eq(c, "ch3");
            eq.setRHS(M * lap(pw(c, fprime) - kappa * lap(c), bcs));
            Solver s(eq, bcs, 0.002, TimeScheme::RK4);
            if (!fused) s.disableFusion();
            s.run(n);
        });
    }
    // 6. VectorSolver: coupled (c, eta), RK4; c is conserved under periodic BCs
    {
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, 64, 1.0, 0.0, 48, 1.0, 0.0);
        VectorField v(mesh, "phi", 2);
        fill_random(v[0], 0.35, 0.45, 3);
        fill_random(v[1], 0.0, 0.1, 4);
        v.allocDevice();
        v.uploadAllToDevice();
        double m0 = 0.0;
        for (int j = 0; j < 48; ++j)
            for (int i = 0; i < 64; ++i) m0 += v[0].curr[v[0].index(i, j)];
        PeriodicBC bx(Axis::X), by(Axis::Y);
        std::vector<BoundaryCondition*> bcs = {&bx, &by};
        VectorEquation eq(v, "chac");
        VectorRHSExpr rhs(2);
        rhs[0] = RHSExpr(lap(pw(v[0], v[1], [] __host__ __device__(double c, double e) {
                                 return 2.0 * c * (1.0 - c) * (1.0 - 2.0 * c) + 2.0 * c * e * e;
                             }) - 0.5 * lap(v[0]), bcs));
        rhs[1] = 0.5 * lap(v[1]) - pw(v[1], v[0], [] __host__ __device__(double e, double c) {
                     return 2.0 * e * (1.0 - e) * (1.0 - 2.0 * e) + 2.0 * c * c * e;
                 });
        eq.setRHS(rhs);
        VectorSolver s(eq, bcs, 0.002, TimeScheme::RK4);
        s.run(50);
        v.downloadCurrFromDevice();
        double m1 = 0.0;
        bool finite = true;
        for (int j = 0; j < 48; ++j)
            for (int i = 0; i < 64; ++i) {
                m1 += v[0].curr[v[0].index(i, j)];
                finite = finite && std::isfinite(v[1].curr[v[1].index(i, j)]);
            }
        char buf[128];
        std::snprintf(buf, sizeof buf, "mass of c %.15e -> %.15e (rel %.2e)", m0, m1, std::fabs(m1 - m0) / m0);
        report("VectorSolver coupled RK4, conserved c", finite && std::fabs(m1 - m0) / m0 < 1e-12, buf);
    }
    // 9. General multi-step Solver (the glass-formation application's form):
    //    mu and D STEADY from pw terms of 2 and 3 fields, c TRANSIENT from
    //    D lap(mu) + grad(D) . grad(mu), phi and eta TRANSIENT from a pw term
    //    plus lap; every step one fused launch.  All stored cells of the five
    //    fields, fused against the unfused sequence, bit for bit.
    for (int dim = 2; dim <= 3; ++dim) {
        Mesh mesh = dim == 2 ? Mesh::makeUniform2D(CoordSys::CARTESIAN, 96, 1.0, 0.0, 70, 0.8, 0.0)
                             : Mesh::makeUniform3D(CoordSys::CARTESIAN, 40, 1.0, 0.0, 24, 1.0, 0.0, 18, 1.2, 0.0);
        auto f2 = [] __host__ __device__(double cv, double pv) { return (1.0 - pv * pv) * (cv - 0.5) * 2.5; };
        auto f3 = [] __host__ __device__(double cv, double pv, double ev) {
            return (0.3 + 0.5 * pv + 0.2 * ev * ev) * cv * (1.0 - cv);
        };
        auto g3 = [] __host__ __device__(double pv, double ev, double cv) {
            return -0.8 * (pv * (1.0 - pv) * (0.5 - pv + 0.1 * cv) + 0.3 * pv * ev * ev);
        };
        auto h2 = [] __host__ __device__(double pv, double ev) { return -0.6 * (ev * (1.0 - ev) * (0.5 - ev) + 0.2 * pv * pv * ev); };
        std::vector<double> got[2][5];
        bool fused_ok = true;
        for (int fused = 1; fused >= 0; --fused) {
            ScalarField c(mesh, "c"), phi(mesh, "phi"), eta(mesh, "eta"), mu(mesh, "mu"), D(mesh, "D");
            fill_random(c, 0.3, 0.7, 41);
            fill_random(phi, 0.0, 1.0, 42);
            fill_random(eta, 0.0, 0.4, 43);
            ScalarField* all[5] = {&c, &phi, &eta, &mu, &D};
            for (auto* f : all) {
                f->allocDevice();
                f->uploadAllToDevice();
            }
            PeriodicBC bx(Axis::X), bz(Axis::Z);
            NoFluxBC by(Axis::Y);
            std::vector<BoundaryCondition*> bcs = {&bx, &by};
            if (dim == 3) bcs.push_back(&bz);
            Equation eq_mu(mu, "mu"), eqD(D, "D"), eqC(c, "c"), eqPhi(phi, "phi"), eqEta(eta, "eta");
            eq_mu.setRHS(pw(c, phi, f2));
            eqD.setRHS(pw(c, phi, eta, f3));
            RHSExpr rc = RHSExpr(D * lap(mu)) + grad(D, 0) * grad(mu, 0) + grad(D, 1) * grad(mu, 1);
            if (dim == 3) rc += grad(D, 2) * grad(mu, 2);
            eqC.setRHS(rc);
            eqPhi.setRHS(pw(phi, eta, c, g3) + 0.3 * lap(phi));
            eqEta.setRHS(pw(phi, eta, h2) + 0.2 * lap(eta));
            Solver s({{&c, bcs, &eq_mu, EquationType::STEADY},
                      {&mu, bcs, &eqD, EquationType::STEADY},
                      {&D, bcs, &eqD, EquationType::STEADY},
                      {&c, bcs, &eqC, EquationType::TRANSIENT},
                      {&phi, bcs, &eqPhi, EquationType::TRANSIENT},
                      {&eta, bcs, &eqEta, EquationType::TRANSIENT}},
                     2e-3, TimeScheme::EULER);
            if (fused) fused_ok = s.fused();
            else s.disableFusion();
            s.run(20);
            for (int q = 0; q < 5; ++q) {
                all[q]->downloadCurrFromDevice();
                got[fused][q] = all[q]->curr;
            }
        }
        bool same = fused_ok;
        const char* names[5] = {"c", "phi", "eta", "mu", "D"};
        std::string which;
        for (int q = 0; q < 5; ++q) {
            bool eq = got[0][q].size() == got[1][q].size();
            for (std::size_t i = 0; eq && i < got[0][q].size(); ++i)
                eq = std::memcmp(&got[0][q][i], &got[1][q][i], sizeof(double)) == 0;
            if (!eq) which += std::string(" ") + names[q];
            same = same && eq;
        }
        report(std::string("general multi-step, 6 steps, 5 fields, ") + (dim == 2 ? "2-D" : "3-D"), same,
               fused_ok ? (which.empty() ? "every stored cell equal, fused vs unfused" : "differs:" + which)
                        : "the solver did not fuse");
    }
    // 11. Single-equation Euler with gradient, product and two-field pw terms
    //     (one flat_step launch per step), zero-flux x, periodic y
    {
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, 77, 1.0, 0.0, 45, 0.9, 0.0);
        ScalarField v(mesh, "v");
        fill_random(v, 0.2, 0.8, 61);
        v.allocDevice();
        v.uploadAllToDevice();
        fused_vs_unfused("Euler, lap + grad*grad + pw(u, v) + grad(v) + u*lap(v)", mesh, 0.2, 0.8, 40,
                         [&](ScalarField& u, bool fused, int n) {
                             NoFluxBC bx(Axis::X);
                             PeriodicBC by(Axis::Y);
                             Equation eq(u, "u");
                             eq.setRHS(RHSExpr(0.5 * lap(u)) + 0.2 * (grad(u, 0) * grad(u, 1)) +
                                       pw(u, v, [] __host__ __device__(double a, double b) { return a * (1.0 - a) * (b - 0.5); }) +
                                       grad(v, 0, 0.1) + u * lap(v));
                             Solver s(eq, {&bx, &by}, 0.01, TimeScheme::EULER);
                             if (!fused) s.disableFusion();
                             if (fused && !s.fused()) report("Euler flat plan", false, "the solver did not fuse");
                             s.run(n);
                         });
    }
    // 10. The same six-step system at 1024^2: ms per time step, fused against
    //     the unfused sequence (one kernel per term, scratch materialisation,
    //     as the reference launches it)
    {
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, 1024, 1.0, 0.0, 1024, 1.0, 0.0);
        auto f2 = [] __host__ __device__(double cv, double pv) { return (1.0 - pv * pv) * (cv - 0.5) * 2.5; };
        auto f3 = [] __host__ __device__(double cv, double pv, double ev) {
            return (0.3 + 0.5 * pv + 0.2 * ev * ev) * cv * (1.0 - cv);
        };
        auto g3 = [] __host__ __device__(double pv, double ev, double cv) {
            return -0.8 * (pv * (1.0 - pv) * (0.5 - pv + 0.1 * cv) + 0.3 * pv * ev * ev);
        };
        auto h2 = [] __host__ __device__(double pv, double ev) { return -0.6 * (ev * (1.0 - ev) * (0.5 - ev) + 0.2 * pv * pv * ev); };
        double ms[2] = {0.0, 0.0};
        for (int fused = 0; fused < 2; ++fused) {
            ScalarField c(mesh, "c"), phi(mesh, "phi"), eta(mesh, "eta"), mu(mesh, "mu"), D(mesh, "D");
            fill_random(c, 0.3, 0.7, 51);
            fill_random(phi, 0.0, 1.0, 52);
            fill_random(eta, 0.0, 0.4, 53);
            for (ScalarField* f : {&c, &phi, &eta, &mu, &D}) {
                f->allocDevice();
                f->uploadAllToDevice();
            }
            PeriodicBC bx(Axis::X);
            NoFluxBC by(Axis::Y);
            std::vector<BoundaryCondition*> bcs = {&bx, &by};
            Equation eq_mu(mu, "mu"), eqD(D, "D"), eqC(c, "c"), eqPhi(phi, "phi"), eqEta(eta, "eta");
            eq_mu.setRHS(pw(c, phi, f2));
            eqD.setRHS(pw(c, phi, eta, f3));
            eqC.setRHS(RHSExpr(D * lap(mu)) + grad(D, 0) * grad(mu, 0) + grad(D, 1) * grad(mu, 1));
            eqPhi.setRHS(pw(phi, eta, c, g3) + 0.3 * lap(phi));
            eqEta.setRHS(pw(phi, eta, h2) + 0.2 * lap(eta));
            Solver s({{&c, bcs, &eq_mu, EquationType::STEADY},
                      {&mu, bcs, &eqD, EquationType::STEADY},
                      {&D, bcs, &eqD, EquationType::STEADY},
                      {&c, bcs, &eqC, EquationType::TRANSIENT},
                      {&phi, bcs, &eqPhi, EquationType::TRANSIENT},
                      {&eta, bcs, &eqEta, EquationType::TRANSIENT}},
                     1e-4, TimeScheme::EULER);
            if (!fused) s.disableFusion();
            s.run(5);
            const int n = 100;
            const auto t0 = std::chrono::steady_clock::now();
            s.run(n);
            ms[fused] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / n;
        }
        char buf[160];
        std::snprintf(buf, sizeof buf, "1024^2, 6 steps over 5 fields: unfused %.3f ms, fused %.3f ms per time step (%.1fx)",
                      ms[0], ms[1], ms[0] / ms[1]);
        report("general multi-step timing", ms[1] > 0.0, buf);
    }
    // 7. OutputWriter: the asynchronous files equal IO::writeField's byte for
    //    byte, for a snapshot taken before the device cells change again
    for (int dim = 2; dim <= 3; ++dim) {
        Mesh mesh = dim == 2 ? Mesh::makeUniform2D(CoordSys::CARTESIAN, 53, 0.5, -1.0, 31, 0.25, 2.0)
                             : Mesh::makeUniform3D(CoordSys::CARTESIAN, 37, 1.0, 0.0, 20, 0.5, 1.0, 6, 2.0, -3.0);
        ScalarField f(mesh, dim == 2 ? "w2" : "w3");
        fill_random(f, -1.0, 1.0, 11 + dim);
        f.allocDevice();
        f.uploadAllToDevice();
        const std::string ref = "ref_" + f.name;
        IO::writeField(f, ref + ".field", FieldFormat::BINARY);
        IO::writeField(f, ref + ".dat", FieldFormat::DAT);
        IO::writeField(f, ref + ".vts", FieldFormat::VTS);
        bool same = true;
        {
            IO::OutputWriter w(nlohmann::json::parse(R"({"print_interval": 1, "write_interval": 1, "format": "ALL"})"));
            w.writeFields(f, 7, 0.25);
            cudaMemset(f.d_curr, 0, f.storedSize * sizeof(double));  // after the snapshot, before the files exist
            w.flush();
        }
        for (const char* ext : {".field", ".dat", ".vts"})
            same = same && slurp(ref + ext) == slurp("output/" + f.name + "_7" + ext) && !slurp(ref + ext).empty();
        report(std::string("OutputWriter async files, ") + (dim == 2 ? "2-D" : "3-D"), same,
               "BINARY / DAT / VTS equal IO::writeField's bytes");
    }
    {
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, 16, 1.0, 0.0, 8, 1.0, 0.0);
        ScalarField f(mesh, "no_such_dir/x");
        f.allocDevice();
        bool thrown = false;
        try {
            IO::OutputWriter w(nlohmann::json::parse(R"({"print_interval": 1, "write_interval": 1, "format": "BINARY"})"));
            w.writeFields(f, 1, 0.0);
            w.flush();
        } catch (const std::runtime_error&) {
            thrown = true;
        }
        report("OutputWriter async error reaches flush()", thrown, "unopenable path -> std::runtime_error");
    }
    // 8. Output overlap: the multi-step CH app loop at 1024^2 with no output,
    //    with a .field file every 200 steps written synchronously (the
    //    reference's order), and the same written asynchronously; wall time
    //    until every file is on disk
    {
        const int n = 1024, nsteps = 4000, every = 200;
        Mesh mesh = Mesh::makeUniform2D(CoordSys::CARTESIAN, n, 1.0, 0.0, n, 1.0, 0.0);
        double ms[3] = {0.0, 0.0, 0.0};
        std::string files[3];
        for (int mode = 0; mode < 3; ++mode) {  // 0 no output, 1 sync, 2 async
            ScalarField c(mesh, mode == 2 ? "ov_async" : "ov_sync"), mu(mesh, "mu");
            fill_random(c, 0.49, 0.51, 21);
            c.allocDevice();
            c.uploadAllToDevice();
            mu.allocDevice();
            PeriodicBC bx(Axis::X), by(Axis::Y);
            std::vector<BoundaryCondition*> bcs = {&bx, &by};
            Equation eqMu(mu, "mu"), eqC(c, "c");
            eqMu.setRHS(pw(c, fprime) - kappa * lap(c));
            eqC.setRHS(M * lap(mu));
            Solver s({{&c, bcs, &eqMu, EquationType::STEADY}, {&mu, bcs, &eqC, EquationType::TRANSIENT}}, 0.005,
                     TimeScheme::EULER);
            nlohmann::json cfg = nlohmann::json::parse(R"({"print_interval": 100000, "write_interval": 1, "format": "BINARY"})");
            cfg["write_interval"] = every;
            cfg["async"] = mode == 2;
            IO::OutputWriter w(cfg);
            s.advance();  // plan and first launch outside the timed loop
            cudaDeviceSynchronize();
            const auto t0 = std::chrono::steady_clock::now();
            for (int st = 1; st < nsteps; ++st) {
                s.advance();
                if (mode > 0 && w.shouldWrite(s.step)) w.writeFields(c, s.step, s.time);
            }
            w.flush();
            cudaDeviceSynchronize();
            ms[mode] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            if (mode > 0) files[mode] = slurp("output/" + c.name + "_" + std::to_string(nsteps - nsteps % every) + ".field");
        }
        const std::size_t cut1 = files[1].find("---\n"), cut2 = files[2].find("---\n");
        const bool same = cut1 != std::string::npos && cut2 != std::string::npos &&
                          files[1].substr(cut1) == files[2].substr(cut2) && files[1].size() > (std::size_t)n * n * 8;
        char buf[200];
        std::snprintf(buf, sizeof buf,
                      "CH 1024^2 multi-step, %d steps, %d .field writes: no output %.1f ms, sync %.1f ms, async %.1f ms "
                      "(%.0f%% of the output time hidden)",
                      nsteps - 1, (nsteps - 1) / every, ms[0], ms[1], ms[2], 100.0 * (ms[1] - ms[2]) / (ms[1] - ms[0]));
        report("OutputWriter overlap, same final cells", same, buf);
    }
    std::printf(g_fail ? "SOME CHECKS FAILED\n" : "ALL CHECKS PASSED\n");
    return g_fail ? 1 : 0;
}
