#pragma once
// Solver -- explicit Euler / RK4 time stepping (API of the reference's
// include/solver/Solver.h), single-equation and multi-step modes.
//
// GPU path.  When the equation's right-hand side is a sum of lap / pw terms of
// the unknown (one pw functor), or M*lap(such a sum, bcs), and every BC is a
// PeriodicBC / NoFluxBC / FixedBC, each RK stage runs as ONE fused kernel
// (BCs folded into the halo loads, the stage combination into the tile load,
// the update into the last stage).  Otherwise the terms run one kernel each,
// as in the reference, on this library's kernels.  The multi-step
// Cahn-Hilliard form (mu STEADY from pw + lap of c, c TRANSIENT from M*lap(mu))
// fuses into one kernel per step.  After advance() returns, unknown.d_curr
// holds the new state; fused steps swap d_curr and d_prev instead of copying,
// so d_prev then holds the previous time level.

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "boundary/BoundaryCondition.h"
#include "equation/Equation.h"
#include "field/ScalarField.h"

namespace PhiX {

enum class TimeScheme { EULER, RK4 };
enum class EquationType { TRANSIENT, STEADY };

struct SolverStep {
    ScalarField* sourceField;
    std::vector<BoundaryCondition*> bcs;
    Equation* equation;
    EquationType type = EquationType::TRANSIENT;
};

struct FusedPlan;  // the compiled fused path (solver/Solver.cu)

class Solver {
public:
    Solver(Equation& equation, std::vector<BoundaryCondition*> bcs, double dt, TimeScheme scheme = TimeScheme::EULER);
    Solver(std::vector<SolverStep> steps, double dt, TimeScheme scheme = TimeScheme::EULER);
    ~Solver();
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    double dt;
    TimeScheme scheme;
    int step = 0;
    double time = 0.0;

    void advance();
    void advanceCPU();
    void run(int nSteps, int callbackEvery = 0, std::function<void(const Solver&)> callback = nullptr);

    const ScalarField& unknown() const { return equation_.unknown; }
    ScalarField& unknown() { return equation_.unknown; }
    const Equation& equation() const { return equation_; }
    const std::vector<BoundaryCondition*>& bcs() const { return bcs_; }

    // True when advance() runs the fused kernels.
    bool fused() const { return plan_ != nullptr; }
    // Force the per-term (unfused) path.
    void disableFusion();

private:
    Equation& equation_;
    std::vector<BoundaryCondition*> bcs_;
    ScalarField rhs_;
    ScalarField k1_, k2_, k3_, k4_;
    ScalarField phi_tmp_;
    bool use_rk4_ = false;
    bool multiStep_ = false;
    std::vector<SolverStep> steps_;
    std::vector<std::unique_ptr<ScalarField>> stepScratch_;
    std::unique_ptr<FusedPlan> plan_;

    void applyBCsGPU();
    void applyBCsCPU();
    void eulerUpdateGPU();
    void eulerUpdateCPU();
    void rk4AdvanceGPU();
    void rk4AdvanceCPU();
    void multiStepAdvanceGPU();
    void multiStepAdvanceCPU();
    void fusedAdvance();
};

}  // namespace PhiX
