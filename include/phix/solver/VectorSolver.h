#pragma once
// VectorSolver -- Euler / RK4 for a VectorEquation with every component
// advanced from one consistent stage state (API of the reference's
// include/solver/VectorSolver.h).

#include <functional>
#include <vector>

#include "boundary/BoundaryCondition.h"
#include "equation/VectorEquation.h"
#include "field/VectorField.h"
#include "solver/Solver.h"

namespace PhiX {

class VectorSolver {
public:
    VectorSolver(VectorEquation& equation, std::vector<BoundaryCondition*> bcs, double dt,
                 TimeScheme scheme = TimeScheme::EULER);
    VectorSolver(const VectorSolver&) = delete;
    VectorSolver& operator=(const VectorSolver&) = delete;

    double dt;
    TimeScheme scheme;
    int step = 0;
    double time = 0.0;

    void advance();
    void advanceCPU();
    void run(int nSteps, int callbackEvery = 0, std::function<void(const VectorSolver&)> callback = nullptr);

    const VectorField& unknown() const { return equation_.unknown; }
    VectorField& unknown() { return equation_.unknown; }
    const VectorEquation& equation() const { return equation_; }
    const std::vector<BoundaryCondition*>& bcs() const { return bcs_; }

private:
    VectorEquation& equation_;
    std::vector<BoundaryCondition*> bcs_;
    bool use_rk4_;
    VectorField rhs_, k1_, k2_, k3_, k4_, phi_tmp_;

    void applyBCsGPU();
    void applyBCsCPU();
    void rk4AdvanceGPU();
    void rk4AdvanceCPU();
};

}  // namespace PhiX
