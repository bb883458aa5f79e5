#pragma once
#include "boundary/BoundaryCondition.h"
namespace PhiX {
// Dirichlet as a constant fill of every ghost layer on the chosen side(s).
class FixedBC : public BoundaryCondition {
public:
    double value;
    FixedBC(Axis axis, Side side, double value);
    using BoundaryCondition::applyOnCPU;
    using BoundaryCondition::applyOnGPU;
    void applyOnCPU(ScalarField& f) const override;
    void applyOnGPU(ScalarField& f) const override;
    int fusedKind() const override;
    double fusedValue() const override { return value; }
};
}  // namespace PhiX
