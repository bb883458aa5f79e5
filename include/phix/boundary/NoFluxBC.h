#pragma once
#include "boundary/BoundaryCondition.h"
namespace PhiX {
// Zero-gradient: every ghost layer <- nearest physical cell.
class NoFluxBC : public BoundaryCondition {
public:
    NoFluxBC(Axis axis, Side side = Side::BOTH);
    using BoundaryCondition::applyOnCPU;
    using BoundaryCondition::applyOnGPU;
    void applyOnCPU(ScalarField& f) const override;
    void applyOnGPU(ScalarField& f) const override;
    int fusedKind() const override;
};
}  // namespace PhiX
