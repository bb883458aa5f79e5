#pragma once
#include "boundary/BoundaryCondition.h"
namespace PhiX {
// Ghost <- opposite physical layer, both sides.
class PeriodicBC : public BoundaryCondition {
public:
    explicit PeriodicBC(Axis axis);
    using BoundaryCondition::applyOnCPU;
    using BoundaryCondition::applyOnGPU;
    void applyOnCPU(ScalarField& f) const override;
    void applyOnGPU(ScalarField& f) const override;
    int fusedKind() const override;
};
}  // namespace PhiX
