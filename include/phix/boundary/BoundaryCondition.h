#pragma once
// BoundaryCondition -- ghost-cell fill of one axis (API of the reference's
// include/boundary/BoundaryCondition.h).  The fused solver path reads the
// built-in kinds (PeriodicBC, NoFluxBC, FixedBC) as halo mappings instead of
// running these fills.

#include "field/ScalarField.h"
#include "field/VectorField.h"

namespace PhiX {

enum class Axis { X = 0, Y = 1, Z = 2 };
enum class Side { LOW, HIGH, BOTH };

class BoundaryCondition {
public:
    Axis axis;
    Side side;
    BoundaryCondition(Axis axis, Side side) : axis(axis), side(side) {}
    virtual ~BoundaryCondition() = default;

    virtual void applyOnCPU(ScalarField& f) const = 0;
    virtual void applyOnGPU(ScalarField& f) const = 0;
    virtual void applyOnCPU(VectorField& vf) const {
        for (int c = 0; c < vf.nComponents(); ++c) applyOnCPU(vf[c]);
    }
    virtual void applyOnGPU(VectorField& vf) const {
        for (int c = 0; c < vf.nComponents(); ++c) applyOnGPU(vf[c]);
    }

    // Kind for the fused path: PHIX_BC_* of phix_b200.h, or -1 for BCs the
    // fused kernels cannot express (user subclasses).
    virtual int fusedKind() const { return -1; }
    virtual double fusedValue() const { return 0.0; }
};

}  // namespace PhiX
