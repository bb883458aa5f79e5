#pragma once
// Equation -- d(unknown)/dt = RHS (API of the reference's
// include/equation/Equation.h).  computeRHS zeroes the whole rhs array, runs
// every term in order and returns with the results complete.

#include <string>
#include <vector>

#include "equation/Term.h"
#include "field/ScalarField.h"

namespace PhiX {

class Equation {
public:
    std::string name;
    ScalarField& unknown;
    std::vector<ScalarField*> auxFields;

    explicit Equation(ScalarField& unknown, const std::string& name = "");

    void setRHS(const RHSExpr& expr);
    void setRHS(const Term& t);

    void computeRHS(ScalarField& rhs) const;
    void computeRHSCPU(ScalarField& rhs) const;
    bool hasRHS() const { return !rhs_expr_.terms.empty(); }

    // The expression set by setRHS (read by the fused Solver path).
    const RHSExpr& rhsExpr() const { return rhs_expr_; }

private:
    RHSExpr rhs_expr_;
    mutable ScratchPool scratch_pool_;
};

}  // namespace PhiX
