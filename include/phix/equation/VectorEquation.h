#pragma once
// VectorEquation -- one scalar Equation per component (API of the
// reference's include/equation/VectorEquation.h).

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "equation/Equation.h"
#include "equation/Term.h"
#include "field/VectorField.h"

namespace PhiX {

class VectorEquation {
public:
    std::string name;
    VectorField& unknown;
    std::map<std::string, double> params;

    explicit VectorEquation(VectorField& unknown, const std::string& name = "");
    void setRHS(const VectorRHSExpr& expr);
    void computeRHS(VectorField& rhs) const;
    void computeRHSCPU(VectorField& rhs) const;
    Equation& componentEquation(int c);
    const Equation& componentEquation(int c) const;
    bool hasRHS() const;

private:
    std::vector<std::unique_ptr<Equation>> equations_;
};

}  // namespace PhiX
