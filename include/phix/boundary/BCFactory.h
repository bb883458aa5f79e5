#pragma once
// buildBCs -- BCs from a JSON block {"x_min": "Periodic"|"NoFlux", ...}
// (API of the reference's include/boundary/BCFactory.h; needs nlohmann/json
// on the include path, as the reference does).

#include <memory>
#include <vector>

#include <nlohmann/json.hpp>

#include "boundary/BoundaryCondition.h"

namespace PhiX {

struct BCSet {
    std::vector<std::unique_ptr<BoundaryCondition>> storage;
    std::vector<BoundaryCondition*> ptrs;
};

BCSet buildBCs(const nlohmann::json& bc_config);

}  // namespace PhiX
