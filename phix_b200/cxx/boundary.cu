// boundary.cu -- PeriodicBC / NoFluxBC / FixedBC and buildBCs of the drop-in
// C++ API.  GPU fills go through phix_bc_apply with a grid that carries only
// this BC; CPU fills walk the same faces on the host.
#include <stdexcept>
#include <string>

#include "boundary/BCFactory.h"
#include "boundary/FixedBC.h"
#include "boundary/NoFluxBC.h"
#include "boundary/PeriodicBC.h"
#include "phix_b200.h"

namespace PhiX {

namespace {

// phix grid of field f with BC kind `kind` on the chosen sides of `axis` only.
phix_grid_t one_bc_grid(const ScalarField& f, Axis axis, Side side, int kind, double value) {
    phix_grid_t g{};
    g.dim = f.mesh.dim;
    for (int a = 0; a < 3; ++a) {
        g.n[a] = f.mesh.n[a];
        g.d[a] = a < f.mesh.dim ? f.mesh.d[a] : 1.0;
    }
    g.ghost = f.ghost;
    const int a = static_cast<int>(axis);
    if (side == Side::LOW || side == Side::BOTH) { g.bc_type[2 * a] = kind; g.bc_val[2 * a] = value; }
    if (side == Side::HIGH || side == Side::BOTH) { g.bc_type[2 * a + 1] = kind; g.bc_val[2 * a + 1] = value; }
    return g;
}

void gpu_fill(ScalarField& f, Axis axis, Side side, int kind, double value, const char* who) {
    if (!f.deviceAllocated()) throw std::runtime_error(std::string(who) + "::applyOnGPU: device not allocated");
    if (static_cast<int>(axis) >= f.mesh.dim) return;
    phix_grid_t g = one_bc_grid(f, axis, side, kind, value);
    const int rc = phix_bc_apply(f.d_curr, &g, nullptr);
    if (rc == PHIX_ERR_ARG) throw std::invalid_argument(phix_last_error());
    if (rc != PHIX_OK) throw std::runtime_error(phix_last_error());
}

// Host fill over the full stored extent of the two other axes, every layer.
void cpu_fill(ScalarField& f, Axis axis, bool lo, bool hi, int kind, double value) {
    const int sx = f.storedDims[0], sy = f.storedDims[1], sz = f.storedDims[2], g = f.ghost;
    int astr, nf0, nf1, fs0, fs1;
    const int a = static_cast<int>(axis);
    const int n = f.mesh.n[a];
    if (a == 0) { astr = 1; nf0 = sy; nf1 = sz; fs0 = sx; fs1 = sx * sy; }
    else if (a == 1) { astr = sx; nf0 = sx; nf1 = sz; fs0 = 1; fs1 = sx * sy; }
    else { astr = sx * sy; nf0 = sx; nf1 = sy; fs0 = 1; fs1 = sx; }
    double* d = f.curr.data();
    for (int t0 = 0; t0 < nf0; ++t0)
        for (int t1 = 0; t1 < nf1; ++t1) {
            const int off = t0 * fs0 + t1 * fs1;
            for (int l = 1; l <= g; ++l) {
                const int ilo = (g - l) * astr + off, ihi = (g + n + l - 1) * astr + off;
                if (kind == PHIX_BC_PERIODIC) {
                    d[ilo] = d[(g + n - l) * astr + off];
                    d[ihi] = d[(g + l - 1) * astr + off];
                } else if (kind == PHIX_BC_NOFLUX) {
                    if (lo) d[ilo] = d[g * astr + off];
                    if (hi) d[ihi] = d[(g + n - 1) * astr + off];
                } else {
                    if (lo) d[ilo] = value;
                    if (hi) d[ihi] = value;
                }
            }
        }
}

bool has_lo(Side s) { return s == Side::LOW || s == Side::BOTH; }
bool has_hi(Side s) { return s == Side::HIGH || s == Side::BOTH; }

}  // namespace

PeriodicBC::PeriodicBC(Axis a) : BoundaryCondition(a, Side::BOTH) {}
void PeriodicBC::applyOnCPU(ScalarField& f) const { cpu_fill(f, axis, true, true, PHIX_BC_PERIODIC, 0.0); }
void PeriodicBC::applyOnGPU(ScalarField& f) const { gpu_fill(f, axis, Side::BOTH, PHIX_BC_PERIODIC, 0.0, "PeriodicBC"); }
int PeriodicBC::fusedKind() const { return PHIX_BC_PERIODIC; }

NoFluxBC::NoFluxBC(Axis a, Side s) : BoundaryCondition(a, s) {}
void NoFluxBC::applyOnCPU(ScalarField& f) const { cpu_fill(f, axis, has_lo(side), has_hi(side), PHIX_BC_NOFLUX, 0.0); }
void NoFluxBC::applyOnGPU(ScalarField& f) const { gpu_fill(f, axis, side, PHIX_BC_NOFLUX, 0.0, "NoFluxBC"); }
int NoFluxBC::fusedKind() const { return PHIX_BC_NOFLUX; }

FixedBC::FixedBC(Axis a, Side s, double v) : BoundaryCondition(a, s), value(v) {}
void FixedBC::applyOnCPU(ScalarField& f) const { cpu_fill(f, axis, has_lo(side), has_hi(side), PHIX_BC_FIXED, value); }
void FixedBC::applyOnGPU(ScalarField& f) const { gpu_fill(f, axis, side, PHIX_BC_FIXED, value, "FixedBC"); }
int FixedBC::fusedKind() const { return PHIX_BC_FIXED; }

// ---------------------------------------------------------------------------
// buildBCs: x_min/x_max (required), y_*, z_* when present; "Periodic" must be
// on both sides of an axis; "NoFlux" per side.
// ---------------------------------------------------------------------------
namespace {
void add_axis(BCSet& set, Axis axis, const std::string& lo, const std::string& hi) {
    const bool pl = lo == "Periodic", ph = hi == "Periodic";
    if (pl != ph) {
        const char* nm = axis == Axis::X ? "X" : axis == Axis::Y ? "Y" : "Z";
        throw std::runtime_error(std::string("buildBCs: Periodic BC must be set on both sides of axis ") + nm +
                                 ", got \"" + lo + "\" / \"" + hi + "\"");
    }
    if (pl) {
        set.storage.push_back(std::make_unique<PeriodicBC>(axis));
        set.ptrs.push_back(set.storage.back().get());
        return;
    }
    for (int s = 0; s < 2; ++s) {
        const std::string& type = s == 0 ? lo : hi;
        if (type != "NoFlux") throw std::runtime_error("buildBCs: unsupported BC type \"" + type + "\"");
        set.storage.push_back(std::make_unique<NoFluxBC>(axis, s == 0 ? Side::LOW : Side::HIGH));
        set.ptrs.push_back(set.storage.back().get());
    }
}
}  // namespace

BCSet buildBCs(const nlohmann::json& c) {
    BCSet set;
    add_axis(set, Axis::X, c.at("x_min").get<std::string>(), c.at("x_max").get<std::string>());
    if (c.contains("y_min") && c.contains("y_max"))
        add_axis(set, Axis::Y, c.at("y_min").get<std::string>(), c.at("y_max").get<std::string>());
    if (c.contains("z_min") && c.contains("z_max"))
        add_axis(set, Axis::Z, c.at("z_min").get<std::string>(), c.at("z_max").get<std::string>());
    return set;
}

}  // namespace PhiX
