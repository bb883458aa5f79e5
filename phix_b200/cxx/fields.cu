// fields.cu -- Mesh, ScalarField, VectorField of the drop-in C++ API.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>

#include "IO/FieldIO.h"
#include "field/ScalarField.h"
#include "field/VectorField.h"
#include "mesh/Mesh.h"

namespace PhiX {

namespace {
void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}
}  // namespace

// ---------------------------------------------------------------------------
// Mesh
// ---------------------------------------------------------------------------
std::string coordSysToString(CoordSys cs) {
    switch (cs) {
        case CoordSys::CYLINDRICAL: return "CYLINDRICAL";
        case CoordSys::SPHERICAL: return "SPHERICAL";
        default: return "CARTESIAN";
    }
}

CoordSys stringToCoordSys(const std::string& s) {
    std::string u = s;
    std::transform(u.begin(), u.end(), u.begin(), [](unsigned char c) { return (char)std::toupper(c); });
    if (u == "CARTESIAN") return CoordSys::CARTESIAN;
    if (u == "CYLINDRICAL") return CoordSys::CYLINDRICAL;
    if (u == "SPHERICAL") return CoordSys::SPHERICAL;
    throw std::invalid_argument("Unknown CoordSys: " + s);
}

Mesh::Mesh() : dim(1), coordSys(CoordSys::CARTESIAN), n{0, 1, 1}, d{0.0, 1.0, 1.0}, origin{0.0, 0.0, 0.0} {}

Mesh::Mesh(int dim_, CoordSys cs, int nx, double dx, double x0, int ny, double dy, double y0, int nz, double dz,
           double z0)
    : dim(dim_), coordSys(cs), n{nx, ny, nz}, d{dx, dy, dz}, origin{x0, y0, z0} {
    validate();
}

Mesh Mesh::makeUniform1D(CoordSys cs, int nx, double dx, double x0) {
    return Mesh(1, cs, nx, dx, x0, 1, 1.0, 0.0, 1, 1.0, 0.0);
}
Mesh Mesh::makeUniform2D(CoordSys cs, int nx, double dx, double x0, int ny, double dy, double y0) {
    return Mesh(2, cs, nx, dx, x0, ny, dy, y0, 1, 1.0, 0.0);
}
Mesh Mesh::makeUniform3D(CoordSys cs, int nx, double dx, double x0, int ny, double dy, double y0, int nz, double dz,
                         double z0) {
    return Mesh(3, cs, nx, dx, x0, ny, dy, y0, nz, dz, z0);
}

void Mesh::validate() const {
    if (dim < 1 || dim > 3) throw std::invalid_argument("Mesh: dim must be 1, 2, or 3");
    for (int a = 0; a < dim; ++a) {
        if (n[a] <= 0) throw std::invalid_argument("Mesh: n[" + std::to_string(a) + "] must be > 0");
        if (d[a] <= 0.0) throw std::invalid_argument("Mesh: d[" + std::to_string(a) + "] must be > 0");
    }
    for (int a = dim; a < 3; ++a)
        if (n[a] != 1) throw std::invalid_argument("Mesh: n[" + std::to_string(a) + "] must be 1 for unused axes");
}

bool Mesh::isValid() const noexcept {
    try {
        validate();
        return true;
    } catch (...) {
        return false;
    }
}

void Mesh::write(const std::string& path) const {
    validate();
    std::ofstream o(path);
    if (!o) throw std::runtime_error("Mesh::write: cannot open file: " + path);
    o << "# PhiX Mesh\n"
      << "dim      " << dim << "\n"
      << "coordSys " << coordSysToString(coordSys) << "\n";
    const char* ax[3] = {"x", "y", "z"};
    for (int a = 0; a < 3; ++a)
        o << "n" << ax[a] << " " << n[a] << "  d" << ax[a] << " " << d[a] << "  " << ax[a] << "0 " << origin[a] << "\n";
}

Mesh Mesh::readFromFile(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("Mesh::readFromFile: cannot open file: " + path);
    int dm = 1;
    CoordSys cs = CoordSys::CARTESIAN;
    int nn[3] = {1, 1, 1};
    double dd[3] = {1.0, 1.0, 1.0}, oo[3] = {0.0, 0.0, 0.0};
    const std::string nk[3] = {"nx", "ny", "nz"}, dk[3] = {"dx", "dy", "dz"}, ok[3] = {"x0", "y0", "z0"};
    std::string line;
    while (std::getline(in, line)) {
        const auto hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        std::istringstream ss(line);
        std::string tok;
        while (ss >> tok) {
            if (tok == "dim") { ss >> dm; continue; }
            if (tok == "coordSys") { std::string v; ss >> v; cs = stringToCoordSys(v); continue; }
            for (int a = 0; a < 3; ++a) {
                if (tok == nk[a]) ss >> nn[a];
                else if (tok == dk[a]) ss >> dd[a];
                else if (tok == ok[a]) ss >> oo[a];
            }
        }
    }
    return Mesh(dm, cs, nn[0], dd[0], oo[0], nn[1], dd[1], oo[1], nn[2], dd[2], oo[2]);
}

void Mesh::print() const {
    std::cout << "=== Mesh ===\n  dim      : " << dim << "\n  coordSys : " << coordSysToString(coordSys) << "\n";
    const char* ax[3] = {"x", "y", "z"};
    for (int a = 0; a < 3; ++a) {
        std::cout << "  " << ax[a] << ": n=" << n[a] << "  d=" << d[a] << "  origin=" << origin[a];
        if (a >= dim) std::cout << "  (inactive)";
        std::cout << "\n";
    }
    std::cout << "  totalSize: " << totalSize() << "\n";
}

// ---------------------------------------------------------------------------
// ScalarField
// ---------------------------------------------------------------------------
ScalarField::ScalarField(const Mesh& m, const std::string& nm, int g) : name(nm), mesh(m), ghost(g) {
    if (g < 0) throw std::invalid_argument("ScalarField: ghost must be >= 0");
    for (int a = 0; a < 3; ++a) storedDims[a] = mesh.n[a] + 2 * ghost;
    storedSize = (std::size_t)storedDims[0] * storedDims[1] * storedDims[2];
    curr.assign(storedSize, 0.0);
    prev.assign(storedSize, 0.0);
}

ScalarField ScalarField::makeShell(const Mesh& m, int g, double* d_buf, const std::string& nm) {
    ScalarField f(m, nm, g);
    f.curr.clear();
    f.curr.shrink_to_fit();
    f.prev.clear();
    f.prev.shrink_to_fit();
    f.d_curr = d_buf;
    f.d_prev = nullptr;
    f.ownsDeviceMemory_ = false;
    return f;
}

ScalarField::ScalarField(ScalarField&& o) noexcept
    : name(std::move(o.name)), mesh(o.mesh), ghost(o.ghost), storedSize(o.storedSize), curr(std::move(o.curr)),
      prev(std::move(o.prev)), d_curr(o.d_curr), d_prev(o.d_prev), ownsDeviceMemory_(o.ownsDeviceMemory_) {
    for (int a = 0; a < 3; ++a) storedDims[a] = o.storedDims[a];
    o.d_curr = o.d_prev = nullptr;
    o.ownsDeviceMemory_ = false;
}

ScalarField& ScalarField::operator=(ScalarField&& o) noexcept {
    if (this == &o) return *this;
    freeDevice();
    name = std::move(o.name);
    ghost = o.ghost;
    for (int a = 0; a < 3; ++a) storedDims[a] = o.storedDims[a];
    storedSize = o.storedSize;
    curr = std::move(o.curr);
    prev = std::move(o.prev);
    d_curr = o.d_curr;
    d_prev = o.d_prev;
    ownsDeviceMemory_ = o.ownsDeviceMemory_;
    o.d_curr = o.d_prev = nullptr;
    o.ownsDeviceMemory_ = false;
    return *this;
}

ScalarField::~ScalarField() { freeDevice(); }

void ScalarField::fill(double v) { fillCurr(v); fillPrev(v); }
void ScalarField::fillCurr(double v) { std::fill(curr.begin(), curr.end(), v); }
void ScalarField::fillPrev(double v) { std::fill(prev.begin(), prev.end(), v); }
void ScalarField::advanceTimeLevelCPU() { std::copy(curr.begin(), curr.end(), prev.begin()); }

void ScalarField::advanceTimeLevelGPU() {
    if (!deviceAllocated()) throw std::runtime_error("ScalarField::advanceTimeLevelGPU: device not allocated");
    cuda_check(cudaMemcpy(d_prev, d_curr, storedSize * sizeof(double), cudaMemcpyDeviceToDevice), "advanceTimeLevelGPU");
}

void ScalarField::allocDevice() {
    if (deviceAllocated()) return;
    const std::size_t b = storedSize * sizeof(double);
    cuda_check(cudaMalloc(&d_curr, b), "allocDevice");
    cuda_check(cudaMalloc(&d_prev, b), "allocDevice");
    cuda_check(cudaMemset(d_curr, 0, b), "allocDevice");
    cuda_check(cudaMemset(d_prev, 0, b), "allocDevice");
    ownsDeviceMemory_ = true;
}

void ScalarField::freeDevice() {
    if (ownsDeviceMemory_) {
        if (d_curr) cudaFree(d_curr);
        if (d_prev) cudaFree(d_prev);
    }
    d_curr = d_prev = nullptr;
}

#define PHIX_FIELD_COPY(fn, dst, src, kind, needs)                                           \
    void ScalarField::fn() needs {                                                           \
        if (!deviceAllocated()) throw std::runtime_error("ScalarField::" #fn ": device not allocated"); \
        cuda_check(cudaMemcpy(dst, src, storedSize * sizeof(double), kind), #fn);            \
    }
PHIX_FIELD_COPY(uploadCurrToDevice, d_curr, curr.data(), cudaMemcpyHostToDevice, const)
PHIX_FIELD_COPY(uploadPrevToDevice, d_prev, prev.data(), cudaMemcpyHostToDevice, const)
PHIX_FIELD_COPY(downloadCurrFromDevice, curr.data(), d_curr, cudaMemcpyDeviceToHost, )
PHIX_FIELD_COPY(downloadPrevFromDevice, prev.data(), d_prev, cudaMemcpyDeviceToHost, )
#undef PHIX_FIELD_COPY

void ScalarField::uploadAllToDevice() const { uploadCurrToDevice(); uploadPrevToDevice(); }
void ScalarField::downloadAllFromDevice() { downloadCurrFromDevice(); downloadPrevFromDevice(); }

void ScalarField::write(const std::string& path, FieldFormat fmt) const { IO::writeField(*this, path, fmt); }
ScalarField ScalarField::readFromFile(const Mesh& m, const std::string& path, int g) {
    return IO::readScalarField(m, path, g);
}

void ScalarField::print() const {
    std::cout << "=== ScalarField ===\n  name       : " << name << "\n  ghost      : " << ghost
              << "\n  storedDims : " << storedDims[0] << " x " << storedDims[1] << " x " << storedDims[2] << "  ("
              << storedSize << " cells)\n  device     : " << (deviceAllocated() ? "allocated" : "not allocated")
              << "\n";
    double mn = std::numeric_limits<double>::max(), mx = std::numeric_limits<double>::lowest(), s = 0.0;
    std::size_t cnt = 0;
    for (int k = 0; k < mesh.n[2]; ++k)
        for (int j = 0; j < mesh.n[1]; ++j)
            for (int i = 0; i < mesh.n[0]; ++i) {
                const double v = curr[index(i, j, k)];
                mn = std::min(mn, v);
                mx = std::max(mx, v);
                s += v;
                ++cnt;
            }
    if (cnt)
        std::cout << "  curr  min  : " << mn << "\n  curr  max  : " << mx << "\n  curr  mean : " << s / (double)cnt
                  << "\n";
}

// ---------------------------------------------------------------------------
// VectorField
// ---------------------------------------------------------------------------
VectorField::VectorField(const Mesh& m, const std::string& nm, int nc, int g) : mesh(m), ghost(g), name(nm) {
    if (nc < 1) throw std::invalid_argument("VectorField: nComponents must be >= 1");
    for (int c = 0; c < nc; ++c) components_.push_back(std::make_unique<ScalarField>(m, componentName(nm, c, nc), g));
}

VectorField::VectorField(VectorField&& o) noexcept
    : mesh(o.mesh), ghost(o.ghost), name(std::move(o.name)), components_(std::move(o.components_)) {}

VectorField& VectorField::operator=(VectorField&& o) noexcept {
    if (this != &o) {
        ghost = o.ghost;
        name = std::move(o.name);
        components_ = std::move(o.components_);
    }
    return *this;
}

// 3-component fields name their components <base>_x/_y/_z, others <base>_<c>.
std::string VectorField::componentName(const std::string& base, int c, int nc) {
    if (nc == 3 && c >= 0 && c < 3) return base + (c == 0 ? "_x" : c == 1 ? "_y" : "_z");
    return base + "_" + std::to_string(c);
}

ScalarField& VectorField::operator[](int c) {
    if (c < 0 || c >= nComponents()) throw std::out_of_range("VectorField: component index out of range");
    return *components_[c];
}
const ScalarField& VectorField::operator[](int c) const {
    if (c < 0 || c >= nComponents()) throw std::out_of_range("VectorField: component index out of range");
    return *components_[c];
}

void VectorField::fill(double v) { for (auto& c : components_) c->fill(v); }
void VectorField::fillCurr(double v) { for (auto& c : components_) c->fillCurr(v); }
void VectorField::fillPrev(double v) { for (auto& c : components_) c->fillPrev(v); }
void VectorField::advanceTimeLevelCPU() { for (auto& c : components_) c->advanceTimeLevelCPU(); }
void VectorField::advanceTimeLevelGPU() { for (auto& c : components_) c->advanceTimeLevelGPU(); }
void VectorField::allocDevice() { for (auto& c : components_) c->allocDevice(); }
void VectorField::freeDevice() { for (auto& c : components_) c->freeDevice(); }
void VectorField::uploadAllToDevice() const { for (auto& c : components_) c->uploadAllToDevice(); }
void VectorField::uploadCurrToDevice() const { for (auto& c : components_) c->uploadCurrToDevice(); }
void VectorField::downloadAllFromDevice() { for (auto& c : components_) c->downloadAllFromDevice(); }
void VectorField::downloadCurrFromDevice() { for (auto& c : components_) c->downloadCurrFromDevice(); }
void VectorField::write(const std::string& path, FieldFormat fmt) const { IO::writeField(*this, path, fmt); }
VectorField VectorField::readFromFile(const Mesh& m, const std::string& path, int g) {
    return IO::readVectorField(m, path, g);
}
void VectorField::print() const {
    std::cout << "=== VectorField " << name << " (" << nComponents() << " components) ===\n";
    for (auto& c : components_) c->print();
}

}  // namespace PhiX
