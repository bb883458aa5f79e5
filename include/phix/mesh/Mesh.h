#pragma once
// Mesh -- uniform Cartesian 1/2/3-D grid (API of the reference's
// include/mesh/Mesh.h: n, d, origin, factories, validate, text IO).

#include <cstddef>
#include <stdexcept>
#include <string>

namespace PhiX {

enum class CoordSys { CARTESIAN, CYLINDRICAL, SPHERICAL };

class Mesh {
public:
    int dim;
    CoordSys coordSys;
    int n[3];          // cells per axis (unused axes = 1)
    double d[3];       // spacing
    double origin[3];  // lower corner

    Mesh();
    Mesh(int dim, CoordSys cs, int nx, double dx, double x0, int ny, double dy, double y0, int nz, double dz,
         double z0);

    static Mesh makeUniform1D(CoordSys cs, int nx, double dx, double x0 = 0.0);
    static Mesh makeUniform2D(CoordSys cs, int nx, double dx, double x0, int ny, double dy, double y0);
    static Mesh makeUniform3D(CoordSys cs, int nx, double dx, double x0, int ny, double dy, double y0, int nz,
                              double dz, double z0);

    static Mesh readFromFile(const std::string& path);
    void write(const std::string& path) const;
    void print() const;

    std::size_t totalSize() const { return static_cast<std::size_t>(n[0]) * n[1] * n[2]; }
    double coord(int axis, int i) const { return origin[axis] + (i + 0.5) * d[axis]; }
    int index(int i, int j, int k) const { return i + n[0] * (j + n[1] * k); }
    int index(int i) const { return i; }
    int index(int i, int j) const { return i + n[0] * j; }

    void validate() const;     // throws std::invalid_argument
    bool isValid() const noexcept;
};

std::string coordSysToString(CoordSys cs);
CoordSys stringToCoordSys(const std::string& s);

}  // namespace PhiX
