// io_format.cu -- writes scalar and vector fields in every format through the
// reference's IO API only (IO::writeField / readField, no device calls), so
// that it builds against the reference library and against libphix_cxx.so
// and the two builds' files can be compared byte for byte on a machine
// without a GPU.  Files go to the current directory; the messages of the
// readers' errors go to stdout, one line each, for the same comparison.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <functional>
#include <iterator>
#include <stdexcept>
#include <string>

#include "IO/FieldIO.h"
#include "field/ScalarField.h"
#include "field/VectorField.h"
#include "mesh/Mesh.h"

using namespace PhiX;

// Values with awkward decimal forms: negative, tiny, huge, exact integers.
static double value(int i, int j, int k, int c) {
    const int q = i + 7 * j + 31 * k + 101 * c;
    switch (q % 5) {
        case 0: return std::sin(0.37 * q) * 1e-7;
        case 1: return -std::exp(0.01 * q);
        case 2: return 1.0 / (q + 1.0);
        case 3: return static_cast<double>(q) * 1e12;
        default: return -0.0 + 0.5 * (q % 3);
    }
}

static void fill(ScalarField& f, int c) {
    const Mesh& m = f.mesh;
    for (int k = 0; k < m.n[2]; ++k)
        for (int j = 0; j < m.n[1]; ++j)
            for (int i = 0; i < m.n[0]; ++i) f.curr[f.index(i, j, k)] = value(i, j, k, c);
}

static void expect_error(const char* what, const std::function<void()>& fn) {
    try {
        fn();
        std::printf("%s: no error\n", what);
    } catch (const std::exception& e) {
        std::printf("%s: %s\n", what, e.what());
    }
}

static void truncate_copy(const std::string& from, const std::string& to, long drop) {
    std::ifstream in(from, std::ios::binary);
    std::string bytes((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    std::ofstream(to, std::ios::binary).write(bytes.data(), static_cast<std::streamsize>(bytes.size() - drop));
}

int main() {
    const Mesh m2 = Mesh::makeUniform2D(CoordSys::CARTESIAN, 13, 0.5, -1.0, 7, 0.25, 2.0);
    const Mesh m3 = Mesh::makeUniform3D(CoordSys::CARTESIAN, 5, 1.0, 0.0, 4, 0.5, 1.0, 3, 2.0, -3.0);
    const struct { const Mesh* m; const char* tag; } meshes[2] = {{&m2, "2d"}, {&m3, "3d"}};
    for (const auto& mt : meshes) {
        const std::string t = mt.tag;
        ScalarField s(*mt.m, "s_" + t);
        fill(s, 0);
        IO::writeField(s, "s_" + t + ".field", FieldFormat::BINARY);
        IO::writeField(s, "s_" + t + ".dat", FieldFormat::DAT);
        IO::writeField(s, "s_" + t + ".vts", FieldFormat::VTS);
        // read back through both readers and write again
        ScalarField r = IO::readScalarField(*mt.m, "s_" + t + ".field");
        IO::writeField(r, "rb_" + t + ".field", FieldFormat::BINARY);
        ScalarField d(*mt.m, "d_" + t);
        IO::readField(d, "s_" + t + ".dat");
        IO::writeField(d, "rd_" + t + ".field", FieldFormat::BINARY);

        VectorField v(*mt.m, "v_" + t, 3);
        for (int c = 0; c < 3; ++c) fill(v[c], c + 1);
        IO::writeField(v, "v_" + t + ".vfield", FieldFormat::BINARY);
        IO::writeField(v, "v_" + t + ".dat", FieldFormat::DAT);
        IO::writeField(v, "v_" + t + ".vts", FieldFormat::VTS);
        VectorField w = IO::readVectorField(*mt.m, "v_" + t + ".vfield");
        IO::writeField(w, "rv_" + t + ".vfield", FieldFormat::BINARY);
        VectorField wd = IO::readVectorField(*mt.m, "v_" + t + ".dat");
        IO::writeField(wd, "rvd_" + t + ".vfield", FieldFormat::BINARY);
        VectorField u(*mt.m, "u_" + t, 3);
        IO::readField(u, "v_" + t + ".dat");
        IO::writeField(u, "ru_" + t + ".vfield", FieldFormat::BINARY);
    }
    // error paths
    const Mesh other = Mesh::makeUniform2D(CoordSys::CARTESIAN, 12, 0.5, -1.0, 7, 0.25, 2.0);
    ScalarField so(other, "so");
    VectorField vo(other, "vo", 3), v2(m2, "v2", 2);
    truncate_copy("s_2d.field", "cut.field", 8);
    truncate_copy("v_2d.vfield", "cut.vfield", 8);
    truncate_copy("s_2d.dat", "cut.dat", 40);
    expect_error("readScalarField mesh", [&] { IO::readScalarField(other, "s_2d.field"); });
    expect_error("readScalarField dat mesh", [&] { IO::readScalarField(other, "s_2d.dat"); });
    expect_error("readField mesh", [&] { IO::readField(so, "s_2d.field"); });
    expect_error("readField dat mesh", [&] { IO::readField(so, "s_2d.dat"); });
    expect_error("readScalarField truncated", [&] { IO::readScalarField(m2, "cut.field"); });
    expect_error("readScalarField dat truncated", [&] { IO::readScalarField(m2, "cut.dat"); });
    expect_error("readVectorField mesh", [&] { IO::readVectorField(other, "v_2d.vfield"); });
    expect_error("readVectorField truncated", [&] { IO::readVectorField(m2, "cut.vfield"); });
    expect_error("readField vector ncomp", [&] { IO::readField(v2, "v_2d.vfield"); });
    expect_error("readField vector mesh", [&] { IO::readField(vo, "v_2d.vfield"); });
    expect_error("readField vector dat ncomp", [&] { IO::readField(v2, "v_2d.dat"); });
    expect_error("readScalarField missing", [&] { IO::readScalarField(m2, "no_such.field"); });
    expect_error("writeField unopenable", [&] { IO::writeField(so, "no_such_dir/x.field", FieldFormat::BINARY); });
    std::printf("io_format done\n");
    return 0;
}
