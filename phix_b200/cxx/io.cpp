// io.cpp -- FieldIO, ConfigFile and OutputWriter of the drop-in C++ API.
// The .field / .vfield binary formats are byte-compatible with the
// reference's (src/IO/FieldIO.cpp:207-235, :318-347).
#include <algorithm>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <vector>

#include "IO/ConfigFile.h"
#include "IO/FieldIO.h"
#include "IO/OutputWriter.h"
#include "field/ScalarField.h"
#include "field/VectorField.h"

namespace PhiX {
namespace IO {

namespace {

struct Header {
    std::string name;
    int nx = 1, ny = 1, nz = 1, ghost = 1, ncomp = 1;
};

bool is_dat(std::ifstream& in) {
    std::string line;
    std::getline(in, line);
    in.clear();
    in.seekg(0);
    return line.find("- DAT") != std::string::npos;
}

Header parse_binary_header(std::ifstream& in, const std::string& path) {
    Header h;
    std::string line;
    bool done = false;
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line == "---") { done = true; break; }
        std::istringstream ss(line);
        std::string tok;
        while (ss >> tok) {
            if (tok[0] == '#') break;
            if (tok == "name") ss >> h.name;
            else if (tok == "ghost") ss >> h.ghost;
            else if (tok == "nComponents") ss >> h.ncomp;
            else if (tok == "nx") ss >> h.nx;
            else if (tok == "ny") ss >> h.ny;
            else if (tok == "nz") ss >> h.nz;
        }
    }
    if (!done) throw std::runtime_error("IO: missing '---' header terminator in " + path);
    return h;
}

Header parse_dat_header(std::ifstream& in) {
    Header h;
    std::string line;
    std::streampos pos = in.tellg();
    while (std::getline(in, line)) {
        if (line.empty() || line[0] != '#') {
            in.clear();
            in.seekg(pos);
            break;
        }
        pos = in.tellg();
        std::istringstream ss(line.substr(1));
        std::string tok;
        while (ss >> tok) {
            if (tok == "name:") ss >> h.name;
            else if (tok == "nx") ss >> h.nx;
            else if (tok == "ny") ss >> h.ny;
            else if (tok == "nz") ss >> h.nz;
        }
    }
    return h;
}

void check_dims(const Header& h, const Mesh& m, const char* who) {
    if (h.nx != m.n[0] || h.ny != m.n[1] || h.nz != m.n[2])
        throw std::runtime_error(std::string(who) + ": mesh dimensions in file (" + std::to_string(h.nx) + "x" +
                                 std::to_string(h.ny) + "x" + std::to_string(h.nz) + ") do not match provided mesh (" +
                                 std::to_string(m.n[0]) + "x" + std::to_string(m.n[1]) + "x" + std::to_string(m.n[2]) +
                                 ")");
}

void gather(const ScalarField& f, std::vector<double>& buf) {
    buf.clear();
    buf.reserve(f.mesh.totalSize());
    for (int k = 0; k < f.mesh.n[2]; ++k)
        for (int j = 0; j < f.mesh.n[1]; ++j)
            for (int i = 0; i < f.mesh.n[0]; ++i) buf.push_back(f.curr[f.index(i, j, k)]);
}

void scatter(ScalarField& f, const std::vector<double>& buf) {
    std::size_t q = 0;
    for (int k = 0; k < f.mesh.n[2]; ++k)
        for (int j = 0; j < f.mesh.n[1]; ++j)
            for (int i = 0; i < f.mesh.n[0]; ++i) f.curr[f.index(i, j, k)] = buf[q++];
}

void read_phys(std::ifstream& in, std::vector<double>& buf, std::size_t n, const std::string& path) {
    buf.resize(n);
    in.read(reinterpret_cast<char*>(buf.data()), static_cast<std::streamsize>(n * sizeof(double)));
    if (!in) throw std::runtime_error("IO: unexpected end of binary data in " + path);
}

void read_dat_values(std::ifstream& in, ScalarField* const* f, int nf, const std::string& path) {
    std::string line;
    const Mesh& m = f[0]->mesh;
    for (int k = 0; k < m.n[2]; ++k)
        for (int j = 0; j < m.n[1]; ++j)
            for (int i = 0; i < m.n[0]; ++i) {
                if (!std::getline(in, line)) throw std::runtime_error("IO: unexpected end of DAT data in " + path);
                std::istringstream ss(line);
                double x, y, z;
                if (!(ss >> x >> y >> z)) throw std::runtime_error("IO: malformed DAT line in " + path);
                for (int c = 0; c < nf; ++c)
                    if (!(ss >> f[c]->curr[f[c]->index(i, j, k)]))
                        throw std::runtime_error("IO: malformed DAT line in " + path);
            }
}

}  // namespace

void writeField(const ScalarField& f, const std::string& path, FieldFormat fmt) {
    const Mesh& m = f.mesh;
    if (fmt == FieldFormat::BINARY) {
        std::ofstream o(path, std::ios::binary);
        if (!o) throw std::runtime_error("IO::writeField: cannot open file: " + path);
        o << "# PhiX ScalarField\nname    " << f.name << "\nnx " << m.n[0] << "  ny " << m.n[1] << "  nz " << m.n[2]
          << "\nghost   " << f.ghost << "\n---\n";
        std::vector<double> buf;
        gather(f, buf);
        o.write(reinterpret_cast<const char*>(buf.data()), static_cast<std::streamsize>(buf.size() * sizeof(double)));
        return;
    }
    std::ofstream o(path);
    if (!o) throw std::runtime_error("IO::writeField: cannot open file: " + path);
    if (fmt == FieldFormat::DAT) {
        o << "# PhiX ScalarField - DAT\n# name: " << f.name << "\n# nx " << m.n[0] << "  ny " << m.n[1] << "  nz "
          << m.n[2] << "\n# x y z value\n";
        o << std::scientific << std::setprecision(12);
        for (int k = 0; k < m.n[2]; ++k)
            for (int j = 0; j < m.n[1]; ++j)
                for (int i = 0; i < m.n[0]; ++i)
                    o << m.coord(0, i) << "  " << m.coord(1, j) << "  " << m.coord(2, k) << "  "
                      << f.curr[f.index(i, j, k)] << "\n";
        return;
    }
    // VTS: corner-node grid + cell data, ASCII
    o << "<?xml version=\"1.0\"?>\n<VTKFile type=\"StructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
      << "  <StructuredGrid WholeExtent=\"0 " << m.n[0] << " 0 " << m.n[1] << " 0 " << m.n[2] << "\">\n"
      << "    <Piece Extent=\"0 " << m.n[0] << " 0 " << m.n[1] << " 0 " << m.n[2] << "\">\n"
      << "      <Points>\n        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    o << std::scientific << std::setprecision(12);
    for (int k = 0; k <= m.n[2]; ++k)
        for (int j = 0; j <= m.n[1]; ++j)
            for (int i = 0; i <= m.n[0]; ++i)
                o << "          " << m.origin[0] + i * m.d[0] << " " << m.origin[1] + j * m.d[1] << " "
                  << m.origin[2] + k * m.d[2] << "\n";
    o << "        </DataArray>\n      </Points>\n      <CellData Scalars=\"" << f.name
      << "\">\n        <DataArray type=\"Float64\" Name=\"" << f.name << "\" format=\"ascii\">\n";
    for (int k = 0; k < m.n[2]; ++k)
        for (int j = 0; j < m.n[1]; ++j)
            for (int i = 0; i < m.n[0]; ++i) o << "          " << f.curr[f.index(i, j, k)] << "\n";
    o << "        </DataArray>\n      </CellData>\n    </Piece>\n  </StructuredGrid>\n</VTKFile>\n";
}

ScalarField readScalarField(const Mesh& mesh, const std::string& path, int ghost) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("IO::readScalarField: cannot open file: " + path);
    if (is_dat(in)) {
        const Header h = parse_dat_header(in);
        check_dims(h, mesh, "IO::readScalarField");
        ScalarField f(mesh, h.name.empty() ? "field" : h.name, ghost);
        ScalarField* fs[1] = {&f};
        read_dat_values(in, fs, 1, path);
        return f;
    }
    const Header h = parse_binary_header(in, path);
    check_dims(h, mesh, "IO::readScalarField");
    ScalarField f(mesh, h.name, ghost);
    std::vector<double> buf;
    read_phys(in, buf, mesh.totalSize(), path);
    scatter(f, buf);
    return f;
}

void readField(ScalarField& f, const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("IO::readField: cannot open file: " + path);
    if (is_dat(in)) {
        const Header h = parse_dat_header(in);
        check_dims(h, f.mesh, "IO::readField");
        ScalarField* fs[1] = {&f};
        read_dat_values(in, fs, 1, path);
        return;
    }
    const Header h = parse_binary_header(in, path);
    check_dims(h, f.mesh, "IO::readField");
    std::vector<double> buf;
    read_phys(in, buf, f.mesh.totalSize(), path);
    scatter(f, buf);
}

void writeField(const VectorField& vf, const std::string& path, FieldFormat fmt) {
    const Mesh& m = vf.mesh;
    if (fmt == FieldFormat::BINARY) {
        std::ofstream o(path, std::ios::binary);
        if (!o) throw std::runtime_error("IO::writeField: cannot open file: " + path);
        o << "# PhiX VectorField\nname         " << vf.name << "\nnComponents  " << vf.nComponents() << "\nnx "
          << m.n[0] << "  ny " << m.n[1] << "  nz " << m.n[2] << "\nghost        " << vf.ghost << "\n---\n";
        std::vector<double> buf;
        for (int c = 0; c < vf.nComponents(); ++c) {
            gather(vf[c], buf);
            o.write(reinterpret_cast<const char*>(buf.data()), static_cast<std::streamsize>(buf.size() * sizeof(double)));
        }
        return;
    }
    for (int c = 0; c < vf.nComponents(); ++c) {
        const std::string ext = fmt == FieldFormat::DAT ? ".dat" : ".vts";
        std::string base = path;
        if (base.size() > ext.size() && base.compare(base.size() - ext.size(), ext.size(), ext) == 0)
            base.resize(base.size() - ext.size());
        writeField(vf[c], base + "_" + std::to_string(c) + ext, fmt);
    }
}

VectorField readVectorField(const Mesh& mesh, const std::string& path, int ghost) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("IO::readVectorField: cannot open file: " + path);
    const Header h = parse_binary_header(in, path);
    check_dims(h, mesh, "IO::readVectorField");
    VectorField vf(mesh, h.name, h.ncomp, ghost);
    std::vector<double> buf;
    for (int c = 0; c < h.ncomp; ++c) {
        read_phys(in, buf, mesh.totalSize(), path);
        scatter(vf[c], buf);
    }
    return vf;
}

void readField(VectorField& vf, const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("IO::readField: cannot open file: " + path);
    const Header h = parse_binary_header(in, path);
    check_dims(h, vf.mesh, "IO::readField");
    if (h.ncomp != vf.nComponents()) throw std::runtime_error("IO::readField: component count mismatch in " + path);
    std::vector<double> buf;
    for (int c = 0; c < h.ncomp; ++c) {
        read_phys(in, buf, vf.mesh.totalSize(), path);
        scatter(vf[c], buf);
    }
}

int resolveStartStep(const std::string& startFrom, const std::string& ref) {
    if (startFrom == "initial_field") return 0;
    const int target = std::stoi(startFrom);
    const std::string prefix = ref + "_";
    std::vector<int> steps;
    namespace fs = std::filesystem;
    if (fs::is_directory("output"))
        for (const auto& e : fs::directory_iterator("output")) {
            const fs::path p = e.path();
            if (p.extension() != ".field") continue;
            const std::string stem = p.stem().string();
            if (stem.rfind(prefix, 0) != 0) continue;
            try {
                steps.push_back(std::stoi(stem.substr(prefix.size())));
            } catch (...) {
            }
        }
    if (steps.empty())
        throw std::runtime_error("IO::resolveStartStep: start_from=\"" + startFrom + "\" but no " + prefix +
                                 "*.field files found in output/");
    return *std::min_element(steps.begin(), steps.end(),
                             [target](int a, int b) { return std::abs(a - target) < std::abs(b - target); });
}

void initField(ScalarField& f, int startStep) {
    const std::string path = startStep == 0 ? "settings/initial_field/" + f.name + ".field"
                                            : "output/" + f.name + "_" + std::to_string(startStep) + ".field";
    std::cout << (startStep == 0 ? "  cold start: loading " : "  warm start: loading ") << path << "\n";
    readField(f, path);
}

// ---------------------------------------------------------------------------
// ConfigFile: `//` comments outside strings are stripped, then JSON.
// ---------------------------------------------------------------------------
std::string ConfigFile::stripLineComment(const std::string& line) {
    bool str = false;
    for (std::size_t i = 0; i < line.size(); ++i) {
        const char c = line[i];
        if (str) {
            if (c == '\\') ++i;
            else if (c == '"') str = false;
        } else if (c == '"') {
            str = true;
        } else if (c == '/' && i + 1 < line.size() && line[i + 1] == '/') {
            return line.substr(0, i);
        }
    }
    return line;
}

ConfigFile::ConfigFile(const std::string& path) {
    std::ifstream in(path);
    if (!in.is_open()) throw std::runtime_error("ConfigFile: cannot open \"" + path + "\"");
    std::ostringstream s;
    std::string line;
    while (std::getline(in, line)) s << stripLineComment(line) << '\n';
    try {
        data_ = nlohmann::json::parse(s.str());
    } catch (const nlohmann::json::parse_error& e) {
        throw std::runtime_error("ConfigFile: JSON parse error in \"" + path + "\": " + e.what());
    }
}

ConfigFile ConfigFile::fromArgs(int argc, char* argv[], const std::string& defaultPath) {
    const std::string path = argc >= 2 ? argv[1] : defaultPath;
    try {
        return ConfigFile(path);
    } catch (const std::exception& e) {
        std::cerr << e.what() << "\n  Usage: " << argv[0] << " [path/to/settings.jsonc]\n";
        std::exit(1);
    }
}

const nlohmann::json& ConfigFile::operator[](const std::string& key) const { return data_.at(key); }
bool ConfigFile::has(const std::string& key) const { return data_.contains(key); }

// ---------------------------------------------------------------------------
// OutputWriter
// ---------------------------------------------------------------------------
OutputWriter::OutputWriter(const nlohmann::json& c)
    : printInterval(c.at("print_interval").get<int>()), writeInterval(c.at("write_interval").get<int>()) {
    const std::string fmt = c.at("format").get<std::string>();
    writeBinary_ = fmt == "BINARY" || fmt == "ALL";
    writeDat_ = fmt == "DAT" || fmt == "ALL";
    writeVtk_ = fmt == "VTK" || fmt == "ALL";
    std::filesystem::create_directories("output");
    resetTimer();
}

void OutputWriter::writeFields(ScalarField& f, int step, double simTime) {
    f.downloadCurrFromDevice();
    const std::string base = "output/" + f.name + "_" + std::to_string(step);
    if (writeBinary_) writeField(f, base + ".field", FieldFormat::BINARY);
    if (writeDat_) writeField(f, base + ".dat", FieldFormat::DAT);
    if (writeVtk_) writeField(f, base + ".vts", FieldFormat::VTS);
    std::cout << "  step " << step << "  t=" << simTime << "  written: " << base << "\n" << std::flush;
}

void OutputWriter::printProgress(int step, double simTime) {
    const double el = std::chrono::duration<double>(Clock::now() - t_start_).count();
    std::cout << "  [progress] step=" << step << "  t=" << simTime << "  elapsed=" << std::fixed
              << std::setprecision(1) << el << "s\n"
              << std::flush;
}

void OutputWriter::resetTimer() { t_start_ = Clock::now(); }

}  // namespace IO
}  // namespace PhiX
