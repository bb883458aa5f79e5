// io.cpp -- FieldIO, ConfigFile and OutputWriter of the drop-in C++ API.
// The .field / .vfield binary formats are byte-compatible with the
// reference's (src/IO/FieldIO.cpp:207-235, :318-347).  OutputWriter writes
// the same files as the reference's (src/IO/OutputWriter.cpp:24-33) but off
// the solver's critical path: device snapshot, side-stream download into
// pinned memory, worker-thread formatting.
#include <algorithm>
#include <condition_variable>
#include <deque>
#include <exception>
#include <mutex>
#include <thread>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <vector>

#include <cuda_runtime.h>

#include "IO/ConfigFile.h"
#include "IO/FieldIO.h"
#include "IO/OutputWriter.h"
#include "field/ScalarField.h"
#include "field/VectorField.h"

namespace PhiX {
namespace IO {

namespace {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

struct Header {
    std::string name;
    int nx = 0, ny = 0, nz = 0, ghost = 0, ncomp = 0;
};

bool is_dat(std::ifstream& in) {
    std::string line;
    std::getline(in, line);
    in.clear();
    in.seekg(0);
    return line.find("- DAT") != std::string::npos;
}

void chomp(std::string& line) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
}

// BINARY header: "key value" lines up to "---", '#' lines are comments, and
// nx / ny / nz may share one line (src/IO/FieldIO.cpp:51-112).
Header parse_binary_header(std::ifstream& in, const std::string& path) {
    Header h;
    std::string line;
    bool done = false;
    while (std::getline(in, line)) {
        chomp(line);
        if (line == "---") {
            done = true;
            break;
        }
        std::istringstream ss(line);
        std::string tok;
        if (!(ss >> tok) || tok[0] == '#') continue;
        if (tok == "name") ss >> h.name;
        else if (tok == "ghost") ss >> h.ghost;
        else if (tok == "nComponents") ss >> h.ncomp;
        else
            for (std::istringstream row(line); row >> tok;) {
                if (tok == "nx") row >> h.nx;
                else if (tok == "ny") row >> h.ny;
                else if (tok == "nz") row >> h.nz;
            }
    }
    if (!done) throw std::runtime_error("IO: missing '---' header terminator in " + path);
    return h;
}

// DAT header: the leading '#' lines; the stream is left at the first data
// line (src/IO/FieldIO.cpp:127-199).
Header parse_dat_header(std::ifstream& in) {
    Header h;
    std::string line;
    for (;;) {
        const std::streampos pos = in.tellg();
        if (!std::getline(in, line)) break;
        chomp(line);
        if (line.empty() || line[0] != '#') {
            in.seekg(pos);
            break;
        }
        std::istringstream row(line.substr(1));
        for (std::string tok; row >> tok;) {
            if (tok == "name:") row >> h.name;
            else if (tok == "nComponents:") row >> h.ncomp;
            else if (tok == "nx") row >> h.nx;
            else if (tok == "ny") row >> h.ny;
            else if (tok == "nz") row >> h.nz;
        }
    }
    return h;
}

std::string dims(int x, int y, int z) { return std::to_string(x) + "x" + std::to_string(y) + "x" + std::to_string(z); }

bool same_dims(const Header& h, const Mesh& m) { return h.nx == m.n[0] && h.ny == m.n[1] && h.nz == m.n[2]; }

// The reference's two wordings of a dimension mismatch for scalar files.
void check_mesh(const Header& h, const Mesh& m) {
    if (!same_dims(h, m))
        throw std::runtime_error("IO::readScalarField: mesh dimensions in file (" + dims(h.nx, h.ny, h.nz) +
                                 ") do not match provided mesh (" + dims(m.n[0], m.n[1], m.n[2]) + ")");
}

void check_field(const Header& h, const ScalarField& f) {
    if (!same_dims(h, f.mesh))
        throw std::runtime_error("IO::readField: file dimensions (" + dims(h.nx, h.ny, h.nz) + ") do not match field \"" +
                                 f.name + "\" mesh (" + dims(f.mesh.n[0], f.mesh.n[1], f.mesh.n[2]) + ")");
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

// BINARY payload of a scalar file: the physical cells, x fastest.
void read_block(std::ifstream& in, ScalarField& f, const std::string& path, const char* msg) {
    std::vector<double> buf(f.mesh.totalSize());
    in.read(reinterpret_cast<char*>(buf.data()), static_cast<std::streamsize>(buf.size() * sizeof(double)));
    if (!in) throw std::runtime_error(msg + path);
    scatter(f, buf);
}

// BINARY payload of a vector file: one such block per component.
void read_vector_blocks(std::ifstream& in, ScalarField* const* f, int nf, const std::string& path, const char* who) {
    std::vector<double> buf(f[0]->mesh.totalSize());
    for (int c = 0; c < nf; ++c) {
        in.read(reinterpret_cast<char*>(buf.data()), static_cast<std::streamsize>(buf.size() * sizeof(double)));
        if (!in)
            throw std::runtime_error(std::string(who) + ": unexpected end of data for component " + std::to_string(c) +
                                     " in " + path);
        scatter(*f[c], buf);
    }
}

// DAT payload: one "x y z v0 [v1 ...]" line per physical cell.
void read_dat_values(std::ifstream& in, ScalarField* const* f, int nf, const std::string& path, const char* who) {
    std::string line;
    const Mesh& m = f[0]->mesh;
    for (int k = 0; k < m.n[2]; ++k)
        for (int j = 0; j < m.n[1]; ++j)
            for (int i = 0; i < m.n[0]; ++i) {
                if (!std::getline(in, line))
                    throw std::runtime_error(std::string(who) + ": unexpected end of DAT data in " + path);
                chomp(line);
                std::istringstream ss(line);
                double x, y, z;
                if (!(ss >> x >> y >> z)) throw std::runtime_error(std::string(who) + ": malformed DAT line in " + path);
                for (int c = 0; c < nf; ++c)
                    if (!(ss >> f[c]->curr[f[c]->index(i, j, k)]))
                        throw std::runtime_error(std::string(who) +
                                                 (nf == 1 ? ": malformed DAT line in "
                                                          : ": missing component " + std::to_string(c) +
                                                                " in DAT line in ") +
                                                 path);
            }
}

// VTS: XML head and the corner-node grid, shared by scalar and vector files.
void vts_head(std::ofstream& o, const Mesh& m) {
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
    o << "        </DataArray>\n      </Points>\n";
}

void vts_tail(std::ofstream& o, const std::string& path) {
    o << "        </DataArray>\n      </CellData>\n    </Piece>\n  </StructuredGrid>\n</VTKFile>\n";
    if (!o) throw std::runtime_error("IO::writeField: write failed: " + path);
}

}  // namespace

// The physical cells of a field, x fastest, formatted as the reference's
// writeField does (src/IO/FieldIO.cpp:207-312).  `phys` holds
// mesh.totalSize() values; both the synchronous writeField and the
// asynchronous OutputWriter format through this one function, so their
// files are the same bytes.
static void write_scalar_cells(const std::string& name, const Mesh& m, int ghost, const double* phys,
                               const std::string& path, FieldFormat fmt) {
    const std::size_t N = m.totalSize();
    if (fmt == FieldFormat::BINARY) {
        std::ofstream o(path, std::ios::binary);
        if (!o) throw std::runtime_error("IO::writeField: cannot open file: " + path);
        o << "# PhiX ScalarField\nname    " << name << "\nnx " << m.n[0] << "  ny " << m.n[1] << "  nz " << m.n[2]
          << "\nghost   " << ghost << "\n---\n";
        o.write(reinterpret_cast<const char*>(phys), static_cast<std::streamsize>(N * sizeof(double)));
        if (!o) throw std::runtime_error("IO::writeField: write failed: " + path);
        return;
    }
    std::ofstream o(path);
    if (!o) throw std::runtime_error("IO::writeField: cannot open file: " + path);
    std::size_t q = 0;
    if (fmt == FieldFormat::DAT) {
        o << "# PhiX ScalarField - DAT\n# name: " << name << "\n# nx " << m.n[0] << "  ny " << m.n[1] << "  nz "
          << m.n[2] << "\n# x y z value\n";
        o << std::scientific << std::setprecision(12);
        for (int k = 0; k < m.n[2]; ++k)
            for (int j = 0; j < m.n[1]; ++j)
                for (int i = 0; i < m.n[0]; ++i)
                    o << m.coord(0, i) << "  " << m.coord(1, j) << "  " << m.coord(2, k) << "  " << phys[q++] << "\n";
        if (!o) throw std::runtime_error("IO::writeField: write failed: " + path);
        return;
    }
    vts_head(o, m);
    o << "      <CellData Scalars=\"" << name << "\">\n        <DataArray type=\"Float64\" Name=\"" << name
      << "\" format=\"ascii\">\n";
    for (; q < N; ++q) o << "          " << phys[q] << "\n";
    vts_tail(o, path);
}

void writeField(const ScalarField& f, const std::string& path, FieldFormat fmt) {
    std::vector<double> buf;
    gather(f, buf);
    write_scalar_cells(f.name, f.mesh, f.ghost, buf.data(), path, fmt);
}

ScalarField readScalarField(const Mesh& mesh, const std::string& path, int ghost) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("IO::readScalarField: cannot open file: " + path);
    const bool dat = is_dat(in);
    const Header h = dat ? parse_dat_header(in) : parse_binary_header(in, path);
    check_mesh(h, mesh);
    ScalarField f(mesh, dat && h.name.empty() ? "field" : h.name, ghost);
    ScalarField* fs[1] = {&f};
    if (dat) read_dat_values(in, fs, 1, path, "IO::readScalarField");
    else read_block(in, f, path, "IO::readScalarField: unexpected end of binary data in ");
    return f;
}

void readField(ScalarField& f, const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("IO::readField: cannot open file: " + path);
    const bool dat = is_dat(in);
    const Header h = dat ? parse_dat_header(in) : parse_binary_header(in, path);
    check_field(h, f);
    ScalarField* fs[1] = {&f};
    if (dat) read_dat_values(in, fs, 1, path, "IO::readField");
    else read_block(in, f, path, "IO::readField: unexpected end of binary data in ");
}

// Vector files (src/IO/FieldIO.cpp:318-440): BINARY holds the components one
// after the other; DAT and VTS interleave them per cell in one file, VTS
// padded with zeros to three components.
void writeField(const VectorField& vf, const std::string& path, FieldFormat fmt) {
    const Mesh& m = vf.mesh;
    const int nc = vf.nComponents();
    if (fmt == FieldFormat::BINARY) {
        std::ofstream o(path, std::ios::binary);
        if (!o) throw std::runtime_error("IO::writeField: cannot open file: " + path);
        o << "# PhiX VectorField\nname         " << vf.name << "\nnComponents  " << nc << "\nnx " << m.n[0]
          << "  ny " << m.n[1] << "  nz " << m.n[2] << "\nghost        " << vf.ghost << "\n---\n";
        std::vector<double> buf;
        for (int c = 0; c < nc; ++c) {
            gather(vf[c], buf);
            o.write(reinterpret_cast<const char*>(buf.data()), static_cast<std::streamsize>(buf.size() * sizeof(double)));
        }
        if (!o) throw std::runtime_error("IO::writeField: write failed: " + path);
        return;
    }
    std::ofstream o(path);
    if (!o) throw std::runtime_error("IO::writeField: cannot open file: " + path);
    if (fmt == FieldFormat::DAT) {
        o << "# PhiX VectorField - DAT\n# name: " << vf.name << "  nComponents: " << nc << "\n# nx " << m.n[0]
          << "  ny " << m.n[1] << "  nz " << m.n[2] << "\n# x y z";
        for (int c = 0; c < nc; ++c) o << " v" << c;
        o << "\n" << std::scientific << std::setprecision(12);
        for (int k = 0; k < m.n[2]; ++k)
            for (int j = 0; j < m.n[1]; ++j)
                for (int i = 0; i < m.n[0]; ++i) {
                    o << m.coord(0, i) << "  " << m.coord(1, j) << "  " << m.coord(2, k);
                    for (int c = 0; c < nc; ++c) o << "  " << vf[c].curr[vf[c].index(i, j, k)];
                    o << "\n";
                }
        if (!o) throw std::runtime_error("IO::writeField: write failed: " + path);
        return;
    }
    const int vtk_nc = nc <= 3 ? 3 : nc;
    vts_head(o, m);
    o << "      <CellData Vectors=\"" << vf.name << "\">\n        <DataArray type=\"Float64\" Name=\"" << vf.name
      << "\" NumberOfComponents=\"" << vtk_nc << "\" format=\"ascii\">\n";
    for (int k = 0; k < m.n[2]; ++k)
        for (int j = 0; j < m.n[1]; ++j)
            for (int i = 0; i < m.n[0]; ++i) {
                o << "         ";
                for (int c = 0; c < nc; ++c) o << " " << vf[c].curr[vf[c].index(i, j, k)];
                for (int c = nc; c < vtk_nc; ++c) o << " 0.0";
                o << "\n";
            }
    vts_tail(o, path);
}

VectorField readVectorField(const Mesh& mesh, const std::string& path, int ghost) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("IO::readVectorField: cannot open file: " + path);
    const bool dat = is_dat(in);
    const Header h = dat ? parse_dat_header(in) : parse_binary_header(in, path);
    if (h.ncomp <= 0) throw std::runtime_error("IO::readVectorField: invalid nComponents in " + path);
    if (!same_dims(h, mesh)) throw std::runtime_error("IO::readVectorField: mesh mismatch in " + path);
    VectorField vf(mesh, dat && h.name.empty() ? "field" : h.name, h.ncomp, ghost);
    std::vector<ScalarField*> fs;
    for (int c = 0; c < h.ncomp; ++c) fs.push_back(&vf[c]);
    if (dat) read_dat_values(in, fs.data(), h.ncomp, path, "IO::readVectorField");
    else read_vector_blocks(in, fs.data(), h.ncomp, path, "IO::readVectorField");
    return vf;
}

void readField(VectorField& vf, const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("IO::readField: cannot open file: " + path);
    const bool dat = is_dat(in);
    const Header h = dat ? parse_dat_header(in) : parse_binary_header(in, path);
    if (h.ncomp != vf.nComponents())
        throw std::runtime_error("IO::readField: file nComponents (" + std::to_string(h.ncomp) +
                                 ") does not match field \"" + vf.name + "\" nComponents (" +
                                 std::to_string(vf.nComponents()) + ")");
    if (!same_dims(h, vf.mesh))
        throw std::runtime_error("IO::readField: mesh mismatch for field \"" + vf.name + "\" in " + path);
    std::vector<ScalarField*> fs;
    for (int c = 0; c < h.ncomp; ++c) fs.push_back(&vf[c]);
    if (dat) read_dat_values(in, fs.data(), h.ncomp, path, "IO::readField");
    else read_vector_blocks(in, fs.data(), h.ncomp, path, "IO::readField");
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

// Snapshots in flight.  Each slot holds one field's physical cells: packed on
// the device by a strided copy on the legacy default stream (which orders it
// after every solver launch and keeps the next steps from overwriting the
// cells before they are copied), downloaded on a non-blocking side stream
// into pinned memory, then written by the worker thread.  The solver's next
// launches run while the download and the file writes proceed.
struct OutputWriter::Async {
    struct Slot {
        double* dev = nullptr;   // packed physical cells (device)
        double* host = nullptr;  // pinned copy of dev
        std::size_t cap = 0;     // doubles
        cudaEvent_t packed = nullptr;
        cudaEvent_t landed = nullptr;
        bool busy = false;
    };
    struct Job {
        int slot;
        std::string name;
        Mesh mesh;
        int ghost;
        std::string base;
    };

    int device = 0;
    bool bin, dat, vtk;
    cudaStream_t side = nullptr;
    std::vector<Slot> slots;
    std::deque<Job> jobs;
    int running = 0;  // jobs taken by the worker and not finished
    bool stop = false;
    std::exception_ptr error;
    std::mutex m;
    std::condition_variable wake;  // worker: a job or stop
    std::condition_variable freed;  // writer: a slot freed or a job finished
    std::thread worker;

    Async(int nslots, bool b, bool d, bool v) : bin(b), dat(d), vtk(v), slots(static_cast<std::size_t>(nslots)) {
        cuda_check(cudaGetDevice(&device), "OutputWriter");
        cuda_check(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking), "OutputWriter: stream");
        for (auto& sl : slots) {
            cuda_check(cudaEventCreateWithFlags(&sl.packed, cudaEventDisableTiming), "OutputWriter: event");
            cuda_check(cudaEventCreateWithFlags(&sl.landed, cudaEventDisableTiming | cudaEventBlockingSync),
                       "OutputWriter: event");
        }
        worker = std::thread([this] { run(); });
    }

    ~Async() {
        {
            std::lock_guard<std::mutex> lk(m);
            stop = true;
        }
        wake.notify_all();
        if (worker.joinable()) worker.join();
        cudaStreamSynchronize(side);
        for (auto& sl : slots) {
            if (sl.dev) cudaFree(sl.dev);
            if (sl.host) cudaFreeHost(sl.host);
            if (sl.packed) cudaEventDestroy(sl.packed);
            if (sl.landed) cudaEventDestroy(sl.landed);
        }
        if (side) cudaStreamDestroy(side);
    }

    // Worker: waits for each snapshot to land in pinned memory, writes its
    // files, frees the slot.  The first error is kept for the writer thread.
    void run() {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lk(m);
        for (;;) {
            wake.wait(lk, [this] { return stop || !jobs.empty(); });
            if (jobs.empty()) return;  // stop, nothing left
            Job job = std::move(jobs.front());
            jobs.pop_front();
            ++running;
            lk.unlock();
            std::exception_ptr err;
            try {
                Slot& sl = slots[static_cast<std::size_t>(job.slot)];
                cuda_check(cudaEventSynchronize(sl.landed), "OutputWriter: download");
                if (bin) write_scalar_cells(job.name, job.mesh, job.ghost, sl.host, job.base + ".field", FieldFormat::BINARY);
                if (dat) write_scalar_cells(job.name, job.mesh, job.ghost, sl.host, job.base + ".dat", FieldFormat::DAT);
                if (vtk) write_scalar_cells(job.name, job.mesh, job.ghost, sl.host, job.base + ".vts", FieldFormat::VTS);
            } catch (...) {
                err = std::current_exception();
            }
            lk.lock();
            if (err && !error) error = err;
            slots[static_cast<std::size_t>(job.slot)].busy = false;
            --running;
            freed.notify_all();
        }
    }

    void rethrow() {
        std::exception_ptr e;
        {
            std::lock_guard<std::mutex> lk(m);
            std::swap(e, error);
        }
        if (e) std::rethrow_exception(e);
    }

    void drain() {
        std::unique_lock<std::mutex> lk(m);
        freed.wait(lk, [this] { return jobs.empty() && running == 0; });
    }

    // A free slot with room for n doubles (waits for the worker if all are busy).
    int acquire(std::size_t n) {
        int s = -1;
        {
            std::unique_lock<std::mutex> lk(m);
            freed.wait(lk, [this] {
                for (auto& sl : slots)
                    if (!sl.busy) return true;
                return false;
            });
            for (std::size_t i = 0; i < slots.size(); ++i)
                if (!slots[i].busy) {
                    s = static_cast<int>(i);
                    break;
                }
            slots[static_cast<std::size_t>(s)].busy = true;
        }
        Slot& sl = slots[static_cast<std::size_t>(s)];
        if (sl.cap < n) {
            try {
                if (sl.dev) cuda_check(cudaFree(sl.dev), "OutputWriter");
                if (sl.host) cuda_check(cudaFreeHost(sl.host), "OutputWriter");
                sl.dev = sl.host = nullptr;
                sl.cap = 0;
                cuda_check(cudaMalloc(&sl.dev, n * sizeof(double)), "OutputWriter: device snapshot");
                cuda_check(cudaMallocHost(&sl.host, n * sizeof(double)), "OutputWriter: pinned buffer");
                sl.cap = n;
            } catch (...) {
                release(s);
                throw;
            }
        }
        return s;
    }

    void release(int s) {
        std::lock_guard<std::mutex> lk(m);
        slots[static_cast<std::size_t>(s)].busy = false;
        freed.notify_all();
    }

    void submit(const ScalarField& f, const std::string& base) {
        const Mesh& msh = f.mesh;
        const std::size_t nx = static_cast<std::size_t>(msh.n[0]), ny = static_cast<std::size_t>(msh.n[1]);
        const std::size_t plane = nx * ny, N = msh.totalSize();
        const int s = acquire(N);
        Slot& sl = slots[static_cast<std::size_t>(s)];
        try {
            const std::size_t pitch = static_cast<std::size_t>(f.storedDims[0]) * sizeof(double);
            for (int k = 0; k < msh.n[2]; ++k)
                cuda_check(cudaMemcpy2DAsync(sl.dev + static_cast<std::size_t>(k) * plane, nx * sizeof(double),
                                             f.d_curr + f.index(0, 0, k), pitch, nx * sizeof(double), ny,
                                             cudaMemcpyDeviceToDevice, 0),
                           "OutputWriter: pack");
            cuda_check(cudaEventRecord(sl.packed, 0), "OutputWriter");
            cuda_check(cudaStreamWaitEvent(side, sl.packed, 0), "OutputWriter");
            cuda_check(cudaMemcpyAsync(sl.host, sl.dev, N * sizeof(double), cudaMemcpyDeviceToHost, side),
                       "OutputWriter: download");
            cuda_check(cudaEventRecord(sl.landed, side), "OutputWriter");
        } catch (...) {
            release(s);
            throw;
        }
        {
            std::lock_guard<std::mutex> lk(m);
            jobs.push_back(Job{s, f.name, msh, f.ghost, base});
        }
        wake.notify_one();
    }
};

OutputWriter::OutputWriter(const nlohmann::json& c)
    : printInterval(c.at("print_interval").get<int>()), writeInterval(c.at("write_interval").get<int>()) {
    const std::string fmt = c.at("format").get<std::string>();
    writeBinary_ = fmt == "BINARY" || fmt == "ALL";
    writeDat_ = fmt == "DAT" || fmt == "ALL";
    writeVtk_ = fmt == "VTK" || fmt == "ALL";
    if (c.contains("async")) async_ = c.at("async").get<bool>();
    if (c.contains("async_buffers")) asyncBuffers_ = c.at("async_buffers").get<int>();
    if (asyncBuffers_ < 1) throw std::invalid_argument("OutputWriter: async_buffers must be >= 1");
    std::filesystem::create_directories("output");
    resetTimer();
}

OutputWriter::~OutputWriter() {
    if (!pending_) return;
    try {
        flush();
    } catch (const std::exception& e) {
        std::cerr << "OutputWriter: " << e.what() << "\n";
    }
    pending_.reset();
}

OutputWriter::OutputWriter(OutputWriter&&) noexcept = default;
OutputWriter& OutputWriter::operator=(OutputWriter&&) noexcept = default;

void OutputWriter::flush() {
    if (!pending_) return;
    pending_->drain();
    pending_->rethrow();
}

void OutputWriter::writeFields(ScalarField& f, int step, double simTime) {
    const std::string base = "output/" + f.name + "_" + std::to_string(step);
    if (async_ && f.deviceAllocated()) {
        if (!pending_) pending_ = std::make_unique<Async>(asyncBuffers_, writeBinary_, writeDat_, writeVtk_);
        pending_->rethrow();
        pending_->submit(f, base);
    } else {
        // the reference's order (src/IO/OutputWriter.cpp:24-33)
        if (pending_) flush();
        f.downloadCurrFromDevice();
        if (writeBinary_) writeField(f, base + ".field", FieldFormat::BINARY);
        if (writeDat_) writeField(f, base + ".dat", FieldFormat::DAT);
        if (writeVtk_) writeField(f, base + ".vts", FieldFormat::VTS);
    }
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
