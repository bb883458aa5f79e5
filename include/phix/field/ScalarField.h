#pragma once
// ScalarField -- FP64 ghost-padded field with host and device copies
// (API of the reference's include/field/ScalarField.h).  Layout:
//   storedDims[a] = mesh.n[a] + 2*ghost on every axis, x fastest,
//   index(i,j,k) = (i+g) + sx*((j+g) + sy*(k+g)).

#include <cstddef>
#include <string>
#include <vector>

#include "IO/FieldFormat.h"
#include "mesh/Mesh.h"

namespace PhiX {

class ScalarField {
public:
    std::string name;
    const Mesh& mesh;
    int ghost;
    int storedDims[3];
    std::size_t storedSize;

    std::vector<double> curr;  // current time level (host)
    std::vector<double> prev;  // previous time level (host)
    double* d_curr = nullptr;  // device copies (nullptr until allocDevice)
    double* d_prev = nullptr;

    explicit ScalarField(const Mesh& mesh, const std::string& name, int ghost = 1);

    // Non-owning wrapper of an external device buffer (no host storage).
    static ScalarField makeShell(const Mesh& mesh, int ghost, double* d_buf, const std::string& name = "shell");

    ScalarField(const ScalarField&) = delete;
    ScalarField& operator=(const ScalarField&) = delete;
    ScalarField(ScalarField&& other) noexcept;
    ScalarField& operator=(ScalarField&& other) noexcept;
    ~ScalarField();

    int index(int i, int j, int k) const { return (i + ghost) + storedDims[0] * ((j + ghost) + storedDims[1] * (k + ghost)); }
    int index(int i, int j) const { return index(i, j, 0); }
    int index(int i) const { return index(i, 0, 0); }

    void fill(double value);
    void fillCurr(double value);
    void fillPrev(double value);

    void advanceTimeLevelCPU();  // prev <- curr
    void advanceTimeLevelGPU();  // d_prev <- d_curr

    bool deviceAllocated() const { return d_curr != nullptr; }
    void allocDevice();
    void freeDevice();

    void uploadCurrToDevice() const;
    void uploadPrevToDevice() const;
    void uploadAllToDevice() const;
    void downloadCurrFromDevice();
    void downloadPrevFromDevice();
    void downloadAllFromDevice();

    bool ownsDeviceMemory() const { return ownsDeviceMemory_; }

    void write(const std::string& path, FieldFormat fmt = FieldFormat::BINARY) const;
    static ScalarField readFromFile(const Mesh& mesh, const std::string& path, int ghost = 1);
    void print() const;

private:
    bool ownsDeviceMemory_ = true;
};

using Field = ScalarField;

}  // namespace PhiX
