#pragma once
// VectorField -- N ScalarField components on one mesh (API of the reference's
// include/field/VectorField.h).

#include <memory>
#include <string>
#include <vector>

#include "IO/FieldFormat.h"
#include "field/ScalarField.h"

namespace PhiX {

class VectorField {
public:
    explicit VectorField(const Mesh& mesh, const std::string& name, int nComponents, int ghost = 1);
    VectorField(const VectorField&) = delete;
    VectorField& operator=(const VectorField&) = delete;
    VectorField(VectorField&& other) noexcept;
    VectorField& operator=(VectorField&& other) noexcept;
    ~VectorField() = default;

    ScalarField& operator[](int c);
    const ScalarField& operator[](int c) const;
    int nComponents() const { return static_cast<int>(components_.size()); }
    ScalarField& x() { return (*this)[0]; }
    ScalarField& y() { return (*this)[1]; }
    ScalarField& z() { return (*this)[2]; }
    const ScalarField& x() const { return (*this)[0]; }
    const ScalarField& y() const { return (*this)[1]; }
    const ScalarField& z() const { return (*this)[2]; }

    const Mesh& mesh;
    int ghost;
    std::string name;

    void fill(double value);
    void fillCurr(double value);
    void fillPrev(double value);
    void advanceTimeLevelCPU();
    void advanceTimeLevelGPU();
    void allocDevice();
    void freeDevice();
    void uploadAllToDevice() const;
    void uploadCurrToDevice() const;
    void downloadAllFromDevice();
    void downloadCurrFromDevice();
    void write(const std::string& path, FieldFormat fmt = FieldFormat::BINARY) const;
    static VectorField readFromFile(const Mesh& mesh, const std::string& path, int ghost = 1);
    void print() const;
    static std::string componentName(const std::string& baseName, int c, int nComp);

private:
    std::vector<std::unique_ptr<ScalarField>> components_;
};

}  // namespace PhiX
