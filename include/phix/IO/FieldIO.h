#pragma once
// Field IO (API of the reference's include/IO/FieldIO.h).  BINARY .field:
// text header ("# PhiX ScalarField", name, nx ny nz, ghost, "---") then the
// physical cells as little-endian FP64, x fastest; DAT: "x y z value" text.

#include <string>

#include "IO/FieldFormat.h"
#include "mesh/Mesh.h"

namespace PhiX {
class ScalarField;
class VectorField;
namespace IO {
void writeField(const ScalarField& f, const std::string& path, FieldFormat fmt = FieldFormat::BINARY);
ScalarField readScalarField(const Mesh& mesh, const std::string& path, int ghost = 1);
void readField(ScalarField& f, const std::string& path);
int resolveStartStep(const std::string& startFrom, const std::string& refFieldName = "c");
void initField(ScalarField& f, int startStep);
void writeField(const VectorField& vf, const std::string& path, FieldFormat fmt = FieldFormat::BINARY);
VectorField readVectorField(const Mesh& mesh, const std::string& path, int ghost = 1);
void readField(VectorField& vf, const std::string& path);
}  // namespace IO
}  // namespace PhiX
