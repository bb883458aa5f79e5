#pragma once
namespace PhiX {
// Output format of field IO: BINARY (.field / .vfield), DAT (x y z value text),
// VTS (VTK XML StructuredGrid).
enum class FieldFormat { BINARY, DAT, VTS };
}  // namespace PhiX
