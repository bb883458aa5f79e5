#pragma once
// Print / write intervals of a driver loop (API of the reference's
// include/IO/OutputWriter.h; needs nlohmann/json on the include path).
#include <chrono>
#include <string>

#include <nlohmann/json.hpp>

#include "IO/FieldFormat.h"
#include "field/ScalarField.h"

namespace PhiX {
namespace IO {
class OutputWriter {
public:
    explicit OutputWriter(const nlohmann::json& output_config);
    int printInterval;
    int writeInterval;
    bool shouldPrint(int step) const { return step % printInterval == 0; }
    bool shouldWrite(int step) const { return step % writeInterval == 0; }
    void writeFields(ScalarField& f, int step, double simTime);
    void printProgress(int step, double simTime);
    void resetTimer();

private:
    bool writeBinary_;
    bool writeDat_;
    bool writeVtk_;
    using Clock = std::chrono::steady_clock;
    Clock::time_point t_start_;
};
}  // namespace IO
}  // namespace PhiX
