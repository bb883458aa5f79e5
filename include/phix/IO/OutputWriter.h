#pragma once
// Print / write intervals of a driver loop (API of the reference's
// include/IO/OutputWriter.h; needs nlohmann/json on the include path).
//
// writeFields overlaps output with the time steps that follow it: the
// physical cells are packed on the device (on the legacy default stream, so
// after every launch that wrote them), copied to pinned host memory on a
// side stream, and formatted and written by a worker thread, through the same
// formatter as IO::writeField, so the files are the same bytes as the
// synchronous path's.  Two departures from the reference, both only in the
// asynchronous mode:
//   * the host copy f.curr is not refreshed (the reference downloads it);
//   * a file error is thrown from a later writeFields or from flush(), and
//     a pending one is printed to stderr by the destructor.
// Optional keys of the output config (ignored by the reference):
//   "async": false        the reference's synchronous download + write
//   "async_buffers": n    snapshots in flight before writeFields waits (3)
#include <chrono>
#include <memory>
#include <string>

#include <nlohmann/json.hpp>

#include "IO/FieldFormat.h"
#include "field/ScalarField.h"

namespace PhiX {
namespace IO {
class OutputWriter {
public:
    explicit OutputWriter(const nlohmann::json& output_config);
    ~OutputWriter();
    OutputWriter(OutputWriter&&) noexcept;
    OutputWriter& operator=(OutputWriter&&) noexcept;
    int printInterval;
    int writeInterval;
    bool shouldPrint(int step) const { return step % printInterval == 0; }
    bool shouldWrite(int step) const { return step % writeInterval == 0; }
    void writeFields(ScalarField& f, int step, double simTime);
    void printProgress(int step, double simTime);
    void resetTimer();
    // Waits until every file of earlier writeFields calls is on disk; throws
    // the first error a background write met.
    void flush();

private:
    bool writeBinary_;
    bool writeDat_;
    bool writeVtk_;
    bool async_ = true;
    int asyncBuffers_ = 3;
    using Clock = std::chrono::steady_clock;
    Clock::time_point t_start_;
    struct Async;
    std::unique_ptr<Async> pending_;
};
}  // namespace IO
}  // namespace PhiX
