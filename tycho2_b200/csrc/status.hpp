// Status codes returned through the C ABI (mirrors include/tycho_cuda.h) and
// the per-thread last-error message.
#pragma once

#include <string>

namespace tycho {

enum Status : int {
    kOk = 0,
    kErrArg = 1,          // invalid argument
    kErrIO = 2,           // file could not be read/written
    kErrFormat = 3,       // malformed mesh / deck
    kErrCuda = 4,         // CUDA runtime error
    kErrOom = 5,          // device memory exhausted
    kErrCycle = 6,        // a direction's dependency graph has a cycle
    kErrNotConverged = 7, // iteration limit reached before the tolerance
    kErrTimeout = 8,      // a bounded device wait gave up
    kErrBusy = 9,         // admission refused (serving)
    kErrMissing = 10,     // required input not set
};

void set_last_error(const std::string &msg);
const std::string &last_error();

}  // namespace tycho
