// Host-side phase timing: with TYCHO_TRACE=1 in the environment, each traced
// scope prints "[tycho] <name> <milliseconds>" to stderr when it ends.
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>

namespace tycho {

inline bool trace_on()
{
    static const bool on = [] {
        const char *v = std::getenv("TYCHO_TRACE");
        return v && *v && *v != '0';
    }();
    return on;
}

class TraceScope {
public:
    explicit TraceScope(const char *name) : name_(name), t0_(std::chrono::steady_clock::now()) {}
    ~TraceScope() { report(); }
    // Ends the current phase (reported now) and starts the next one.
    void next(const char *name)
    {
        report();
        name_ = name;
        t0_ = std::chrono::steady_clock::now();
    }
    TraceScope(const TraceScope &) = delete;
    TraceScope &operator=(const TraceScope &) = delete;

private:
    void report() const
    {
        if (!trace_on()) return;
        const double ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
        std::fprintf(stderr, "[tycho] %s %.3f\n", name_, ms);
    }
    const char *name_;
    std::chrono::steady_clock::time_point t0_;
};

}  // namespace tycho
