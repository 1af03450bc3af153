// Optional per-kernel timing: when enabled, library entry points bracket each kernel launch
// with CUDA events on the caller's stream; hb_timing_read sums the elapsed times per name.
#pragma once

#include <cuda_runtime.h>

namespace hb {

bool timing_on();
void timing_begin(const char* name, cudaStream_t s);
void timing_end(cudaStream_t s);

// RAII bracket around one launch (no-op when timing is off).
struct TimedSection {
    cudaStream_t s;
    bool on;
    TimedSection(const char* name, cudaStream_t st) : s(st), on(timing_on()) {
        if (on) timing_begin(name, s);
    }
    ~TimedSection() {
        if (on) timing_end(s);
    }
};

}  // namespace hb
