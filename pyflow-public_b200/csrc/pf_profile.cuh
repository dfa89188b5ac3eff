// pf_profile.cuh -- launch-bracketing hooks of the per-kernel timers.
#pragma once
#include <cuda_runtime.h>

#include "../../include/pyflow_b200.h"

namespace pf {

bool prof_on();
void prof_suspend(bool on);
void prof_begin(const char* name, cudaStream_t s);
void prof_end(cudaStream_t s);

// Brackets one kernel launch statement with timing events when enabled.
#define PF_LAUNCH(name, stream, ...)                   \
    do {                                               \
        const bool _pf_p = ::pf::prof_on();            \
        if (_pf_p) ::pf::prof_begin(name, stream);     \
        __VA_ARGS__;                                   \
        if (_pf_p) ::pf::prof_end(stream);             \
    } while (0)

}  // namespace pf
