/*
 * Named NVTX ranges around the stages of a problem and of a scene (problem,
 * pyramid level, PatchMatch pass, geometric iteration, network, fusion), so
 * that a profiler's timeline shows the flow's structure.  NVTX v3 is
 * header-only; with no tool attached a range costs a branch and, for a
 * formatted name, one snprintf.
 */
#pragma once

#include <nvtx3/nvToolsExt.h>
#include <stdarg.h>
#include <stdio.h>

namespace hpm {

class Range {
public:
    explicit Range(const char *fmt, ...) __attribute__((format(printf, 2, 3)))
    {
        char name[96];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(name, sizeof(name), fmt, ap);
        va_end(ap);
        nvtxRangePushA(name);
    }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};

}  // namespace hpm
