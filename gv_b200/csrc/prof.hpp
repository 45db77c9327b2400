// Per-kernel CUDA-event timing, enabled through gv_profile_enable().  Replaces
// the reference's wall-clock Profiler singleton (src/util/profiler.cu:20-40,
// include/util/profiler.cuh:11-54): events are recorded on the stream the
// kernel is launched on, so the numbers are device time of that kernel.
#pragma once
#include <cuda_runtime.h>

namespace gv {

enum ProfSlot {
    PROF_RADIX = 0,
    PROF_SEGMENT,
    PROF_MEMBER,
    PROF_APPLY,
    PROF_COMPACT,
    PROF_PULL,
    PROF_TC_SNAPSHOT,
    PROF_TC_COUNT,
    PROF_BFS_LEVEL,
    PROF_BC_DEP,
    PROF_WPR_BUILD,
    PROF_WPR_SWEEP,
    PROF_WPR_GRAD,
    PROF_TC_CORE,
    PROF_TC_PROBE,
    PROF_TC_SORT,
    PROF_NSLOTS
};

int prof_begin(int slot, cudaStream_t s);  // -1 when profiling is off
void prof_end(int token, cudaStream_t s);

struct ProfScope {
    int tok;
    cudaStream_t s;
    ProfScope(int slot, cudaStream_t st) : tok(prof_begin(slot, st)), s(st) {}
    ~ProfScope() { prof_end(tok, s); }
};

}  // namespace gv
