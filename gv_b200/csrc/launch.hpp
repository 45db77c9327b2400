// Launch bookkeeping shared by every translation unit: each kernel launch goes
// through GV_LAUNCH so the library can report how many of its kernels ran.
#pragma once
#include <atomic>
#include <cstdint>

namespace gv {
extern std::atomic<unsigned long long> g_launches;
}

#define GV_LAUNCH(kernel, grid, block, smem, stream, ...)                 \
    do {                                                                  \
        kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);       \
        ::gv::g_launches.fetch_add(1, std::memory_order_relaxed);         \
    } while (0)
