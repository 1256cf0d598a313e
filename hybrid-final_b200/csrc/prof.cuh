// prof.cuh -- per-kernel device times of op-by-op steps (hp_profile_step).
//
// Every launch wrapper marks its stream with the kernel's name just before
// the launch.  While a profile is being recorded a mark is a CUDA event on
// that stream, and the time from one mark to the next is the kernel named by
// the first; otherwise a mark is a flag test.  Marks inside a stream capture
// are skipped (the graph path is not profiled).  One recording at a time
// per process.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace hp {
namespace prof {
extern bool g_on;
void mark_slow(cudaStream_t st, const char *name);
inline void mark(cudaStream_t st, const char *name) {
    if (g_on) mark_slow(st, name);
}
// hp_profile_step's recording: begin, the op-by-op steps, a closing mark,
// then end() adds every kernel's time to its name's entry (false when an
// event failed)
void begin();
bool end(std::vector<std::string> &names, std::vector<int> &launches, std::vector<double> &ms);
} // namespace prof
} // namespace hp
