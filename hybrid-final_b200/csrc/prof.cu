// prof.cu -- the per-kernel recorder behind hp_profile_step (prof.cuh).
#include <string>
#include <vector>

#include "prof.cuh"

namespace hp {
namespace prof {

bool g_on = false;

struct Mark {
    const char *name;
    cudaEvent_t ev;
};
std::vector<Mark> g_marks;
std::vector<cudaEvent_t> g_pool; // events kept for the next recording
bool g_failed = false;

void mark_slow(cudaStream_t st, const char *name) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
    cudaEvent_t ev;
    if (!g_pool.empty()) {
        ev = g_pool.back();
        g_pool.pop_back();
    } else if (cudaEventCreate(&ev) != cudaSuccess) {
        g_failed = true;
        return;
    }
    if (cudaEventRecord(ev, st) != cudaSuccess) g_failed = true;
    g_marks.push_back({name, ev});
}

void begin() {
    g_marks.clear();
    g_failed = false;
    g_on = true;
}

// stop recording (the last mark closes the last kernel) and add each
// kernel's time to its name's entry; returns false when an event failed
bool end(std::vector<std::string> &names, std::vector<int> &launches, std::vector<double> &ms) {
    g_on = false;
    bool ok = !g_failed;
    if (!g_marks.empty() && cudaEventSynchronize(g_marks.back().ev) != cudaSuccess) ok = false;
    for (size_t k = 0; ok && k + 1 < g_marks.size(); k++) {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, g_marks[k].ev, g_marks[k + 1].ev) != cudaSuccess) {
            ok = false;
            break;
        }
        const std::string nm = g_marks[k].name ? g_marks[k].name : "";
        size_t i = 0;
        while (i < names.size() && names[i] != nm) i++;
        if (i == names.size()) {
            names.push_back(nm);
            launches.push_back(0);
            ms.push_back(0.0);
        }
        launches[i]++;
        ms[i] += t;
    }
    for (auto &m : g_marks) g_pool.push_back(m.ev);
    g_marks.clear();
    return ok;
}

} // namespace prof
} // namespace hp
