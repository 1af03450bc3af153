// Event-based per-kernel timing for benchmarks (see timing.cuh).
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "timing.cuh"

namespace hb {

namespace {
struct Section {
    std::string name;
    cudaEvent_t b = nullptr, e = nullptr;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Section> g_sections;
std::vector<size_t> g_open;  // indices of sections begun but not yet ended
}  // namespace

bool timing_on() { return g_on; }

void timing_begin(const char* name, cudaStream_t s) {
    std::lock_guard<std::mutex> lk(g_mu);
    Section sec;
    sec.name = name;
    cudaEventCreate(&sec.b);
    cudaEventCreate(&sec.e);
    cudaEventRecord(sec.b, s);
    g_open.push_back(g_sections.size());
    g_sections.push_back(sec);
}

void timing_end(cudaStream_t s) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_open.empty()) return;
    const size_t i = g_open.back();
    g_open.pop_back();
    if (i < g_sections.size()) cudaEventRecord(g_sections[i].e, s);
}

}  // namespace hb

extern "C" {

int hb_timing_enable(int on) {
    std::lock_guard<std::mutex> lk(hb::g_mu);
    hb::g_on = on != 0;
    return HB_OK;
}

int hb_timing_read(char* names, size_t names_cap, float* ms, int cap, int* n_sections, int* n_launches) {
    std::lock_guard<std::mutex> lk(hb::g_mu);
    std::vector<std::string> order;
    std::vector<double> tot;
    std::vector<int> cnt;
    int launches = 0;
    int status = HB_OK;
    for (auto& sec : hb::g_sections) {
        const std::string& nm = sec.name;
        float t = 0.f;
        if (cudaEventSynchronize(sec.e) != cudaSuccess || cudaEventElapsedTime(&t, sec.b, sec.e) != cudaSuccess) {
            status = HB_ERR_CUDA;
            hb::set_error("hb_timing_read: event query failed");
        }
        size_t k = 0;
        for (; k < order.size(); ++k)
            if (order[k] == nm) break;
        if (k == order.size()) {
            order.push_back(nm);
            tot.push_back(0.0);
            cnt.push_back(0);
        }
        tot[k] += t;
        cnt[k] += 1;
        ++launches;
        cudaEventDestroy(sec.b);
        cudaEventDestroy(sec.e);
    }
    hb::g_sections.clear();
    hb::g_open.clear();
    std::string joined;
    for (size_t k = 0; k < order.size(); ++k) {
        if (k) joined += "\n";
        joined += order[k];
        if ((int)k < cap && ms) ms[k] = (float)tot[k];
    }
    if (names && names_cap) {
        std::strncpy(names, joined.c_str(), names_cap - 1);
        names[names_cap - 1] = '\0';
    }
    if (n_sections) *n_sections = (int)order.size();
    if (n_launches) *n_launches = launches;
    return status;
}

}  // extern "C"
