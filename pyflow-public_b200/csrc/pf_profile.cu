// pf_profile.cu -- optional per-kernel device-time accounting.
//
// When enabled, every kernel launch of the library is bracketed by a pair of
// CUDA events recorded on the launching stream; pf_profile_read() waits for
// the pending events and returns, per kernel name, the number of launches and
// the summed device time.  Disabled (the default), the hooks cost one branch.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pf_profile.cuh"

namespace pf {

namespace {

struct Pending {
    int slot;
    cudaEvent_t a, b;
};

struct Entry {
    std::string name;
    long long launches = 0;
    double ms = 0.0;
};

std::mutex g_mu;
bool g_on = false;
std::vector<Entry> g_entries;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_pool;

cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

int slot_of(const char* name) {
    for (size_t i = 0; i < g_entries.size(); ++i)
        if (g_entries[i].name == name) return (int)i;
    g_entries.push_back(Entry{name});
    return (int)g_entries.size() - 1;
}

void flush_locked() {
    for (auto& p : g_pending) {
        cudaEventSynchronize(p.b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p.a, p.b);
        g_entries[p.slot].launches += 1;
        g_entries[p.slot].ms += ms;
        g_pool.push_back(p.a);
        g_pool.push_back(p.b);
    }
    g_pending.clear();
}

thread_local cudaEvent_t t_open = nullptr;
thread_local int t_slot = -1;

}  // namespace

// profiling is suspended while a step graph is being captured: event records
// are not allowed inside conditional graph bodies
static thread_local int t_suspend = 0;

bool prof_on() { return g_on && t_suspend == 0; }

void prof_suspend(bool on) { t_suspend += on ? 1 : -1; }

void prof_begin(const char* name, cudaStream_t s) {
    std::lock_guard<std::mutex> lk(g_mu);
    t_slot = slot_of(name);
    t_open = take_event();
    cudaEventRecord(t_open, s);
}

void prof_end(cudaStream_t s) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!t_open) return;
    cudaEvent_t b = take_event();
    cudaEventRecord(b, s);
    g_pending.push_back(Pending{t_slot, t_open, b});
    t_open = nullptr;
    if (g_pending.size() > 4096) flush_locked();
}

}  // namespace pf

extern "C" {

int pf_profile_enable(int enable) {
    std::lock_guard<std::mutex> lk(pf::g_mu);
    pf::flush_locked();
    if (enable && !pf::g_on) pf::g_entries.clear();
    pf::g_on = enable != 0;
    return PF_OK;
}

int pf_profile_read(pf_kernel_time* out, int max_entries, int* count) {
    std::lock_guard<std::mutex> lk(pf::g_mu);
    pf::flush_locked();
    const int n = (int)pf::g_entries.size();
    if (count) *count = n;
    if (!out) return PF_OK;
    for (int i = 0; i < n && i < max_entries; ++i) {
        std::memset(out[i].name, 0, sizeof(out[i].name));
        std::strncpy(out[i].name, pf::g_entries[i].name.c_str(), sizeof(out[i].name) - 1);
        out[i].launches = pf::g_entries[i].launches;
        out[i].ms = pf::g_entries[i].ms;
    }
    return PF_OK;
}

}  // extern "C"
