// The autotuner's choices (z-chunk lengths per level shape, smoothing schedules per
// problem class), kept for the process and, when a cache file is set
// (uaamg_set_tune_cache), in a small JSON file so later processes reuse them:
//
//   {"entries": {"<key>": [v, ...], ...}}
//
// Keys name the GPU (device name and SM count), the precision and the shape, so one
// file can serve several GPUs and problems.  There is no counterpart in the
// reference: its kernels fix their tile shapes and smoothing at compile time
// (cuda_uaamg_preconditioner_3d_opt_f.cu:444, NU = 1).
#include <cuda_runtime.h>

#include <cstdio>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/uaamg.h"
#include "engine.h"

namespace uaamg {
namespace {

std::mutex g_mu;
std::map<std::string, std::vector<int>> g_entries;
std::string g_path;

// Reads the entries of a cache file written by save(): "key": [ints] pairs.
void load(const std::string& path) {
    std::ifstream f(path);
    if (!f) return;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string t = ss.str();
    size_t p = t.find("\"entries\"");
    if (p == std::string::npos) return;
    p = t.find('{', p);
    while (p != std::string::npos) {
        const size_t k0 = t.find('"', p + 1);
        if (k0 == std::string::npos) break;
        const size_t k1 = t.find('"', k0 + 1);
        const size_t a0 = t.find('[', k1);
        const size_t a1 = t.find(']', a0);
        if (k1 == std::string::npos || a0 == std::string::npos || a1 == std::string::npos) break;
        std::vector<int> v;
        std::stringstream vs(t.substr(a0 + 1, a1 - a0 - 1));
        std::string item;
        while (std::getline(vs, item, ',')) {
            try { v.push_back(std::stoi(item)); } catch (...) { v.clear(); break; }
        }
        if (!v.empty()) g_entries[t.substr(k0 + 1, k1 - k0 - 1)] = v;
        p = a1;
        const size_t nx = t.find_first_of(",}", p);
        if (nx == std::string::npos || t[nx] == '}') break;
        p = nx;
    }
}

void save() {
    if (g_path.empty()) return;
    const std::string tmp = g_path + ".tmp";
    {
        std::ofstream f(tmp);
        if (!f) return;
        f << "{\"entries\": {";
        bool first = true;
        for (const auto& kv : g_entries) {
            f << (first ? "\n " : ",\n ") << '"' << kv.first << "\": [";
            for (size_t q = 0; q < kv.second.size(); ++q) f << (q ? ", " : "") << kv.second[q];
            f << ']';
            first = false;
        }
        f << "\n}}\n";
    }
    std::rename(tmp.c_str(), g_path.c_str());
}

}  // namespace

std::string tune_gpu_id() {
    static std::mutex mu;
    static std::map<int, std::string> ids;  // per device ordinal
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return "gpu?";
    }
    std::lock_guard<std::mutex> lk(mu);
    auto it = ids.find(dev);
    if (it != ids.end()) return it->second;
    cudaDeviceProp pr;
    if (cudaGetDeviceProperties(&pr, dev) != cudaSuccess) {
        cudaGetLastError();
        return "gpu?";
    }
    std::string n = pr.name;
    for (char& c : n)
        if (c == ' ' || c == '"' || c == '|') c = '_';
    return ids[dev] = n + "/" + std::to_string(pr.multiProcessorCount);
}

bool tune_lookup(const std::string& key, std::vector<int>* val) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_entries.find(key);
    if (it == g_entries.end()) return false;
    *val = it->second;
    return true;
}

void tune_store(const std::string& key, const std::vector<int>& val) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_entries[key] = val;
    save();
}

}  // namespace uaamg

extern "C" uaamg_status uaamg_set_tune_cache(const char* path) {
    std::lock_guard<std::mutex> lk(uaamg::g_mu);
    uaamg::g_path = path ? path : "";
    if (!uaamg::g_path.empty()) uaamg::load(uaamg::g_path);
    return UAAMG_OK;
}
