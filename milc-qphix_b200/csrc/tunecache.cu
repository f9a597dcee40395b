// Persistent autotuner choices (tunecache.h).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

#include "tunecache.h"

namespace qb {

namespace {

std::mutex g_mu;
std::map<std::string, std::vector<double>> g_entries;
bool g_loaded = false;

const char *cache_path()
{
    const char *p = std::getenv("QPHIX_B200_TUNECACHE");
    return (p && p[0]) ? p : nullptr;
}

// lines "key v0 v1 ..."; later lines for the same key win
void load_locked()
{
    if (g_loaded) return;
    g_loaded = true;
    const char *path = cache_path();
    if (!path) return;
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string key;
        if (!(ls >> key) || key.empty() || key[0] == '#') continue;
        std::vector<double> v;
        double x;
        while (ls >> x) v.push_back(x);
        if (!v.empty()) g_entries[key] = v;
    }
}

}  // namespace

bool tune_cache_get(const std::string &key, std::vector<double> &vals)
{
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    auto it = g_entries.find(key);
    if (it == g_entries.end()) return false;
    vals = it->second;
    return true;
}

void tune_cache_put(const std::string &key, const std::vector<double> &vals)
{
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    g_entries[key] = vals;
    const char *path = cache_path();
    if (!path) return;
    std::ofstream out(path, std::ios::app);
    if (!out) return;  // an unwritable cache only costs the re-tuning
    out << key;
    char buf[32];
    for (double v : vals) {
        std::snprintf(buf, sizeof buf, " %.9g", v);
        out << buf;
    }
    out << '\n';
}

std::string tune_device_tag()
{
    int dev = 0;
    cudaDeviceProp p{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&p, dev) != cudaSuccess) return "unknown";
    std::string name(p.name);
    for (char &ch : name)
        if (ch == ' ' || ch == '\t') ch = '_';
    return name + "/" + std::to_string(p.multiProcessorCount);
}

}  // namespace qb
