// autotune.cu -- the table of tuned launch configurations, its JSON cache file, and the extern "C"
// controls (autotune.h describes what is tuned and when).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "autotune.h"
#include "capi_util.h"
#include "../../include/rhmc_b200.h"

namespace rhmc {

namespace {
struct Entry {
    int choice;
    std::vector<DsShape> shapes;
    std::vector<float> us;
};
std::mutex g_mu;
std::map<std::string, Entry> g_table;
std::string g_cache;     // file the table is saved to after every new entry ("" = none)
bool g_env_read = false;  // RHMC_TUNE_CACHE consulted
int g_enabled = -1;
int g_override = -1;

std::string json_escape(const std::string &s)
{
    std::string o;
    for (char ch : s) o += (ch == '"' || ch == '\\') ? '\'' : ch;
    return o;
}

std::string to_json_locked()
{
    std::ostringstream o;
    o << "{\"version\": 1, \"entries\": [";
    bool first = true;
    for (const auto &kv : g_table) {
        o << (first ? "\n" : ",\n") << "  {\"key\": \"" << json_escape(kv.first) << "\", \"choice\": " << kv.second.choice
          << ", \"shapes\": [";
        for (size_t i = 0; i < kv.second.shapes.size(); i++)
            o << (i ? ", " : "") << "[" << kv.second.shapes[i].block << ", " << kv.second.shapes[i].minb << "]";
        o << "], \"us\": [";
        for (size_t i = 0; i < kv.second.us.size(); i++) {
            char b[32];
            snprintf(b, sizeof(b), "%.2f", kv.second.us[i]);
            o << (i ? ", " : "") << b;
        }
        o << "]}";
        first = false;
    }
    o << "\n]}\n";
    return o.str();
}

// numbers of the bracketed list that starts at s[p] == '[' (nested brackets flattened)
std::vector<double> parse_numbers(const std::string &s, size_t p, size_t *end)
{
    std::vector<double> v;
    int depth = 0;
    size_t i = p;
    for (; i < s.size(); i++) {
        const char ch = s[i];
        if (ch == '[') depth++;
        else if (ch == ']') {
            if (--depth == 0) break;
        } else if ((ch >= '0' && ch <= '9') || ch == '-' || ch == '.') {
            char *e = nullptr;
            v.push_back(strtod(s.c_str() + i, &e));
            i = (size_t)(e - s.c_str()) - 1;
        }
    }
    if (end) *end = i;
    return v;
}

// reads the entries of a file written by to_json_locked (entries already in the table win)
int load_locked(const std::string &path)
{
    std::ifstream in(path);
    if (!in) return -1;
    std::stringstream ss;
    ss << in.rdbuf();
    const std::string s = ss.str();
    int n = 0;
    size_t p = 0;
    while ((p = s.find("\"key\": \"", p)) != std::string::npos) {
        p += 8;
        const size_t q = s.find('"', p);
        if (q == std::string::npos) break;
        const std::string key = s.substr(p, q - p);
        const size_t c = s.find("\"choice\": ", q), sh = s.find("\"shapes\": [", q), us = s.find("\"us\": [", q);
        if (c == std::string::npos || sh == std::string::npos || us == std::string::npos) break;
        Entry e;
        e.choice = atoi(s.c_str() + c + 10);
        size_t endp = 0;
        const std::vector<double> shp = parse_numbers(s, sh + 10, &endp);
        const std::vector<double> t = parse_numbers(s, us + 6, &endp);
        for (size_t i = 0; i + 1 < shp.size(); i += 2) e.shapes.push_back(DsShape{(int)shp[i], (int)shp[i + 1]});
        for (double x : t) e.us.push_back((float)x);
        if (e.choice >= 0 && e.choice < (int)e.shapes.size() && !g_table.count(key)) {
            g_table[key] = e;
            n++;
        }
        p = endp;
    }
    return n;
}

int save_locked(const std::string &path)
{
    std::ofstream out(path);
    if (!out) return -1;
    out << to_json_locked();
    return out ? 0 : -1;
}

void read_env_locked()
{
    if (g_env_read) return;
    g_env_read = true;
    const char *p = getenv("RHMC_TUNE_CACHE");
    if (p && *p) {
        g_cache = p;
        load_locked(g_cache);
    }
}

std::string device_name()
{
    static std::mutex mu;
    static std::map<int, std::string> names;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return "unknown";
    std::lock_guard<std::mutex> lock(mu);
    auto it = names.find(dev);
    if (it != names.end()) return it->second;
    cudaDeviceProp prop;
    const std::string n = cudaGetDeviceProperties(&prop, dev) == cudaSuccess ? std::string(prop.name) : "unknown";
    names[dev] = n;
    return n;
}
}  // namespace

bool autotune_enabled()
{
    if (g_enabled < 0) {
        const char *e = getenv("RHMC_AUTOTUNE");
        g_enabled = (e && e[0] == '0') ? 0 : 1;
    }
    return g_enabled != 0;
}

int autotune_override() { return g_override; }

int tune_get(const std::string &key)
{
    std::lock_guard<std::mutex> lock(g_mu);
    read_env_locked();
    auto it = g_table.find(key);
    return it == g_table.end() ? -1 : it->second.choice;
}

void tune_put(const std::string &key, int choice, const float *us, const DsShape *shapes, int n)
{
    std::lock_guard<std::mutex> lock(g_mu);
    read_env_locked();
    Entry e;
    e.choice = choice;
    for (int i = 0; i < n; i++) {
        e.shapes.push_back(shapes[i]);
        e.us.push_back(us[i]);
    }
    g_table[key] = e;
    if (!g_cache.empty()) save_locked(g_cache);
}

std::string tune_key(long vh, const std::string &what) { return device_name() + "|vh=" + std::to_string(vh) + "|" + what; }

bool stream_capturing(cudaStream_t s)
{
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) return true;  // do not time on a stream we cannot query
    return st != cudaStreamCaptureStatusNone;
}

int persistent_grid(const void *kern, int block, int ntiles)
{
    static std::mutex mu;
    static std::map<std::pair<int, std::pair<const void *, int>>, int> waves;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return ntiles;
    const auto key = std::make_pair(dev, std::make_pair(kern, block));
    int wave;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = waves.find(key);
        if (it != waves.end()) {
            wave = it->second;
        } else {
            int nsm = 0, nb = 0;
            if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, block, 0) == cudaSuccess)
                wave = nsm * nb;
            else
                wave = 0;
            cudaGetLastError();
            waves[key] = wave;
        }
    }
    return (wave > 0 && ntiles > wave) ? wave : ntiles;
}

}  // namespace rhmc

using namespace rhmc;

extern "C" {

int rhmc_autotune(int enable)
{
    const int prev = autotune_enabled() ? 1 : 0;
    g_enabled = enable ? 1 : 0;
    return prev;
}

int rhmc_autotune_override(int candidate)
{
    const int prev = g_override;
    g_override = candidate < 0 ? -1 : (candidate > 2 ? 2 : candidate);
    return prev;
}

int rhmc_tune_cache_load(const char *path)
{
    if (!path || !*path) return fail(RHMC_ERR_ARG, "rhmc_tune_cache_load: no path");
    std::lock_guard<std::mutex> lock(g_mu);
    g_env_read = true;
    g_cache = path;
    load_locked(g_cache);  // a missing file is an empty cache, written after the first tuning
    return RHMC_OK;
}

int rhmc_tune_cache_save(const char *path)
{
    std::lock_guard<std::mutex> lock(g_mu);
    const std::string p = (path && *path) ? std::string(path) : g_cache;
    if (p.empty()) return fail(RHMC_ERR_ARG, "rhmc_tune_cache_save: no path");
    if (save_locked(p)) return fail(RHMC_ERR_ARG, "rhmc_tune_cache_save: cannot write %s", p.c_str());
    return RHMC_OK;
}

long rhmc_tune_report(char *buf, long len)
{
    std::lock_guard<std::mutex> lock(g_mu);
    read_env_locked();
    const std::string s = to_json_locked();
    if (buf && len > 0) {
        const size_t n = s.size() < (size_t)(len - 1) ? s.size() : (size_t)(len - 1);
        memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return (long)s.size() + 1;
}

int rhmc_tune_clear(void)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_table.clear();
    return RHMC_OK;
}

}  // extern "C"
