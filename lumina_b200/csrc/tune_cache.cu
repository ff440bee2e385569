// tune_cache.cu -- persistent choices of the pair-kernel tuner.
//
// The tuner (otf.cu) times every build of the FP32 and FP64 pair kernels on
// a new geometry and keeps the fastest.  Its choices are kept in process
// memory and in a small JSON file, one flat object of "key": variant, so a
// later process on the same GPU model and library build starts with them.
// The key names the device (model, SM count), the build (compile time of the
// kernels), the kernel family and the geometry class (N, trig flavour,
// flags).  The file is $LUMINA_TUNE_CACHE, else
// $XDG_CACHE_HOME/lumina_b200/tune.json, else ~/.cache/lumina_b200/tune.json;
// LUMINA_TUNE_CACHE=off keeps the choices in memory only.  An unreadable or
// malformed file is ignored and rewritten.
#include "lumina_internal.cuh"

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <sys/stat.h>
#include <unistd.h>

namespace lum {
namespace {

std::mutex g_mu;
std::map<std::string, int> g_map;
bool g_loaded = false;

std::string cache_path() {
  const char* env = std::getenv("LUMINA_TUNE_CACHE");
  if (env && *env) {
    std::string v(env);
    if (v == "off" || v == "0") return std::string();
    return v;
  }
  std::string base;
  const char* xdg = std::getenv("XDG_CACHE_HOME");
  const char* home = std::getenv("HOME");
  if (xdg && *xdg)
    base = xdg;
  else if (home && *home)
    base = std::string(home) + "/.cache";
  else
    return std::string();
  return base + "/lumina_b200/tune.json";
}

void make_parent_dirs(const std::string& path) {
  for (size_t p = 1; p < path.size(); ++p)
    if (path[p] == '/') mkdir(path.substr(0, p).c_str(), 0755);
}

// Parses {"key": int, ...} as written by save_locked(); anything else yields
// nothing.
void load_locked() {
  g_loaded = true;
  const std::string path = cache_path();
  if (path.empty()) return;
  FILE* f = std::fopen(path.c_str(), "r");
  if (!f) return;
  std::string text;
  char buf[4096];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
  std::fclose(f);
  std::map<std::string, int> parsed;
  size_t i = text.find('{');
  if (i == std::string::npos) return;
  ++i;
  while (true) {
    const size_t q0 = text.find('"', i);
    if (q0 == std::string::npos) break;
    const size_t q1 = text.find('"', q0 + 1);
    if (q1 == std::string::npos) return;
    const size_t colon = text.find(':', q1);
    if (colon == std::string::npos) return;
    char* end = nullptr;
    const long v = std::strtol(text.c_str() + colon + 1, &end, 10);
    if (end == text.c_str() + colon + 1) return;
    parsed[text.substr(q0 + 1, q1 - q0 - 1)] = (int)v;
    i = (size_t)(end - text.c_str());
  }
  for (auto& kv : parsed) g_map.insert(kv);
}

void save_locked() {
  const std::string path = cache_path();
  if (path.empty()) return;
  make_parent_dirs(path);
  const std::string tmp = path + ".tmp." + std::to_string((long)getpid());
  FILE* f = std::fopen(tmp.c_str(), "w");
  if (!f) return;
  std::fprintf(f, "{\n");
  size_t c = 0;
  for (auto& kv : g_map)
    std::fprintf(f, "  \"%s\": %d%s\n", kv.first.c_str(), kv.second,
                 ++c < g_map.size() ? "," : "");
  std::fprintf(f, "}\n");
  if (std::fclose(f) == 0)
    std::rename(tmp.c_str(), path.c_str());
  else
    std::remove(tmp.c_str());
}

}  // namespace

std::string tune_device_tag() {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
  std::string name(prop.name);
  for (char& ch : name)
    if (ch == '"' || ch == '\\' || ch == ' ') ch = '_';
  return name + "_sm" + std::to_string(prop.multiProcessorCount);
}

bool tune_lookup(const std::string& key, int* value) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_loaded) load_locked();
  auto it = g_map.find(key);
  if (it == g_map.end()) return false;
  *value = it->second;
  return true;
}

void tune_store(const std::string& key, int value) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_loaded) load_locked();
  g_map[key] = value;
  save_locked();
}

}  // namespace lum
