// tune.cpp -- persistent cache of autotuned launch choices (see tune.h).
// File format: one entry per line, "key v1 v2 ...", the key without spaces;
// a later line for the same key wins.
#include "tune.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

#include "common.cuh"

namespace dage {
namespace {

std::mutex g_mutex;
std::map<std::string, std::vector<int>> g_cache;
std::string g_path;
bool g_env_checked = false;

void load_file_locked(const std::string &path) {
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::string key;
    if (!(is >> key)) continue;
    std::vector<int> v;
    int x;
    while (is >> x) v.push_back(x);
    if (!v.empty()) g_cache[key] = v;
  }
}

void check_env_locked() {
  if (g_env_checked) return;
  g_env_checked = true;
  const char *e = std::getenv("DAGE_TUNE_CACHE");
  if (e && *e && g_path.empty()) {
    g_path = e;
    load_file_locked(g_path);
  }
}

}  // namespace

std::string tune_device_key() {
  int dev = 0;
  cudaDeviceProp prop{};
  if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
    return "dev?";
  std::string name = prop.name;
  for (char &c : name)
    if (c == ' ') c = '_';
  return name + "/sm" + std::to_string(prop.multiProcessorCount);
}

bool tune_lookup(const std::string &key, std::vector<int> &val) {
  std::lock_guard<std::mutex> lock(g_mutex);
  check_env_locked();
  auto it = g_cache.find(key);
  if (it == g_cache.end()) return false;
  val = it->second;
  return true;
}

void tune_store(const std::string &key, const std::vector<int> &val) {
  std::lock_guard<std::mutex> lock(g_mutex);
  check_env_locked();
  g_cache[key] = val;
  if (g_path.empty()) return;
  if (FILE *f = std::fopen(g_path.c_str(), "a")) {
    std::fprintf(f, "%s", key.c_str());
    for (int v : val) std::fprintf(f, " %d", v);
    std::fprintf(f, "\n");
    std::fclose(f);
  }
}

}  // namespace dage

extern "C" int dage_set_tune_cache(const char *path) {
  dage::clear_error();
  std::lock_guard<std::mutex> lock(dage::g_mutex);
  dage::g_env_checked = true;  // an explicit path overrides the environment
  dage::g_path = path ? path : "";
  if (!dage::g_path.empty()) {
    // the file must be writable (created when missing)
    FILE *f = std::fopen(dage::g_path.c_str(), "a");
    if (!f) return dage::fail(DAGE_E_INVALID, "cannot open tune cache file %s", path);
    std::fclose(f);
    dage::load_file_locked(dage::g_path);
  }
  return 0;
}
