// The autotuner's host side: candidates, size buckets, and the cache of picked shapes.
#include "tune.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

namespace wsb {

namespace {

std::mutex g_mu;
std::map<std::string, ws_shape> g_cache;
bool g_loaded = false;

// half-octave bucket of a positive count
int bucket(long long x) { return x <= 0 ? -1 : int(std::floor(2.0 * std::log2(double(x)))); }

const char *cacheFile() {
  const char *p = std::getenv("WEAVESIM_TUNE_CACHE");
  return (p && *p) ? p : nullptr;
}

// one line a shape: key, then threads cta_state wide_cluster wide_min plain_launch trials trial_ms default_ms
std::string encode(const std::string &key, const ws_shape &s) {
  std::ostringstream o;
  o << key << ' ' << s.threads << ' ' << s.cta_state << ' ' << s.wide_cluster << ' ' << s.wide_min << ' ' << s.plain_launch
    << ' ' << s.trials << ' ' << s.trial_ms << ' ' << s.default_ms;
  return o.str();
}
bool decode(const std::string &line, std::string &key, ws_shape &s) {
  std::istringstream in(line);
  std::memset(&s, 0, sizeof(s));
  if (!(in >> key >> s.threads >> s.cta_state >> s.wide_cluster >> s.wide_min >> s.plain_launch >> s.trials >> s.trial_ms >>
        s.default_ms))
    return false;
  return true;
}

void loadLocked() {
  if (g_loaded) return;
  g_loaded = true;
  const char *f = cacheFile();
  if (!f) return;
  std::ifstream in(f);
  std::string line, key;
  ws_shape s;
  while (std::getline(in, line))
    if (decode(line, key, s)) g_cache[key] = s;       // a later line for the same key wins
}

ws_shape shape(int threads, int state, int cl, int wmin, int plain) {
  ws_shape s;
  std::memset(&s, 0, sizeof(s));
  s.threads = threads; s.cta_state = state; s.wide_cluster = cl; s.wide_min = wmin; s.plain_launch = plain;
  return s;
}

}  // namespace

std::string tuneKey(const std::string &device, const TuneInfo &t) {
  std::ostringstream o;
  std::string dev = device;
  for (char &ch : dev)
    if (ch == ' ' || ch == '|') ch = '_';
  o << dev << "|f" << t.form << "|p" << t.prec << "|s" << t.shortSides << "|e" << t.ext << "|b" << bucket(t.nInst) << "|x"
    << bucket(t.maxElems) << "|t" << bucket(t.totalElems);
  return o.str();
}

std::vector<ws_shape> tuneStage1(const TuneInfo &t) {
  std::vector<ws_shape> out;
  if (t.form == WS_FORM_PLAIN) {
    for (int mode = 0; mode < 3; mode++) out.push_back(shape(0, 0, 1, 0, mode));
  } else if (t.form == WS_FORM_CTA) {
    for (int thr : {256, 512, 128})
      for (int state : {WS_CTA_AUTO, WS_CTA_GLOBAL}) out.push_back(shape(thr, state, 1, 0, 0));
  } else {
    out.push_back(shape(0, 0, 1, 0, 0));          // the grid form has one shape: every co-resident block
  }
  return out;
}

std::vector<ws_shape> tuneStage2(const TuneInfo &t, const ws_shape &b) {
  std::vector<ws_shape> out;
  if (t.form != WS_FORM_CTA) return out;
  for (int wmin : {65536, 32768, 16384, 8192}) {
    if (t.maxElems < wmin) continue;              // no instance would be wide
    for (int cl : {2, 4, 8}) out.push_back(shape(b.threads, b.cta_state, cl, wmin, 0));
  }
  return out;
}

bool tuneLookup(const std::string &key, ws_shape *out) {
  std::lock_guard<std::mutex> lock(g_mu);
  loadLocked();
  auto it = g_cache.find(key);
  if (it == g_cache.end()) return false;
  if (out) *out = it->second;
  return true;
}

void tuneStore(const std::string &key, const ws_shape &s) {
  std::lock_guard<std::mutex> lock(g_mu);
  loadLocked();
  g_cache[key] = s;
  if (const char *f = cacheFile()) {
    std::ofstream o(f, std::ios::app);
    if (o) o << encode(key, s) << '\n';
  }
}

void tuneClear() {
  std::lock_guard<std::mutex> lock(g_mu);
  g_cache.clear();
  g_loaded = true;           // the file is not read again in this process
}

}  // namespace wsb
