// Autotuner of launch shapes: which tile runs per CTA, CTAs per SM, scan cluster
// size and window length, and filter-bank run length each kernel family uses for a
// given problem class on a given GPU.
//
// A choice is one integer per key.  Keys name the operation, the parameters that
// change the best shape (taps, stages, form, dtype exactly; batch, channels and
// lengths as power-of-two classes) and the device's SM count, e.g.
//     fir_bf16x3|T=256|tiles=2^3|batch=2^10|sms=148
// Entries live in a process-wide table, loaded from and saved to a JSON cache file
// ({"format": "dsplib_b200 autotune 1", "entries": {"<key>": <choice>, ...}}).
// Modes: OFF (the built-in rules only), CACHED (default: a cached choice when there is
// one, else the built-in rule), MEASURE (as CACHED, and a class without an entry is
// measured when a handle or plan is initialised: every candidate launched on scratch
// buffers of the problem's shape, timed with CUDA events, the fastest stored and the
// cache file rewritten).  The reference selects its kernel variants by fixed size
// classes in init (DSPLIB_fir_ci.cpp:350-405, DSPLIB_cascadeBiquad.cpp:480-615).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "dsplib_internal.h"

namespace dsplib {

namespace {

struct TuneTable {
   std::mutex mu;
   std::map<std::string, int> entries;
   std::string path;
   bool pathFromEnv = false;
   int mode = DSPLIB_GPU_TUNE_CACHED;
   bool modeFromEnv = false;
   unsigned generation = 1;
};

TuneTable &table()
{
   static TuneTable t;
   return t;
}

// Parse the cache file's entries: every "key": integer pair inside "entries".  Returns
// false (and leaves out) when the text is not such a file.
bool parseCache(const std::string &text, std::map<std::string, int> &out)
{
   const size_t e = text.find("\"entries\"");
   if (text.find("dsplib_b200 autotune 1") == std::string::npos || e == std::string::npos) return false;
   size_t i = text.find('{', e);
   if (i == std::string::npos) return false;
   std::map<std::string, int> got;
   bool closed = false;
   i++;
   while (i < text.size()) {
      while (i < text.size() && (text[i] == ' ' || text[i] == '\n' || text[i] == '\r' || text[i] == '\t' ||
                                 text[i] == ','))
         i++;
      if (i >= text.size()) return false;
      if (text[i] == '}') {
         closed = true;
         break;
      }
      if (text[i] != '"') return false;
      const size_t k1 = text.find('"', i + 1);
      if (k1 == std::string::npos) return false;
      const std::string key = text.substr(i + 1, k1 - i - 1);
      i = text.find(':', k1);
      if (i == std::string::npos) return false;
      i++;
      while (i < text.size() && text[i] == ' ') i++;
      char *end = nullptr;
      const long v = std::strtol(text.c_str() + i, &end, 10);
      if (end == text.c_str() + i) return false;
      i = (size_t) (end - text.c_str());
      got[key] = (int) v;
   }
   if (!closed) return false;
   out.swap(got);
   return true;
}

void loadLocked(TuneTable &t)
{
   if (t.path.empty()) return;
   FILE *f = std::fopen(t.path.c_str(), "rb");
   if (!f) return;
   std::string text;
   char buf[4096];
   size_t n;
   while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
   std::fclose(f);
   std::map<std::string, int> got;
   if (parseCache(text, got))
      for (auto &kv : got) t.entries[kv.first] = kv.second; // entries set in this process win on save
}

bool saveLocked(TuneTable &t)
{
   if (t.path.empty()) return true;
   const std::string tmp = t.path + ".tmp";
   FILE *f = std::fopen(tmp.c_str(), "wb");
   if (!f) return false;
   std::fprintf(f, "{\n  \"format\": \"dsplib_b200 autotune 1\",\n  \"entries\": {");
   bool first = true;
   for (auto &kv : t.entries) {
      std::fprintf(f, "%s\n    \"%s\": %d", first ? "" : ",", kv.first.c_str(), kv.second);
      first = false;
   }
   std::fprintf(f, "\n  }\n}\n");
   const bool ok = std::fclose(f) == 0;
   return ok && std::rename(tmp.c_str(), t.path.c_str()) == 0;
}

// The environment's settings, read once: DSPLIB_GPU_TUNE_CACHE (cache file) and
// DSPLIB_GPU_AUTOTUNE (0, 1 or 2: the mode).
void initFromEnv(TuneTable &t)
{
   static bool done = false;
   if (done) return;
   done = true;
   if (const char *p = std::getenv("DSPLIB_GPU_TUNE_CACHE")) {
      if (*p) {
         t.path = p;
         t.pathFromEnv = true;
         loadLocked(t);
      }
   }
   if (const char *m = std::getenv("DSPLIB_GPU_AUTOTUNE")) {
      const int v = std::atoi(m);
      if (v >= DSPLIB_GPU_TUNE_OFF && v <= DSPLIB_GPU_TUNE_MEASURE) {
         t.mode = v;
         t.modeFromEnv = true;
      }
   }
}

} // namespace

int tuneMode()
{
   TuneTable &t = table();
   std::lock_guard<std::mutex> lock(t.mu);
   initFromEnv(t);
   return t.mode;
}

unsigned tuneGeneration()
{
   TuneTable &t = table();
   std::lock_guard<std::mutex> lock(t.mu);
   initFromEnv(t);
   return t.generation;
}

bool tuneLookup(const std::string &key, int *choice)
{
   TuneTable &t = table();
   std::lock_guard<std::mutex> lock(t.mu);
   initFromEnv(t);
   if (t.mode == DSPLIB_GPU_TUNE_OFF) return false;
   auto it = t.entries.find(key);
   if (it == t.entries.end()) return false;
   *choice = it->second;
   return true;
}

void tuneStore(const std::string &key, int choice, bool save)
{
   TuneTable &t = table();
   std::lock_guard<std::mutex> lock(t.mu);
   initFromEnv(t);
   t.entries[key] = choice;
   t.generation++;
   if (save) (void) saveLocked(t);
}

int tuneClass(long long v)
{
   int c = 0;
   while (c < 62 && (1LL << c) < v) c++;
   return c;
}

int deviceSms()
{
   static int cached[64] = {}; // per device ordinal, read once
   int dev = 0;
   if (cudaGetDevice(&dev) != cudaSuccess) {
      (void) cudaGetLastError();
      return 0;
   }
   if (dev >= 0 && dev < 64 && cached[dev] > 0) return cached[dev];
   int sms = 0;
   if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
      (void) cudaGetLastError();
      return 0;
   }
   if (dev >= 0 && dev < 64) cached[dev] = sms;
   return sms;
}

// L2 flush between timed launches: a write larger than the L2 cache, outside the events,
// so that every candidate reads its inputs from HBM as a call in a pipeline does.
constexpr size_t kFlushBytes = 256u << 20;

float tuneTime(const std::function<cudaError_t(cudaStream_t)> &launch, cudaStream_t s, int reps, void *flush)
{
   cudaEvent_t e0 = nullptr, e1 = nullptr;
   if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      (void) cudaGetLastError();
      if (e0) cudaEventDestroy(e0);
      return -1.0f;
   }
   float best = -1.0f;
   bool ok = launch(s) == cudaSuccess && cudaStreamSynchronize(s) == cudaSuccess; // warm-up
   std::vector<float> times;
   for (int r = 0; ok && r < reps; r++) {
      ok = (!flush || cudaMemsetAsync(flush, r & 0xff, kFlushBytes, s) == cudaSuccess) &&
           cudaEventRecord(e0, s) == cudaSuccess && launch(s) == cudaSuccess && cudaEventRecord(e1, s) == cudaSuccess &&
           cudaEventSynchronize(e1) == cudaSuccess;
      float ms = 0.0f;
      if (ok && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) times.push_back(ms);
   }
   if (ok && !times.empty()) {
      std::sort(times.begin(), times.end());
      best = times[times.size() / 2];
   }
   (void) cudaGetLastError();
   cudaEventDestroy(e0);
   cudaEventDestroy(e1);
   return best;
}

bool tuneFill(void *p, size_t bytes, bool asFloat)
{
   cudaStream_t s = nullptr;
   if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      (void) cudaGetLastError();
      return false;
   }
   const bool ok = launchTuneFill(p, bytes, asFloat, s) == cudaSuccess && cudaStreamSynchronize(s) == cudaSuccess;
   cudaStreamDestroy(s);
   (void) cudaGetLastError();
   return ok;
}

int tunePick(const std::string &key, const std::vector<int> &cands,
             const std::function<cudaError_t(int, cudaStream_t)> &launch)
{
   if (cands.empty()) return -1;
   cudaStream_t s = nullptr;
   if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      (void) cudaGetLastError();
      return -1;
   }
   void *flush = nullptr;
   if (cudaMalloc(&flush, kFlushBytes) != cudaSuccess) {
      (void) cudaGetLastError();
      flush = nullptr;
   }
   int best = -1;
   float bestMs = 0.0f;
   for (int c : cands) {
      const float ms = tuneTime([&](cudaStream_t st) { return launch(c, st); }, s, 5, flush);
      if (ms >= 0.0f && (best < 0 || ms < bestMs)) {
         best = c;
         bestMs = ms;
      }
   }
   (void) cudaStreamSynchronize(s);
   if (flush) cudaFree(flush);
   cudaStreamDestroy(s);
   (void) cudaGetLastError();
   if (best >= 0) tuneStore(key, best, true);
   return best;
}

} // namespace dsplib

using namespace dsplib;

extern "C" {

DSPLIB_STATUS DSPLIB_gpu_autotuneSetMode(int32_t mode)
{
   if (mode < DSPLIB_GPU_TUNE_OFF || mode > DSPLIB_GPU_TUNE_MEASURE) return DSPLIB_ERR_INVALID_VALUE;
   TuneTable &t = table();
   std::lock_guard<std::mutex> lock(t.mu);
   initFromEnv(t);
   t.mode = mode;
   t.generation++;
   return DSPLIB_SUCCESS;
}

int32_t DSPLIB_gpu_autotuneGetMode(void) { return tuneMode(); }

DSPLIB_STATUS DSPLIB_gpu_autotuneSetCachePath(const char *path)
{
   TuneTable &t = table();
   std::lock_guard<std::mutex> lock(t.mu);
   initFromEnv(t);
   t.path = path ? path : "";
   t.pathFromEnv = false;
   loadLocked(t);
   t.generation++;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_autotuneSave(void)
{
   TuneTable &t = table();
   std::lock_guard<std::mutex> lock(t.mu);
   initFromEnv(t);
   if (t.path.empty()) return DSPLIB_ERR_INVALID_VALUE;
   return saveLocked(t) ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

DSPLIB_STATUS DSPLIB_gpu_autotuneClear(void)
{
   TuneTable &t = table();
   std::lock_guard<std::mutex> lock(t.mu);
   initFromEnv(t);
   t.entries.clear();
   t.generation++;
   return DSPLIB_SUCCESS;
}

int32_t DSPLIB_gpu_autotuneLookup(const char *key)
{
   if (!key) return -1;
   TuneTable &t = table();
   std::lock_guard<std::mutex> lock(t.mu);
   initFromEnv(t);
   auto it = t.entries.find(key);
   return it == t.entries.end() ? -1 : it->second;
}

DSPLIB_STATUS DSPLIB_gpu_autotuneStore(const char *key, int32_t choice)
{
   if (!key || !*key || choice < 0) return DSPLIB_ERR_INVALID_VALUE;
   tuneStore(key, choice, false);
   return DSPLIB_SUCCESS;
}

static std::string handleKey(DSPLIB_kernelHandle handle, std::vector<int> *cands)
{
   if (!handle) return std::string();
   const uint32_t magic = ((const HandleCommon *) handle)->magic;
   if (magic == kMagicFir) return firHandleTuneKey(handle, cands);
   if (magic == kMagicBiquad) return biquadHandleTuneKey(handle, cands);
   return std::string();
}

DSPLIB_STATUS DSPLIB_gpu_autotune(DSPLIB_kernelHandle handle)
{
   if (!handle) return DSPLIB_ERR_NULL_POINTER;
   const uint32_t magic = ((const HandleCommon *) handle)->magic;
   if (magic == kMagicFir) return firHandleTune(handle);
   if (magic == kMagicBiquad) return biquadHandleTune(handle);
   return DSPLIB_ERR_NOT_IMPLEMENTED;
}

int32_t DSPLIB_gpu_autotuneHandleKey(DSPLIB_kernelHandle handle, char *buf, int32_t len)
{
   std::vector<int> cands;
   const std::string key = handleKey(handle, &cands);
   if (buf && len > 0) {
      const size_t n = key.size() < (size_t) len - 1 ? key.size() : (size_t) len - 1;
      std::memcpy(buf, key.data(), n);
      buf[n] = 0;
   }
   return key.empty() ? 0 : (int32_t) cands.size();
}

int32_t DSPLIB_gpu_autotuneHandleCandidate(DSPLIB_kernelHandle handle, int32_t i)
{
   std::vector<int> cands;
   if (handleKey(handle, &cands).empty() || i < 0 || i >= (int32_t) cands.size()) return -1;
   return cands[i];
}

int32_t DSPLIB_gpu_autotuneCount(void)
{
   TuneTable &t = table();
   std::lock_guard<std::mutex> lock(t.mu);
   initFromEnv(t);
   return (int32_t) t.entries.size();
}

} // extern "C"
