#include "common.cuh"

#include <atomic>
#include <cstdarg>
#include <map>
#include <mutex>
#include <vector>

namespace tcb {

static std::atomic<uint64_t> g_launches{0};
void count_launch(unsigned k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

namespace {
struct Rec {
  std::string name;
  cudaEvent_t a, b;
  double bytes, flops;
};
std::mutex g_prof_mu;
std::atomic<bool> g_prof_on{false};
std::vector<Rec> g_recs;
}  // namespace

StageTimer::StageTimer(const char *n, cudaStream_t s, double bytes, double flops)
    : name(n), stream(s), slot(-1) {
  if (!g_prof_on.load(std::memory_order_relaxed)) return;
  Rec r{n, nullptr, nullptr, bytes, flops};
  if (cudaEventCreate(&r.a) != cudaSuccess) return;
  if (cudaEventCreate(&r.b) != cudaSuccess) {
    cudaEventDestroy(r.a);
    return;
  }
  cudaEventRecord(r.a, s);
  std::lock_guard<std::mutex> lk(g_prof_mu);
  slot = (int)g_recs.size();
  g_recs.push_back(r);
}

StageTimer::~StageTimer() {
  if (slot < 0) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (slot < (int)g_recs.size()) cudaEventRecord(g_recs[slot].b, stream);
}

static void clear_recs() {
  for (auto &r : g_recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  g_recs.clear();
}

static thread_local char g_last_error[1024] = {0};

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

int sm_count() {
  static int cached = -1;
  if (cached < 0) {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) ==
            cudaSuccess && v > 0)
      cached = v;
    else
      cached = 148;
  }
  return cached;
}

}  // namespace tcb

extern "C" const char *tcb_last_error(void) { return tcb::g_last_error; }
extern "C" int tcb_version(void) { return 100; }

extern "C" int tcb_profile_enable(int on) {
  std::lock_guard<std::mutex> lk(tcb::g_prof_mu);
  tcb::clear_recs();
  tcb::g_prof_on.store(on != 0);
  return TCB_OK;
}

extern "C" int tcb_profile_report(char *buf, size_t len) {
  TCB_CHECK_ARG(buf && len > 2, "tcb_profile_report: bad buffer");
  std::lock_guard<std::mutex> lk(tcb::g_prof_mu);
  struct Sum {
    long count = 0;
    double ms = 0.0, bytes = 0.0, flops = 0.0;
  };
  std::map<std::string, Sum> acc;
  for (auto &r : tcb::g_recs) {
    TCB_CUDA(cudaEventSynchronize(r.b));
    float ms = 0.f;
    TCB_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    auto &e = acc[r.name];
    e.count += 1;
    e.ms += ms;
    e.bytes += r.bytes;
    e.flops += r.flops;
  }
  std::string out = "{";
  bool first = true;
  char tmp[384];
  for (auto &kv : acc) {
    snprintf(tmp, sizeof(tmp),
             "%s\"%s\": {\"count\": %ld, \"ms\": %.6f, \"bytes\": %.17g, \"flops\": %.17g}",
             first ? "" : ", ", kv.first.c_str(), kv.second.count, kv.second.ms, kv.second.bytes,
             kv.second.flops);
    out += tmp;
    first = false;
  }
  out += "}";
  TCB_CHECK_ARG(out.size() + 1 <= len, "tcb_profile_report: buffer too small (%zu needed)",
                out.size() + 1);
  memcpy(buf, out.c_str(), out.size() + 1);
  return TCB_OK;
}

extern "C" int tcb_launch_count(uint64_t *out) {
  TCB_CHECK_ARG(out, "tcb_launch_count: null out");
  *out = tcb::g_launches.load();
  return TCB_OK;
}

extern "C" int tcb_copy2d(void *dst, size_t dpitch, const void *src, size_t spitch,
                          size_t width_bytes, size_t height, void *stream) {
  TCB_CHECK_ARG(dst && src, "tcb_copy2d: null pointer");
  TCB_CHECK_ARG(dpitch >= width_bytes && spitch >= width_bytes, "tcb_copy2d: pitch < width");
  if (width_bytes == 0 || height == 0) return TCB_OK;
  TCB_CUDA(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width_bytes, height,
                             cudaMemcpyDefault, (cudaStream_t)stream));
  return TCB_OK;
}
