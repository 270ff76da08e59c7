// Library runtime: error text, per-device stream, stream-ordered allocation,
// device status word.
#include <cstdarg>
#include <mutex>

#include "hp_runtime.cuh"

namespace hp {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char* last_error() { return g_err; }

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
cudaStream_t g_stream[kMaxDevices] = {};
cudaStream_t g_copy_stream[kMaxDevices][2] = {};
bool g_pool_ready[kMaxDevices] = {};
// One sticky status word per device: kernels OR bits into it, and the host
// entry points read and clear it at their synchronisation points
// (consume_device_status), so no launch needs a memset in front of it.
uint32_t* g_status[kMaxDevices] = {};

int cur_dev() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}
void ensure_pool(int d) {
  if (g_pool_ready[d]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, d) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  g_pool_ready[d] = true;
}
}  // namespace

cudaStream_t library_stream() {
  std::lock_guard<std::mutex> lk(g_mu);
  int d = cur_dev();
  if (!g_stream[d]) cudaStreamCreateWithFlags(&g_stream[d], cudaStreamNonBlocking);
  ensure_pool(d);
  return g_stream[d];
}

cudaStream_t library_copy_stream(int which) {
  std::lock_guard<std::mutex> lk(g_mu);
  int d = cur_dev();
  cudaStream_t& st = g_copy_stream[d][which & 1];
  if (!st) cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  return st;
}

void* dev_alloc(size_t bytes, cudaStream_t s) {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    ensure_pool(cur_dev());
  }
  void* p = nullptr;
  if (cudaMallocAsync(&p, bytes, s) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
void dev_free(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

uint32_t* device_status(cudaStream_t) {
  int d = cur_dev();
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_status[d]) {
    if (cudaMalloc(&g_status[d], 64 * sizeof(uint32_t)) != cudaSuccess ||
        cudaMemset(g_status[d], 0, 64 * sizeof(uint32_t)) != cudaSuccess) {
      cudaGetLastError();
      g_status[d] = nullptr;
      return nullptr;
    }
  }
  return g_status[d];
}

int consume_device_status(cudaStream_t s) {
  uint32_t* w = device_status(s);
  if (!w) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  uint32_t h = 0;
  HP_CUDA_TRY(cudaMemcpyAsync(&h, w, sizeof(h), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (h == 0) return HP_OK;
  HP_CUDA_TRY(cudaMemsetAsync(w, 0, sizeof(uint32_t), s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (h & DEV_STATUS_TIMEOUT) {
    set_error("a bounded device-side wait gave up (status 0x%x)", h);
    return HP_ERR_TIMEOUT;
  }
  set_error("device status 0x%x", h);
  return HP_ERR_CUDA;
}

namespace {
struct ProfState {
  bool on = false;
  int count = 0;
  cudaEvent_t ev[32];
  const char* name[32];
  bool created = false;
};
ProfState g_prof;
}  // namespace

bool profiling_on() { return g_prof.on; }

void profile_mark(cudaStream_t s, const char* name) {
  if (!g_prof.on || g_prof.count >= 32) return;
  if (!g_prof.created) {
    for (int i = 0; i < 32; i++) cudaEventCreate(&g_prof.ev[i]);
    g_prof.created = true;
  }
  g_prof.name[g_prof.count] = name;
  cudaEventRecord(g_prof.ev[g_prof.count], s);
  g_prof.count++;
}

}  // namespace hp

extern "C" {

void hp_profile_enable(int on) {
  hp::g_prof.on = on != 0;
  hp::g_prof.count = 0;
}

int hp_profile_read(double* ms, int max_phases, char* names, size_t names_len) {
  using hp::g_prof;
  if (g_prof.count < 2) return 0;
  cudaEventSynchronize(g_prof.ev[g_prof.count - 1]);
  int n = g_prof.count - 1 < max_phases ? g_prof.count - 1 : max_phases;
  size_t off = 0;
  for (int i = 0; i < n; i++) {
    float t = 0;
    cudaEventElapsedTime(&t, g_prof.ev[i], g_prof.ev[i + 1]);
    ms[i] = t;
    if (names && off < names_len) {
      int w = snprintf(names + off, names_len - off, "%s%s", i ? "," : "", g_prof.name[i + 1]);
      if (w > 0) off += (size_t)w;
    }
  }
  g_prof.count = 0;
  return n;
}

int hp_device_status(void* stream, uint32_t* bits, int clear) {
  using namespace hp;
  cudaStream_t s = (cudaStream_t)stream;
  uint32_t* w = device_status(s);
  if (!w) {
    set_error("status word allocation failed");
    return HP_ERR_CUDA;
  }
  uint32_t h = 0;
  HP_CUDA_TRY(cudaMemcpyAsync(&h, w, sizeof(h), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (bits) *bits = h;
  if (clear && h) {
    HP_CUDA_TRY(cudaMemsetAsync(w, 0, sizeof(uint32_t), s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (h & DEV_STATUS_TIMEOUT) {
    set_error("a bounded device-side wait gave up (status 0x%x)", h);
    return HP_ERR_TIMEOUT;
  }
  if (h & DEV_STATUS_NOT_SPD) {
    set_error("a Cholesky pivot was not positive (status 0x%x)", h);
    return HP_ERR_NOT_SPD;
  }
  if (h) {
    set_error("device status 0x%x", h);
    return HP_ERR_CUDA;
  }
  return HP_OK;
}

const char* hp_last_error(void) { return hp::last_error(); }
const char* hp_version(void) { return "hyperprec-b200 0.1.0 (sm_100a)"; }

int hp_device_ok(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return 0;
  }
  int d = 0, major = 0, minor = 0;
  cudaGetDevice(&d);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, d);
  return (major == 10 && minor == 0) ? 1 : 0;
}

}  // extern "C"
