// Context, status and error plumbing of the C ABI; the shared start-vector
// generator.
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include "internal.cuh"

namespace fame {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void count_launch(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_last_error(int code, const std::string& msg) {
  g_last_error = std::string(fame_status_string(code)) + ": " + msg;
}

int fail(int code, const std::string& msg) {
  set_last_error(code, msg);
  return code;
}

// Stream-ordered allocation for this host thread (StreamOrderedAlloc): device
// memory then comes from the device's default memory pool on that stream, and a
// free waits for that stream only instead of the whole device.
static thread_local bool t_ordered = false;
static thread_local cudaStream_t t_alloc_stream = nullptr;

StreamOrderedAlloc::StreamOrderedAlloc(cudaStream_t s) : prev_on(t_ordered), prev(t_alloc_stream) {
  t_ordered = true;
  t_alloc_stream = s;
}
StreamOrderedAlloc::~StreamOrderedAlloc() {
  t_ordered = prev_on;
  t_alloc_stream = prev;
}

// Per-device state shared by all handles: the device fault word that bounded
// in-kernel waits set when they give up, the SM count, and the stream on which
// the library's device allocations are ordered.
constexpr int kMaxDevices = 64;
static std::atomic<unsigned*> g_fault[kMaxDevices];
static std::atomic<int> g_sms[kMaxDevices];
static std::mutex g_dev_mu;

static int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) return -1;
  return d;
}
static std::atomic<cudaStream_t> g_pool_stream[kMaxDevices];

// Device memory of the library comes from a memory pool the library creates per
// device (not the device's default pool, so the retention set here affects no other
// user of the process), kept cached between a free and the next allocation (creating
// and destroying handles then costs no new mappings of device memory);
// fame_device_trim_memory returns it to the driver.
static std::atomic<cudaMemPool_t> g_pool[kMaxDevices];

static cudaStream_t pool_stream(int dev) {
  if (dev < 0) return nullptr;
  cudaStream_t s = g_pool_stream[dev].load();
  if (s) return s;
  std::lock_guard<std::mutex> lk(g_dev_mu);
  s = g_pool_stream[dev].load();
  if (!s) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      cudaMemPoolDestroy(pool);
      return nullptr;
    }
    cudaGetLastError();
    g_pool[dev].store(pool);
    g_pool_stream[dev].store(s);
  }
  return s;
}

int dalloc(void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return FAME_OK;
  cudaError_t e;
  const int dev = current_device();
  cudaStream_t ps = pool_stream(dev);
  cudaMemPool_t pool = dev >= 0 ? g_pool[dev].load() : nullptr;
  if (!ps || !pool) {
    e = cudaErrorNotReady;
  } else if (t_ordered) {
    // usable on every stream once the (host-side) pool allocation is ordered
    e = cudaMallocFromPoolAsync(p, bytes, pool, t_alloc_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t_alloc_stream);
  } else {
    // the host wait makes the block usable on every stream
    e = cudaMallocFromPoolAsync(p, bytes, pool, ps);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ps);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(e == cudaErrorMemoryAllocation ? FAME_ERR_OOM : FAME_ERR_CUDA,
                std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
  }
  return FAME_OK;
}

void dfree(void* p) {
  if (!p) return;
  if (t_ordered) {
    // every use of the block was queued on this thread's stream: wait for it, then free in order
    cudaStreamSynchronize(t_alloc_stream);
    cudaFreeAsync(p, t_alloc_stream);
  } else {
    // the same device-wide wait as cudaFree, then back to the pool instead of the driver,
    // on the device that owns the block (which need not be the current one)
    int owner = current_device(), prev = owner;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) == cudaSuccess && at.device >= 0) owner = at.device;
    cudaGetLastError();
    if (owner != prev) cudaSetDevice(owner);
    cudaDeviceSynchronize();
    cudaFreeAsync(p, pool_stream(owner));
    if (owner != prev) cudaSetDevice(prev);
  }
}


int ensure_device_state(int device) {
  if (device < 0 || device >= kMaxDevices) return fail(FAME_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (g_fault[device].load() == nullptr) {
    unsigned* p = nullptr;
    FAME_CUDA_TRY(cudaMalloc(&p, sizeof(unsigned)));
    FAME_CUDA_TRY(cudaMemset(p, 0, sizeof(unsigned)));
    g_fault[device].store(p);
  }
  if (g_sms[device].load() == 0) {
    int v = 0;
    FAME_CUDA_TRY(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
    g_sms[device].store(v);
  }
  return FAME_OK;
}

unsigned* fault_word() {
  const int d = current_device();
  return d < 0 ? nullptr : g_fault[d].load();
}

int num_sms() {
  const int d = current_device();
  const int v = d < 0 ? 0 : g_sms[d].load();
  return v > 0 ? v : 148;
}

int check_fault(fame_ctx* ctx) {
  unsigned* p = g_fault[ctx->device].load();
  if (!p) return FAME_OK;
  FAME_CUDA_TRY(cudaMemcpyAsync(ctx->pinned, p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
  FAME_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  unsigned v = 0;
  std::memcpy(&v, ctx->pinned, sizeof(unsigned));
  if (v == 0) return FAME_OK;
  FAME_CUDA_TRY(cudaMemsetAsync(p, 0, sizeof(unsigned), ctx->stream));
  return fail(FAME_ERR_CUDA, "a bounded device-side wait gave up (bulk copy never completed); results are invalid");
}

int ctx_workspace(fame_ctx* ctx, size_t bytes, void** out) {
  if (bytes > ctx->ws_bytes) {
    FAME_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    dfree(ctx->ws);
    ctx->ws = nullptr;
    ctx->ws_bytes = 0;
    FAME_TRY(dalloc(&ctx->ws, bytes));
    ctx->ws_bytes = bytes;
  }
  *out = ctx->ws;
  return FAME_OK;
}

int read_back(fame_ctx* ctx, const void* dsrc, void* hdst, size_t bytes) {
  if (bytes > 4096) return fail(FAME_ERR_INVALID, "read_back larger than staging area");
  FAME_CUDA_TRY(cudaMemcpyAsync(ctx->pinned, dsrc, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  FAME_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  std::memcpy(hdst, ctx->pinned, bytes);
  return FAME_OK;
}

// splitmix64 over the counter; shared with the oracle's start_vector.
__global__ void k_start_vector(unsigned long long seed, long long n, double2* v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double u[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      unsigned long long c = 2ull * (unsigned long long)i + h;
      unsigned long long z = seed + (c + 1ull) * 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z = z ^ (z >> 31);
      u[h] = 2.0 * ((double)(z >> 11) * 0x1.0p-53) - 1.0;
    }
    v[i] = make_double2(u[0], u[1]);
  }
}

}  // namespace fame

using namespace fame;

extern "C" {

const char* fame_status_string(int s) {
  switch (s) {
    case FAME_OK: return "FAME_OK";
    case FAME_ERR_INVALID: return "FAME_ERR_INVALID";
    case FAME_ERR_CUDA: return "FAME_ERR_CUDA";
    case FAME_ERR_OOM: return "FAME_ERR_OOM";
    case FAME_ERR_NOT_CONVERGED: return "FAME_ERR_NOT_CONVERGED";
    case FAME_ERR_NONFINITE: return "FAME_ERR_NONFINITE";
    case FAME_ERR_BUDGET: return "FAME_ERR_BUDGET";
    case FAME_ERR_SINGULAR: return "FAME_ERR_SINGULAR";
    case FAME_ERR_UNSUPPORTED: return "FAME_ERR_UNSUPPORTED";
    case FAME_ERR_BREAKDOWN: return "FAME_ERR_BREAKDOWN";
    default: return "FAME_ERR_UNKNOWN";
  }
}

const char* fame_last_error(void) { return g_last_error.c_str(); }

int fame_version(void) { return 100; }

long long fame_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

int fame_device_trim_memory(int device) {
  int prev = 0, count = 0;
  FAME_CUDA_TRY(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(FAME_ERR_INVALID, "bad device index");
  FAME_CUDA_TRY(cudaGetDevice(&prev));
  FAME_CUDA_TRY(cudaSetDevice(device));
  cudaMemPool_t pool = g_pool[device].load();
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess && pool) e = cudaMemPoolTrimTo(pool, 0);
  cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(FAME_ERR_CUDA, std::string("fame_device_trim_memory: ") + cudaGetErrorString(e));
  return FAME_OK;
}

int fame_ctx_create(int device, fame_ctx** out) {
  if (!out) return fail(FAME_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int count = 0;
  FAME_CUDA_TRY(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(FAME_ERR_INVALID, "bad device index");
  FAME_CUDA_TRY(cudaSetDevice(device));
  FAME_TRY(ensure_device_state(device));
  fame_ctx* c = new fame_ctx();
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaMallocHost(&c->pinned, 4096) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return fail(FAME_ERR_CUDA, "context resources");
  }
  c->stream = c->own;
  *out = c;
  return FAME_OK;
}

int fame_ctx_destroy(fame_ctx* c) {
  if (!c) return FAME_OK;
  cudaStreamSynchronize(c->stream);
  if (c->pinned) cudaFreeHost(c->pinned);
  dfree(c->ws);
  if (c->ev) cudaEventDestroy(c->ev);
  if (c->capture) cudaStreamDestroy(c->capture);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return FAME_OK;
}

int fame_ctx_set_stream(fame_ctx* c, void* stream) {
  if (!c) return fail(FAME_ERR_INVALID, "ctx is NULL");
  c->stream = (cudaStream_t)stream;  // NULL: the legacy default stream, as everywhere in CUDA
  return FAME_OK;
}

int fame_ctx_use_own_stream(fame_ctx* c) {
  if (!c) return fail(FAME_ERR_INVALID, "ctx is NULL");
  c->stream = c->own;
  return FAME_OK;
}

int fame_ctx_sync(fame_ctx* c) {
  if (!c) return fail(FAME_ERR_INVALID, "ctx is NULL");
  FAME_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return check_fault(c);
}

int fame_start_vector(fame_ctx* c, unsigned long long seed, long long n, void* v) {
  if (!c || !v || n <= 0) return fail(FAME_ERR_INVALID, "fame_start_vector arguments");
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 16);
  k_start_vector<<<blocks, 256, 0, c->stream>>>(seed, n, (double2*)v);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

}  // extern "C"
