// Allocation-free Morton ordering.
//
// tlr_morton_order() takes its working memory (sort keys and the per-key counters) from the
// stream-ordered allocator on every call.  Some callers cannot allocate device memory at that
// point: code that runs while another framework's caching allocator holds the device's memory
// and forbids outside allocations, service loops that must not allocate after start-up, or
// callers that only hand in buffers they already own.  tlr_morton_order_noalloc() serves them:
// it runs the same kernels with their working memory in one fixed array that lives in this
// library's device image, so the call itself allocates nothing.
#include "../../include/tlr_b200.h"
#include "tlr_kernels.h"

#include <mutex>

constexpr int kMaxSites = 1 << 20;      // n <= 1,048,576
constexpr int kMaxOrder = 10;           // bits per axis (the reference's order)
constexpr size_t kBuckets = (size_t)1 << (2 * kMaxOrder);
// keys[n] + counts, offsets and cursors for every key value: 4 x 2^20 x 4 bytes = 16 MiB.
// Every GPU that loads the library holds this array until the process exits.  In host code the
// name g_morton_scratch is only a host-side stand-in; kernels get the device address below.
constexpr size_t kScratchWords = (size_t)kMaxSites + 3 * kBuckets;
static __device__ __align__(256) unsigned g_morton_scratch[kScratchWords];

namespace {

constexpr int kMaxDevices = 64;
unsigned* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

// Device address of the array on the current device, looked up once per device.
int scratch_for_current_device(unsigned** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return tlr::set_error(TLR_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return tlr::set_error(TLR_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_morton_scratch);
    if (e != cudaSuccess || p == nullptr)
      return tlr::set_error(TLR_ERR_CUDA, e != cudaSuccess ? cudaGetErrorString(e) : "no symbol address");
    g_scratch_addr[dev] = static_cast<unsigned*>(p);
  }
  *out = g_scratch_addr[dev];
  return 0;
}

}  // namespace

extern "C" int tlr_morton_order_noalloc(const double* xy_dev, int n, int order, long long* perm_dev, void* stream) {
  if (!xy_dev || !perm_dev) return tlr::set_error(TLR_ERR_ARG, "xy and perm must be device pointers");
  if (n < 1 || n > kMaxSites)
    return tlr::set_error(TLR_ERR_ARG, "tlr_morton_order_noalloc: n must be in [1, 1048576]");
  if (order < 1 || order > kMaxOrder)
    return tlr::set_error(TLR_ERR_ARG, "tlr_morton_order_noalloc: order must be in [1, 10]");
  unsigned* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc != 0) return rc;
  unsigned* keys = scratch;
  unsigned* cnt = keys + kMaxSites;
  unsigned* off = cnt + kBuckets;
  unsigned* cur = off + kBuckets;
  // launch_morton clears the counters it needs (cnt) before use; keys, offsets and cursors are
  // fully rewritten, so what an earlier call left in the array does not matter.
  const int lr = tlr::launch_morton(xy_dev, n, order, keys, cnt, off, cur, perm_dev, static_cast<cudaStream_t>(stream));
  if (lr != 0) return tlr::set_error(TLR_ERR_CUDA, cudaGetErrorString((cudaError_t)lr));
  return 0;
}
