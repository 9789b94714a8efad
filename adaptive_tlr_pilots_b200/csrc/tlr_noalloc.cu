// Allocation-free Morton ordering.
//
// tlr_morton_order() takes its working memory (sort keys, indices and digit counts) from the
// stream-ordered allocator on every call.  Some callers cannot allocate device memory at that
// point: code that runs while another framework's caching allocator holds the device's memory
// and forbids outside allocations, service loops that must not allocate after start-up, or
// callers that only hand in buffers they already own.  tlr_morton_order_noalloc() serves them:
// it runs the same kernels with their working memory in one fixed array that lives in this
// library's device image, so the call itself allocates nothing.
#include "../../include/tlr_b200.h"
#include "tlr_kernels.h"

constexpr int kMaxSites = 1 << 20;  // n <= 1,048,576
constexpr int kMaxOrder = 10;       // bits per axis (the reference's order)
// keys and indices of n sites plus the digit counts of every 2,048-site tile (at most 256 digit
// values): 2 x 2^20 + 256 x 512 words = 8.5 MiB.  Every GPU that loads the library holds this
// array until the process exits.  In host code the name g_morton_scratch is only a host-side
// stand-in; kernels get the device address below.
constexpr size_t kScratchWords = 2 * (size_t)kMaxSites + 256 * ((size_t)kMaxSites / 2048);
static __device__ __align__(256) unsigned g_morton_scratch[kScratchWords];

namespace {

// Device address of the array on the current device.  Looked up on every call (the lookup is
// cheap and allocates nothing), so a cached address can never outlive its context.
int scratch_for_current_device(unsigned** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_morton_scratch);
  if (e != cudaSuccess || p == nullptr)
    return tlr::set_error(TLR_ERR_CUDA, e != cudaSuccess ? cudaGetErrorString(e) : "no symbol address");
  *out = static_cast<unsigned*>(p);
  return 0;
}

}  // namespace

extern "C" int tlr_morton_order_noalloc(const double* xy_dev, int n, int order, long long* perm_dev, void* stream) {
  if (!xy_dev || !perm_dev) return tlr::set_error(TLR_ERR_ARG, "xy and perm must be device pointers");
  if (n < 1 || n > kMaxSites)
    return tlr::set_error(TLR_ERR_ARG, "tlr_morton_order_noalloc: n must be in [1, 1048576]");
  if (order < 1 || order > kMaxOrder)
    return tlr::set_error(TLR_ERR_ARG, "tlr_morton_order_noalloc: order must be in [1, 10]");
  if (tlr::morton_work_words(n, order) > kScratchWords)
    return tlr::set_error(TLR_ERR_ARG, "tlr_morton_order_noalloc: working set exceeds the static array");
  unsigned* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc != 0) return rc;
  // Every word the kernels read is written earlier in the same call (keys and indices by the key
  // kernel, each pass's digit counts by its histogram kernel), so what an earlier call left in the
  // array does not matter.
  const int lr = tlr::launch_morton(xy_dev, n, order, scratch, perm_dev, static_cast<cudaStream_t>(stream));
  if (lr != 0) return tlr::set_error(TLR_ERR_CUDA, cudaGetErrorString((cudaError_t)lr));
  return 0;
}
