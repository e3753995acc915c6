// sk_noalloc.cu — a radix sort entry point that allocates nothing.
//
// Some callers cannot allocate device memory at all: code running inside a
// host callback or a driver hook where cudaMalloc is not permitted, embedders
// whose allocator owns every byte of the device and forbids other libraries
// from allocating, and real-time loops that must not block on the allocator.
// For them strata_sort_u32_noalloc sorts caller-owned buffers using only a
// fixed scratch area compiled into this library.
//
// The scratch is the file-scope array below.  Its host-side name is only a
// stand-in for the device symbol, so its device address is looked up once per
// device with cudaGetSymbolAddress (with that device current) and cached.
// That lookup happens inside the first call made on each device; make that
// first call before any stream capture.
//
// Every call shares the one array and it keeps the last call's contents, so
// each call clears the parts that must start at zero.  Calls whose GPU work
// overlaps (two host threads, or two streams, on the same device) race on the
// array: callers must serialize them.
#include "sk_ops.cuh"

#include <mutex>

namespace {

// Largest input of one call: 2^20 keys (4 MiB of keys).
constexpr uint64_t kNoAllocMaxKeys = 1ull << 20;
// Histograms, bin offsets, counters, status word, look-back table (274 tiles)
// and the ping-pong half: 4,483,200 bytes, held by every GPU that loads the
// library until the process exits.
constexpr uint64_t kScratchBytes = 4 * 256 * 4 + 4 * 256 * 4 + 64 + 64 + 274 * 256 * 4 + kNoAllocMaxKeys * 4;

static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_sort_scratch on the current device (set-up once per device).
cudaError_t scratch_for_current_device(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" strata_status strata_sort_u32_noalloc(const uint32_t* d_keys_in, uint32_t* d_keys_out, uint64_t n,
                                                 int key_bits, void* stream) {
  if (n > kNoAllocMaxKeys) return STRATA_E_INVALID;  // beyond STRATA_NOALLOC_SORT_MAX_KEYS
  if (key_bits < 0 || key_bits > 32) return STRATA_E_INVALID;
  if (n && (!d_keys_in || !d_keys_out)) return STRATA_E_INVALID;
  // The passes scatter into d_keys_out while other tiles still read their
  // input: overlapping buffers would corrupt the keys without an error.
  if (n) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(d_keys_in), b = reinterpret_cast<uintptr_t>(d_keys_out);
    if (a < b + n * 4 && b < a + n * 4) return STRATA_E_INVALID;
  }
  if (sk::radix_sort_u32_static_bytes(kNoAllocMaxKeys) > kScratchBytes) return STRATA_E_CUDA;
  if (n == 0) return STRATA_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char* scratch = nullptr;
  if (scratch_for_current_device(&scratch) != cudaSuccess) {
    cudaGetLastError();
    return STRATA_E_CUDA;
  }
  try {
    if (key_bits == 0) {
      sk::check_cuda(cudaMemcpyAsync(d_keys_out, d_keys_in, n * 4, cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync");
      sk::check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
      return STRATA_OK;
    }
    uint32_t h_status = 0;
    sk::radix_sort_u32_static(s, d_keys_in, d_keys_out, n, key_bits, scratch, kNoAllocMaxKeys, &h_status);
    sk::check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (h_status & sk::ST_LOOKBACK_TIMEOUT) return STRATA_E_TIMEOUT;
    if (h_status) return STRATA_E_CUDA;
  } catch (const sk::SkError& err) {
    cudaGetLastError();
    return err.code;
  }
  return STRATA_OK;
}
