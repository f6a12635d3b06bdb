// libpqi: an allocation-free single-bit-flip pass.
//
// Some callers cannot hand the library a workspace: a host process whose device
// memory belongs to another framework's allocator (which forbids raw cudaMalloc
// next to it), or a latency-bound loop that must not call cudaMalloc because it
// can synchronise the whole device. pqi_single_bit_flips_noalloc serves them: it
// is pqi_single_bit_flips with its scratch (the selection key and the n float32
// gains) in a fixed array compiled into the library instead of in a caller
// workspace. The caller still passes the weights, the state and the outputs.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds it (PQI_NOALLOC_BYTES) until the process exits. In host code its
// name is only a host-side stand-in, so the device address is looked up once
// per device with cudaGetSymbolAddress, with that device current, on the first
// call made there; that first call should come before any stream capture.
// All calls share the array and it keeps the last call's contents (the key is
// cleared at the start of every call); calls that overlap on the GPU, from two
// streams or two host threads on one device, race on it.
#include <mutex>

#include "pqi_common.cuh"

namespace pqi {

constexpr int kNoAllocMaxN = PQI_NOALLOC_MAX_N;
constexpr size_t kNoAllocKeyBytes = 256;
constexpr size_t kNoAllocBytes = kNoAllocKeyBytes + (size_t)kNoAllocMaxN * sizeof(float);
static_assert(kNoAllocBytes == PQI_NOALLOC_BYTES, "header and library disagree on the array size");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
static void* g_noalloc_addr[kMaxDevices] = {nullptr};
static std::mutex g_noalloc_mu;

// Device address of g_noalloc_scratch on the current device (looked up once).
static pqi_status noalloc_scratch(void** out) {
  int dev = 0;
  PQI_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error_text("pqi_single_bit_flips_noalloc: device ordinal above 63");
    return PQI_ENOTSUP;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
      return PQI_ECUDA;
    }
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return PQI_OK;
}

}  // namespace pqi

using namespace pqi;

extern "C" pqi_status pqi_single_bit_flips_noalloc(const pqi_weights* w, const uint32_t* theta,
                                                   int is_spin_glass, int global_size,
                                                   int local_size, float* best_energy,
                                                   int* best_index, void* stream) {
  PQI_CHECK_ARG(w && theta);
  if (w->n < 1 || w->n > kNoAllocMaxN) {
    set_error_text("pqi_single_bit_flips_noalloc: n must be in [1, PQI_NOALLOC_MAX_N = 65536]");
    return PQI_EINVAL;
  }
  SelGeom geo;
  PQI_CHECK_ARG(make_sel_geom(w->n, global_size, local_size, &geo));
  void* scratch = nullptr;
  pqi_status rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  unsigned long long* key = static_cast<unsigned long long*>(scratch);
  float* g32 = reinterpret_cast<float*>(static_cast<char*>(scratch) + kNoAllocKeyBytes);
  cudaStream_t s = as_stream(stream);
  rc = launch_gains(w, theta, 1, g32, nullptr, s);
  if (rc) return rc;
  // launch_select clears the key before the reduction
  return launch_select(g32, w->n, is_spin_glass ? 2.0f : 1.0f, geo, key, best_energy, best_index,
                       s);
}
