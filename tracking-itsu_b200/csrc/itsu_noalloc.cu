// itsu_noalloc.cu - the clustering stage of one primary vertex with no allocation at all.
//
// Some callers cannot call cudaMalloc: an online reconstruction process that reserves the
// device's memory through its own pool when it starts (a cudaMalloc would fail or fight the
// pool), or a latency-critical loop where an allocation's implicit device synchronisation is not
// acceptable. itsu_pvc_initialize_noalloc serves them: the caller passes device inputs and
// outputs, and the only scratch the kernel needs (the transformed clusters in input order, the
// coordinate copies the sort writes beside its output, and the status word) lives in the
// file-scope array below, which every GPU that loads the library holds until the process exits.
//
// In host code, itsu_noalloc_scratch names a host-side stand-in, not the device array: its
// device address is obtained once per device with cudaGetSymbolAddress, with that device current,
// on the first call made on that device, and cached. No call can be captured into a CUDA graph:
// each one reads the layer offsets back and waits for its stream. The cached address belongs to the device's context at that time: a
// cudaDeviceReset (or anything else that destroys the primary context) leaves it stale, so the
// entry point must not be used on a device after it has been reset while the library stays
// loaded. All calls share the one array and it keeps the last call's
// contents; the status word is cleared at the start of each call, everything else is written
// before it is read. Calls whose work overlaps on the GPU (concurrent streams, or threads calling
// at the same time) race on the array.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "itsu.h"
#include "itsu_internal.h"

namespace {

constexpr int64_t kMaxClusters = ITSU_NOALLOC_MAX_CLUSTERS;
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }
// layout: DevStatus | transformed clusters | xyzr | phi | per-cluster id, alpha, MC id, bin
constexpr size_t kStatusOff = 0;
constexpr size_t kTmpOff = align_up(sizeof(itsu::DevStatus));
constexpr size_t kXyzrOff = kTmpOff + align_up(sizeof(itsu_cluster) * kMaxClusters);
constexpr size_t kPhiOff = kXyzrOff + align_up(sizeof(float4) * kMaxClusters);
constexpr size_t kAuxOff = kPhiOff + align_up(sizeof(float) * kMaxClusters);
constexpr size_t kScratchBytes = kAuxOff + align_up(sizeof(int4) * kMaxClusters);

static __device__ __align__(256) unsigned char itsu_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned char *g_scratch[kMaxDevices] = {};  // device address of the array, per device

// The message is reported through itsu_last_error(NULL), the calling thread's last error.
itsu_status noalloc_fail(itsu_status st, const char *fmt, ...)
{
  char buf[384];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  itsu::set_thread_error(buf);
  return st;
}

}  // namespace

extern "C" itsu_status itsu_pvc_initialize_noalloc(const itsu_cluster *clusters, const int32_t *layer_offsets,
                                                   const float *vertex, int64_t n_clusters, itsu_cluster *sorted,
                                                   int32_t *index_tables, void *cuda_stream)
{
  if (n_clusters < 0 || n_clusters > kMaxClusters) {
    return noalloc_fail(ITSU_ERR_CAPACITY, "itsu_pvc_initialize_noalloc: %lld clusters, at most %lld fit the static scratch",
                        (long long)n_clusters, (long long)kMaxClusters);
  }
  if (!layer_offsets || !vertex || !index_tables || (n_clusters > 0 && (!clusters || !sorted))) {
    return noalloc_fail(ITSU_ERR_INVALID, "itsu_pvc_initialize_noalloc: null pointer");
  }
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess || device < 0 || device >= kMaxDevices) {
    return noalloc_fail(ITSU_ERR_CUDA, "itsu_pvc_initialize_noalloc: no current device (%s)", cudaGetErrorString(err));
  }
  unsigned char *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch[device]) {
      void *p = nullptr;
      err = cudaGetSymbolAddress(&p, itsu_noalloc_scratch);
      if (err != cudaSuccess) {
        return noalloc_fail(ITSU_ERR_CUDA, "itsu_pvc_initialize_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(err));
      }
      g_scratch[device] = static_cast<unsigned char *>(p);
    }
    scratch = g_scratch[device];
  }
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);

  // The offsets bound every index the kernel touches: check them before launching.
  int32_t off[ITSU_LAYERS + 1];
  if ((err = cudaMemcpyAsync(off, layer_offsets, sizeof off, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
      (err = cudaStreamSynchronize(stream)) != cudaSuccess) {
    return noalloc_fail(ITSU_ERR_CUDA, "itsu_pvc_initialize_noalloc: reading layer offsets: %s", cudaGetErrorString(err));
  }
  if (off[0] != 0 || off[ITSU_LAYERS] != n_clusters) {
    return noalloc_fail(ITSU_ERR_INVALID, "itsu_pvc_initialize_noalloc: layer offsets must run from 0 to n_clusters");
  }
  for (int l = 0; l < ITSU_LAYERS; ++l) {
    if (off[l + 1] < off[l]) return noalloc_fail(ITSU_ERR_INVALID, "itsu_pvc_initialize_noalloc: layer offsets decrease");
  }

  itsu::Arena a{};
  a.n_events = 1;
  a.n_clusters = n_clusters;
  a.raw = clusters;
  a.layer_off = layer_offsets;
  a.vtx = vertex;
  a.sorted = sorted;
  a.index_tables = index_tables;
  a.status = reinterpret_cast<itsu::DevStatus *>(scratch + kStatusOff);
  a.tmp = reinterpret_cast<itsu_cluster *>(scratch + kTmpOff);
  a.xyzr = reinterpret_cast<float4 *>(scratch + kXyzrOff);
  a.phi = reinterpret_cast<float *>(scratch + kPhiOff);
  a.clu_aux = reinterpret_cast<int4 *>(scratch + kAuxOff);
  const itsu::Launch l{stream, 0, 256, 8};
  itsu::launch_status_init(a, l);
  itsu::launch_cluster_sort(a, l);
  if ((err = cudaGetLastError()) != cudaSuccess) {
    return noalloc_fail(ITSU_ERR_CUDA, "itsu_pvc_initialize_noalloc: launch: %s", cudaGetErrorString(err));
  }
  itsu::DevStatus status;
  if ((err = cudaMemcpyAsync(&status, a.status, sizeof status, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
      (err = cudaStreamSynchronize(stream)) != cudaSuccess) {
    return noalloc_fail(ITSU_ERR_CUDA, "itsu_pvc_initialize_noalloc: %s", cudaGetErrorString(err));
  }
  if (status.flags & itsu::kFlagInvalid) {
    return noalloc_fail(ITSU_ERR_INVALID, "itsu_pvc_initialize_noalloc: malformed %s (index %d)",
                        status.invalid_event != INT32_MAX ? "primary vertex" : "cluster", status.invalid_index);
  }
  return ITSU_OK;
}
