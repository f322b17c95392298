// itsu_report.cu - the road report on the device: IOUtils::writeRoadsReport (src/CA/IOUtils.cxx:
// 125-170) classifies every road of an event against the event's labels map.
//
// Per event an open-addressing hash table (linear probing, power-of-two size at least twice the
// event's labels) holds the map's Monte Carlo ids; each slot keeps the first label entry with its
// id (std::unordered_map::emplace keeps the first) and the first non-fake road that carries it.
// Roads are numbered in the batch's run-major order, which within an event is the reference's
// vertex-then-road order, so "first" is an atomicMin. Three passes: insert the labels, look up
// every road (recording the first non-fake road per slot), classify every road and count.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "itsu.h"
#include "itsu_internal.h"

namespace itsu {
namespace {

constexpr int kReportThreads = 256;
constexpr int32_t kEmptyKey = INT32_MIN;

__device__ __forceinline__ uint32_t hash_id(int32_t id)
{
  uint32_t h = (uint32_t)id * 0x9E3779B1u;  // Fibonacci hashing, then a final mix of the high bits
  return h ^ (h >> 15);
}

__device__ __forceinline__ int64_t global_index() { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int64_t global_stride() { return (int64_t)gridDim.x * blockDim.x; }

__global__ void k_report_clear(ReportArgs r)
{
  for (int64_t i = global_index(); i < r.table_size; i += global_stride()) {
    r.keys[i] = kEmptyKey;
    r.first_label[i] = INT32_MAX;
    r.first_road[i] = INT64_MAX;
  }
  for (int64_t e = global_index(); e < r.n_events; e += global_stride()) {
    r.counts[e] = itsu_report_counts{0, 0, 0, 0};
  }
}

// Slot of key in event e's table: found (>= 0), absent (-1) or, when inserting, the slot it was
// put in. The probe sequence is bounded by the table size.
__global__ void k_report_insert(ReportArgs r)
{
  for (int64_t i = global_index(); i < r.n_labels; i += global_stride()) {
    const int e = r.label_event[i];
    const int32_t key = r.labels[i].mc_id;
    const int64_t base = r.table_base[e];
    const uint32_t mask = (uint32_t)(r.table_base[e + 1] - base - 1);
    uint32_t h = hash_id(key) & mask;
    for (uint32_t probe = 0; probe <= mask; ++probe, h = (h + 1) & mask) {
      const int32_t prev = atomicCAS(&r.keys[base + h], kEmptyKey, key);
      if (prev == kEmptyKey || prev == key) {
        if (prev == kEmptyKey) {
          atomicAdd(&r.counts[e].labels, 1);
        }
        atomicMin(&r.first_label[base + h], (int32_t)i);
        break;
      }
    }
  }
}

__device__ __forceinline__ int run_of(const int32_t *run_offsets, int n_runs, int64_t road)
{
  int lo = 0, hi = n_runs;  // the last run r with run_offsets[r] <= road
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (run_offsets[mid] <= road) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  return lo;
}

__device__ __forceinline__ int64_t find_slot(const ReportArgs &r, int e, int32_t key)
{
  const int64_t base = r.table_base[e];
  const uint32_t mask = (uint32_t)(r.table_base[e + 1] - base - 1);
  uint32_t h = hash_id(key) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe, h = (h + 1) & mask) {
    const int32_t k = r.keys[base + h];
    if (k == key) {
      return base + h;
    }
    if (k == kEmptyKey) {
      return -1;
    }
  }
  return -1;
}

__global__ void k_report_lookup(ReportArgs r)
{
  for (int64_t i = global_index(); i < r.n_roads; i += global_stride()) {
    const int run = run_of(r.run_offsets, r.n_runs, i);
    const int e = r.run_event ? r.run_event[run] : run;
    const itsu_road road = r.roads[i];
    const int64_t slot = road.label == kEmptyKey ? -1 : find_slot(r, e, road.label);
    r.road_slot[i] = slot;
    r.road_event[i] = e;
    if (slot >= 0 && !road.is_fake) {
      atomicMin(reinterpret_cast<unsigned long long *>(&r.first_road[slot]), (unsigned long long)i);
    }
  }
}

__global__ void k_report_classify(ReportArgs r)
{
  for (int64_t i = global_index(); i < r.n_roads; i += global_stride()) {
    const int64_t slot = r.road_slot[i];
    const int e = r.road_event[i];
    uint8_t cls = ITSU_ROAD_UNREPORTED;
    if (slot >= 0) {
      if (r.roads[i].is_fake) {
        cls = ITSU_ROAD_FAKE;
        atomicAdd(&r.counts[e].fake, 1);
      } else if (r.first_road[slot] == i) {
        cls = ITSU_ROAD_CORRECT;
        atomicAdd(&r.counts[e].correct, 1);
      } else {
        cls = ITSU_ROAD_DUPLICATE;
        atomicAdd(&r.counts[e].duplicate, 1);
      }
    }
    r.road_class[i] = cls;
  }
}

unsigned grid_for(int64_t n, int num_sms)
{
  const int64_t blocks = (n + kReportThreads - 1) / kReportThreads;
  const int64_t cap = (int64_t)num_sms * 8;
  return (unsigned)(blocks < 1 ? 1 : (blocks < cap ? blocks : cap));
}

}  // namespace

void launch_report(const ReportArgs &r, cudaStream_t stream, int num_sms)
{
  const int64_t n_clear = r.table_size > r.n_events ? r.table_size : r.n_events;
  k_report_clear<<<grid_for(n_clear, num_sms), kReportThreads, 0, stream>>>(r);
  if (r.n_labels > 0) {
    k_report_insert<<<grid_for(r.n_labels, num_sms), kReportThreads, 0, stream>>>(r);
  }
  if (r.n_roads > 0) {
    k_report_lookup<<<grid_for(r.n_roads, num_sms), kReportThreads, 0, stream>>>(r);
    k_report_classify<<<grid_for(r.n_roads, num_sms), kReportThreads, 0, stream>>>(r);
  }
}

}  // namespace itsu
