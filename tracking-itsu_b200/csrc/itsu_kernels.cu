// itsu_kernels.cu - sm_100a kernels of the ITS CA track finder.
//
// Every stage is a deterministic count -> exclusive scan -> write sequence over flat,
// event-major arrays, so the output order is the reference's emission order with no atomics on
// the output path (the only atomics fill neighbour rows, which are then sorted):
//   clustering   one CTA per (event, layer): vertex-relative transform, stable counting sort by
//                bin (per-warp histograms, warp-match ranks), index table (PVC.cxx:31-142)
//   tracklets    one thread per inner cluster walking the reference's bin window (Tracker.cxx:45-117)
//   cells        one thread per tracklet walking the next-layer tracklets of its outer cluster
//                (Tracker.cxx:120-235)
//   neighbours   one thread per cell walking the next-layer cells of its outer tracklet; rows
//                keyed by the next-layer cell, sorted ascending (Tracker.cxx:417-474)
//   levels       layer-ordered longest-chain DP plus the number of level-decreasing chains
//   roads        one thread per level-5 cell: depth-first enumeration in the reference's order,
//                Moore-vote labels (Tracker.cxx:477-652)
// Capacity overflow never writes out of bounds: the write passes check the scanned totals
// against the arena capacities, record the requirement and skip; the host grows and re-runs.
#include <climits>

#include "itsu_device.cuh"
#include "itsu_internal.h"

namespace itsu {
namespace {

constexpr int kThreads = 256;
constexpr int kSortThreads = 512;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kBuckets = kTableSize + 1;  // bucket 0: negative bins; bucket b+1: bin b
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr float kMaxAbsCoordinate = 1.0e6f;

__device__ __forceinline__ bool capacity_failed(const DevStatus *s) { return (*(volatile const int32_t *)&s->flags & kCapacityMask) != 0; }

// Largest s in [0, nseg) with off[s] <= i, for off[0] <= i < off[nseg]; never an empty segment.
__device__ __forceinline__ int find_segment(const int32_t *__restrict__ off, int nseg, int64_t i)
{
  int lo = 0, hi = nseg;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(off + mid) <= i) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  return lo;
}

__device__ __forceinline__ int grid_threads() { return gridDim.x * blockDim.x; }
__device__ __forceinline__ int64_t global_thread() { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }

// ------------------------------------------------------------------------------------------
// status

__global__ void k_status_init(DevStatus *s)
{
  s->flags = 0;
  s->invalid_index = INT_MAX;
  s->invalid_event = INT_MAX;
  for (int k = 0; k < 4; ++k) {
    s->total[k] = 0;
  }
}

// ------------------------------------------------------------------------------------------
// exclusive scan of int32 counts (three kernels: tile sums, scan of tile sums, tile scans)

__device__ __forceinline__ int64_t scan_length(const int64_t *n_dev, int64_t n_host) { return n_dev ? *n_dev : n_host; }

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *warp_totals, T &block_total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const T t = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) {
      inc += t;
    }
  }
  if (lane == 31) {
    warp_totals[warp] = inc;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    T w = lane < nw ? warp_totals[lane] : T(0);
    T winc = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const T t = __shfl_up_sync(0xffffffffu, winc, d);
      if (lane >= d) {
        winc += t;
      }
    }
    if (lane < nw) {
      warp_totals[lane] = winc - w;
    }
    if (lane == nw - 1) {
      warp_totals[32] = winc;
    }
  }
  __syncthreads();
  const T res = warp_totals[warp] + inc - v;
  block_total = warp_totals[32];
  __syncthreads();
  return res;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int32_t *__restrict__ in, const int64_t *n_dev,
                                                             int64_t n_host, int64_t *partials, const DevStatus *status)
{
  __shared__ int64_t warp_totals[33];
  if (capacity_failed(status)) {
    return;
  }
  const int64_t n = scan_length(n_dev, n_host);
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int64_t base = t * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (base + k < n) {
        sum += in[base + k];
      }
    }
    int64_t total;
    block_exclusive_scan<int64_t>(sum, warp_totals, total);
    if (threadIdx.x == 0) {
      partials[t] = total;
    }
  }
}

__global__ void __launch_bounds__(1024) k_scan_partials(int64_t *partials, const int64_t *n_dev, int64_t n_host,
                                                        int32_t *out, int64_t *total_out, DevStatus *status)
{
  __shared__ int64_t warp_totals[33];
  if (capacity_failed(status)) {
    return;
  }
  const int64_t n = scan_length(n_dev, n_host);
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  int64_t carry = 0;
  for (int64_t t0 = 0; t0 < tiles; t0 += blockDim.x) {
    const int64_t t = t0 + threadIdx.x;
    const int64_t v = t < tiles ? partials[t] : 0;
    int64_t total;
    const int64_t ex = block_exclusive_scan<int64_t>(v, warp_totals, total);
    if (t < tiles) {
      partials[t] = carry + ex;
    }
    carry += total;
  }
  if (threadIdx.x == 0) {
    *total_out = carry;
    out[n] = (int32_t)carry;
    if (carry > INT_MAX) {
      atomicOr(&status->flags, kFlagCountOverflow);
    }
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int32_t *__restrict__ in, int32_t *__restrict__ out,
                                                            const int64_t *n_dev, int64_t n_host,
                                                            const int64_t *__restrict__ partials, const DevStatus *status)
{
  __shared__ int64_t warp_totals[33];
  if (capacity_failed(status)) {
    return;
  }
  const int64_t n = scan_length(n_dev, n_host);
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int64_t base = t * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    if (base + kScanItems <= n) {
      const int4 a = *reinterpret_cast<const int4 *>(in + base);
      const int4 b = *reinterpret_cast<const int4 *>(in + base + 4);
      v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
    } else {
#pragma unroll
      for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
      }
    }
    int64_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      sum += v[k];
    }
    int64_t total;
    int64_t run = partials[t] + block_exclusive_scan<int64_t>(sum, warp_totals, total);
    int32_t o[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      o[k] = (int32_t)run;
      run += v[k];
    }
    if (base + kScanItems <= n) {
      *reinterpret_cast<int4 *>(out + base) = make_int4(o[0], o[1], o[2], o[3]);
      *reinterpret_cast<int4 *>(out + base + 4) = make_int4(o[4], o[5], o[6], o[7]);
    } else {
#pragma unroll
      for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) {
          out[base + k] = o[k];
        }
      }
    }
  }
}

int scan_grid(const Launch &l) { return l.num_sms * 4; }

// The four scans of a run: tracklets per cluster, cells per tracklet, neighbours per cell, roads
// per cell. Each is three kernels (tile sums, scan of tile sums, tile scans).
struct ScanArgs {
  const int32_t *in;
  int32_t *out;
  const int64_t *n_dev;
  int64_t n_host;
  int64_t *total;
};

template <int kWhich>
ScanArgs scan_args(const Arena &a)
{
  switch (kWhich) {
  case 0: return ScanArgs{a.trk_count, a.trk_off, nullptr, a.n_clusters, &a.status->total[kTracklets]};
  case 1: return ScanArgs{a.cell_count, a.cell_off, &a.status->total[kTracklets], 0, &a.status->total[kCells]};
  case 2: return ScanArgs{a.nb_count, a.nb_off, &a.status->total[kCells], 0, &a.status->total[kNeighbours]};
  default: return ScanArgs{a.road_count, a.road_off, &a.status->total[kCells], 0, &a.status->total[kRoads]};
  }
}

template <int kWhich>
void step_scan_reduce(const Arena &a, const Launch &l)
{
  const ScanArgs s = scan_args<kWhich>(a);
  k_scan_reduce<<<scan_grid(l), kScanThreads, 0, l.stream>>>(s.in, s.n_dev, s.n_host, a.scan_partials, a.status);
}

template <int kWhich>
void step_scan_partials(const Arena &a, const Launch &l)
{
  const ScanArgs s = scan_args<kWhich>(a);
  k_scan_partials<<<1, 1024, 0, l.stream>>>(a.scan_partials, s.n_dev, s.n_host, s.out, s.total, a.status);
}

template <int kWhich>
void step_scan_apply(const Arena &a, const Launch &l)
{
  const ScanArgs s = scan_args<kWhich>(a);
  k_scan_apply<<<scan_grid(l), kScanThreads, 0, l.stream>>>(s.in, s.out, s.n_dev, s.n_host, a.scan_partials, a.status);
}

// ------------------------------------------------------------------------------------------
// (a) clustering: PrimaryVertexContext::initialize (PrimaryVertexContext.cxx:31-142)

__device__ __forceinline__ int bucket_of(int bin) { return bin < 0 ? 0 : bin + 1; }

__device__ __forceinline__ void store_sorted(const Arena &a, int64_t at, const itsu_cluster &c)
{
  a.sorted[at] = c;
  a.xyzr[at] = make_float4(c.x, c.y, c.z, c.r);
  a.phi[at] = c.phi;
}

__global__ void __launch_bounds__(kSortThreads) k_cluster_sort(Arena a)
{
  __shared__ int hist[kSortWarps][kBuckets];
  __shared__ int bucket_total[kBuckets];
  __shared__ int bucket_base[kBuckets];

  const int seg = blockIdx.x;
  const int e = seg / ITSU_LAYERS, layer = seg % ITSU_LAYERS;
  const int64_t begin = a.layer_off[seg];
  const int n = (int)(a.layer_off[seg + 1] - begin);
  const float vx = a.vtx[3 * e], vy = a.vtx[3 * e + 1], vz = a.vtx[3 * e + 2];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0 && layer == 0) {
    const bool ok = isfinite(vx) && isfinite(vy) && isfinite(vz) && fabsf(vx) <= kMaxAbsCoordinate &&
                    fabsf(vy) <= kMaxAbsCoordinate && fabsf(vz) <= kMaxAbsCoordinate;
    if (!ok) {
      atomicOr(&a.status->flags, kFlagInvalid);
      atomicMin(&a.status->invalid_event, e);
    }
  }
  for (int k = tid; k < kSortWarps * kBuckets; k += kSortThreads) {
    (&hist[0][0])[k] = 0;
  }
  __syncthreads();

  // Pass 1: transform every cluster (input order), per-warp bucket histograms.
  const int chunk = (n + kSortWarps - 1) / kSortWarps;
  const int wb = min(n, warp * chunk), we = min(n, wb + chunk);
  for (int i = wb + lane; i < we; i += 32) {
    itsu_cluster c = a.raw[begin + i];
    const Transformed t = transform_cluster(layer, c.x, c.y, c.z, vx, vy);
    c.phi = t.phi;
    c.r = t.r;
    c.bin = t.bin;
    const bool ok = isfinite(c.x) && isfinite(c.y) && isfinite(c.z) && fabsf(c.x) <= kMaxAbsCoordinate &&
                    fabsf(c.y) <= kMaxAbsCoordinate && fabsf(c.z) <= kMaxAbsCoordinate && !(t.r == 0.0f && c.z == vz);
    if (!ok) {
      atomicOr(&a.status->flags, kFlagInvalid);
      atomicMin(&a.status->invalid_index, (int)(begin + i));
    }
    a.tmp[begin + i] = c;
    atomicAdd(&hist[warp][bucket_of(t.bin)], 1);
  }
  __syncthreads();

  // Pass 2: per-bucket prefix over warps, exclusive scan over buckets, index table.
  for (int b = tid; b < kBuckets; b += kSortThreads) {
    int s = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      const int v = hist[w][b];
      hist[w][b] = s;
      s += v;
    }
    bucket_total[b] = s;
  }
  __syncthreads();
  if (warp == 0) {
    constexpr int per = (kBuckets + 31) / 32;
    const int b0 = lane * per, b1 = min(kBuckets, b0 + per);
    int local = 0;
    for (int b = b0; b < b1; ++b) {
      local += bucket_total[b];
    }
    int inc = local;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) {
        inc += t;
      }
    }
    int run = inc - local;
    for (int b = b0; b < b1; ++b) {
      bucket_base[b] = run;
      run += bucket_total[b];
    }
  }
  __syncthreads();
  for (int b = tid; b < kBuckets; b += kSortThreads) {
    const int base = bucket_base[b];
    for (int w = 0; w < kSortWarps; ++w) {
      hist[w][b] += base;
    }
  }
  if (layer > 0) {
    // table[b] = first sorted index with bin >= b = #clusters with bin < b for b >= 1; table[0] = 0
    // (PrimaryVertexContext.cxx:90-119: negative bins never move the fill cursor off bin 0).
    int32_t *table = a.index_tables + ((int64_t)e * ITSU_TRACKLET_LAYERS + layer - 1) * kTableSize;
    for (int b = tid; b < kTableSize; b += kSortThreads) {
      table[b] = b == 0 ? 0 : bucket_base[b + 1];
    }
  }
  __syncthreads();

  // Pass 3: stable scatter. Warps own consecutive input ranges whose bucket offsets were
  // prefixed in warp order; inside a warp, lanes of equal bucket rank by lane order.
  for (int i0 = wb; i0 < we; i0 += 32) {
    const int i = i0 + lane;
    const bool valid = i < we;
    itsu_cluster c;
    int bucket = -1 - lane;
    if (valid) {
      c = a.tmp[begin + i];
      bucket = bucket_of(c.bin);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, bucket);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    int pos = 0;
    if (valid) {
      pos = hist[warp][bucket] + rank;
    }
    __syncwarp();
    if (valid && lane == 31 - __clz(peers)) {
      hist[warp][bucket] += __popc(peers);
    }
    __syncwarp();
    if (valid) {
      store_sorted(a, begin + pos, c);
    }
  }

  // Pass 4: negative bins share bucket 0 in input order; order them by bin, stably.
  const int m = bucket_total[0];
  if (m > 1) {
    __syncthreads();
    for (int i = tid; i < m; i += kSortThreads) {
      const itsu_cluster c = a.sorted[begin + i];
      int rank = 0;
      for (int j = 0; j < m; ++j) {
        const int kj = a.sorted[begin + j].bin;
        rank += (kj < c.bin) || (kj == c.bin && j < i);
      }
      a.tmp[begin + rank] = c;
    }
    __syncthreads();
    for (int i = tid; i < m; i += kSortThreads) {
      store_sorted(a, begin + i, a.tmp[begin + i]);
    }
  }
}

// ------------------------------------------------------------------------------------------
// (b) tracklets: TrackerTraits<false>::computeLayerTracklets (Tracker.cxx:45-117)

// Tracklet layer L of event e runs only if every layer pair up to L has clusters (:49-52).
__device__ __forceinline__ bool tracklets_active(const int32_t *lo, int layer)
{
  for (int l = 0; l <= layer; ++l) {
    if (lo[l + 1] - lo[l] <= 0 || lo[l + 2] - lo[l + 1] <= 0) {
      return false;
    }
  }
  return true;
}

// Tracklet.cxx:32-40 for a queued pair (out slot, inner flat index, outer flat index, cluster
// segment of the inner cluster).
__device__ __forceinline__ void write_tracklet(const Arena &a, int4 q)
{
  const int seg = q.w;
  const int e = seg / ITSU_LAYERS, layer = seg % ITSU_LAYERS;
  const float4 c = a.xyzr[q.y];
  const float4 d = a.xyzr[q.z];
  itsu_tracklet t;
  t.first_cluster = q.y - a.layer_off[seg];
  t.second_cluster = q.z - a.layer_off[seg + 1];
  t.tan_lambda = (c.z - d.z) / (c.w - d.w);
  t.phi = itsu_atan2f(c.y - d.y, c.x - d.x);
  a.tracklets[q.x] = t;
  a.trk_seg_id[q.x] = e * ITSU_TRACKLET_LAYERS + layer;
}

// Walks the reference's candidate sequence of one inner cluster (Tracker.cxx:73-89): the phi
// rows of its bin window in wrap-around order, and in each row the sorted clusters from the
// row's first bin to the first cluster at or after the window's end (inclusive, P1/P5 bounds).
struct CandidateWalk {
  const int32_t *table;
  int n_next;
  int z_min, z_span;  // first z bin, number of z bins + 1
  int phi_bin, rows_left;
  int j, last;

  __device__ __forceinline__ bool next()
  {
    ++j;
    while (j > last) {
      if (rows_left == 0) {
        return false;
      }
      const int first_bin = bin_index(z_min, phi_bin);
      const int max_bin = min(first_bin + z_span, kTableBins);
      j = table[first_bin];
      last = min(table[max_bin], n_next - 1);
      phi_bin = (phi_bin + 1 == kPhiBins) ? 0 : phi_bin + 1;
      --rows_left;
    }
    return true;
  }
};

constexpr int kQueue = 64;  // per-warp queue of accepted pairs, drained 32 at a time

// One thread per inner cluster; the warp advances its 32 candidate walks in lock step so that
// accepted pairs can be compacted (ballot) into a per-warp queue. The write pass drains the queue
// with all 32 lanes converged, so the double-precision azimuth of each new tracklet runs without
// divergence. Output slots come from the scan of the count pass: emission order is the
// reference's (inner cluster, phi row, candidate).
template <bool kWrite>
__global__ void __launch_bounds__(kThreads) k_tracklets(Arena a)
{
  __shared__ int4 queue[kWrite ? kThreads / 32 : 1][kQueue];
  if (kWrite && capacity_failed(a.status)) {
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i = global_thread();
  const bool in_range = i < a.n_clusters;
  int seg = 0, e = 0, layer = ITSU_LAYERS - 1;
  const int32_t *lo = a.layer_off;
  if (in_range) {
    seg = find_segment(a.layer_off, a.n_events * ITSU_LAYERS, i);
    e = seg / ITSU_LAYERS;
    layer = seg % ITSU_LAYERS;
    lo = a.layer_off + e * ITSU_LAYERS;
  }
  float4 c = make_float4(0, 0, 0, 0);
  float phi1 = 0, tan_lambda = 0;
  int64_t next_begin = 0;
  CandidateWalk walk{nullptr, 0, 0, 0, 0, 0, 0, -1};
  bool has = false;
  if (in_range && layer < ITSU_LAYERS - 1 && tracklets_active(lo, layer)) {
    c = a.xyzr[i];
    phi1 = a.phi[i];
    const float vz = a.vtx[3 * e + 2];
    tan_lambda = (c.z - vz) / c.w;
    const float dir_z = tan_lambda * (kC.r[layer + 1] - c.w) + c.z;
    const int4 rect = bins_rect(phi1, layer, dir_z);
    if (!(rect.x == 0 && rect.y == 0 && rect.z == 0 && rect.w == 0)) {
      int phi_bins = rect.w - rect.y + 1;
      if (phi_bins < 0) {
        phi_bins += kPhiBins;
      }
      walk.table = a.index_tables + ((int64_t)e * ITSU_TRACKLET_LAYERS + layer) * kTableSize;
      walk.n_next = lo[layer + 2] - lo[layer + 1];
      walk.z_min = rect.x;
      walk.z_span = rect.z - rect.x + 1;
      walk.phi_bin = rect.y;
      walk.rows_left = phi_bins;
      next_begin = lo[layer + 1];
      has = walk.next();
    }
  }
  int count = 0;
  int out = 0;
  int queued = 0;
  if (kWrite && in_range) {
    out = a.trk_off[i];
  }
  const float max_dz = kC.trk_max_dz[layer < ITSU_TRACKLET_LAYERS ? layer : 0];
  while (__any_sync(0xffffffffu, has)) {
    bool pass = false;
    if (has) {
      const int64_t jf = next_begin + walk.j;
      const float4 d = a.xyzr[jf];
      const float phi2 = a.phi[jf];
      const float delta_z = fabsf(tan_lambda * (d.w - c.w) + c.z - d.z);
      const float delta_phi = fabsf(phi1 - phi2);
      pass = delta_z < max_dz && (delta_phi < kPhiCoordinateCut || fabsf(delta_phi - kTwoPi) < kPhiCoordinateCut);
    }
    if (kWrite) {
      const unsigned m = __ballot_sync(0xffffffffu, pass);
      if (pass) {
        queue[warp][queued + __popc(m & ((1u << lane) - 1u))] = make_int4(out, (int)i, (int)(next_begin + walk.j), seg);
        ++out;
      }
      queued += __popc(m);
      if (queued >= 32) {
        __syncwarp();
        write_tracklet(a, queue[warp][lane]);
        __syncwarp();
        if (lane < queued - 32) {
          queue[warp][lane] = queue[warp][lane + 32];
        }
        __syncwarp();
        queued -= 32;
      }
    } else {
      count += pass;
    }
    if (has) {
      has = walk.next();
    }
  }
  if (kWrite) {
    __syncwarp();
    if (lane < queued) {
      write_tracklet(a, queue[warp][lane]);
    }
    if (in_range) {
      const int32_t first = a.trk_off[i];
      a.trk_lookup[i] = (layer >= 1 && layer <= ITSU_CELL_LAYERS && a.trk_off[i + 1] > first)
                            ? first - a.trk_seg[e * ITSU_TRACKLET_LAYERS + layer]
                            : ITSU_UNUSED_INDEX;
    }
  } else if (in_range) {
    a.trk_count[i] = count;
  }
}

// trk_seg[6e+L] = first tracklet of (e, L); capacity check of the tracklet total.
__global__ void k_tracklet_segments(Arena a)
{
  const int nseg = a.n_events * ITSU_TRACKLET_LAYERS;
  for (int s = (int)global_thread(); s <= nseg; s += grid_threads()) {
    if (s == nseg) {
      const int64_t total = a.status->total[kTracklets];
      a.trk_seg[s] = (int32_t)total;
      if (total > a.cap_tracklets) {
        atomicOr(&a.status->flags, kFlagCapTracklets);
      }
    } else {
      const int e = s / ITSU_TRACKLET_LAYERS, layer = s % ITSU_TRACKLET_LAYERS;
      a.trk_seg[s] = a.trk_off[a.layer_off[e * ITSU_LAYERS + layer]];
    }
  }
}

// ------------------------------------------------------------------------------------------
// (c) cells: TrackerTraits<false>::computeLayerCells (Tracker.cxx:120-235)

// Cell layer L of event e runs only if tracklet layers 0..L+1 are all non-empty (:124-128).
__device__ __forceinline__ bool cells_active(const int32_t *ts, int layer)
{
  for (int l = 0; l <= layer; ++l) {
    if (ts[l + 1] - ts[l] <= 0 || ts[l + 2] - ts[l + 1] <= 0) {
      return false;
    }
  }
  return true;
}

template <bool kWrite>
__global__ void __launch_bounds__(kThreads) k_cells(Arena a)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int64_t n = a.status->total[kTracklets];
  for (int64_t k = global_thread(); k < n; k += grid_threads()) {
    const int sid = a.trk_seg_id[k];
    const int e = sid / ITSU_TRACKLET_LAYERS, layer = sid % ITSU_TRACKLET_LAYERS;
    const int32_t *ts = a.trk_seg + e * ITSU_TRACKLET_LAYERS;
    int count = 0;
    int64_t out = kWrite ? a.cell_off[k] : 0;
    if (layer < ITSU_CELL_LAYERS && cells_active(ts, layer)) {
      const int32_t *lo = a.layer_off + e * ITSU_LAYERS;
      const itsu_tracklet t1 = a.tracklets[k];
      const float4 c1 = a.xyzr[lo[layer] + t1.first_cluster];
      const int64_t c2i = lo[layer + 1] + t1.second_cluster;
      const float4 c2 = a.xyzr[c2i];
      const int32_t j0 = a.trk_off[c2i], j1 = a.trk_off[c2i + 1];
      const float vx = a.vtx[3 * e], vy = a.vtx[3 * e + 1], vz = a.vtx[3 * e + 2];
      for (int32_t j = j0; j < j1; ++j) {
        const itsu_tracklet t2 = a.tracklets[j];
        if (!cell_precut(layer, t1.tan_lambda, t1.phi, t2.tan_lambda, t2.phi, c1, vz)) {
          continue;
        }
        const float4 c3 = a.xyzr[lo[layer + 2] + t2.second_cluster];
        float3 normal;
        float curvature;
        if (cell_geometry(layer, c1, c2, c3, vx, vy, normal, curvature)) {
          if (kWrite) {
            itsu_cell cell;
            cell.first_cluster = t1.first_cluster;
            cell.second_cluster = t2.first_cluster;
            cell.third_cluster = t2.second_cluster;
            cell.first_tracklet = (int32_t)(k - ts[layer]);
            cell.second_tracklet = j - ts[layer + 1];
            cell.nx = normal.x;
            cell.ny = normal.y;
            cell.nz = normal.z;
            cell.curvature = curvature;
            cell.level = 1;
            a.cells[out] = cell;
            a.cell_seg_id[out] = e * ITSU_CELL_LAYERS + layer;
            ++out;
          } else {
            ++count;
          }
        }
      }
    }
    if (!kWrite) {
      a.cell_count[k] = count;
    } else {
      const int32_t first = a.cell_off[k];
      a.cell_lookup[k] = (layer >= 1 && layer < ITSU_CELL_LAYERS && a.cell_off[k + 1] > first)
                             ? first - a.cell_seg[e * ITSU_CELL_LAYERS + layer]
                             : ITSU_UNUSED_INDEX;
    }
  }
}

__global__ void k_cell_segments(Arena a)
{
  if (capacity_failed(a.status)) {
    return;  // tracklet offsets beyond the arena: nothing downstream runs
  }
  const int nseg = a.n_events * ITSU_CELL_LAYERS;
  for (int s = (int)global_thread(); s <= nseg; s += grid_threads()) {
    if (s == nseg) {
      const int64_t total = a.status->total[kCells];
      a.cell_seg[s] = (int32_t)total;
      if (total > a.cap_cells) {
        atomicOr(&a.status->flags, kFlagCapCells);
      }
    } else {
      const int e = s / ITSU_CELL_LAYERS, layer = s % ITSU_CELL_LAYERS;
      a.cell_seg[s] = a.cell_off[a.trk_seg[e * ITSU_TRACKLET_LAYERS + layer]];
    }
  }
}

// ------------------------------------------------------------------------------------------
// (d) neighbours and CA levels: Tracker<IsGPU>::findCellsNeighbours (Tracker.cxx:417-474)

// Per-cell state of the neighbour and road stages, reset so that the stage can be re-run.
__global__ void __launch_bounds__(kThreads) k_neighbour_reset(Arena a)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int64_t n = a.status->total[kCells];
  for (int64_t c = global_thread(); c < n; c += grid_threads()) {
    a.nb_count[c] = 0;
    a.nb_fill[c] = 0;
    a.road_count[c] = 0;
    a.paths[c] = a.cell_seg_id[c] % ITSU_CELL_LAYERS == 0 ? 1 : 0;
  }
}

template <bool kWrite>
__global__ void __launch_bounds__(kThreads) k_neighbours(Arena a)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int64_t n = a.status->total[kCells];
  for (int64_t c = global_thread(); c < n; c += grid_threads()) {
    const int sid = a.cell_seg_id[c];
    const int e = sid / ITSU_CELL_LAYERS, layer = sid % ITSU_CELL_LAYERS;
    if (layer >= ITSU_NEIGHBOUR_LAYERS) {
      continue;
    }
    const itsu_cell cell = a.cells[c];
    const int64_t ft = a.trk_seg[e * ITSU_TRACKLET_LAYERS + layer + 1] + cell.second_tracklet;
    const int32_t j0 = a.cell_off[ft], j1 = a.cell_off[ft + 1];
    const float3 n1 = make_float3(cell.nx, cell.ny, cell.nz);
    const int32_t c_local = (int32_t)(c - a.cell_seg[e * ITSU_CELL_LAYERS + layer]);
    for (int32_t j = j0; j < j1; ++j) {
      const itsu_cell next = a.cells[j];
      if (neighbour_cut(layer, n1, cell.curvature, make_float3(next.nx, next.ny, next.nz), next.curvature)) {
        if (kWrite) {
          const int slot = atomicAdd(&a.nb_fill[j], 1);
          a.nb[a.nb_off[j] + slot] = c_local;
        } else {
          atomicAdd(&a.nb_count[j], 1);
        }
      }
    }
  }
}

__global__ void k_neighbour_check(Arena a)
{
  if (global_thread() == 0 && !capacity_failed(a.status) && a.status->total[kNeighbours] > a.cap_neighbours) {
    atomicOr(&a.status->flags, kFlagCapNeighbours);
  }
}

// Rows of layer `layer` cells: sort ascending (the reference pushes in cell order), then the
// level (Tracker.cxx:463-468: 1 + the highest neighbour level) and the number of
// level-decreasing chains down to layer 0 (the roads a level-5 cell starts, Tracker.cxx:477-571).
__global__ void __launch_bounds__(kThreads) k_levels(Arena a, int layer)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int64_t n = a.status->total[kCells];
  for (int64_t c = global_thread(); c < n; c += grid_threads()) {
    const int sid = a.cell_seg_id[c];
    if (sid % ITSU_CELL_LAYERS != layer) {
      continue;
    }
    const int e = sid / ITSU_CELL_LAYERS;
    const int32_t b = a.nb_off[c], en = a.nb_off[c + 1];
    int32_t *row = a.nb + b;
    const int len = en - b;
    for (int p = 1; p < len; ++p) {
      const int32_t v = row[p];
      int q = p - 1;
      while (q >= 0 && row[q] > v) {
        row[q + 1] = row[q];
        --q;
      }
      row[q + 1] = v;
    }
    const int64_t prev_base = a.cell_seg[e * ITSU_CELL_LAYERS + layer - 1];
    int level = 1;
    for (int p = 0; p < len; ++p) {
      level = max(level, a.cells[prev_base + row[p]].level + 1);
    }
    int64_t paths = 0;
    bool overflow = false;
    for (int p = 0; p < len; ++p) {
      const int64_t nbi = prev_base + row[p];
      if (a.cells[nbi].level == level - 1) {
        paths += a.paths[nbi];
        if (paths > INT_MAX) {
          paths = INT_MAX;
          overflow = true;
        }
      }
    }
    a.cells[c].level = level;
    a.paths[c] = paths;
    if (layer == ITSU_CELL_LAYERS - 1 && level == kCellsMinLevel) {
      a.road_count[c] = (int32_t)paths;
      if (overflow) {
        atomicOr(&a.status->flags, kFlagCountOverflow);
      }
    }
  }
}

// ------------------------------------------------------------------------------------------
// (e) roads: Tracker<IsGPU>::findTracks / traverseCellsTree / computeMontecarloLabels

__global__ void k_road_segments(Arena a)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int nseg = a.n_events;
  for (int s = (int)global_thread(); s <= nseg; s += grid_threads()) {
    if (s == nseg) {
      const int64_t total = a.status->total[kRoads];
      a.road_seg[s] = (int32_t)total;
      if (total > a.cap_roads) {
        atomicOr(&a.status->flags, kFlagCapRoads);
      }
    } else {
      a.road_seg[s] = a.road_off[a.cell_seg[s * ITSU_CELL_LAYERS + ITSU_CELL_LAYERS - 1]];
    }
  }
}

__device__ __forceinline__ int32_t cluster_mc(const Arena &a, const int32_t *lo, int layer, int32_t idx)
{
  return a.sorted[lo[layer] + idx].mc_id;
}

__global__ void __launch_bounds__(kThreads) k_roads(Arena a)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int64_t n = a.status->total[kCells];
  for (int64_t c = global_thread(); c < n; c += grid_threads()) {
    int64_t out = a.road_off[c];
    if (a.road_off[c + 1] == out) {
      continue;
    }
    const int sid = a.cell_seg_id[c];
    const int e = sid / ITSU_CELL_LAYERS;
    const int32_t *cs = a.cell_seg + e * ITSU_CELL_LAYERS;
    const int32_t *lo = a.layer_off + e * ITSU_LAYERS;
    int32_t cur[ITSU_CELL_LAYERS];  // local cell index per layer along the current chain
    int32_t it[ITSU_CELL_LAYERS];   // next neighbour slot per layer
    int level[ITSU_CELL_LAYERS];
    int l = ITSU_CELL_LAYERS - 1;
    cur[l] = (int32_t)(c - cs[l]);
    it[l] = a.nb_off[c];
    level[l] = a.cells[c].level;
    while (true) {
      if (l == 0) {
        // a complete chain: one road, labelled by Moore's vote over its 7 clusters (:574-652)
        itsu_road road;
        int max_value = ITSU_UNUSED_INDEX, count = 0;
        bool fake = false;
        for (int k = 0; k < ITSU_CELL_LAYERS; ++k) {
          road.cell_ids[k] = cur[k];
          const itsu_cell &cell = a.cells[cs[k] + cur[k]];
          if (k == 0) {
            max_value = cluster_mc(a, lo, 0, cell.first_cluster);
            count = 1;
            const int second = cluster_mc(a, lo, 1, cell.second_cluster);
            if (second == max_value) {
              ++count;
            } else {
              max_value = second;
              count = 1;
              fake = true;
            }
          }
          const int current = cluster_mc(a, lo, k + 2, cell.third_cluster);
          if (current == max_value) {
            ++count;
          } else {
            --count;
            fake = true;
          }
          if (count == 0) {
            max_value = current;
            count = 1;
          }
        }
        road.size = ITSU_CELL_LAYERS;
        road.label = max_value;
        road.is_fake = fake ? 1 : 0;
        road.pad_[0] = road.pad_[1] = road.pad_[2] = 0;
        a.roads[out++] = road;
        ++l;
        continue;
      }
      const int64_t flat = cs[l] + cur[l];
      const int32_t end = a.nb_off[flat + 1];
      bool descended = false;
      while (it[l] < end) {
        const int32_t nb = a.nb[it[l]++];
        const int64_t nflat = cs[l - 1] + nb;
        const int nlevel = a.cells[nflat].level;
        if (nlevel == level[l] - 1) {
          cur[l - 1] = nb;
          it[l - 1] = a.nb_off[nflat];
          level[l - 1] = nlevel;
          --l;
          descended = true;
          break;
        }
      }
      if (!descended) {
        if (l == ITSU_CELL_LAYERS - 1) {
          break;
        }
        ++l;
      }
    }
  }
}

int fixed_grid(const Launch &l) { return l.num_sms * 8; }

void step_status_init(const Arena &a, const Launch &l) { k_status_init<<<1, 1, 0, l.stream>>>(a.status); }

void step_cluster_sort(const Arena &a, const Launch &l)
{
  if (a.n_events > 0) {
    k_cluster_sort<<<a.n_events * ITSU_LAYERS, kSortThreads, 0, l.stream>>>(a);
  }
}

template <bool kWrite>
void step_tracklets(const Arena &a, const Launch &l)
{
  const int64_t blocks = (a.n_clusters + kThreads - 1) / kThreads;
  if (blocks > 0) {
    k_tracklets<kWrite><<<(unsigned)blocks, kThreads, 0, l.stream>>>(a);
  }
}

void step_tracklet_segments(const Arena &a, const Launch &l)
{
  k_tracklet_segments<<<(a.n_events * ITSU_TRACKLET_LAYERS + kThreads) / kThreads, kThreads, 0, l.stream>>>(a);
}

template <bool kWrite>
void step_cells(const Arena &a, const Launch &l) { k_cells<kWrite><<<fixed_grid(l), kThreads, 0, l.stream>>>(a); }

void step_cell_segments(const Arena &a, const Launch &l)
{
  k_cell_segments<<<(a.n_events * ITSU_CELL_LAYERS + kThreads) / kThreads, kThreads, 0, l.stream>>>(a);
}

void step_neighbour_reset(const Arena &a, const Launch &l) { k_neighbour_reset<<<fixed_grid(l), kThreads, 0, l.stream>>>(a); }

template <bool kWrite>
void step_neighbours(const Arena &a, const Launch &l) { k_neighbours<kWrite><<<fixed_grid(l), kThreads, 0, l.stream>>>(a); }

void step_neighbour_check(const Arena &a, const Launch &l) { k_neighbour_check<<<1, 32, 0, l.stream>>>(a); }

template <int kLayer>
void step_levels(const Arena &a, const Launch &l) { k_levels<<<fixed_grid(l), kThreads, 0, l.stream>>>(a, kLayer); }

void step_road_segments(const Arena &a, const Launch &l)
{
  k_road_segments<<<(a.n_events + kThreads) / kThreads, kThreads, 0, l.stream>>>(a);
}

void step_roads(const Arena &a, const Launch &l) { k_roads<<<fixed_grid(l), kThreads, 0, l.stream>>>(a); }

// The whole run, kernel by kernel, in launch order.
const KernelStep kSteps[] = {
    {"status_init", step_status_init},                   // 0
    {"cluster_sort", step_cluster_sort},                 // 1  (a)
    {"tracklets_count", step_tracklets<false>},          // 2  (b)
    {"scan_reduce_tracklets", step_scan_reduce<0>},      // 3
    {"scan_partials_tracklets", step_scan_partials<0>},  // 4
    {"scan_apply_tracklets", step_scan_apply<0>},        // 5
    {"tracklet_segments", step_tracklet_segments},       // 6
    {"tracklets_write", step_tracklets<true>},           // 7
    {"cells_count", step_cells<false>},                  // 8  (c)
    {"scan_reduce_cells", step_scan_reduce<1>},          // 9
    {"scan_partials_cells", step_scan_partials<1>},      // 10
    {"scan_apply_cells", step_scan_apply<1>},            // 11
    {"cell_segments", step_cell_segments},               // 12
    {"cells_write", step_cells<true>},                   // 13
    {"neighbour_reset", step_neighbour_reset},           // 14 (d)
    {"neighbours_count", step_neighbours<false>},        // 15
    {"scan_reduce_neighbours", step_scan_reduce<2>},     // 16
    {"scan_partials_neighbours", step_scan_partials<2>}, // 17
    {"scan_apply_neighbours", step_scan_apply<2>},       // 18
    {"neighbour_check", step_neighbour_check},           // 19
    {"neighbours_write", step_neighbours<true>},         // 20
    {"levels_1", step_levels<1>},                        // 21
    {"levels_2", step_levels<2>},                        // 22
    {"levels_3", step_levels<3>},                        // 23
    {"levels_4", step_levels<4>},                        // 24
    {"scan_reduce_roads", step_scan_reduce<3>},          // 25 (e)
    {"scan_partials_roads", step_scan_partials<3>},      // 26
    {"scan_apply_roads", step_scan_apply<3>},            // 27
    {"road_segments", step_road_segments},               // 28
    {"roads_write", step_roads},                         // 29
};
constexpr int kNumSteps = sizeof(kSteps) / sizeof(kSteps[0]);

void run_steps(int first, int last, const Arena &a, const Launch &l)
{
  for (int k = first; k <= last; ++k) {
    kSteps[k].launch(a, l);
  }
}

}  // namespace

const KernelStep *pipeline_steps(int *count)
{
  *count = kNumSteps;
  return kSteps;
}

void launch_status_init(const Arena &a, const Launch &l) { run_steps(0, 0, a, l); }
void launch_cluster_sort(const Arena &a, const Launch &l) { run_steps(1, 1, a, l); }
void launch_tracklets_count(const Arena &a, const Launch &l) { run_steps(2, 6, a, l); }
void launch_tracklets_write(const Arena &a, const Launch &l) { run_steps(7, 7, a, l); }
void launch_cells_count(const Arena &a, const Launch &l) { run_steps(8, 12, a, l); }
void launch_cells_write(const Arena &a, const Launch &l) { run_steps(13, 13, a, l); }
void launch_neighbours_count(const Arena &a, const Launch &l) { run_steps(14, 19, a, l); }
void launch_neighbours_write(const Arena &a, const Launch &l) { run_steps(20, 24, a, l); }
void launch_roads_count(const Arena &a, const Launch &l) { run_steps(25, 28, a, l); }
void launch_roads_write(const Arena &a, const Launch &l) { run_steps(29, 29, a, l); }

int kernels_per_run() { return kNumSteps; }

}  // namespace itsu
