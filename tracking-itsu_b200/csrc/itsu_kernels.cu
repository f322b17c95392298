// itsu_kernels.cu - sm_100a kernels of the ITS CA track finder.
//
// Every stage is a deterministic count -> exclusive scan -> write sequence over flat,
// event-major arrays, so the output order is the reference's emission order (where a count pass
// uses atomics, to reserve scratch or fill neighbour rows, the write pass restores the order):
//   clustering   one CTA per (event, layer): vertex-relative transform, stable counting sort by
//                bin (per-warp histograms, warp-match ranks), index table, z-sorted bin lists
//                for the tracklet pruning (PVC.cxx:31-142)
//   tracklets    count: one thread per inner cluster walking the reference's bin window,
//                z-pruned (Tracker.cxx:45-117); tail: lookup, owners, crowded clusters; write:
//                a map over tracklets (slope and correctly rounded azimuth)
//   cells        count: a warp per 32 first tracklets, their outgoing-tracklet pairs flattened
//                over the lanes, exact cuts, one 32-byte entry per found cell (Tracker.cxx:
//                120-235); learned form: the prefilter scores the entries; write: the entries
//                scattered to their scanned slots, then the lookup table
//   neighbours   one thread per cell walking the next-layer cells of its outer tracklet; rows
//                keyed by the next-layer cell, sorted ascending (Tracker.cxx:417-474)
//   levels       layer-ordered longest-chain DP plus the number of level-decreasing chains
//   roads        one thread per level-5 cell: depth-first enumeration in the reference's order,
//                Moore-vote labels (Tracker.cxx:477-652)
// Capacity overflow never writes out of bounds: the passes check the scanned totals and scratch
// reservations against the arena capacities, record the requirement and skip; the host grows
// and re-runs.
#include <climits>

#include "itsu_device.cuh"
#include "itsu_internal.h"
#include "itsu_mlp.cuh"

namespace itsu {
namespace {

constexpr int kThreads = 256;     // threads per block of the fixed-shape helper kernels
constexpr int kMaxThreads = 512;  // upper bound of the tunable per-item kernels' block size
constexpr int kSortThreads = 512;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kBuckets = kTableSize + 1;  // bucket 0: negative bins; bucket b+1: bin b
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
// The tracklet and cell count passes add each warp's total to the tile sum of the warp's first
// item, which is only right if no warp straddles two tiles: whole warps (block sizes are
// multiples of 32, checked at launch) over tiles of a whole number of warps.
static_assert(kScanTile % 32 == 0, "a warp's 32 items lie in one scan tile");
constexpr float kMaxAbsCoordinate = 1.0e6f;
constexpr int kMaxPruneBin = 256;  // larger bins disable pruning for their layer
constexpr int kPruneWords = kMaxPruneBin / 64;  // a pruned column's passes: a mask of this many 64-bit words
static_assert(kMaxPruneBin % 64 == 0, "a pruned column's passes are whole 64-bit words");

__device__ __forceinline__ bool capacity_failed(const DevStatus *s) { return (*(volatile const int32_t *)&s->flags & kCapacityMask) != 0; }

__device__ __forceinline__ int grid_threads() { return gridDim.x * blockDim.x; }
__device__ __forceinline__ int64_t global_thread() { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }

// ------------------------------------------------------------------------------------------
// status

// Status reset of a run; the tracklet scan's tile sums start at zero too (the tracklet count
// pass adds each warp's tracklets to them).
__global__ void k_status_init(Arena a)
{
  if (a.scan_partials) {
    for (int64_t t = global_thread(); t < (a.n_clusters + kScanTile - 1) / kScanTile; t += grid_threads()) {
      a.scan_partials[t] = 0;
    }
  }
  if (global_thread() != 0) {
    return;
  }
  DevStatus *s = a.status;
  s->flags = 0;
  s->invalid_index = INT_MAX;
  s->invalid_event = INT_MAX;
  for (int k = 0; k < 4; ++k) {
    s->total[k] = 0;
  }
  s->cell_entries = 0;
  s->crowded = 0;
  s->trk_crowded = 0;
}

// A launch shape the per-item passes cannot run: the run stops and reports it.
__global__ void k_flag_bad_launch(DevStatus *s) { atomicOr(&s->flags, kFlagLaunchShape); }

// ------------------------------------------------------------------------------------------
// exclusive scan of int32 counts (tile sums, scan of tile sums, tile scans; the tracklet and
// cell count passes fill their scans' tile sums themselves)

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
// per cell. The neighbour and road scans are three kernels (tile sums, scan of tile sums, tile
// scans); the tracklet and cell scans are two, their tile sums added up by the count passes.
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

// A warp's 32 consecutive 36-byte clusters move between global and shared memory as 288 words,
// each load or store instruction covering 128 contiguous bytes; a lane then reads or writes its
// own record in the stage (word stride 9, odd: no bank conflicts).
constexpr int kClusterWords = sizeof(itsu_cluster) / 4;
static_assert(sizeof(itsu_cluster) == 36 && alignof(itsu_cluster) == 4, "cluster layout");

__device__ __forceinline__ void stage_in(int32_t *stage, const itsu_cluster *src, int count)
{
  const int32_t *w = reinterpret_cast<const int32_t *>(src);
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < kClusterWords; ++k) {
    const int at = k * 32 + lane;
    if (at < count * kClusterWords) {
      stage[at] = w[at];
    }
  }
  __syncwarp();
}

__device__ __forceinline__ void stage_out(itsu_cluster *dst, const int32_t *stage, int count)
{
  __syncwarp();
  int32_t *w = reinterpret_cast<int32_t *>(dst);
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < kClusterWords; ++k) {
    const int at = k * 32 + lane;
    if (at < count * kClusterWords) {
      w[at] = stage[at];
    }
  }
}

// The 24-byte input record (itsu_cluster_in) in 4-byte words.
constexpr int kClusterInWords = sizeof(itsu_cluster_in) / 4;
static_assert(sizeof(itsu_cluster_in) == 24 && alignof(itsu_cluster_in) == 4, "input record layout");
static_assert(sizeof(itsu_cluster_track) == 16, "track record layout");

// A warp's 32 consecutive records of kWords words each, moved into its stage with coalesced loads.
template <int kWords, typename Record>
__device__ __forceinline__ void stage_in_words(int32_t *stage, const Record *src, int count)
{
  const int32_t *w = reinterpret_cast<const int32_t *>(src);
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < kWords; ++k) {
    const int at = k * 32 + lane;
    if (at < count * kWords) {
      stage[at] = w[at];
    }
  }
  __syncwarp();
}

// A lane's 24-byte input record from the stage, as a cluster whose phi, r and bin clustering fills.
__device__ __forceinline__ itsu_cluster stage_get_in(const int32_t *stage, int lane)
{
  const int32_t *w = stage + lane * kClusterInWords;  // word stride 6: each access a 2-way bank conflict at most
  itsu_cluster c;
  c.x = __int_as_float(w[0]);
  c.y = __int_as_float(w[1]);
  c.z = __int_as_float(w[2]);
  c.phi = 0.0f;
  c.r = 0.0f;
  c.cluster_id = w[3];
  c.alpha = __int_as_float(w[4]);
  c.mc_id = w[5];
  c.bin = 0;
  return c;
}

__device__ __forceinline__ itsu_cluster stage_get(const int32_t *stage, int lane)
{
  itsu_cluster c;
  int32_t *w = reinterpret_cast<int32_t *>(&c);
#pragma unroll
  for (int k = 0; k < kClusterWords; ++k) {
    w[k] = stage[lane * kClusterWords + k];
  }
  return c;
}

__device__ __forceinline__ void stage_put(int32_t *stage, int lane, const itsu_cluster &c)
{
  const int32_t *w = reinterpret_cast<const int32_t *>(&c);
#pragma unroll
  for (int k = 0; k < kClusterWords; ++k) {
    stage[lane * kClusterWords + k] = w[k];
  }
}

__global__ void __launch_bounds__(kSortThreads) k_cluster_sort(Arena a)
{
  __shared__ int hist[kSortWarps][kBuckets];
  __shared__ int bucket_total[kBuckets];
  __shared__ int bucket_base[kBuckets];
  __shared__ int32_t stages[kSortWarps][32 * kClusterWords];

  const int seg = blockIdx.x;
  const int e = seg / ITSU_LAYERS, layer = seg % ITSU_LAYERS;
  const int64_t begin = a.layer_off[seg];
  const int n = (int)(a.layer_off[seg + 1] - begin);
  const int64_t raw_begin = a.raw_off ? a.raw_off[seg] : begin;  // frames share raw clusters
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

  // Pass 1: transform every cluster (input order), per-warp bucket histograms. Each warp owns a
  // consecutive input range and moves it through its stage 32 clusters at a time.
  int32_t *stage = stages[warp];
  const int chunk = (n + kSortWarps - 1) / kSortWarps;
  const int wb = min(n, warp * chunk), we = min(n, wb + chunk);
  for (int i0 = wb; i0 < we; i0 += 32) {
    const int count = min(32, we - i0);
    itsu_cluster c{};
    if (a.raw_track) {
      // 16-byte input records (x, y, z, MC id): one aligned 16-byte load per lane; the cluster id
      // is the record's index in its layer's input order, alpha 0
      if (lane < count) {
        const float4 q = reinterpret_cast<const float4 *>(a.raw_track + raw_begin + i0)[lane];
        c.x = q.x;
        c.y = q.y;
        c.z = q.z;
        c.cluster_id = i0 + lane;
        c.alpha = 0.0f;
        c.mc_id = __float_as_int(q.w);
      }
    } else if (a.raw_in) {
      // 24-byte input records (x, y, z, id, alpha, MC id): read in 6-word strides, then the stage
      // is reused for the 36-byte records once every lane has read its own
      stage_in_words<kClusterInWords>(stage, a.raw_in + raw_begin + i0, count);
      if (lane < count) {
        c = stage_get_in(stage, lane);
      }
      __syncwarp();
    } else {
      stage_in(stage, a.raw + raw_begin + i0, count);
      if (lane < count) {
        c = stage_get(stage, lane);
      }
    }
    if (lane < count) {
      const Transformed t = transform_cluster(layer, c.x, c.y, c.z, vx, vy);
      c.phi = t.phi;
      c.r = t.r;
      c.bin = t.bin;
      const bool ok = isfinite(c.x) && isfinite(c.y) && isfinite(c.z) && fabsf(c.x) <= kMaxAbsCoordinate &&
                      fabsf(c.y) <= kMaxAbsCoordinate && fabsf(c.z) <= kMaxAbsCoordinate && !(t.r == 0.0f && c.z == vz);
      if (!ok) {
        atomicOr(&a.status->flags, kFlagInvalid);
        atomicMin(&a.status->invalid_index, (int)(begin + i0 + lane));
      }
      stage_put(stage, lane, c);
      atomicAdd(&hist[warp][bucket_of(t.bin)], 1);
    }
    stage_out(a.tmp + begin + i0, stage, count);
    __syncwarp();  // the stage is refilled next
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
    const int count = min(32, we - i0);
    stage_in(stage, a.tmp + begin + i0, count);
    const bool valid = lane < count;
    itsu_cluster c;
    int bucket = -1 - lane;
    if (valid) {
      c = stage_get(stage, lane);
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
      const int64_t at = begin + pos;
      a.xyzr[at] = make_float4(c.x, c.y, c.z, c.r);
      a.phi[at] = c.phi;
      a.clu_aux[at] = make_int4(c.cluster_id, __float_as_int(c.alpha), c.mc_id, c.bin);
    }
  }
  __syncthreads();

  // Pass 3b: the sorted records (reference layout) assembled from the scattered fields, in
  // output order, through the stages: coalesced stores instead of nine scattered ones per cluster.
  for (int i0 = warp * 32; i0 < n; i0 += kSortThreads) {
    const int count = min(32, n - i0);
    if (lane < count) {
      const int64_t at = begin + i0 + lane;
      const float4 p = a.xyzr[at];
      const int4 x = a.clu_aux[at];
      itsu_cluster c;
      c.x = p.x;
      c.y = p.y;
      c.z = p.z;
      c.phi = a.phi[at];
      c.r = p.w;
      c.cluster_id = x.x;
      c.alpha = __int_as_float(x.y);
      c.mc_id = x.z;
      c.bin = x.w;
      stage_put(stage, lane, c);
      if (a.clu_seg) {
        a.clu_seg[at] = seg;
      }
    }
    stage_out(a.sorted + begin + i0, stage, count);
    __syncwarp();  // the stage is refilled next
  }

  // Pass 4: negative bins share bucket 0 in input order; order them by bin, stably. A bottom-up
  // merge sort between the sorted segment and tmp: in each round, runs of `width` are merged in
  // pairs, every cluster moving to (its place in its run) + (the clusters of the partner run that
  // go before it: smaller bins, and for the right run equal bins too), so ties keep input order.
  // O(m log^2 m) work over the block, for layers with many clusters beyond the z range.
  const int m = bucket_total[0];
  if (m > 1) {
    itsu_cluster *src = a.sorted + begin, *dst = a.tmp + begin;
    for (int width = 1; width < m; width *= 2) {
      __syncthreads();
      for (int i = tid; i < m; i += kSortThreads) {
        const int run = i / width;
        const bool left = (run & 1) == 0;
        const int own_start = run * width;
        const int other_start = left ? own_start + width : own_start - width;
        const int other_end = min(other_start + width, m);
        const itsu_cluster c = src[i];
        int lo = other_start, hi = max(other_start, other_end);  // an empty partner run: no move
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          const int k = src[mid].bin;
          if (k < c.bin || (!left && k == c.bin)) {
            lo = mid + 1;
          } else {
            hi = mid;
          }
        }
        dst[min(own_start, other_start) + (i - own_start) + (lo - other_start)] = c;
      }
      itsu_cluster *t = src;
      src = dst;
      dst = t;
    }
    __syncthreads();
    for (int i = tid; i < m; i += kSortThreads) {
      const itsu_cluster c = src[i];
      if (src != a.sorted + begin) {
        a.sorted[begin + i] = c;
      }
      a.xyzr[begin + i] = make_float4(c.x, c.y, c.z, c.r);
      a.phi[begin + i] = c.phi;
    }
  }

  // Pass 5: the tracklet stage's candidate-pruning index. A layer is regular when every cluster
  // has a z bin and a phi bin inside the 20 x 20 table (then a bin's column is its clusters' z
  // bin) and no bin holds more than kMaxPruneBin clusters; for regular layers, each bin's
  // clusters are listed again sorted by (z, sorted index), with the layer's r range beside.
  if (a.zs == nullptr || layer == 0) {
    return;  // no index wanted, or layer 0 (never the outer layer of a tracklet)
  }
  __shared__ int s_irregular;
  __shared__ int s_rmin, s_rmax;  // float bits; r >= 0 orders like its bits
  __shared__ int s_largest;       // the largest bin
  if (tid == 0) {
    s_irregular = m > 0 || bucket_total[kBuckets - 1] > 0;  // negative bins or bin 400
    s_rmin = 0x7f800000;
    s_rmax = 0;
    s_largest = 0;
  }
  __syncthreads();
  int irregular = 0, rmin = 0x7f800000, rmax = 0;
  for (int i = tid; i < n; i += kSortThreads) {
    const float4 c = a.xyzr[begin + i];
    const int zb = z_bin_index(layer, c.z);
    const int pb = phi_bin_index(a.phi[begin + i]);
    irregular |= zb < 0 || zb >= kZBins || pb < 0 || pb >= kPhiBins;
    rmin = min(rmin, __float_as_int(c.w));
    rmax = max(rmax, __float_as_int(c.w));
  }
  if (irregular) {
    atomicOr(&s_irregular, 1);
  }
  atomicMin(&s_rmin, rmin);
  atomicMax(&s_rmax, rmax);
  int largest = 0;
  for (int b = tid; b < kTableBins; b += kSortThreads) {
    largest = max(largest, bucket_total[b + 1]);
  }
  if (largest > kMaxPruneBin) {
    atomicOr(&s_irregular, 1);
  }
  atomicMax(&s_largest, largest);
  // each cluster's rank in its bin by (z, sorted index): a warp per bin of at most kMaxPruneBin
  // (256) clusters, the bin's z values staged in the warp's record stage (free in this pass)
  static_assert(kMaxPruneBin <= 32 * kClusterWords, "a bin's z values fit a warp's stage");
  float *zstage = reinterpret_cast<float *>(stage);
  for (int bin = warp; bin < kTableBins; bin += kSortWarps) {
    const int st = bucket_base[bin + 1], cnt = bucket_total[bin + 1];
    if (cnt == 0 || cnt > kMaxPruneBin) {
      continue;  // warp-uniform
    }
    for (int k = lane; k < cnt; k += 32) {
      zstage[k] = a.xyzr[begin + st + k].z;
    }
    __syncwarp();
    for (int k = lane; k < cnt; k += 32) {
      const float4 c = a.xyzr[begin + st + k];
      int rank = 0;
      for (int j = 0; j < cnt; ++j) {
        const float zj = zstage[j];
        rank += zj < c.z || (zj == c.z && j < k);
      }
      a.zs[begin + st + rank] = make_float4(c.z, c.w, a.phi[begin + st + k], __int_as_float(st + k));
    }
    __syncwarp();  // the stage is refilled for the warp's next bin
  }
  __syncthreads();
  if (tid == 0) {
    // 0: not regular; else the 64-bit words of a pass mask over its largest bin (1, 2 or 4)
    a.seg_regular[seg] = s_irregular ? 0 : (s_largest <= 64 ? 1 : (s_largest <= 128 ? 2 : kPruneWords));
    a.seg_rrange[seg] = make_float2(__int_as_float(s_rmin), __int_as_float(s_rmax));
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

// Tracklet.cxx:32-40: the tracklet from inner cluster c to outer cluster d (local indices given);
// write_tracklet stores the one from flat cluster i_flat to j_flat.
__device__ __forceinline__ itsu_tracklet make_tracklet(float4 c, float4 d, int32_t c_local, int32_t d_local)
{
  itsu_tracklet t;
  t.first_cluster = c_local;
  t.second_cluster = d_local;
  t.tan_lambda = (c.z - d.z) / (c.w - d.w);
  t.phi = itsu_atan2f(c.y - d.y, c.x - d.x);
  return t;
}

__device__ __forceinline__ void store_tracklet(const Arena &a, int64_t out, const itsu_tracklet &t)
{
  a.tracklets[out] = t;
  a.trk_slope[out] = make_float2(t.tan_lambda, t.phi);
}

__device__ __forceinline__ void write_tracklet(const Arena &a, int out, int64_t i_flat, int64_t j_flat, int seg)
{
  store_tracklet(a, out, make_tracklet(a.xyzr[i_flat], a.xyzr[j_flat], (int32_t)(i_flat - a.layer_off[seg]),
                                       (int32_t)(j_flat - a.layer_off[seg + 1])));
}

constexpr int kTrackletSlots = kTrackletSlotsPerCluster;
constexpr int kMaxMaskedOut = 64;  // out-degrees up to this are evaluated pair-parallel with a pass mask

// The reference's candidate sequence of one inner cluster (Tracker.cxx:73-113), calling
// on_pass(j) for every next-layer cluster j that passes the cut, in emission order: the phi
// rows of the bin window in wrap-around order and, in each row, the sorted clusters from the
// row's first bin through the first cluster at or after the window's end (inclusive bound, with
// the P1/P5 guards).
//
// On a regular next layer the row is walked through the pruning index instead, which is exact:
// a pass needs |P - z2| < dz with P = (tanL (r2 - r1) + z1) in binary32, P is monotone in r2, so
// every passing z2 lies within [P(rmin) - dz, P(rmax) + dz] (widened by 1e-3 cm for the rounding
// of the bounds); only the z bins of the row that meet that interval can hold passes, and in each
// such bin only the clusters listed there between the two z values. Their passes are put back
// into index order before on_pass. The row's last candidate (the inclusive bound, past the
// window's z bins) is always evaluated. Irregular layers take the reference walk.
struct TrackletProbe {
  float4 c;      // inner cluster (x, y, z, r)
  float phi1, tan_lambda, max_dz;
  const float4 *xyzr;  // next layer
  const float *phi;
  GateWindow win;      // kGate: the learned form's first-stage windows

  // Tracker.cxx:93-100 for a next-layer cluster at z2, r2, phi2; kGate: and inside the windows
  template <bool kGate>
  __device__ __forceinline__ bool pass(float z2, float r2, float phi2) const
  {
    const float delta_z = fabsf(tan_lambda * (r2 - c.w) + c.z - z2);
    const float delta_phi = fabsf(phi1 - phi2);
    const bool cut = delta_z < max_dz && (delta_phi < kPhiCoordinateCut || delta_phi > kPhiWrapTracklet);
    if constexpr (kGate) {
      return cut && gate_window_pass(win, make_float4(0.0f, 0.0f, z2, r2), phi2);
    }
    return cut;
  }

  template <bool kGate>
  __device__ __forceinline__ bool pass(int j) const
  {
    const float4 d = xyzr[j];
    return pass<kGate>(d.z, d.w, phi[j]);
  }
};

// win_row, win_rows: the phi rows whose candidates are walked (win_rows = kPhiBins: every row); of
// the other rows only the bound candidate is tested (the first cluster of the first bin after the
// row's last z column: past empty bins it can lie in any later row).
template <int kWords, bool kGate, typename OnPass>
__device__ __forceinline__ void walk_candidates(const int32_t *table, int n_next, int4 rect, int layer, const TrackletProbe &probe,
                                                bool prune, float zlo, float zhi, const float4 *zs, int zs_off,
                                                int win_row, int win_rows, OnPass &&on_pass)
{
  // zs[k - zs_off] is the k-th entry of the next layer's z-sorted bin lists (zs_off > 0: a staged
  // copy in shared memory that starts at entry zs_off)
  static_assert(kWords >= 1 && kWords <= kPruneWords, "mask words");
  int phi_bins = rect.w - rect.y + 1;
  if (phi_bins < 0) {
    phi_bins += kPhiBins;
  }
  const int zb_lo = prune ? max(rect.x, z_bin_index(layer + 1, zlo)) : 0;
  const int zb_top = prune ? z_bin_index(layer + 1, zhi) : 0;  // clusters of higher z bins have z > zhi
  const int zb_hi = prune ? min(rect.z, zb_top) : -1;
  for (int phi_bin = rect.y, phi_count = 0; phi_count < phi_bins;
       phi_bin = (phi_bin + 1 == kPhiBins) ? 0 : phi_bin + 1, ++phi_count) {
    const int first_bin = bin_index(rect.x, phi_bin);
    const int max_bin = min(first_bin + rect.z - rect.x + 1, kTableBins);  // P5
    const bool walk_row = win_rows >= kPhiBins ||
                          (phi_bin < kPhiBins && (phi_bin - win_row + kPhiBins) % kPhiBins < win_rows);
    if (prune && phi_bin < kPhiBins) {
      for (int col = zb_lo; walk_row && col <= zb_hi; ++col) {
        const int bin = phi_bin * kPhiBins + col;
        const int k0 = table[bin], k1 = table[bin + 1];
        int lo = k0, hi = k1;  // first listed cluster with z >= zlo
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (zs[mid - zs_off].x < zlo) {
            lo = mid + 1;
          } else {
            hi = mid;
          }
        }
        // a pruned column holds at most 64 * kWords clusters (the layer's largest bin chose
        // kWords): its passes as a mask over their positions in the column, in registers,
        // emitted in index order
        unsigned long long hit[kWords];
#pragma unroll
        for (int w = 0; w < kWords; ++w) {
          hit[w] = 0ull;
        }
        for (int k = lo; k < k1; ++k) {
          const float4 q = zs[k - zs_off];  // z, r, phi and the sorted index of the k-th cluster by z
          if (!(q.x <= zhi)) {
            break;
          }
          if (probe.pass<kGate>(q.x, q.y, q.z)) {
            const int pos = __float_as_int(q.w) - k0;
            const unsigned long long bit = 1ull << (pos & 63);
            if constexpr (kWords == 1) {
              hit[0] |= bit;  // a single-word layer's columns hold at most 64 clusters
            } else {
#pragma unroll
              for (int w = 0; w < kWords; ++w) {
                hit[w] |= (pos >> 6) == w ? bit : 0ull;
              }
            }
          }
        }
#pragma unroll
        for (int w = 0; w < kWords; ++w) {
          while (hit[w]) {
            const int b = __ffsll((long long)hit[w]) - 1;
            hit[w] &= hit[w] - 1ull;
            on_pass(k0 + 64 * w + b);
          }
        }
      }
      // The inclusive bound's candidate (P1: inside the layer): the first cluster of bin
      // max_bin, the row's next z column. When that bin is not empty and its z column lies
      // beyond zhi's (z bins are monotone in z; a regular layer's clusters sit in exactly their
      // bins), the candidate's z exceeds zhi and it fails the Δz cut: it is not read.
      const int x = table[max_bin];
      const bool beyond = rect.z + 1 < kZBins && rect.z + 1 > zb_top && table[max_bin + 1] > x;
      if (!beyond && x < n_next && probe.pass<kGate>(x)) {
        on_pass(x);
      }
    } else {
      const int first_row = table[first_bin];
      const int last_row = min(table[max_bin], n_next - 1);  // inclusive bound, P1
      for (int j = walk_row ? first_row : last_row; j <= last_row; ++j) {
        if (probe.pass<kGate>(j) && (walk_row || j == table[max_bin])) {
          on_pass(j);
        }
      }
    }
  }
}

// The walk state of one inner cluster i (flat index): whether its layer runs the tracklet
// stage, and the probe, window and pruning bounds of its candidate walk.
struct InnerCluster {
  bool walk;
  int win_row, win_rows;  // the phi rows its |dphi| window reaches (win_rows = kPhiBins: every row)
  int seg, e, layer;
  int4 rect;
  TrackletProbe probe;
  bool prune;
  int words;
  float zlo, zhi;
  const int32_t *table;
  int n_next;
  int64_t next_begin;
};

// The phi rows that hold the azimuths within half_width of phi (the window's rows, clamped into
// 0..kPhiBins - 1): first row and count, in the walk's cyclic order.
__device__ __forceinline__ void window_rows(float phi, float half_width, int *first, int *rows)
{
  float lo = phi - half_width, hi = phi + half_width;
  lo = lo < 0.0f ? lo + kTwoPi : lo;
  hi = hi >= kTwoPi ? hi - kTwoPi : hi;
  const int r_lo = min(phi_bin_index(lo), kPhiBins - 1), r_hi = min(phi_bin_index(hi), kPhiBins - 1);
  int n = r_hi - r_lo + 1;
  *first = r_lo;
  *rows = n <= 0 ? n + kPhiBins : n;
}

// With a tracklet gate (learned form), its first stage's windows for the layer narrow the walk: a
// tracklet outside them is not kept. The walk keeps the plain rect and its row sequence (with the
// reference's edge behaviour, e.g. a first row of 20 when the window's lower edge rounds to 2pi),
// but of a row outside the |dphi| window (widened by 1e-3 rad against rounding) it only tests the
// row's bound candidate (P1), which can lie in the next row; the pruned columns take the narrower
// z range of the |dz| window (widened by 1e-3 cm). In a regular layer every cluster sits in its
// own bin, so the walk still meets every plain candidate inside the windows, in the plain order;
// other layers are walked whole. Every candidate's cut includes the windows themselves
// (gate_window_pass): the gated tracklets are exactly the plain tracklets inside the windows.
// kGate: the learned form with a tracklet gate (a.gate set); the plain form's instantiation has
// none of the windows' code.
template <bool kGate>
__device__ __forceinline__ InnerCluster inner_cluster(const Arena &a, int64_t i)
{
  InnerCluster s;
  s.walk = false;
  s.seg = a.clu_seg[i];
  s.e = s.seg / ITSU_LAYERS;
  s.layer = s.seg % ITSU_LAYERS;
  const int32_t *lo = a.layer_off + s.e * ITSU_LAYERS;
  if (s.layer >= ITSU_LAYERS - 1 || !tracklets_active(lo, s.layer)) {
    return s;
  }
  s.probe.c = a.xyzr[i];
  s.probe.phi1 = a.phi[i];
  const float vz = a.vtx[3 * s.e + 2];
  s.probe.tan_lambda = (s.probe.c.z - vz) / s.probe.c.w;
  const float dir_z = s.probe.tan_lambda * (kC.r[s.layer + 1] - s.probe.c.w) + s.probe.c.z;
  s.rect = bins_rect(s.probe.phi1, s.layer, dir_z);
  if (s.rect.x == 0 && s.rect.y == 0 && s.rect.z == 0 && s.rect.w == 0) {
    return s;  // the reference's "no bins" rect (Tracker.cxx:66-70)
  }
  s.walk = true;
  s.next_begin = lo[s.layer + 1];
  s.probe.xyzr = a.xyzr + s.next_begin;
  s.probe.phi = a.phi + s.next_begin;
  s.probe.max_dz = kC.trk_max_dz[s.layer];
  const int next_seg = s.seg + 1;
  s.words = a.seg_regular[next_seg];  // 0: not regular, else the mask words its largest bin needs
  s.win_row = 0;
  s.win_rows = kPhiBins;
  if constexpr (kGate) {
    s.probe.win = gate_window(*a.gate, s.layer, s.probe.c, s.probe.phi1, vz);
    if (s.words != 0 && s.probe.win.dphi + 1e-3f < kPhiCoordinateCut) {  // a wider window narrows nothing
      window_rows(s.probe.phi1, s.probe.win.dphi + 1e-3f, &s.win_row, &s.win_rows);
    }
  }
  s.prune = a.prune_tracklets && s.words != 0;
  s.zlo = s.zhi = 0;
  if (s.prune) {
    const float2 rr = a.seg_rrange[next_seg];
    const float p1 = s.probe.tan_lambda * (rr.x - s.probe.c.w) + s.probe.c.z;
    const float p2 = s.probe.tan_lambda * (rr.y - s.probe.c.w) + s.probe.c.z;
    const float half = kGate ? fminf(s.probe.max_dz, s.probe.win.dz + 1e-3f) : s.probe.max_dz;
    s.zlo = fminf(p1, p2) - half - 1e-3f;
    s.zhi = fmaxf(p1, p2) + half + 1e-3f;
    s.prune = isfinite(s.zlo) && isfinite(s.zhi);
  }
  s.table = a.index_tables + ((int64_t)s.e * ITSU_TRACKLET_LAYERS + s.layer) * kTableSize;
  s.n_next = lo[s.layer + 2] - lo[s.layer + 1];
  return s;
}

// staged: the block's copy in shared memory of the next layer's z-sorted entries from staged_off on
// (null: read them from global memory)
template <bool kGate, typename OnPass>
__device__ __forceinline__ void walk_inner(const Arena &a, const InnerCluster &s, OnPass &&on_pass,
                                           const float4 *staged = nullptr, int staged_off = 0)
{
  const float4 *zs = staged ? staged : a.zs + s.next_begin;
  const int off = staged ? staged_off : 0;
  if (s.words <= 1) {  // unpruned, or bins of at most 64 clusters
    walk_candidates<1, kGate>(s.table, s.n_next, s.rect, s.layer, s.probe, s.prune, s.zlo, s.zhi, zs, off, s.win_row,
                              s.win_rows, on_pass);
  } else if (s.words == 2) {
    walk_candidates<2, kGate>(s.table, s.n_next, s.rect, s.layer, s.probe, s.prune, s.zlo, s.zhi, zs, off, s.win_row,
                              s.win_rows, on_pass);
  } else {
    walk_candidates<kPruneWords, kGate>(s.table, s.n_next, s.rect, s.layer, s.probe, s.prune, s.zlo, s.zhi, zs, off,
                                        s.win_row, s.win_rows, on_pass);
  }
}

// ---- bulk copies into shared memory (cp.async.bulk, this GPU's memory, no multicast) ----

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global to shared
// memory, completing on `bar` (the calling thread also arrives on it, expecting those bytes).
__device__ __forceinline__ void bulk_copy_to_shared(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(bytes), "r"(b)
               : "memory");
}

// Waits for phase `parity` of `bar` to complete, at most `limit` tries; false if it did not.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int limit)
{
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  for (int t = 0; t < limit; ++t) {
    unsigned done;
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                 : "=r"(done)
                 : "r"(b), "r"(parity)
                 : "memory");
    if (done) {
      return true;
    }
  }
  return false;
}

constexpr int kStageEntries = 2048;  // the staged walk's shared copy: up to 2048 entries (32 KB) per block
constexpr int kStageRows = 4;        // and up to 4 phi rows of the next layer
constexpr int kWaitTries = 1 << 20;  // bounded waits: each try_wait suspends for a bounded time

// The staged walk's set-up, block-wide: when every walking thread of the block walks pruned rows
// of the same next layer, without a wrap around phi, and their rows (at most kStageRows) hold at
// most kStageEntries entries, one bulk copy brings those entries into shared memory. Returns the
// first staged entry's index in the layer (its *staged_count entries), or -1 with nothing staged.
// A copy that does not complete within the bounded wait sets the timeout flag.
__device__ int stage_rows(const Arena &a, const InnerCluster &s, float4 *stage, uint64_t *bar, int *staged_count)
{
  __shared__ int s_lo, s_hi, s_seg, s_ok, s_k0, s_m;
  if (threadIdx.x == 0) {
    s_lo = kPhiBins;
    s_hi = -1;
    s_seg = -1;
    s_ok = 1;
  }
  __syncthreads();
  if (s.walk) {
    if (!s.prune || s.rect.y > s.rect.w) {
      atomicAnd(&s_ok, 0);  // unpruned, or a window that wraps around phi
    }
    atomicMin(&s_lo, s.rect.y);
    atomicMax(&s_hi, s.rect.w);
    atomicMax(&s_seg, s.seg + 1);
  }
  __syncthreads();
  if (s.walk && s.seg + 1 != s_seg) {
    atomicAnd(&s_ok, 0);  // more than one next layer
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s_m = 0;
    s_k0 = -1;
    if (s_ok && s_hi >= s_lo && s_hi - s_lo < kStageRows) {
      const int e = s_seg / ITSU_LAYERS, next_layer = s_seg % ITSU_LAYERS;
      const int32_t *table = a.index_tables + ((int64_t)e * ITSU_TRACKLET_LAYERS + next_layer - 1) * kTableSize;
      const int k0 = table[s_lo * kPhiBins], k1 = table[min((s_hi + 1) * kPhiBins, kTableBins)];
      if (k1 > k0 && k1 - k0 <= kStageEntries) {
        s_k0 = k0;
        s_m = k1 - k0;
        mbar_init(bar, 1);
        bulk_copy_to_shared(stage, a.zs + a.layer_off[s_seg] + k0, (unsigned)(s_m * sizeof(float4)), bar);
      }
    }
  }
  __syncthreads();
  if (s_k0 < 0) {
    return -1;
  }
  if (!mbar_wait(bar, 0, kWaitTries)) {
    atomicOr(&a.status->flags, kFlagTimeout);
    mbar_wait(bar, 0, kWaitTries);  // the copy may still land: wait once more before leaving
    return -1;
  }
  *staged_count = s_m;
  return s_k0;
}

constexpr int kCountThreads = 256;

// Count pass, one thread per inner cluster: the number of tracklets, and the outer clusters of
// the first kTrackletSlots of them in emission order. kStaged: the block's walks read the next
// layer's z-sorted entries from a shared-memory copy made by one bulk copy (stage_rows), where
// they allow it. kGate: the learned form's first stage (inner_cluster). At most kCountThreads
// threads per block; measured per 128 events: the plain instantiation at 40 registers (6 blocks
// per SM) 0.64 ms, at 48 0.66, at 54 0.72; the learned one at 48 (5 blocks) 0.39 ms, at 56 0.43.
template <bool kStaged, bool kGate>
__global__ void __launch_bounds__(kCountThreads, kGate ? 5 : 6) k_tracklets_count(Arena a)
{
  extern __shared__ float4 stage[];  // kStaged: kStageEntries entries
  __shared__ uint64_t bar;
  const int64_t i = global_thread();
  const bool valid = i < a.n_clusters;
  int count = 0;
  InnerCluster s;
  s.walk = false;
  if (valid) {
    s = inner_cluster<kGate>(a, i);
  }
  const float4 *staged = nullptr;
  int staged_off = 0;
  if constexpr (kStaged) {
    int m = 0;
    staged_off = stage_rows(a, s, stage, &bar, &m);
    staged = staged_off >= 0 ? stage : nullptr;
  }
  if (s.walk && !(a.status->flags & kFlagTimeout)) {
    walk_inner<kGate>(
        a, s,
        [&](int j) {
          if (count < kTrackletSlots) {
            a.trk_slots[count * a.slot_stride + i] = j;
          }
          ++count;
        },
        staged, staged_off);
  }
  // the warp's 32 clusters lie in one scan tile: their tracklets go to its sum (the tracklet
  // scan has no reduce pass)
  const int warp_count = (int)__reduce_add_sync(0xffffffffu, (unsigned)count);
  if ((threadIdx.x & 31) == 0 && warp_count != 0) {
    atomicAdd(reinterpret_cast<unsigned long long *>(&a.scan_partials[i / kScanTile]), (unsigned long long)warp_count);
  }
  if (!valid) {
    return;
  }
  a.trk_count[i] = count;
  if (count > kTrackletSlots) {  // rare: the write pass leaves this cluster to k_tracklets_crowded
    const unsigned long long q = atomicAdd(reinterpret_cast<unsigned long long *>(&a.status->trk_crowded), 1ull);
    if ((int64_t)q < a.n_clusters) {
      a.clu_crowded[q] = (int32_t)i;
    }
  }
}

__device__ __forceinline__ float4 shfl4(float4 v, int src)
{
  return make_float4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                     __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}

__device__ __forceinline__ int warp_exclusive_sum(int v, int &total)
{
  const int lane = threadIdx.x & 31;
  int inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) {
      inc += t;
    }
  }
  total = __shfl_sync(0xffffffffu, inc, 31);
  return inc - v;
}

// Owner lane of flattened item t given the lanes' exclusive prefix sums: the last lane whose
// prefix is <= t (for t < total this lane holds item t). All lanes must call it together.
__device__ __forceinline__ int owner_of(int excl, int t)
{
  int owner = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1) {
    const int v = __shfl_sync(0xffffffffu, excl, owner + step);
    if (v <= t) {
      owner += step;
    }
  }
  return owner;
}

// Learned form: the tracklet gate. After the count pass and before the tracklet scan, a warp per
// 32 consecutive inner clusters scores their tracklets (the outer clusters the count pass kept in
// their slots), 32 at a time on the tensor cores (8 -> 16 -> 16 -> 1, ReLU, BF16 / FP32, the
// network in registers), keeps those whose logit is not below the gate's threshold (a NaN logit
// keeps its tracklet), moves the kept slots to the front in their order and lowers the cluster's
// count and its scan tile's sum by the dropped ones. The write pass then writes the kept tracklets
// in emission order, as in the plain form. Inner clusters with more than kTrackletSlots tracklets
// keep all of them, unscored (the crowded pass writes them), and so do those of the layers the
// network does not score (the model's mlp_layers).
//
// Per warp and group of 32 clusters, the flattened tracklets' owners and ranks are listed once in
// shared memory (each cluster's lane writes its own entries), and each cluster's gate state (what
// its features need of it) sits beside them, so that a tile reads its rows' owners, states and
// slots without searches or shuffles; the lanes holding a row's logit keep or drop it.
constexpr int kGateThreads = 256;
constexpr int kGateWarps = kGateThreads / 32;

struct __align__(16) GateLane {
  GateInner g;
  int32_t next;  // first cluster of the next layer
  int32_t pad_;
};

// The gate pass's per-warp shared memory.
struct GateShared {
  __align__(16) __nv_bfloat16 rows[kGateWarps][32][kMlpIn];
  unsigned long long keep[kGateWarps][32];
  uint16_t owner_rank[kGateWarps][32 * kTrackletSlots];  // owner lane * 64 + rank
  GateLane lanes[kGateWarps][32];
};

// One warp group of k_tracklets_gate: the inner clusters base .. base + 31 of which those in
// [start, end) take part (event e).
__device__ __forceinline__ void gate_group(const Arena &a, const GateSmem &net, const GateRegs &R, GateShared &sh, int warp,
                                           int64_t base, int64_t start, int64_t end, int e)
{
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  __nv_bfloat16 (&rows)[32][kMlpIn] = sh.rows[warp];
  unsigned long long (&keep)[32] = sh.keep[warp];
  uint16_t (&owner_rank)[32 * kTrackletSlots] = sh.owner_rank[warp];
  GateLane (&lanes)[32] = sh.lanes[warp];
  const int64_t i = base + lane;
  int count = 0;
  bool scored = false;  // by the network: in the range, and not crowded
  if (i >= start && i < end) {
    count = a.trk_count[i];
    if (count > 0 && count <= kTrackletSlots) {
      const int seg = a.clu_seg[i];
      scored = true;
      GateLane &s = lanes[lane];
      s.g = gate_inner(seg % ITSU_LAYERS, a.xyzr[i], a.phi[i], a.vtx[3 * e], a.vtx[3 * e + 1], a.vtx[3 * e + 2]);
      s.next = a.layer_off[seg + 1];
    }
  }
  const int mine = scored ? count : 0;
  keep[lane] = 0ull;
  int total = 0;
  const int excl = warp_exclusive_sum(mine, total);
  for (int r = 0; r < mine; ++r) {
    owner_rank[excl + r] = (uint16_t)(lane * 64 + r);
  }
  __syncwarp();
  for (int p0 = 0; p0 < total; p0 += 32) {
    const int p = p0 + lane;
    float f[kMlpIn];
    if (p < total) {
      const int orank = owner_rank[p], owner = orank >> 6, rank = orank & 63;
      const GateLane &o = lanes[owner];
      const int64_t j = o.next + a.trk_slots[(int64_t)rank * a.slot_stride + base + owner];
      gate_features(o.g, a.xyzr[j], a.phi[j], f);
    } else {
#pragma unroll
      for (int k = 0; k < kMlpIn; ++k) {
        f[k] = net.mean[k];
      }
    }
    *reinterpret_cast<uint4 *>(&rows[lane][0]) = gate_row(net.mean, net.inv_std, f);
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      float lo, hi;
      gate_forward_m16(R, rows, mt, lo, hi);
      if (t == 0) {  // this lane holds the logits of rows 16 mt + g and 16 mt + g + 8
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int q = p0 + mt * 16 + g + 8 * h;
          const float logit = h ? hi : lo;
          if (q < total && !(logit < net.threshold)) {
            const int orank = owner_rank[q];
            atomicOr(&keep[orank >> 6], 1ull << (orank & 63));
          }
        }
      }
    }
    __syncwarp();  // the rows are refilled for the next tile
  }
  // kept slots to the front, in order (coalesced across the warp's clusters, slot by slot)
  const unsigned long long m = keep[lane];
  const int scan_to = __reduce_max_sync(0xffffffffu, (unsigned)mine);
  int kept = 0;
  for (int q = 0; q < scan_to; ++q) {
    if (q < count && ((m >> q) & 1ull)) {
      if (kept != q) {
        a.trk_slots[(int64_t)kept * a.slot_stride + i] = a.trk_slots[(int64_t)q * a.slot_stride + i];
      }
      ++kept;
    }
  }
  int dropped = 0;
  if (scored) {
    a.trk_count[i] = kept;
    dropped = count - kept;
  }
  // the warp's 32 clusters lie in one scan tile (the count pass added their tracklets to its sum)
  const int warp_dropped = (int)__reduce_add_sync(0xffffffffu, (unsigned)dropped);
  if (lane == 0 && warp_dropped != 0) {
    atomicAdd(reinterpret_cast<unsigned long long *>(&a.scan_partials[base / kScanTile]),
              (unsigned long long)(-(int64_t)warp_dropped));
  }
  __syncwarp();
}

__global__ void __launch_bounds__(kGateThreads) k_tracklets_gate(Arena a)
{
  __shared__ GateSmem net;
  __shared__ GateShared sh;
  load_mlp(net, *a.gate);
  __syncthreads();
  const GateRegs R = gate_regs(net);
  const int warp = threadIdx.x >> 5;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t first_warp = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  for (int e = blockIdx.y; e < a.n_events; e += gridDim.y) {
    for (int l0 = 0; l0 < ITSU_TRACKLET_LAYERS; ++l0) {
      if (!((net.layers >> l0) & 1u) || (l0 > 0 && ((net.layers >> (l0 - 1)) & 1u))) {
        continue;  // not the first layer of a run of scored layers
      }
      int l1 = l0;
      while (l1 + 1 < ITSU_TRACKLET_LAYERS && ((net.layers >> (l1 + 1)) & 1u)) {
        ++l1;
      }
      // the inner clusters of layers l0..l1 of event e, in warp groups aligned to 32 (so that each
      // group lies in one scan tile; a group's lanes outside the range take no part)
      const int64_t start = a.layer_off[e * ITSU_LAYERS + l0], end = a.layer_off[e * ITSU_LAYERS + l1 + 1];
      for (int64_t base = (start & ~(int64_t)31) + first_warp * 32; base < end; base += warps * 32) {
        gate_group(a, net, R, sh, warp, base, start, end, e);
      }
    }
  }
}

// Write pass, a warp per 32 consecutive inner clusters: their tracklets form one contiguous range
// (the scan of the counts), which the warp's lanes fill together: each lane takes the next
// tracklet of the range, finds its inner cluster (owner) and rank there, reads the outer cluster
// the count pass kept in that slot, and writes the tracklet (Tracklet.cxx:32-40) and its segment
// id with coalesced stores; all lanes compute their binary64 azimuths together. Each cluster's
// tracklets lookup entry is written here too. The tracklets of an inner cluster with more than
// kTrackletSlots of them (not kept by the count pass) get their segment ids here and the rest
// from k_tracklets_crowded.
// Runs over the inner clusters [c0, c1) (c0 a multiple of 32, so that warps hold whole aligned
// groups of 32 clusters): all of them, or one event group's share of them.
__global__ void __launch_bounds__(kMaxThreads, 2) k_tracklets_write(Arena a, int64_t c0, int64_t c1)  // 64 registers: 4 blocks of 256 per SM
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int64_t i = c0 + global_thread();
  const int lane = threadIdx.x & 31;
  const bool valid = i < c1;
  int32_t first = 0, count = 0, local = 0, next_begin = 0;
  int seg = 0, sid = 0;
  float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (valid) {
    first = a.trk_off[i];
    count = a.trk_off[i + 1] - first;
    seg = a.clu_seg[i];
    const int e = seg / ITSU_LAYERS, layer = seg % ITSU_LAYERS;
    a.trk_lookup[i] = (layer >= 1 && layer <= ITSU_CELL_LAYERS && count > 0)
                          ? first - a.trk_seg[e * ITSU_TRACKLET_LAYERS + layer]
                          : ITSU_UNUSED_INDEX;
    sid = e * ITSU_TRACKLET_LAYERS + layer;
    if (count > 0) {
      c = a.xyzr[i];
      local = (int32_t)(i - a.layer_off[seg]);
      next_begin = a.layer_off[seg + 1];
    }
  }
  int total = 0;
  const int excl = warp_exclusive_sum(count, total);
  const int32_t base = __shfl_sync(0xffffffffu, first, 0);
  const int64_t i0 = i - lane;
  for (int p0 = 0; p0 < total; p0 += 32) {
    const int p = p0 + lane;
    const int owner = owner_of(excl, p);
    const int rank = p - __shfl_sync(0xffffffffu, excl, owner);
    const int owner_sid = __shfl_sync(0xffffffffu, sid, owner);
    const int owner_count = __shfl_sync(0xffffffffu, count, owner);
    const int32_t owner_local = __shfl_sync(0xffffffffu, local, owner);
    const int32_t owner_next = __shfl_sync(0xffffffffu, next_begin, owner);
    const float4 oc = shfl4(c, owner);
    if (p < total) {
      a.trk_seg_id[base + p] = owner_sid;
      if (owner_count <= kTrackletSlots) {
        const int32_t j = a.trk_slots[(int64_t)rank * a.slot_stride + i0 + owner];
        const float4 d = a.xyzr[owner_next + j];
        store_tracklet(a, base + p, make_tracklet(oc, d, owner_local, j));
      }
    }
  }
}

// Write pass, part 2: the inner clusters with more than kTrackletSlots tracklets (listed by the
// count pass, a handful per batch) walk their candidates again and write their tracklets in order.
template <bool kGate>
__global__ void __launch_bounds__(kMaxThreads) k_tracklets_crowded(Arena a)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int64_t listed = min(a.status->trk_crowded, (int64_t)a.n_clusters);
  for (int64_t q = global_thread(); q < listed; q += grid_threads()) {
    const int64_t i = a.clu_crowded[q];
    const InnerCluster s = inner_cluster<kGate>(a, i);
    int out = a.trk_off[i];
    walk_inner<kGate>(a, s, [&](int j) { write_tracklet(a, out++, i, s.next_begin + j, s.seg); });
  }
}

// Cell layer L of event e runs only if tracklet layers 0..L+1 are all non-empty
// (Tracker.cxx:124-128); ts holds the event's first tracklet of each layer and the next event's.
__device__ __forceinline__ bool cells_active(const int32_t *ts, int layer)
{
  for (int l = 0; l <= layer; ++l) {
    if (ts[l + 1] - ts[l] <= 0 || ts[l + 2] - ts[l + 1] <= 0) {
      return false;
    }
  }
  return true;
}

// trk_seg[6e+L] = first tracklet of (e, L); capacity check of the tracklet total. For the cell
// layers, the segment's cell-stage record too (cell_seginfo[2s], [2s+1]): the first cluster of
// layers L, L+1, L+2 (the first -1 when cell layer L of the event does not run), the first
// tracklet of layers L and L+1 and the vertex, so that each first tracklet's setup in the cell
// count pass is two 16-byte loads of one record instead of a dozen loads of per-event offsets.
__global__ void k_tracklet_segments(Arena a)
{
  // the cells scan's tile sums start at zero: the cell count pass adds each warp's cells there
  const int64_t n_trk = a.status->total[kTracklets];
  if (n_trk <= a.cap_tracklets) {
    for (int64_t t = global_thread(); t < (n_trk + kScanTile - 1) / kScanTile; t += grid_threads()) {
      a.scan_partials[t] = 0;
    }
  }
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
      if (layer < ITSU_CELL_LAYERS) {
        const int32_t *lo = a.layer_off + e * ITSU_LAYERS;
        int32_t ts[ITSU_LAYERS];
        for (int l = 0; l < ITSU_LAYERS; ++l) {
          ts[l] = a.trk_off[lo[l]];
        }
        const bool active = cells_active(ts, layer);
        a.cell_seginfo[2 * s] = make_int4(active ? lo[layer] : -1, lo[layer + 1], lo[layer + 2], ts[layer]);
        a.cell_seginfo[2 * s + 1] = make_int4(ts[layer + 1], __float_as_int(a.vtx[3 * e]), __float_as_int(a.vtx[3 * e + 1]),
                                              __float_as_int(a.vtx[3 * e + 2]));
      }
    }
  }
}

// ------------------------------------------------------------------------------------------
// (c) cells: TrackerTraits<false>::computeLayerCells (Tracker.cxx:120-235)

// Per-lane state of the warp-parallel cell stage: lane l owns first tracklet k = base + l.
struct CellLane {
  int64_t k;
  int layer, e;
  float t1_tan_lambda, t1_phi;
  float4 c1, c2;
  float vx, vy, vz;
  int32_t j0, n_out;     // the outgoing tracklets of the tracklet's outer cluster: [j0, j0 + n_out)
  int32_t c3_base;       // first cluster of layer L + 2
  int32_t t1_local, t1_first, t1_second, t2_base;  // tracklet index in its layer, its clusters, first tracklet of layer L + 1
};

__device__ __forceinline__ CellLane cell_lane(const Arena &a, int64_t k, int64_t n)
{
  CellLane s;
  s.k = k;
  s.n_out = 0;
  s.layer = ITSU_CELL_LAYERS;
  s.e = 0;
  if (k >= n) {
    return s;
  }
  // both loads first: neither depends on the other
  const int sid = a.trk_seg_id[k];
  const itsu_tracklet t1 = a.tracklets[k];
  s.e = sid / ITSU_TRACKLET_LAYERS;
  s.layer = sid % ITSU_TRACKLET_LAYERS;
  if (s.layer >= ITSU_CELL_LAYERS) {
    s.layer = ITSU_CELL_LAYERS;
    return s;
  }
  const int4 A = a.cell_seginfo[2 * sid], B = a.cell_seginfo[2 * sid + 1];
  if (A.x < 0) {
    s.layer = ITSU_CELL_LAYERS;
    return s;
  }
  s.t1_tan_lambda = t1.tan_lambda;
  s.t1_phi = t1.phi;
  s.t1_first = t1.first_cluster;
  s.t1_second = t1.second_cluster;
  s.c1 = a.xyzr[A.x + t1.first_cluster];
  const int64_t c2i = A.y + t1.second_cluster;
  s.c2 = a.xyzr[c2i];
  s.j0 = a.trk_off[c2i];
  s.n_out = a.trk_off[c2i + 1] - s.j0;
  s.vx = __int_as_float(B.y);
  s.vy = __int_as_float(B.z);
  s.vz = __int_as_float(B.w);
  s.c3_base = A.z;
  s.t1_local = (int32_t)(k - A.w);
  s.t2_base = B.x;
  return s;
}

__device__ __forceinline__ void write_cell(const Arena &a, int64_t out, const CellLane &s, const itsu_tracklet &t2, int32_t j,
                                           float3 normal, float curvature)
{
  itsu_cell cell;
  cell.first_cluster = s.t1_first;
  cell.second_cluster = t2.first_cluster;
  cell.third_cluster = t2.second_cluster;
  cell.first_tracklet = s.t1_local;
  cell.second_tracklet = j - s.t2_base;
  cell.nx = normal.x;
  cell.ny = normal.y;
  cell.nz = normal.z;
  cell.curvature = curvature;
  cell.level = 1;
  a.cells[out] = cell;
  a.cell_seg_id[out] = s.e * ITSU_CELL_LAYERS + s.layer;
}

// Count pass: for each first tracklet, a mask of which of its (<= 64) outgoing tracklets make a
// cell, and their number. Each lane runs the cheap cuts of its own tracklet's outgoing tracklets
// (Tracker.cxx:155-173) on their (tanL, phi), one independent 8-byte load each; the
// pairs that pass (about one in eighteen candidates) are then flattened across the warp's lanes so
// that the circle geometry runs with the lanes converged. Each pair that passes the geometry
// becomes a cell entry (its tracklets, normal, curvature and DCA) in the warp's current chunk of
// the entry scratch, so the write pass needs no geometry.
//
// Runs over the first tracklets of events [e0, e1), or of all events when e1 is 0. Warps hold
// aligned groups of 32 tracklets (their cells go to one scan tile); a group that straddles the
// range's ends has its lanes outside the range idle.
__global__ void __launch_bounds__(kMaxThreads) k_cells_count(Arena a, int32_t e0, int32_t e1)
{
  __shared__ unsigned long long masks[kMaxThreads / 32][32];
  if (capacity_failed(a.status)) {
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t n = a.status->total[kTracklets];
  const int64_t t0 = e1 > 0 ? a.trk_seg[(int64_t)e0 * ITSU_TRACKLET_LAYERS] : 0;
  const int64_t t1 = e1 > 0 ? a.trk_seg[(int64_t)e1 * ITSU_TRACKLET_LAYERS] : n;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  int64_t chunk_pos = 0, chunk_end = 0;  // this warp's reserved cell entries (warp-uniform)
  for (int64_t base = (t0 & ~int64_t(31)) + ((int64_t)blockIdx.x * (blockDim.x >> 5) + warp) * 32; base < t1;
       base += warps * 32) {
    const int64_t k_lane = base + lane;
    const bool active = k_lane >= t0 && k_lane < t1;
    const CellLane s = cell_lane(a, active ? k_lane : n, n);
    const bool big = s.n_out > kMaxMaskedOut;
    unsigned long long window = 0;  // the outgoing tracklets that pass the cheap cuts
    if (!big && s.n_out > 0) {
      const float max_dz = kC.cell_max_dz[s.layer];  // n_out > 0: an active cell layer
      // (tanL, phi) of the outgoing tracklets, packed 8 bytes each; the window's two 32-bit
      // halves are filled by two loops (a 64-bit variable shift per candidate costs more)
      const float2 *tp = a.trk_slope + s.j0;
      unsigned lo = 0u, hi = 0u;
      const int n_lo = s.n_out < 32 ? s.n_out : 32;
#pragma unroll 4
      for (int q = 0; q < n_lo; ++q) {
        const float2 t2 = tp[q];
        lo |= (unsigned)cell_precut_dz(s.t1_tan_lambda, s.t1_phi, t2.x, t2.y, s.c1, s.vz, max_dz) << q;
      }
#pragma unroll 4
      for (int q = 32; q < s.n_out; ++q) {
        const float2 t2 = tp[q];
        hi |= (unsigned)cell_precut_dz(s.t1_tan_lambda, s.t1_phi, t2.x, t2.y, s.c1, s.vz, max_dz) << (q - 32);
      }
      window = ((unsigned long long)hi << 32) | lo;
    }
    masks[warp][lane] = 0ull;
    int total = 0;
    const int excl = warp_exclusive_sum(__popcll(window), total);
    __syncwarp();
    for (int p0 = 0; p0 < total; p0 += 32) {
      const int p = p0 + lane;
      const int owner = owner_of(excl, p);
      const int r = p - __shfl_sync(0xffffffffu, excl, owner);
      const unsigned long long wmask = __shfl_sync(0xffffffffu, window, owner);
      const int32_t j0 = __shfl_sync(0xffffffffu, s.j0, owner);
      // the circle geometry reads x, y and r of the first two clusters, not z
      const int32_t c3_base = __shfl_sync(0xffffffffu, s.c3_base, owner);
      const float4 c1 = make_float4(__shfl_sync(0xffffffffu, s.c1.x, owner), __shfl_sync(0xffffffffu, s.c1.y, owner), 0.0f,
                                    __shfl_sync(0xffffffffu, s.c1.w, owner));
      const float4 c2 = make_float4(__shfl_sync(0xffffffffu, s.c2.x, owner), __shfl_sync(0xffffffffu, s.c2.y, owner), 0.0f,
                                    __shfl_sync(0xffffffffu, s.c2.w, owner));
      const float vx = __shfl_sync(0xffffffffu, s.vx, owner), vy = __shfl_sync(0xffffffffu, s.vy, owner);
      const int layer = __shfl_sync(0xffffffffu, s.layer, owner);
      bool pass = false;
      int b = 0;
      int32_t c3 = 0;
      float3 normal = make_float3(0.0f, 0.0f, 0.0f);
      float curvature = 0.0f, dca = 0.0f;
      if (p < total) {
        {
          // the owner's r-th passing outgoing tracklet: the r-th set bit of its window, found in
          // the 32-bit half that holds it
          const unsigned wlo = (unsigned)wmask;
          const int plo = __popc(wlo);
          const bool in_lo = r < plo;
          unsigned m = in_lo ? wlo : (unsigned)(wmask >> 32);
          for (int q = in_lo ? r : r - plo; q > 0; --q) {
            m &= m - 1u;
          }
          b = __ffs(m) - 1 + (in_lo ? 0 : 32);
        }
        c3 = a.tracklets[j0 + b].second_cluster;
        pass = cell_geometry(layer, c1, c2, a.xyzr[c3_base + c3], vx, vy, normal, curvature, dca);
        if (pass) {
          atomicOr(&masks[warp][owner], 1ull << b);
        }
      }
      // entries: the passing lanes' slots, contiguous in the warp's chunk
      const unsigned m = __ballot_sync(0xffffffffu, pass);
      const int need = __popc(m);
      const int rank = __popc(m & ((1u << lane) - 1u));
      int64_t slot = chunk_pos + rank;
      if (need > chunk_end - chunk_pos) {
        const int room = (int)(chunk_end - chunk_pos);
        unsigned long long fresh = 0;
        if (lane == 0) {
          fresh = atomicAdd(reinterpret_cast<unsigned long long *>(&a.status->cell_entries), (unsigned long long)kCellChunk);
          if ((int64_t)fresh + kCellChunk > a.cap_cell_entries) {
            atomicOr(&a.status->flags, kFlagCapScratch);
          }
        }
        const int64_t fresh_base = (int64_t)__shfl_sync(0xffffffffu, fresh, 0);
        slot = rank < room ? chunk_pos + rank : fresh_base + (rank - room);
        chunk_pos = fresh_base + (need - room);
        chunk_end = fresh_base + kCellChunk;
      } else {
        chunk_pos += need;
      }
      if (pass && slot < a.cap_cell_entries) {
        // the rest of the cell record, read again (cached since cell_lane) rather than kept in
        // registers through the pair loops
        const int64_t t1 = base + owner;
        const int2 t1_clusters = *reinterpret_cast<const int2 *>(a.tracklets + t1);
        const int e = a.trk_seg_id[t1] / ITSU_TRACKLET_LAYERS;
        const int32_t *ts = a.trk_seg + e * ITSU_TRACKLET_LAYERS;
        int4 *dst = reinterpret_cast<int4 *>(a.cell_entries + slot);
        dst[0] = make_int4((int)t1, b, e * ITSU_CELL_LAYERS + layer, t1_clusters.x);
        dst[1] = make_int4(t1_clusters.y, c3, (int)(t1 - ts[layer]), j0 + b - ts[layer + 1]);
        dst[2] = make_int4(__float_as_int(normal.x), __float_as_int(normal.y), __float_as_int(normal.z), __float_as_int(curvature));
        if (a.mlp) {
          a.cell_dca[slot] = dca;
        }
      }
    }
    __syncwarp();
    int count = __popcll(masks[warp][lane]);
    if (big) {  // a crowded outer cluster: this lane evaluates its pairs in order
      count = 0;
      for (int b = 0; b < s.n_out; ++b) {
        const itsu_tracklet t2 = a.tracklets[s.j0 + b];
        float3 normal;
        float curvature;
        count += cell_precut(s.layer, s.t1_tan_lambda, s.t1_phi, t2.tan_lambda, t2.phi, s.c1, s.vz) &&
                 cell_geometry(s.layer, s.c1, s.c2, a.xyzr[s.c3_base + t2.second_cluster], s.vx, s.vy, normal, curvature);
      }
    }
    // the warp's 32 tracklets lie in one scan tile: their cells go to its sum (the cells scan
    // has no reduce pass)
    const int batch_cells = (int)__reduce_add_sync(0xffffffffu, (unsigned)count);
    if (lane == 0 && batch_cells != 0) {
      atomicAdd(reinterpret_cast<unsigned long long *>(&a.scan_partials[base / kScanTile]), (unsigned long long)batch_cells);
    }
    if (active) {
      a.cell_count[s.k] = count;
      a.cell_mask[s.k] = big ? 0ull : masks[warp][lane];
      a.cell_lookup[s.k] = ITSU_UNUSED_INDEX;  // the write pass fills it for tracklets with cells
      if (big && count > 0) {
        const unsigned long long q = atomicAdd(reinterpret_cast<unsigned long long *>(&a.status->crowded), 1ull);
        if ((int64_t)q < n) {
          a.cell_crowded[q] = (int32_t)s.k;
        }
      }
    }
    __syncwarp();
  }
  // the unused rest of the last chunk is marked empty
  for (int64_t i = chunk_pos + lane; i < chunk_end && i < a.cap_cell_entries; i += 32) {
    a.cell_entries[i].t1 = -1;
  }
}

// Learned prefilter: scores the count pass's cell entries, 32 per warp on the tensor cores, and
// drops those whose logit is below the model's threshold from their tracklet's mask and count
// before the scan. The score and the exact cuts are combined with AND, so scoring only the pairs
// that passed the cuts (whose geometry also gave the DCA feature) keeps the same cells as scoring
// every candidate first. A NaN logit keeps its cell. The pairs of a tracklet with more than
// kMaxMaskedOut outgoing tracklets are counted in order on one lane and are kept unscored.
constexpr int kPrefilterThreads = 256;

__global__ void __launch_bounds__(kPrefilterThreads) k_cells_prefilter(Arena a)
{
  __shared__ MlpSmem mlp;
  __shared__ __align__(16) __nv_bfloat16 rows[kPrefilterThreads / 32][32][kRowPitch];
  load_mlp(mlp, *a.mlp);
  __syncthreads();
  if (capacity_failed(a.status)) {
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t reserved = a.status->cell_entries;
  const int64_t n = reserved < a.cap_cell_entries ? reserved : a.cap_cell_entries;
  const int64_t tiles = (n + 31) / 32;
  for (int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; tile < tiles; tile += (int64_t)gridDim.x * (blockDim.x >> 5)) {
    const int64_t i = tile * 32 + lane;
    int4 h = make_int4(-1, 0, 0, 0);
    if (i < n) {
      h = reinterpret_cast<const int4 *>(a.cell_entries + i)[0];
    }
    float f[kMlpIn];
    if (h.x >= 0) {
      const int4 g = reinterpret_cast<const int4 *>(a.cell_entries + i)[1];  // c2, c3, t1 local, t2 local
      const int e = h.z / ITSU_CELL_LAYERS, layer = h.z % ITSU_CELL_LAYERS;
      const int32_t *lo = a.layer_off + e * ITSU_LAYERS;
      const itsu_tracklet t1 = a.tracklets[h.x];
      const itsu_tracklet t2 = a.tracklets[a.trk_seg[e * ITSU_TRACKLET_LAYERS + layer + 1] + g.w];
      const float4 c1 = a.xyzr[lo[layer] + h.w];
      const float4 c2 = a.xyzr[lo[layer + 1] + g.x];
      const float4 c3 = a.xyzr[lo[layer + 2] + g.y];
      pair_features(layer, t1.tan_lambda, t1.phi, t2.tan_lambda, t2.phi, c1, c2, c3, a.vtx[3 * e], a.vtx[3 * e + 1],
                    a.vtx[3 * e + 2], a.cell_dca[i], f);
    } else {
      for (int k = 0; k < kMlpIn; ++k) {
        f[k] = mlp.mean[k];
      }
    }
    feature_row(mlp.mean, mlp.inv_std, f, rows[warp][lane]);
    __syncwarp();
    const float logit = mlp_logits_warp<false>(mlp, rows[warp], nullptr);
    if (h.x >= 0 && logit < mlp.threshold) {
      atomicAnd(&a.cell_mask[h.x], ~(1ull << h.y));
      atomicSub(&a.cell_count[h.x], 1);
      atomicAdd(reinterpret_cast<unsigned long long *>(&a.scan_partials[h.x / kScanTile]), ~0ull);  // its tile sum - 1
    }
    __syncwarp();
  }
}

// Write pass, part 1: every cell entry whose bit survived goes to its scanned slot, in
// outgoing-tracklet order within its first tracklet (the rank of its bit in the mask).
__global__ void __launch_bounds__(kMaxThreads) k_cells_scatter(Arena a)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int64_t reserved = a.status->cell_entries;
  const int64_t n = reserved < a.cap_cell_entries ? reserved : a.cap_cell_entries;
  const int64_t stride = grid_threads();
  constexpr int kPer = 4;  // entries per thread per round, their loads in flight together
  for (int64_t i0 = global_thread(); i0 < n; i0 += kPer * stride) {
    int4 h[kPer], g[kPer], q[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int64_t i = i0 + u * stride;
      h[u] = make_int4(-1, 0, 0, 0);
      if (i < n) {
        const int4 *src = reinterpret_cast<const int4 *>(a.cell_entries + i);
        h[u] = src[0];  // t1, bit, segment, c1
        g[u] = src[1];  // c2, c3, t1 local, t2 local
        q[u] = src[2];  // normal, curvature
      }
    }
    unsigned long long m[kPer];
    int32_t off[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      if (h[u].x >= 0) {
        m[u] = a.cell_mask[h[u].x];
        off[u] = a.cell_off[h[u].x];
      }
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      if (h[u].x < 0 || !((m[u] >> h[u].y) & 1ull)) {
        continue;  // an unused slot, or a pair removed by the learned prefilter
      }
      const int32_t rank = __popcll(m[u] & ((1ull << h[u].y) - 1ull));
      const int32_t out = off[u] + rank;
      if (rank == 0 && h[u].z % ITSU_CELL_LAYERS >= 1) {  // the tracklet's first cell: its cells lookup entry
        a.cell_lookup[h[u].x] = out - a.cell_seg[h[u].z];
      }
      int2 *dst = reinterpret_cast<int2 *>(a.cells + out);
      dst[0] = make_int2(h[u].w, g[u].x);
      dst[1] = make_int2(g[u].y, g[u].z);
      dst[2] = make_int2(g[u].w, q[u].x);
      dst[3] = make_int2(q[u].y, q[u].z);
      dst[4] = make_int2(q[u].w, 1);
      a.cell_seg_id[out] = h[u].z;
    }
  }
}

// Write pass, part 2: the tracklets whose outer cluster was too crowded for the pair-parallel
// count (listed by the count pass; their mask is empty): their cells in order on one lane, and
// their cells lookup entry.
__global__ void __launch_bounds__(kMaxThreads) k_cells_crowded(Arena a)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int64_t n = a.status->total[kTracklets];
  const int64_t listed = min(a.status->crowded, n);
  for (int64_t q = global_thread(); q < listed; q += grid_threads()) {
    const int32_t k = a.cell_crowded[q];
    const CellLane s = cell_lane(a, k, n);
    const int32_t first = a.cell_off[k];
    if (s.layer >= 1 && s.layer < ITSU_CELL_LAYERS) {
      a.cell_lookup[k] = first - a.cell_seg[s.e * ITSU_CELL_LAYERS + s.layer];
    }
    int64_t out = first;
    for (int b = 0; b < s.n_out; ++b) {
      const int32_t j = s.j0 + b;
      const itsu_tracklet t2 = a.tracklets[j];
      float3 normal;
      float curvature;
      if (cell_precut(s.layer, s.t1_tan_lambda, s.t1_phi, t2.tan_lambda, t2.phi, s.c1, s.vz) &&
          cell_geometry(s.layer, s.c1, s.c2, a.xyzr[s.c3_base + t2.second_cluster], s.vx, s.vy, normal, curvature)) {
        write_cell(a, out++, s, t2, j, normal, curvature);
      }
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
// A cell's CA level and its number of level-decreasing chains down to layer 0, in one word
// (chains << 3 | level; levels are 1..5 and chain counts are capped at INT_MAX).
__device__ __forceinline__ int64_t chain_word(int64_t paths, int level) { return (paths << 3) | level; }
__device__ __forceinline__ int chain_level(int64_t w) { return (int)(w & 7); }
__device__ __forceinline__ int64_t chain_paths(int64_t w) { return w >> 3; }

__global__ void __launch_bounds__(kMaxThreads) k_neighbour_reset(Arena a)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int64_t n = a.status->total[kCells];
  for (int64_t c = global_thread(); c < n; c += grid_threads()) {
    a.nb_count[c] = 0;
    a.nb_fill[c] = 0;
    a.road_count[c] = 0;
    a.paths[c] = a.cell_seg_id[c] % ITSU_CELL_LAYERS == 0 ? chain_word(1, 1) : 0;  // layer 0: one chain, level 1
  }
}

// Tracker.cxx:416-474 (findCellsNeighbours): a cell of layer L and the cells of layer L + 1 built
// on its second tracklet. The count pass evaluates the cut, counts each passing pair in its row
// and keeps the passing candidates as a mask (rows of up to kMaxMaskedOut candidates); the write
// pass, after the scan of the counts, fills the rows from the mask (re-evaluating the cut only for
// cells with more candidates). Row order is restored by k_levels' sort.
template <bool kWrite>
__global__ void __launch_bounds__(kMaxThreads) k_neighbours(Arena a)
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
    const int32_t second = a.cells[c].second_tracklet;
    const int64_t ft = a.trk_seg[e * ITSU_TRACKLET_LAYERS + layer + 1] + second;
    const int32_t j0 = a.cell_off[ft], j1 = a.cell_off[ft + 1];
    const bool masked = j1 - j0 <= kMaxMaskedOut;
    if (kWrite && masked) {
      const int32_t c_local = (int32_t)(c - a.cell_seg[e * ITSU_CELL_LAYERS + layer]);
      for (unsigned long long m = a.nb_mask[c]; m; m &= m - 1ull) {
        const int32_t j = j0 + __ffsll((long long)m) - 1;
        const int slot = atomicAdd(&a.nb_fill[j], 1);
        a.nb[a.nb_off[j] + slot] = c_local;
      }
      continue;
    }
    const itsu_cell cell = a.cells[c];
    const float3 n1 = make_float3(cell.nx, cell.ny, cell.nz);
    const int32_t c_local = (int32_t)(c - a.cell_seg[e * ITSU_CELL_LAYERS + layer]);
    unsigned long long mask = 0ull;
    for (int32_t j = j0; j < j1; ++j) {
      const itsu_cell next = a.cells[j];
      if (neighbour_cut(layer, n1, cell.curvature, make_float3(next.nx, next.ny, next.nz), next.curvature)) {
        if (kWrite) {
          const int slot = atomicAdd(&a.nb_fill[j], 1);
          a.nb[a.nb_off[j] + slot] = c_local;
        } else {
          atomicAdd(&a.nb_count[j], 1);
          if (masked) {
            mask |= 1ull << (j - j0);
          }
        }
      }
    }
    if (!kWrite && masked) {
      a.nb_mask[c] = mask;
    }
  }
}

__global__ void k_neighbour_check(Arena a)
{
  if (global_thread() == 0 && !capacity_failed(a.status) && a.status->total[kNeighbours] > a.cap_neighbours) {
    atomicOr(&a.status->flags, kFlagCapNeighbours);
  }
}

// One cell of k_levels (below): its row sorted, its level and its number of chains (read from and
// written to the neighbours' chain words, one 8-byte gather per neighbour).
__device__ __forceinline__ void level_of(const Arena &a, int64_t c, int64_t prev_base, int layer)
{
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
  int level = 1;
  for (int p = 0; p < len; ++p) {
    level = max(level, chain_level(a.paths[prev_base + row[p]]) + 1);
  }
  int64_t paths = 0;
  bool overflow = false;
  for (int p = 0; p < len; ++p) {
    const int64_t w = a.paths[prev_base + row[p]];
    if (chain_level(w) == level - 1) {
      paths += chain_paths(w);
      if (paths > INT_MAX) {
        paths = INT_MAX;
        overflow = true;
      }
    }
  }
  a.cells[c].level = level;
  a.paths[c] = chain_word(paths, level);
  if (layer == ITSU_CELL_LAYERS - 1 && level == kCellsMinLevel) {
    a.road_count[c] = (int32_t)paths;
    if (overflow) {
      atomicOr(&a.status->flags, kFlagCountOverflow);
    }
  }
}

// Rows of layer `layer` cells: sort ascending (the reference pushes in cell order), then the
// level (Tracker.cxx:463-468: 1 + the highest neighbour level) and the number of
// level-decreasing chains down to layer 0 (the roads a level-5 cell starts, Tracker.cxx:477-571).
// The blocks of grid row y take the layer's cells of events y, y + gridDim.y, ... (each event's
// cells of a layer are one range).
__global__ void __launch_bounds__(kMaxThreads) k_levels(Arena a, int layer)
{
  if (capacity_failed(a.status)) {
    return;
  }
  for (int e = blockIdx.y; e < a.n_events; e += gridDim.y) {
    const int32_t *cs = a.cell_seg + e * ITSU_CELL_LAYERS;
    const int64_t prev_base = cs[layer - 1];
    for (int64_t c = cs[layer] + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cs[layer + 1];
         c += (int64_t)gridDim.x * blockDim.x) {
      level_of(a, c, prev_base, layer);
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

// A sorted cluster's MC id, from its 16-byte auxiliary record (the batch's 36-byte sorted records
// are twice the footprint, and the road vote's gathers hit L2 less often there).
__device__ __forceinline__ int32_t cluster_mc(const Arena &a, const int32_t *lo, int layer, int32_t idx)
{
  return a.clu_aux[lo[layer] + idx].z;
}

// One road per lane: the roads of a warp's 32 consecutive cells form one contiguous range (the
// scan of the roots' chain counts), which the lanes fill together, each lane taking the next road
// of the range, finding its root cell (owner) and its rank k among the root's roads. The traversal
// of Tracker.cxx:477-571 visits a cell's neighbours in row order and descends into those one level
// down, so the root's k-th road is found by walking down the layers: at each, skip the neighbours
// one level down whose whole subtrees (their chain counts, k_levels) lie before k, and descend into
// the one holding it. A complete chain is labelled by Moore's vote over its 7 clusters
// (Tracker.cxx:574-652) and stored with coalesced writes. The roots are the last layer's cells:
// the blocks of grid row y take those of events y, y + gridDim.y, ...
__global__ void __launch_bounds__(kMaxThreads) k_roads(Arena a)
{
  if (capacity_failed(a.status)) {
    return;
  }
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t warp = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (int e = blockIdx.y; e < a.n_events; e += gridDim.y) {
    const int32_t *cs = a.cell_seg + e * ITSU_CELL_LAYERS;
    const int32_t *lo = a.layer_off + e * ITSU_LAYERS;
    const int64_t n = cs[ITSU_CELL_LAYERS];  // the event's last cell + 1
    for (int64_t base = cs[ITSU_CELL_LAYERS - 1] + warp * 32; base < n; base += warps * 32) {
      const int64_t c = base + lane;
      int32_t first = 0, count = 0;
      if (c < n) {
        first = a.road_off[c];
        count = a.road_off[c + 1] - first;
      }
      int total = 0;
      const int excl = warp_exclusive_sum(count, total);
      if (total == 0) {
        continue;
      }
      const int64_t out0 = __shfl_sync(0xffffffffu, first, 0);
      for (int p0 = 0; p0 < total; p0 += 32) {
        const int p = p0 + lane;
        const int owner = owner_of(excl, p);
        int64_t k = p - __shfl_sync(0xffffffffu, excl, owner);
        if (p >= total) {
          continue;
        }
        int64_t flat = base + owner;
        int32_t cur[ITSU_CELL_LAYERS];  // local cell index per layer along the chain
        cur[ITSU_CELL_LAYERS - 1] = (int32_t)(flat - cs[ITSU_CELL_LAYERS - 1]);
        int level = kCellsMinLevel;
        bool found = true;
#pragma unroll
        for (int l = ITSU_CELL_LAYERS - 1; l >= 1; --l) {
          const int32_t j1 = a.nb_off[flat + 1];
          bool down = false;
          cur[l - 1] = 0;
          for (int32_t j = a.nb_off[flat]; j < j1; ++j) {
            const int32_t nb = a.nb[j];
            const int64_t nflat = cs[l - 1] + nb;
            const int64_t w = a.paths[nflat];
            if (chain_level(w) == level - 1) {
              const int64_t below = chain_paths(w);
              if (k < below) {
                cur[l - 1] = nb;
                flat = nflat;
                down = true;
                break;
              }
              k -= below;
            }
          }
          found = found && down;
          --level;
        }
        if (!found) {  // only when a chain count was capped (the count overflow flag is set)
          atomicOr(&a.status->flags, kFlagCountOverflow);
        }
        itsu_road road;
        int max_value = ITSU_UNUSED_INDEX, votes = 0;
        bool fake = false;
#pragma unroll
        for (int l = 0; l < ITSU_CELL_LAYERS; ++l) {
          road.cell_ids[l] = cur[l];
          const itsu_cell &cell = a.cells[cs[l] + cur[l]];
          if (l == 0) {
            max_value = cluster_mc(a, lo, 0, cell.first_cluster);
            votes = 1;
            const int second = cluster_mc(a, lo, 1, cell.second_cluster);
            if (second == max_value) {
              ++votes;
            } else {
              max_value = second;
              votes = 1;
              fake = true;
            }
          }
          const int current = cluster_mc(a, lo, l + 2, cell.third_cluster);
          if (current == max_value) {
            ++votes;
          } else {
            --votes;
            fake = true;
          }
          if (votes == 0) {
            max_value = current;
            votes = 1;
          }
        }
        road.size = ITSU_CELL_LAYERS;
        road.label = max_value;
        road.is_fake = fake ? 1 : 0;
        road.pad_[0] = road.pad_[1] = road.pad_[2] = 0;
        a.roads[out0 + p] = road;
      }
    }
  }
}

__global__ void k_atan2f(const float *y, const float *x, float *out, int64_t n)
{
  for (int64_t i = global_thread(); i < n; i += grid_threads()) {
    out[i] = itsu_atan2f(y[i], x[i]);
  }
}

// Grid of the grid-stride kernels: the tuned number of resident blocks per SM, scaled to the
// block size so that the number of resident threads stays comparable.
int fixed_grid(const Launch &l) { return l.num_sms * l.blocks_per_sm; }

// Grid of the per-event kernels (a row of blocks per event, events beyond 65535 rows taken in
// turn): about the same blocks in all as the grid-stride kernels.
dim3 event_grid(const Arena &a, const Launch &l)
{
  const int rows = std::min(a.n_events, 65535);
  return dim3((unsigned)std::max(1, (fixed_grid(l) + rows - 1) / rows), (unsigned)rows);
}

void step_status_init(const Arena &a, const Launch &l)
{
  const int64_t tiles = (a.n_clusters + kScanTile - 1) / kScanTile;
  const int64_t blocks = a.scan_partials ? std::min<int64_t>((tiles + kThreads - 1) / kThreads, l.num_sms) : 0;
  k_status_init<<<(unsigned)std::max<int64_t>(blocks, 1), kThreads, 0, l.stream>>>(a);
}

void step_cluster_sort(const Arena &a, const Launch &l)
{
  if (a.n_events > 0) {
    k_cluster_sort<<<a.n_events * ITSU_LAYERS, kSortThreads, 0, l.stream>>>(a);
  }
}

// The per-item count passes need whole warps: each warp adds its items' total to one scan tile.
bool whole_warps(const Arena &a, const Launch &l)
{
  if (l.block % 32 == 0) {
    return true;
  }
  k_flag_bad_launch<<<1, 1, 0, l.stream>>>(a.status);
  return false;
}

void step_tracklets_count(const Arena &a, const Launch &l)
{
  if (!whole_warps(a, l)) {
    return;
  }
  const int64_t blocks = (a.n_clusters + l.block - 1) / l.block;
  if (blocks <= 0) {
    return;
  }
  const size_t stage_bytes = kStageEntries * sizeof(float4);
  // the count pass takes at most kCountThreads threads per block (any whole warps give the same
  // results)
  const int block = std::min(l.block, kCountThreads);
  const unsigned grid = (unsigned)((a.n_clusters + block - 1) / block);
  if (a.prune_tracklets == 2) {  // the staged walk (tuning knob; results are identical)
    if (a.gate) {
      k_tracklets_count<true, true><<<grid, block, stage_bytes, l.stream>>>(a);
    } else {
      k_tracklets_count<true, false><<<grid, block, stage_bytes, l.stream>>>(a);
    }
  } else if (a.gate) {
    k_tracklets_count<false, true><<<grid, block, 0, l.stream>>>(a);
  } else {
    k_tracklets_count<false, false><<<grid, block, 0, l.stream>>>(a);
  }
}

// Launches only in the learned form with the tracklet gate (a.gate set).
void step_tracklets_gate(const Arena &a, const Launch &l)
{
  if (a.gate && a.n_clusters > 0 && a.n_events > 0) {
    const int rows = std::min(a.n_events, 65535);
    const int per_event = std::max(1, (l.num_sms * 8 + rows - 1) / rows);
    k_tracklets_gate<<<dim3((unsigned)per_event, (unsigned)rows), kGateThreads, 0, l.stream>>>(a);
  }
}

void launch_write_range(const Arena &a, const Launch &l, int64_t c0, int64_t c1)
{
  const int64_t blocks = (c1 - c0 + l.block - 1) / l.block;
  if (blocks > 0) {
    k_tracklets_write<<<(unsigned)blocks, l.block, 0, l.stream>>>(a, c0, c1);
  }
}

// The write and cell count passes over all events at once (launches with no event groups).
void step_tracklets_write(const Arena &a, const Launch &l)
{
  if (l.n_groups == 0) {
    launch_write_range(a, l, 0, a.n_clusters);
  }
}

void step_tracklets_crowded(const Arena &a, const Launch &l)
{
  if (a.gate) {
    k_tracklets_crowded<true><<<l.num_sms, 128, 0, l.stream>>>(a);
  } else {
    k_tracklets_crowded<false><<<l.num_sms, 128, 0, l.stream>>>(a);
  }
}

void step_tracklet_segments(const Arena &a, const Launch &l)
{
  k_tracklet_segments<<<(a.n_events * ITSU_TRACKLET_LAYERS + kThreads) / kThreads, kThreads, 0, l.stream>>>(a);
}

void step_cells_count(const Arena &a, const Launch &l)
{
  if (l.n_groups == 0 && whole_warps(a, l)) {
    k_cells_count<<<fixed_grid(l), l.block, 0, l.stream>>>(a, 0, 0);
  }
}

// Event groups: the write pass of a group's inner clusters, then the cell count pass of its
// tracklets, group after group, so that the tracklets a group's count pass gathers were written
// moments before and are still in L2. Group g's clusters are [groups[g], groups[g + 1]) (multiples
// of 32 up to the last), its events [g * group_events, (g + 1) * group_events).
void step_write_count_groups(const Arena &a, const Launch &l)
{
  if (l.n_groups == 0 || !whole_warps(a, l)) {
    return;
  }
  for (int g = 0; g < l.n_groups; ++g) {
    launch_write_range(a, l, l.groups[g], l.groups[g + 1]);
    const int32_t e0 = g * l.group_events, e1 = std::min(a.n_events, (g + 1) * l.group_events);
    k_cells_count<<<fixed_grid(l), l.block, 0, l.stream>>>(a, e0, e1);
  }
}

// Launches only in the learned form (a.mlp set).
void step_cells_prefilter(const Arena &a, const Launch &l)
{
  if (a.mlp) {
    k_cells_prefilter<<<l.num_sms * 3, kPrefilterThreads, 0, l.stream>>>(a);  // one wave (3 blocks per SM by registers)
  }
}

void step_cells_scatter(const Arena &a, const Launch &l) { k_cells_scatter<<<fixed_grid(l), l.block, 0, l.stream>>>(a); }

void step_cells_crowded(const Arena &a, const Launch &l) { k_cells_crowded<<<l.num_sms, 128, 0, l.stream>>>(a); }

void step_cell_segments(const Arena &a, const Launch &l)
{
  k_cell_segments<<<(a.n_events * ITSU_CELL_LAYERS + kThreads) / kThreads, kThreads, 0, l.stream>>>(a);
}

void step_neighbour_reset(const Arena &a, const Launch &l) { k_neighbour_reset<<<fixed_grid(l), l.block, 0, l.stream>>>(a); }

template <bool kWrite>
void step_neighbours(const Arena &a, const Launch &l) { k_neighbours<kWrite><<<fixed_grid(l), l.block, 0, l.stream>>>(a); }

void step_neighbour_check(const Arena &a, const Launch &l) { k_neighbour_check<<<1, 32, 0, l.stream>>>(a); }

template <int kLayer>
void step_levels(const Arena &a, const Launch &l)
{
  if (a.n_events > 0) {
    k_levels<<<event_grid(a, l), l.block, 0, l.stream>>>(a, kLayer);
  }
}

void step_road_segments(const Arena &a, const Launch &l)
{
  k_road_segments<<<(a.n_events + kThreads) / kThreads, kThreads, 0, l.stream>>>(a);
}

void step_roads(const Arena &a, const Launch &l)
{
  if (a.n_events > 0) {
    k_roads<<<event_grid(a, l), l.block, 0, l.stream>>>(a);
  }
}

// The whole run, kernel by kernel, in launch order.
const KernelStep kSteps[] = {
    {"status_init", step_status_init, 0},                    // 0
    {"cluster_sort", step_cluster_sort, 0},                  // 1  (a)
    {"tracklets_count", step_tracklets_count, 0},            // 2  (b)
    {"tracklets_gate", step_tracklets_gate, kGateStep},      // 3  (learned form with the gate)
    {"scan_partials_tracklets", step_scan_partials<0>, 0},   // 4
    {"scan_apply_tracklets", step_scan_apply<0>, 0},         // 5
    {"tracklet_segments", step_tracklet_segments, 0},        // 6
    {"tracklets_crowded", step_tracklets_crowded, 0},        // 7
    {"tracklets_write", step_tracklets_write, kUngroupedStep},  // 8
    {"cells_count", step_cells_count, kUngroupedStep},       // 9  (c)
    {"write_count_by_event_group", step_write_count_groups, kGroupedStep},  // 10 (tracklet write + cell count per group)
    {"cells_prefilter", step_cells_prefilter, kPairPrefilterStep},  // 11 (learned form with the pair prefilter)
    {"scan_partials_cells", step_scan_partials<1>, 0},       // 12
    {"scan_apply_cells", step_scan_apply<1>, 0},             // 13
    {"cell_segments", step_cell_segments, 0},                // 14
    {"cells_scatter", step_cells_scatter, 0},                // 15
    {"cells_crowded", step_cells_crowded, 0},                // 16
    {"neighbour_reset", step_neighbour_reset, 0},            // 17 (d)
    {"neighbours_count", step_neighbours<false>, 0},         // 18
    {"scan_reduce_neighbours", step_scan_reduce<2>, 0},      // 19
    {"scan_partials_neighbours", step_scan_partials<2>, 0},  // 20
    {"scan_apply_neighbours", step_scan_apply<2>, 0},        // 21
    {"neighbour_check", step_neighbour_check, 0},            // 22
    {"neighbours_write", step_neighbours<true>, 0},          // 23
    {"levels_1", step_levels<1>, 0},                         // 24
    {"levels_2", step_levels<2>, 0},                         // 25
    {"levels_3", step_levels<3>, 0},                         // 26
    {"levels_4", step_levels<4>, 0},                         // 27
    {"scan_reduce_roads", step_scan_reduce<3>, 0},           // 28 (e)
    {"scan_partials_roads", step_scan_partials<3>, 0},       // 29
    {"scan_apply_roads", step_scan_apply<3>, 0},             // 30
    {"road_segments", step_road_segments, 0},                // 31
    {"roads_write", step_roads, 0},                          // 32
};
constexpr int kNumSteps = sizeof(kSteps) / sizeof(kSteps[0]);

void run_steps(int first, int last, const Arena &a, const Launch &l)
{
  for (int k = first; k <= last; ++k) {
    kSteps[k].launch(a, l);
  }
}

}  // namespace

// Streamed host runs: appends the last run's roads and road offsets to the batch-wide output at
// event e0. The chunk's first road index is dst_off[e0], written by the previous chunk (or zeroed
// by the host); a chunk that overflowed or does not fit leaves its roads out and passes its base
// on, so the next chunk stays in bounds. The run's status goes to *snap for the host.
__global__ void k_append_roads(Arena a, itsu_road *dst, int32_t *dst_off, int32_t e0, int64_t cap, DevStatus *snap)
{
  const bool ok = !capacity_failed(a.status);
  int64_t base = dst_off[e0];
  base = base < 0 ? 0 : base;
  const int64_t total = ok ? a.status->total[kRoads] : 0;
  const bool fits = base + total <= cap;
  const int64_t tid = global_thread(), threads = grid_threads();
  if (ok && fits) {
    for (int64_t r = tid; r < total; r += threads) {
      dst[base + r] = a.roads[r];
    }
    for (int64_t e = tid + 1; e <= a.n_events; e += threads) {
      dst_off[e0 + e] = (int32_t)(base + a.road_seg[e]);
    }
  } else {
    for (int64_t e = tid + 1; e <= a.n_events; e += threads) {
      dst_off[e0 + e] = (int32_t)base;
    }
  }
  if (tid == 0) {
    DevStatus st = *a.status;
    if (ok && !fits) {
      st.flags |= kFlagCapRoads;
    }
    *snap = st;
  }
}

void launch_append_roads(const Arena &a, const Launch &l, itsu_road *dst, int32_t *dst_off, int32_t e0, int64_t cap, DevStatus *snap)
{
  k_append_roads<<<l.num_sms * 2, 256, 0, l.stream>>>(a, dst, dst_off, e0, cap, snap);
}

const KernelStep *pipeline_steps(int *count)
{
  *count = kNumSteps;
  return kSteps;
}

void launch_status_init(const Arena &a, const Launch &l) { run_steps(0, 0, a, l); }
void launch_cluster_sort(const Arena &a, const Launch &l) { run_steps(1, 1, a, l); }
void launch_tracklets_count(const Arena &a, const Launch &l) { run_steps(2, 6, a, l); }

void launch_atan2f(const float *y, const float *x, float *out, int64_t n, int num_sms, cudaStream_t stream)
{
  if (n > 0) {
    k_atan2f<<<num_sms * 4, 256, 0, stream>>>(y, x, out, n);
  }
}
void launch_tracklets_write(const Arena &a, const Launch &l) { run_steps(7, 8, a, l); }
void launch_cells_count(const Arena &a, const Launch &l) { run_steps(9, 14, a, l); }
void launch_cells_write(const Arena &a, const Launch &l) { run_steps(15, 16, a, l); }
void launch_neighbours_count(const Arena &a, const Launch &l) { run_steps(17, 22, a, l); }
void launch_neighbours_write(const Arena &a, const Launch &l) { run_steps(23, 27, a, l); }
void launch_roads_count(const Arena &a, const Launch &l) { run_steps(28, 31, a, l); }
void launch_roads_write(const Arena &a, const Launch &l) { run_steps(32, 32, a, l); }

int kernels_per_run()
{
  int n = 0;
  for (const KernelStep &k : kSteps) {
    n += (k.learned_only == 0 || k.learned_only == kUngroupedStep) ? 1 : 0;
  }
  return n;
}

}  // namespace itsu
