// itsu_capi.cu - C ABI of the track finder: context, device arena, stage orchestration.
//
// The per-vertex entry points mirror the reference's seam (PrimaryVertexContext::initialize,
// TrackerTraits::computeLayerTracklets / computeLayerCells, Tracker::findCellsNeighbours /
// findTracks / computeMontecarloLabels) and are synchronous like the reference GPU backend
// (src/CA/gpu/cuda/Tracker.cu synchronises after every stage). Each stage counts, scans, and
// sizes its outputs exactly before writing them (two-pass sizing). The whole-path and batch
// entry points enqueue every stage back to back without host round trips (replayed as a CUDA
// graph), then check the device status once; an output that overflowed the arena is grown to the
// reported requirement and the run repeated.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <type_traits>
#include <vector>

#include "itsu.h"
#include "itsu_internal.h"
#include "itsu_mlp.cuh"

using itsu::Arena;
using itsu::DevStatus;
using itsu::Launch;

namespace {

thread_local std::string g_thread_error;

enum Stage { kNone = 0, kInitialized, kTracklets, kCells, kNeighbours, kRoads };

}  // namespace

void itsu::set_thread_error(const char *message) { g_thread_error = message; }

namespace {
// Launch shape of a run; tuned per multiplicity band (itsu_autotune).
struct Tune {
  int block = 256;
  int blocks_per_sm = 8;
  int prune = 1;
  float ms = 0.0f;
  bool set = false;
  int group = 0;  // events per group of the interleaved tracklet write / cell count passes (0: no groups)
};
constexpr int kBands = 32;

// Band of a run: log2 of its mean cluster count per event.
int band_of(int64_t n_clusters, int32_t n_events)
{
  const int64_t mean = n_clusters / (n_events > 0 ? n_events : 1);
  int band = 0;
  while (band + 1 < kBands && (int64_t(1) << (band + 1)) <= mean) {
    ++band;
  }
  return band;
}
}  // namespace

struct itsu_context {
  int device = 0;
  uint32_t flags = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;

  // capacities
  int64_t cap_clusters = 0;
  int32_t cap_events = 0;
  int64_t cap_tracklets = 0, cap_cells = 0, cap_neighbours = 0, cap_roads = 0, cap_partials = 0;
  int64_t init_tracklets = 0, init_cells = 0, init_neighbours = 0, init_roads = 0;

  // device buffers: cluster class
  itsu_cluster *raw = nullptr, *sorted = nullptr, *tmp = nullptr;
  float4 *xyzr = nullptr;
  float *phi = nullptr;
  int32_t *trk_count = nullptr, *trk_off = nullptr, *trk_lookup = nullptr;
  float4 *zs = nullptr;
  int32_t *clu_seg = nullptr;
  int4 *clu_aux = nullptr;
  int32_t *clu_crowded = nullptr;
  int32_t *trk_slots = nullptr;
  // event class
  float2 *seg_rrange = nullptr;
  int32_t *seg_regular = nullptr;
  int32_t *layer_off = nullptr, *index_tables = nullptr, *trk_seg = nullptr, *cell_seg = nullptr, *road_seg = nullptr;
  int4 *cell_seginfo = nullptr;
  float *vtx = nullptr;
  // tracklet class
  itsu_tracklet *tracklets = nullptr;
  float2 *trk_slope = nullptr;  // (tanL, phi) of each tracklet, beside the records
  int32_t *trk_seg_id = nullptr, *cell_count = nullptr, *cell_off = nullptr, *cell_lookup = nullptr, *cell_crowded = nullptr;
  unsigned long long *cell_mask = nullptr;
  // cell class
  itsu_cell *cells = nullptr;
  itsu::CellEntry *cell_entries = nullptr;
  float *cell_dca = nullptr;
  int64_t cap_cell_entries = 0;
  int32_t *cell_seg_id = nullptr, *nb_count = nullptr, *nb_off = nullptr, *nb_fill = nullptr, *road_count = nullptr,
          *road_off = nullptr;
  int64_t *paths = nullptr;
  unsigned long long *nb_mask = nullptr;  // per cell, its passing candidates (neighbour count pass)
  // neighbour and road classes
  int32_t *nb = nullptr;
  itsu_road *roads = nullptr;
  int64_t *scan_partials = nullptr;
  DevStatus *d_status = nullptr;
  DevStatus *h_status = nullptr;

  // current run
  int32_t n_events = 0;
  int64_t n_clusters = 0;
  std::vector<int32_t> h_layer_off;
  std::vector<int64_t> group_bounds;  // event groups of the current whole run (whole_run_launch)
  const itsu_cluster *in_raw = nullptr;
  const itsu_cluster_in *in_raw_in = nullptr;  // the 24-byte input records instead of in_raw (compact host calls)
  itsu_cluster_in *raw_in = nullptr;           // their device copy
  int64_t cap_raw_in = 0;
  const itsu_cluster_track *in_raw_track = nullptr;  // the 16-byte input records instead (track host calls)
  itsu_cluster_track *raw_track = nullptr;            // their device copy
  int64_t cap_raw_track = 0;
  const int32_t *in_raw_off = nullptr;
  const int32_t *in_layer_off = nullptr;
  int32_t *raw_off = nullptr;  // arena copy of a frames run's raw offsets (event class)
  const float *in_vtx = nullptr;
  int stage = kNone;

  // CUDA graph of the whole batch sequence
  cudaGraphExec_t graph = nullptr;
  uint64_t graph_generation = 0;
  uint64_t generation = 1;  // bumped whenever a buffer is reallocated
  const void *graph_key[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int32_t graph_events = -1;
  int64_t graph_clusters = -1;

  // launch shapes per multiplicity band, and the candidate under test while tuning
  Tune tunes[kBands];
  Tune override_tune;
  bool tuning = false;
  int graph_tune[4] = {0, 0, -1, -1};
  bool graph_prefilter = false;
  bool graph_gate = false;

  // streamed host runs (ITSU_FLAG_STREAM_HOST): upload stream, per-chunk events, batch-wide roads
  cudaStream_t copy_stream = nullptr;   // uploads
  cudaStream_t d2h_stream = nullptr;    // road downloads
  cudaEvent_t chunk_ready[16] = {};     // a chunk's upload is done ([15]: the call's start)
  cudaEvent_t chunk_done[16] = {};      // a chunk's roads, road end and status are on the host side
  int32_t *h_road_end = nullptr;        // pinned: each chunk's end in the batch-wide roads
  int32_t *chunk_off = nullptr;   // each chunk's layer offsets, rebased to the chunk
  int64_t cap_chunk_off = 0;
  int32_t *h_chunk_off = nullptr;  // pinned staging of chunk_off
  int64_t cap_h_chunk_off = 0;
  int64_t chunk_clusters = 0;
  itsu_road *roads_all = nullptr;
  int64_t cap_roads_all = 0;
  int32_t *road_off_all = nullptr;
  int64_t cap_road_off_all = 0;
  DevStatus *chunk_status = nullptr;  // 16 snapshots
  DevStatus *h_chunk_status = nullptr;

  // streamed host runs: a second arena with its own stream, created on first use, so that two
  // chunks are in flight (one's small tail kernels overlapping the next one's work)
  itsu_context *twin = nullptr;

  // learned prefilter: FP32 master model and the device model the kernels read
  itsu_prefilter_model *d_master = nullptr;
  itsu::MlpDevice *d_mlp = nullptr;
  bool has_model = false;
  // learned tracklet gate: its FP32 master and device model, and whether the learned form uses it
  itsu_gate_model *d_gate_master = nullptr;
  itsu::GateDevice *d_gate = nullptr;
  bool has_gate = false;
  bool gate = false;
  bool prefilter = false;

  // road report scratch (itsu_roads_report)
  unsigned char *report_scratch = nullptr;
  int64_t cap_report_scratch = 0;

  // device bytes of the arena's buffers (alloc), for itsu_memory_usage
  std::unordered_map<const void *, size_t> arena_sizes;
  int64_t arena_bytes = 0;

  std::string error;
};

namespace {

itsu_status fail(itsu_context *ctx, itsu_status st, const char *fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (ctx) {
    ctx->error = buf;
  }
  g_thread_error = buf;
  return st;
}

#define ITSU_CUDA(ctx, call)                                                                                   \
  do {                                                                                                         \
    cudaError_t err_ = (call);                                                                                 \
    if (err_ != cudaSuccess) {                                                                                 \
      return fail((ctx), err_ == cudaErrorMemoryAllocation ? ITSU_ERR_NOMEM : ITSU_ERR_CUDA, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(err_), __FILE__, __LINE__);                                        \
    }                                                                                                          \
  } while (0)

template <typename T>
void release(T *&p)
{
  if (p) {
    cudaFree((void *)p);
    p = nullptr;
  }
}

// Arena allocation: replaces p by a buffer of count elements and keeps the context's byte count.
template <typename T>
cudaError_t alloc(itsu_context *ctx, T *&p, int64_t count)
{
  if (p) {
    auto it = ctx->arena_sizes.find((const void *)p);
    if (it != ctx->arena_sizes.end()) {
      ctx->arena_bytes -= (int64_t)it->second;
      ctx->arena_sizes.erase(it);
    }
  }
  release(p);
  const size_t bytes = (size_t)std::max<int64_t>(count, 1) * sizeof(T);
  const cudaError_t err = cudaMalloc((void **)&p, bytes);
  if (err == cudaSuccess) {
    ctx->arena_sizes[(const void *)p] = bytes;
    ctx->arena_bytes += (int64_t)bytes;
  }
  return err;
}

Tune current_tune(const itsu_context *ctx)
{
  if (ctx->tuning) {
    return ctx->override_tune;
  }
  const Tune &t = ctx->tunes[band_of(ctx->n_clusters, ctx->n_events)];
  return t.set ? t : Tune{};
}

Launch launch_of(const itsu_context *ctx)
{
  const Tune t = current_tune(ctx);
  Launch l{};
  l.stream = ctx->stream;
  l.num_sms = ctx->num_sms;
  l.block = t.block;
  l.blocks_per_sm = t.blocks_per_sm;
  return l;
}

// Event groups of a run of n_events events with host layer offsets off[n_events * 7 + 1]: group g
// holds events [g * group, (g + 1) * group) and, for the write pass, the inner clusters from the
// first multiple of 32 at or after its first cluster (the previous group's write covers the few
// before it, which only makes their tracklets exist sooner). No groups for one group or fewer.
void group_bounds(const int32_t *off, int32_t n_events, int64_t n_clusters, int group, std::vector<int64_t> &out)
{
  out.clear();
  if (group <= 0 || n_events <= group) return;
  const int n_groups = (n_events + group - 1) / group;
  out.push_back(0);
  for (int g = 1; g < n_groups; ++g) {
    const int64_t first = off[(int64_t)g * group * ITSU_LAYERS] - off[0];
    out.push_back(std::min<int64_t>((first + 31) & ~int64_t(31), n_clusters));
  }
  out.push_back(n_clusters);
}

void attach_groups(Launch &l, const std::vector<int64_t> &bounds, int group)
{
  l.n_groups = bounds.empty() ? 0 : (int)bounds.size() - 1;
  l.group_events = group;
  l.groups = bounds.empty() ? nullptr : bounds.data();
}

// The launch shape of a whole run of the context's current inputs, with its event groups.
Launch whole_run_launch(itsu_context *ctx)
{
  Launch l = launch_of(ctx);
  const int group = current_tune(ctx).group;
  if (group > 0 && (int64_t)ctx->h_layer_off.size() == (int64_t)ctx->n_events * ITSU_LAYERS + 1) {
    group_bounds(ctx->h_layer_off.data(), ctx->n_events, ctx->n_clusters, group, ctx->group_bounds);
  } else {
    ctx->group_bounds.clear();
  }
  attach_groups(l, ctx->group_bounds, group);
  return l;
}

Arena arena_of(const itsu_context *ctx)
{
  Arena a{};
  a.n_events = ctx->n_events;
  a.n_clusters = ctx->n_clusters;
  a.raw = ctx->in_raw;
  a.raw_in = ctx->in_raw_in;
  a.raw_track = ctx->in_raw_track;
  a.raw_off = ctx->in_raw_off;
  a.layer_off = ctx->in_layer_off;
  a.vtx = ctx->in_vtx;
  a.sorted = ctx->sorted;
  a.xyzr = ctx->xyzr;
  a.phi = ctx->phi;
  a.tmp = ctx->tmp;
  a.index_tables = ctx->index_tables;
  a.zs = ctx->zs;
  a.clu_seg = ctx->clu_seg;
  a.clu_aux = ctx->clu_aux;
  a.clu_crowded = ctx->clu_crowded;
  a.seg_rrange = ctx->seg_rrange;
  a.seg_regular = ctx->seg_regular;
  a.prune_tracklets = current_tune(ctx).prune;
  a.trk_count = ctx->trk_count;
  a.trk_slots = ctx->trk_slots;
  a.slot_stride = ctx->cap_clusters;
  a.trk_off = ctx->trk_off;
  a.trk_lookup = ctx->trk_lookup;
  a.trk_seg = ctx->trk_seg;
  a.cell_seginfo = ctx->cell_seginfo;
  a.tracklets = ctx->tracklets;
  a.trk_slope = ctx->trk_slope;
  a.trk_seg_id = ctx->trk_seg_id;
  a.cell_count = ctx->cell_count;
  a.cell_mask = ctx->cell_mask;
  a.cell_off = ctx->cell_off;
  a.cell_lookup = ctx->cell_lookup;
  a.cell_crowded = ctx->cell_crowded;
  a.cell_seg = ctx->cell_seg;
  a.cells = ctx->cells;
  a.cell_seg_id = ctx->cell_seg_id;
  a.cell_entries = ctx->cell_entries;
  a.cell_dca = ctx->cell_dca;
  a.cap_cell_entries = ctx->cap_cell_entries;
  a.nb_count = ctx->nb_count;
  a.nb_off = ctx->nb_off;
  a.nb_fill = ctx->nb_fill;
  a.nb_mask = ctx->nb_mask;
  a.nb = ctx->nb;
  a.paths = ctx->paths;
  a.road_count = ctx->road_count;
  a.road_off = ctx->road_off;
  a.road_seg = ctx->road_seg;
  a.roads = ctx->roads;
  a.mlp = ctx->prefilter ? ctx->d_mlp : nullptr;
  a.gate = ctx->gate ? ctx->d_gate : nullptr;
  a.scan_partials = ctx->scan_partials;
  a.status = ctx->d_status;
  a.cap_tracklets = ctx->cap_tracklets;
  a.cap_cells = ctx->cap_cells;
  a.cap_neighbours = ctx->cap_neighbours;
  a.cap_roads = ctx->cap_roads;
  return a;
}

int64_t grow_to(int64_t need) { return need + need / 4 + 1024; }

// With ITSU_FLAG_NO_GROW the arena keeps the capacities the context was created with.
itsu_status growth_allowed(itsu_context *ctx, const char *what, int64_t need, int64_t cap)
{
  if ((ctx->flags & ITSU_FLAG_NO_GROW) && ctx->stage != -1) {
    return fail(ctx, ITSU_ERR_CAPACITY, "%s: %lld needed, arena holds %lld (ITSU_FLAG_NO_GROW)", what, (long long)need,
                (long long)cap);
  }
  return ITSU_OK;
}

itsu_status ensure_partials(itsu_context *ctx)
{
  const int64_t need = std::max({ctx->cap_clusters, ctx->cap_tracklets, ctx->cap_cells}) / 2048 + 2;
  if (need > ctx->cap_partials) {
    ITSU_CUDA(ctx, alloc(ctx, ctx->scan_partials, need));
    ctx->cap_partials = need;
    ctx->generation++;
  }
  return ITSU_OK;
}

itsu_status ensure_clusters(itsu_context *ctx, int64_t n_clusters, int32_t n_events)
{
  if (n_clusters > ctx->cap_clusters) {
    itsu_status st = growth_allowed(ctx, "clusters", n_clusters, ctx->cap_clusters);
    if (st != ITSU_OK) return st;
    const int64_t cap = grow_to(n_clusters);
    ITSU_CUDA(ctx, alloc(ctx, ctx->raw, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->sorted, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->tmp, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->xyzr, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->phi, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->trk_count, cap + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->trk_off, cap + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->trk_lookup, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->zs, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->clu_seg, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->clu_aux, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->clu_crowded, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->trk_slots, cap * itsu::kTrackletSlotsPerCluster));
    ctx->cap_clusters = cap;
    ctx->generation++;
  }
  if (n_events > ctx->cap_events) {
    itsu_status st = growth_allowed(ctx, "events", n_events, ctx->cap_events);
    if (st != ITSU_OK) return st;
    const int32_t cap = n_events + n_events / 4 + 4;
    ITSU_CUDA(ctx, alloc(ctx, ctx->layer_off, (int64_t)cap * ITSU_LAYERS + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->vtx, (int64_t)cap * 3));
    ITSU_CUDA(ctx, alloc(ctx, ctx->index_tables, (int64_t)cap * ITSU_TRACKLET_LAYERS * ITSU_INDEX_TABLE_SIZE));
    ITSU_CUDA(ctx, alloc(ctx, ctx->trk_seg, (int64_t)cap * ITSU_TRACKLET_LAYERS + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->cell_seginfo, (int64_t)cap * ITSU_TRACKLET_LAYERS * 2));
    ITSU_CUDA(ctx, alloc(ctx, ctx->cell_seg, (int64_t)cap * ITSU_CELL_LAYERS + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->road_seg, (int64_t)cap + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->seg_rrange, (int64_t)cap * ITSU_LAYERS));
    ITSU_CUDA(ctx, alloc(ctx, ctx->seg_regular, (int64_t)cap * ITSU_LAYERS));
    ITSU_CUDA(ctx, alloc(ctx, ctx->raw_off, (int64_t)cap * ITSU_LAYERS));
    ctx->cap_events = cap;
    ctx->generation++;
  }
  return ensure_partials(ctx);
}

itsu_status ensure_tracklets(itsu_context *ctx, int64_t need)
{
  if (need > ctx->cap_tracklets) {
    itsu_status st = growth_allowed(ctx, "tracklets", need, ctx->cap_tracklets);
    if (st != ITSU_OK) return st;
    const int64_t cap = grow_to(need);
    ITSU_CUDA(ctx, alloc(ctx, ctx->tracklets, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->trk_slope, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->trk_seg_id, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->cell_count, cap + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->cell_mask, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->cell_off, cap + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->cell_lookup, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->cell_crowded, cap));
    ctx->cap_tracklets = cap;
    ctx->generation++;
  }
  return ensure_partials(ctx);
}

// Entries the cell count pass may reserve beyond the cells it finds: every warp of its grid can
// leave part of one chunk unused. Sized for the larger of the current launch shape and the
// largest shape the autotuner tries (16 blocks of 512 threads per SM).
int64_t cell_entry_slack(const itsu_context *ctx)
{
  const Tune t = current_tune(ctx);
  const int64_t warps = std::max<int64_t>((int64_t)t.blocks_per_sm * (t.block / 32), 16 * (512 / 32));
  return (int64_t)ctx->num_sms * warps * itsu::kCellChunk;
}

itsu_status ensure_cell_entries(itsu_context *ctx, int64_t need)
{
  if (need > ctx->cap_cell_entries) {
    itsu_status st = growth_allowed(ctx, "cell entries", need, ctx->cap_cell_entries);
    if (st != ITSU_OK) return st;
    const int64_t cap = grow_to(need);
    ITSU_CUDA(ctx, alloc(ctx, ctx->cell_entries, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->cell_dca, cap));
    ctx->cap_cell_entries = cap;
    ctx->generation++;
  }
  return ITSU_OK;
}

itsu_status ensure_cells(itsu_context *ctx, int64_t need)
{
  if (need > ctx->cap_cells) {
    itsu_status st = growth_allowed(ctx, "cells", need, ctx->cap_cells);
    if (st != ITSU_OK) return st;
    const int64_t cap = grow_to(need);
    ITSU_CUDA(ctx, alloc(ctx, ctx->cells, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->cell_seg_id, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->nb_count, cap + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->nb_off, cap + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->nb_fill, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->nb_mask, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->paths, cap));
    ITSU_CUDA(ctx, alloc(ctx, ctx->road_count, cap + 1));
    ITSU_CUDA(ctx, alloc(ctx, ctx->road_off, cap + 1));
    ctx->cap_cells = cap;
    ctx->generation++;
  }
  itsu_status st = ensure_cell_entries(ctx, ctx->cap_cells + cell_entry_slack(ctx));
  if (st != ITSU_OK) return st;
  return ensure_partials(ctx);
}

itsu_status ensure_neighbours(itsu_context *ctx, int64_t need)
{
  if (need > ctx->cap_neighbours) {
    itsu_status st = growth_allowed(ctx, "neighbours", need, ctx->cap_neighbours);
    if (st != ITSU_OK) return st;
    const int64_t cap = grow_to(need);
    ITSU_CUDA(ctx, alloc(ctx, ctx->nb, cap));
    ctx->cap_neighbours = cap;
    ctx->generation++;
  }
  return ITSU_OK;
}

itsu_status ensure_roads(itsu_context *ctx, int64_t need)
{
  if (need > ctx->cap_roads) {
    itsu_status st = growth_allowed(ctx, "roads", need, ctx->cap_roads);
    if (st != ITSU_OK) return st;
    const int64_t cap = grow_to(need);
    ITSU_CUDA(ctx, alloc(ctx, ctx->roads, cap));
    ctx->cap_roads = cap;
    ctx->generation++;
  }
  return ITSU_OK;
}

// Initial output capacities for a run of n_clusters clusters (Pb-Pb-like events produce about
// 8 tracklets, 1 cell and 0.2 roads per cluster; the arena grows past these when needed).
itsu_status ensure_outputs_for(itsu_context *ctx, int64_t n_clusters)
{
  if ((ctx->flags & ITSU_FLAG_NO_GROW) && ctx->stage != -1) {
    return ITSU_OK;  // fixed arena: overflow is reported by the run itself
  }
  // configured capacities are floors; a fixed arena takes them as given
  const bool fixed = (ctx->flags & ITSU_FLAG_NO_GROW) != 0;
  auto pick = [fixed](int64_t configured, int64_t dflt) { return fixed && configured > 0 ? configured : std::max(configured, dflt); };
  itsu_status st;
  if ((st = ensure_tracklets(ctx, pick(ctx->init_tracklets, 10 * n_clusters + 4096))) != ITSU_OK) return st;
  if ((st = ensure_cells(ctx, pick(ctx->init_cells, 2 * n_clusters + 4096))) != ITSU_OK) return st;
  if ((st = ensure_neighbours(ctx, pick(ctx->init_neighbours, 2 * n_clusters + 4096))) != ITSU_OK) return st;
  return ensure_roads(ctx, pick(ctx->init_roads, n_clusters / 2 + 4096));
}

itsu_status check_launch(itsu_context *ctx)
{
  ITSU_CUDA(ctx, cudaGetLastError());
  return ITSU_OK;
}

// Copies the device status to the host and waits for the stream.
itsu_status sync_status(itsu_context *ctx)
{
  ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, ctx->stream));
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->h_status->flags & itsu::kFlagLaunchShape) {
    return fail(ctx, ITSU_ERR_INVALID, "launch shape: the per-item passes need a block size that is a multiple of 32");
  }
  if (ctx->h_status->flags & itsu::kFlagTimeout) {
    return fail(ctx, ITSU_ERR_TIMEOUT, "a bounded device wait (a shared-memory bulk copy) gave up");
  }
  return ITSU_OK;
}

itsu_status check_invalid(itsu_context *ctx)
{
  const DevStatus &s = *ctx->h_status;
  if (s.flags & itsu::kFlagInvalid) {
    if (s.invalid_event != INT32_MAX) {
      return fail(ctx, ITSU_ERR_INVALID, "primary vertex of event %d is not finite or beyond 1e6 cm", s.invalid_event);
    }
    return fail(ctx, ITSU_ERR_INVALID,
                "cluster %d is malformed: a coordinate is not finite or beyond 1e6 cm, or it sits on the beam line "
                "at the vertex z (r == 0 and z == vertex z)",
                s.invalid_index);
  }
  return ITSU_OK;
}

itsu_status clear_flags(itsu_context *ctx)
{
  ITSU_CUDA(ctx, cudaMemsetAsync(&ctx->d_status->flags, 0, sizeof(int32_t), ctx->stream));
  return ITSU_OK;
}

itsu_status count_overflow(itsu_context *ctx)
{
  return fail(ctx, ITSU_ERR_CAPACITY, "a result count exceeds the 32-bit index range of the reference layouts");
}

// Enqueues every stage of the current inputs (no host synchronisation).
void enqueue_run(const Arena &a, const Launch &l)
{
  itsu::launch_status_init(a, l);
  itsu::launch_cluster_sort(a, l);
  itsu::launch_tracklets_count(a, l);
  itsu::launch_tracklets_write(a, l);
  itsu::launch_cells_count(a, l);
  itsu::launch_cells_write(a, l);
  itsu::launch_neighbours_count(a, l);
  itsu::launch_neighbours_write(a, l);
  itsu::launch_roads_count(a, l);
  itsu::launch_roads_write(a, l);
}

void enqueue_all(itsu_context *ctx) { enqueue_run(arena_of(ctx), whole_run_launch(ctx)); }

void drop_graph(itsu_context *ctx)
{
  if (ctx->graph) {
    cudaGraphExecDestroy(ctx->graph);
    ctx->graph = nullptr;
  }
}

// Launches the whole sequence, through a CUDA graph that is re-captured when the inputs,
// sizes or arena buffers change.
itsu_status launch_all(itsu_context *ctx)
{
  const Tune tune = current_tune(ctx);
  const bool same = ctx->graph && ctx->graph_generation == ctx->generation && ctx->graph_key[0] == ctx->in_raw &&
                    ctx->graph_tune[0] == tune.block && ctx->graph_tune[1] == tune.blocks_per_sm &&
                    ctx->graph_tune[2] == tune.prune && ctx->graph_tune[3] == tune.group && ctx->graph_prefilter == ctx->prefilter &&
                    ctx->graph_gate == ctx->gate &&
                    ctx->graph_key[1] == ctx->in_layer_off && ctx->graph_key[2] == ctx->in_vtx &&
                    ctx->graph_key[3] == ctx->in_raw_off && ctx->graph_key[4] == ctx->in_raw_in &&
                    ctx->graph_key[5] == ctx->in_raw_track &&
                    ctx->graph_events == ctx->n_events && ctx->graph_clusters == ctx->n_clusters;
  if (!same) {
    drop_graph(ctx);
    cudaGraph_t g = nullptr;
    ITSU_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_all(ctx);
    const cudaError_t launch_err = cudaGetLastError();
    const cudaError_t end_err = cudaStreamEndCapture(ctx->stream, &g);
    if (launch_err != cudaSuccess || end_err != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return fail(ctx, ITSU_ERR_CUDA, "graph capture failed: %s / %s", cudaGetErrorString(launch_err),
                  cudaGetErrorString(end_err));
    }
    const cudaError_t inst_err = cudaGraphInstantiate(&ctx->graph, g, 0);
    cudaGraphDestroy(g);
    if (inst_err != cudaSuccess) {
      ctx->graph = nullptr;
      return fail(ctx, ITSU_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(inst_err));
    }
    ctx->graph_generation = ctx->generation;
    ctx->graph_key[0] = ctx->in_raw;
    ctx->graph_key[1] = ctx->in_layer_off;
    ctx->graph_key[2] = ctx->in_vtx;
    ctx->graph_key[3] = ctx->in_raw_off;
    ctx->graph_key[4] = ctx->in_raw_in;
    ctx->graph_key[5] = ctx->in_raw_track;
    ctx->graph_tune[0] = tune.block;
    ctx->graph_tune[1] = tune.blocks_per_sm;
    ctx->graph_tune[2] = tune.prune;
    ctx->graph_tune[3] = tune.group;
    ctx->graph_prefilter = ctx->prefilter;
    ctx->graph_gate = ctx->gate;
    ctx->graph_events = ctx->n_events;
    ctx->graph_clusters = ctx->n_clusters;
  }
  ITSU_CUDA(ctx, cudaGraphLaunch(ctx->graph, ctx->stream));
  return ITSU_OK;
}

// Runs every stage, growing the arena and repeating after an overflow.
itsu_status run_all(itsu_context *ctx)
{
  itsu_status st;
  for (int attempt = 0; attempt < 8; ++attempt) {
    if ((st = launch_all(ctx)) != ITSU_OK) return st;
    if ((st = sync_status(ctx)) != ITSU_OK) return st;
    if ((st = check_invalid(ctx)) != ITSU_OK) return st;
    const DevStatus &s = *ctx->h_status;
    if (!(s.flags & itsu::kCapacityMask)) {
      ctx->stage = kRoads;
      return ITSU_OK;
    }
    if (s.flags & itsu::kFlagCountOverflow) return count_overflow(ctx);
    if (ctx->flags & ITSU_FLAG_NO_GROW) {
      return fail(ctx, ITSU_ERR_CAPACITY, "result exceeds the arena (tracklets %lld/%lld cells %lld/%lld neighbours %lld/%lld roads %lld/%lld)",
                  (long long)s.total[0], (long long)ctx->cap_tracklets, (long long)s.total[1], (long long)ctx->cap_cells,
                  (long long)s.total[2], (long long)ctx->cap_neighbours, (long long)s.total[3], (long long)ctx->cap_roads);
    }
    if (s.flags & itsu::kFlagCapTracklets) {
      // cells, neighbours and roads scale with the tracklets: grow them in proportion too
      const double f = (double)s.total[0] / (double)std::max<int64_t>(ctx->cap_tracklets, 1);
      if ((st = ensure_tracklets(ctx, s.total[0])) != ITSU_OK) return st;
      if ((st = ensure_cells(ctx, (int64_t)(ctx->cap_cells * f))) != ITSU_OK) return st;
      if ((st = ensure_neighbours(ctx, (int64_t)(ctx->cap_neighbours * f))) != ITSU_OK) return st;
      if ((st = ensure_roads(ctx, (int64_t)(ctx->cap_roads * f))) != ITSU_OK) return st;
    }
    if ((s.flags & itsu::kFlagCapCells) && (st = ensure_cells(ctx, s.total[1])) != ITSU_OK) return st;
    if ((s.flags & itsu::kFlagCapScratch) && (st = ensure_cell_entries(ctx, s.cell_entries + cell_entry_slack(ctx))) != ITSU_OK) {
      return st;
    }
    if ((s.flags & itsu::kFlagCapNeighbours) && (st = ensure_neighbours(ctx, s.total[2])) != ITSU_OK) return st;
    if ((s.flags & itsu::kFlagCapRoads) && (st = ensure_roads(ctx, s.total[3])) != ITSU_OK) return st;
  }
  return fail(ctx, ITSU_ERR_CAPACITY, "arena growth did not converge");
}

itsu_status stage_count_then_write(itsu_context *ctx, void (*count)(const Arena &, const Launch &),
                                   void (*write)(const Arena &, const Launch &), int total_index,
                                   itsu_status (*ensure)(itsu_context *, int64_t))
{
  itsu_status st;
  for (int attempt = 0;; ++attempt) {
    if ((st = clear_flags(ctx)) != ITSU_OK) return st;
    // the entry reservation, the crowded lists and the tile sums of the tracklet and cell scans
    // (the count passes add to them) start empty for every count, also a retry
    ITSU_CUDA(ctx, cudaMemsetAsync(&ctx->d_status->cell_entries, 0, 3 * sizeof(int64_t), ctx->stream));
    ITSU_CUDA(ctx, cudaMemsetAsync(ctx->scan_partials, 0, sizeof(int64_t) * ctx->cap_partials, ctx->stream));
    count(arena_of(ctx), launch_of(ctx));
    if ((st = check_launch(ctx)) != ITSU_OK) return st;
    if ((st = sync_status(ctx)) != ITSU_OK) return st;
    // the cell count pass keeps its entries for the write: if they overflowed their scratch,
    // grow it and count again
    if (!(ctx->h_status->flags & itsu::kFlagCapScratch) || (ctx->h_status->flags & itsu::kFlagCountOverflow)) break;
    if (attempt == 4) return fail(ctx, ITSU_ERR_CAPACITY, "cell entry scratch growth did not converge");
    if ((st = ensure_cell_entries(ctx, ctx->h_status->cell_entries + cell_entry_slack(ctx))) != ITSU_OK) return st;
  }
  const DevStatus &s = *ctx->h_status;
  if (s.flags & itsu::kFlagCountOverflow) return count_overflow(ctx);
  if (s.flags & itsu::kCapacityMask) {
    if (ctx->flags & ITSU_FLAG_NO_GROW) {
      return fail(ctx, ITSU_ERR_CAPACITY, "stage output of %lld exceeds the arena", (long long)s.total[total_index]);
    }
    // exact two-pass sizing: grow the stage's outputs to the counted total. Growth reallocates
    // only buffers the write pass fills, never the counts and offsets just computed, so the
    // write proceeds on the existing counts.
    if ((st = ensure(ctx, s.total[total_index])) != ITSU_OK) return st;
    if ((st = clear_flags(ctx)) != ITSU_OK) return st;
  }
  write(arena_of(ctx), launch_of(ctx));
  if ((st = check_launch(ctx)) != ITSU_OK) return st;
  if ((st = sync_status(ctx)) != ITSU_OK) return st;
  if (ctx->h_status->flags & itsu::kCapacityMask) {
    return fail(ctx, ITSU_ERR_CAPACITY, "stage output exceeds the arena after growth");
  }
  return ITSU_OK;
}

itsu_status require_stage(itsu_context *ctx, int stage, const char *what)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "%s: null context", what);
  if (ctx->stage < stage) {
    return fail(ctx, ITSU_ERR_STATE, "%s called before the stage it depends on", what);
  }
  return ITSU_OK;
}

// Host inputs of one vertex -> device arena.
itsu_status upload_vertex(itsu_context *ctx, const itsu_cluster *const layers[ITSU_LAYERS], const int32_t counts[ITSU_LAYERS],
                          const float vertex[3])
{
  if (!layers || !counts || !vertex) return fail(ctx, ITSU_ERR_INVALID, "null argument");
  std::vector<int32_t> off(ITSU_LAYERS + 1, 0);
  for (int l = 0; l < ITSU_LAYERS; ++l) {
    if (counts[l] < 0) return fail(ctx, ITSU_ERR_INVALID, "negative cluster count on layer %d", l);
    if (counts[l] > 0 && !layers[l]) return fail(ctx, ITSU_ERR_INVALID, "null cluster array on layer %d", l);
    if ((int64_t)off[l] + counts[l] > INT32_MAX) return fail(ctx, ITSU_ERR_INVALID, "too many clusters");
    off[l + 1] = off[l] + counts[l];
  }
  itsu_status st;
  if ((st = ensure_clusters(ctx, off[ITSU_LAYERS], 1)) != ITSU_OK) return st;
  for (int l = 0; l < ITSU_LAYERS; ++l) {
    if (counts[l] > 0) {
      ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->raw + off[l], layers[l], sizeof(itsu_cluster) * counts[l], cudaMemcpyHostToDevice,
                                     ctx->stream));
    }
  }
  ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->layer_off, off.data(), sizeof(int32_t) * off.size(), cudaMemcpyHostToDevice, ctx->stream));
  ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->vtx, vertex, sizeof(float) * 3, cudaMemcpyHostToDevice, ctx->stream));
  ctx->n_events = 1;
  ctx->n_clusters = off[ITSU_LAYERS];
  ctx->h_layer_off = off;
  ctx->in_raw = ctx->raw;
  ctx->in_raw_in = nullptr;
  ctx->in_raw_track = nullptr;
  ctx->in_raw_off = nullptr;
  ctx->in_layer_off = ctx->layer_off;
  ctx->in_vtx = ctx->vtx;
  ctx->stage = kNone;
  return ITSU_OK;
}

template <typename T>
itsu_status copy_range(itsu_context *ctx, T *dst, const T *src, int64_t count)
{
  if (dst && count > 0) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyDeviceToHost, ctx->stream));
  }
  return ITSU_OK;
}

struct EventSegments {
  int32_t lo[ITSU_LAYERS + 1];
  int32_t ts[ITSU_TRACKLET_LAYERS + 1];
  int32_t cs[ITSU_CELL_LAYERS + 1];
  int32_t rs[2];
  int32_t nbo[ITSU_CELL_LAYERS + 1];  // nb_off at cs[0..5]
};

itsu_status event_segments(itsu_context *ctx, int32_t e, EventSegments &seg)
{
  if (e < 0 || e >= ctx->n_events) return fail(ctx, ITSU_ERR_INVALID, "event %d out of range", e);
  // Only the segments of stages that have run exist: the others read as empty.
  std::memset(&seg, 0, sizeof seg);
  std::memcpy(seg.lo, ctx->h_layer_off.data() + (int64_t)e * ITSU_LAYERS, sizeof seg.lo);
  if (ctx->stage >= kTracklets) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(seg.ts, ctx->trk_seg + (int64_t)e * ITSU_TRACKLET_LAYERS, sizeof seg.ts, cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (ctx->stage >= kCells) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(seg.cs, ctx->cell_seg + (int64_t)e * ITSU_CELL_LAYERS, sizeof seg.cs, cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (ctx->stage >= kRoads) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(seg.rs, ctx->road_seg + e, sizeof seg.rs, cudaMemcpyDeviceToHost, ctx->stream));
  }
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->stage >= kNeighbours) {
    for (int l = 0; l <= ITSU_CELL_LAYERS; ++l) {
      ITSU_CUDA(ctx, cudaMemcpyAsync(&seg.nbo[l], ctx->nb_off + seg.cs[l], sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    }
    ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return ITSU_OK;
}

void counts_from(const itsu_context *ctx, const EventSegments &s, itsu_counts *out)
{
  for (int l = 0; l < ITSU_LAYERS; ++l) out->clusters[l] = s.lo[l + 1] - s.lo[l];
  for (int l = 0; l < ITSU_TRACKLET_LAYERS; ++l) out->tracklets[l] = ctx->stage >= kTracklets ? s.ts[l + 1] - s.ts[l] : 0;
  for (int l = 0; l < ITSU_CELL_LAYERS; ++l) out->cells[l] = ctx->stage >= kCells ? s.cs[l + 1] - s.cs[l] : 0;
  for (int l = 0; l < ITSU_NEIGHBOUR_LAYERS; ++l) {
    out->neighbours[l] = ctx->stage >= kNeighbours ? s.nbo[l + 2] - s.nbo[l + 1] : 0;
  }
  out->roads = ctx->stage >= kRoads ? s.rs[1] - s.rs[0] : 0;
}

}  // namespace

// ============================================================================================
// C ABI

extern "C" {

const char *itsu_version(void) { return "itsu-b200 1.0 (sm_100a)"; }

const char *itsu_status_string(itsu_status status)
{
  switch (status) {
  case ITSU_OK: return "ok";
  case ITSU_ERR_INVALID: return "invalid input";
  case ITSU_ERR_CAPACITY: return "capacity exceeded";
  case ITSU_ERR_TIMEOUT: return "device wait timed out";
  case ITSU_ERR_CUDA: return "CUDA error";
  case ITSU_ERR_NOMEM: return "out of memory";
  case ITSU_ERR_STATE: return "call out of order";
  }
  return "unknown status";
}

const char *itsu_last_error(const itsu_context *ctx) { return ctx ? ctx->error.c_str() : g_thread_error.c_str(); }

void itsu_config_default(itsu_config *cfg)
{
  if (cfg) {
    std::memset(cfg, 0, sizeof *cfg);
  }
}

itsu_status itsu_context_create(const itsu_config *cfg, itsu_context **out)
{
  if (!out) return fail(nullptr, ITSU_ERR_INVALID, "itsu_context_create: null output");
  *out = nullptr;
  itsu_config c;
  itsu_config_default(&c);
  if (cfg) c = *cfg;
  int n_dev = 0;
  cudaError_t err = cudaGetDeviceCount(&n_dev);
  if (err != cudaSuccess || n_dev == 0) {
    return fail(nullptr, ITSU_ERR_CUDA, "no CUDA device: %s", cudaGetErrorString(err));
  }
  if (c.device < 0 || c.device >= n_dev) return fail(nullptr, ITSU_ERR_INVALID, "device %d out of range", c.device);
  auto *ctx = new itsu_context();
  ctx->device = c.device;
  ctx->flags = c.flags;
  ctx->init_tracklets = c.max_tracklets;
  ctx->init_cells = c.max_cells;
  ctx->init_neighbours = c.max_neighbours;
  ctx->init_roads = c.max_roads;
  if (c.stream_chunk_clusters < 0) {
    delete ctx;
    return fail(nullptr, ITSU_ERR_INVALID, "itsu_context_create: negative stream chunk size");
  }
  ctx->chunk_clusters = c.stream_chunk_clusters;
  itsu_status st = ITSU_OK;
  do {
    if ((err = cudaSetDevice(c.device)) != cudaSuccess) break;
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, c.device);
    if (major != 10) {
      st = fail(nullptr, ITSU_ERR_CUDA, "device %d has compute capability %d.x; this build targets sm_100a", c.device, major);
      break;
    }
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, c.device);
    if ((err = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) break;
    ctx->own_stream = true;
    if ((err = cudaMalloc((void **)&ctx->d_status, sizeof(DevStatus))) != cudaSuccess) break;
    if ((err = cudaMallocHost((void **)&ctx->h_status, sizeof(DevStatus))) != cudaSuccess) break;
    std::memset(ctx->h_status, 0, sizeof(DevStatus));
    if (c.max_clusters > 0 || c.max_events > 0) {
      ctx->stage = -1;  // initial allocation: allowed even with ITSU_FLAG_NO_GROW
      if ((st = ensure_clusters(ctx, c.max_clusters, c.max_events)) != ITSU_OK) break;
      if ((st = ensure_outputs_for(ctx, c.max_clusters)) != ITSU_OK) break;
      ctx->stage = kNone;
    }
  } while (false);
  if (err != cudaSuccess && st == ITSU_OK) {
    st = fail(nullptr, err == cudaErrorMemoryAllocation ? ITSU_ERR_NOMEM : ITSU_ERR_CUDA, "context setup: %s",
              cudaGetErrorString(err));
  }
  if (st != ITSU_OK) {
    g_thread_error = ctx->error.empty() ? g_thread_error : ctx->error;
    itsu_context_destroy(ctx);
    return st;
  }
  *out = ctx;
  return ITSU_OK;
}

void itsu_context_destroy(itsu_context *ctx)
{
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->twin) itsu_context_destroy(ctx->twin);
  drop_graph(ctx);
  release(ctx->raw); release(ctx->raw_in); release(ctx->raw_track); release(ctx->sorted); release(ctx->tmp); release(ctx->xyzr); release(ctx->phi);
  release(ctx->trk_count); release(ctx->trk_off); release(ctx->trk_lookup); release(ctx->zs); release(ctx->clu_seg); release(ctx->clu_aux); release(ctx->clu_crowded); release(ctx->trk_slots);
  release(ctx->seg_rrange); release(ctx->seg_regular); release(ctx->raw_off);
  release(ctx->layer_off); release(ctx->index_tables); release(ctx->trk_seg); release(ctx->cell_seginfo); release(ctx->cell_seg);
  release(ctx->road_seg); release(ctx->vtx);
  release(ctx->tracklets); release(ctx->trk_slope); release(ctx->trk_seg_id); release(ctx->cell_count); release(ctx->cell_mask); release(ctx->cell_off); release(ctx->cell_lookup); release(ctx->cell_crowded);
  release(ctx->cells); release(ctx->cell_entries); release(ctx->cell_dca); release(ctx->cell_seg_id); release(ctx->nb_count); release(ctx->nb_off); release(ctx->nb_fill);
  release(ctx->nb_mask);
  release(ctx->road_count); release(ctx->road_off); release(ctx->paths);
  release(ctx->nb); release(ctx->roads); release(ctx->scan_partials); release(ctx->d_status);
  release(ctx->d_master); release(ctx->d_mlp);
  release(ctx->d_gate_master); release(ctx->d_gate);
  release(ctx->report_scratch); release(ctx->chunk_off); release(ctx->roads_all); release(ctx->road_off_all); release(ctx->chunk_status);
  if (ctx->h_chunk_status) cudaFreeHost(ctx->h_chunk_status);
  if (ctx->h_chunk_off) cudaFreeHost(ctx->h_chunk_off);
  for (cudaEvent_t &e : ctx->chunk_ready) {
    if (e) cudaEventDestroy(e);
  }
  for (cudaEvent_t &e : ctx->chunk_done) {
    if (e) cudaEventDestroy(e);
  }
  if (ctx->h_road_end) cudaFreeHost(ctx->h_road_end);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->d2h_stream) cudaStreamDestroy(ctx->d2h_stream);
  if (ctx->h_status) cudaFreeHost(ctx->h_status);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

itsu_status itsu_context_set_stream(itsu_context *ctx, void *cuda_stream)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "null context");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->own_stream) {
    cudaStreamDestroy(ctx->stream);
    ctx->own_stream = false;
    ctx->stream = nullptr;
  }
  if (cuda_stream) {
    ctx->stream = (cudaStream_t)cuda_stream;
  } else {
    ITSU_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  drop_graph(ctx);
  return ITSU_OK;
}

void *itsu_context_stream(const itsu_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

itsu_status itsu_pvc_initialize(itsu_context *ctx, const itsu_cluster *const layers[ITSU_LAYERS], const int32_t counts[ITSU_LAYERS],
                                const float vertex[3])
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "null context");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  itsu_status st;
  if ((st = upload_vertex(ctx, layers, counts, vertex)) != ITSU_OK) return st;
  const Arena a = arena_of(ctx);
  itsu::launch_status_init(a, launch_of(ctx));
  itsu::launch_cluster_sort(a, launch_of(ctx));
  if ((st = check_launch(ctx)) != ITSU_OK) return st;
  if ((st = sync_status(ctx)) != ITSU_OK) return st;
  if ((st = check_invalid(ctx)) != ITSU_OK) return st;
  ctx->stage = kInitialized;
  return ITSU_OK;
}

itsu_status itsu_compute_layer_tracklets(itsu_context *ctx)
{
  itsu_status st;
  if ((st = require_stage(ctx, kInitialized, "itsu_compute_layer_tracklets")) != ITSU_OK) return st;
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  if ((st = ensure_tracklets(ctx, 1)) != ITSU_OK) return st;
  if ((st = stage_count_then_write(ctx, itsu::launch_tracklets_count, itsu::launch_tracklets_write, itsu::kTracklets,
                                   ensure_tracklets)) != ITSU_OK) {
    return st;
  }
  ctx->stage = kTracklets;
  return ITSU_OK;
}

itsu_status itsu_compute_layer_cells(itsu_context *ctx)
{
  itsu_status st;
  if ((st = require_stage(ctx, kTracklets, "itsu_compute_layer_cells")) != ITSU_OK) return st;
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  if ((st = ensure_cells(ctx, 1)) != ITSU_OK) return st;
  if ((st = stage_count_then_write(ctx, itsu::launch_cells_count, itsu::launch_cells_write, itsu::kCells, ensure_cells)) != ITSU_OK) {
    return st;
  }
  ctx->stage = kCells;
  return ITSU_OK;
}

itsu_status itsu_find_cells_neighbours(itsu_context *ctx)
{
  itsu_status st;
  if ((st = require_stage(ctx, kCells, "itsu_find_cells_neighbours")) != ITSU_OK) return st;
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  if ((st = ensure_neighbours(ctx, 1)) != ITSU_OK) return st;
  if ((st = stage_count_then_write(ctx, itsu::launch_neighbours_count, itsu::launch_neighbours_write, itsu::kNeighbours,
                                   ensure_neighbours)) != ITSU_OK) {
    return st;
  }
  ctx->stage = kNeighbours;
  return ITSU_OK;
}

itsu_status itsu_find_tracks(itsu_context *ctx)
{
  itsu_status st;
  if ((st = require_stage(ctx, kNeighbours, "itsu_find_tracks")) != ITSU_OK) return st;
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  if ((st = ensure_roads(ctx, 1)) != ITSU_OK) return st;
  if ((st = stage_count_then_write(ctx, itsu::launch_roads_count, itsu::launch_roads_write, itsu::kRoads, ensure_roads)) != ITSU_OK) {
    return st;
  }
  ctx->stage = kRoads;
  return ITSU_OK;
}

itsu_status itsu_compute_montecarlo_labels(itsu_context *ctx)
{
  // The road kernel votes the labels of every road it writes (Moore's vote over the road's
  // clusters), so the labels already exist once the roads do.
  return require_stage(ctx, kRoads, "itsu_compute_montecarlo_labels");
}

itsu_status itsu_get_counts(itsu_context *ctx, int32_t event, itsu_counts *out)
{
  itsu_status st;
  if ((st = require_stage(ctx, kInitialized, "itsu_get_counts")) != ITSU_OK) return st;
  if (!out) return fail(ctx, ITSU_ERR_INVALID, "null output");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  EventSegments s;
  if ((st = event_segments(ctx, event, s)) != ITSU_OK) return st;
  counts_from(ctx, s, out);
  return ITSU_OK;
}

itsu_status itsu_copy_results(itsu_context *ctx, int32_t event, const itsu_results *out)
{
  itsu_status st;
  if ((st = require_stage(ctx, kInitialized, "itsu_copy_results")) != ITSU_OK) return st;
  if (!out) return fail(ctx, ITSU_ERR_INVALID, "null output");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  EventSegments s;
  if ((st = event_segments(ctx, event, s)) != ITSU_OK) return st;
  itsu_counts n;
  counts_from(ctx, s, &n);
  for (int l = 0; l < ITSU_LAYERS; ++l) {
    if ((st = copy_range(ctx, out->clusters[l], ctx->sorted + s.lo[l], n.clusters[l])) != ITSU_OK) return st;
  }
  for (int l = 0; l < ITSU_TRACKLET_LAYERS; ++l) {
    if ((st = copy_range(ctx, out->index_tables[l], ctx->index_tables + ((int64_t)event * ITSU_TRACKLET_LAYERS + l) * ITSU_INDEX_TABLE_SIZE,
                         ITSU_INDEX_TABLE_SIZE)) != ITSU_OK) {
      return st;
    }
  }
  if (ctx->stage >= kTracklets) {
    for (int l = 0; l < ITSU_TRACKLET_LAYERS; ++l) {
      if ((st = copy_range(ctx, out->tracklets[l], ctx->tracklets + s.ts[l], n.tracklets[l])) != ITSU_OK) return st;
    }
    for (int l = 0; l < ITSU_CELL_LAYERS; ++l) {
      if ((st = copy_range(ctx, out->tracklets_lookup[l], ctx->trk_lookup + s.lo[l + 1], n.clusters[l + 1])) != ITSU_OK) return st;
    }
  } else {
    for (int l = 0; l < ITSU_CELL_LAYERS; ++l) {
      if (out->tracklets_lookup[l]) std::fill(out->tracklets_lookup[l], out->tracklets_lookup[l] + n.clusters[l + 1], ITSU_UNUSED_INDEX);
    }
  }
  if (ctx->stage >= kCells) {
    for (int l = 0; l < ITSU_CELL_LAYERS; ++l) {
      if ((st = copy_range(ctx, out->cells[l], ctx->cells + s.cs[l], n.cells[l])) != ITSU_OK) return st;
    }
    for (int l = 0; l < ITSU_NEIGHBOUR_LAYERS; ++l) {
      if ((st = copy_range(ctx, out->cells_lookup[l], ctx->cell_lookup + s.ts[l + 1], n.tracklets[l + 1])) != ITSU_OK) return st;
    }
  } else {
    for (int l = 0; l < ITSU_NEIGHBOUR_LAYERS; ++l) {  // no cells yet: every lookup entry unused
      if (out->cells_lookup[l]) std::fill(out->cells_lookup[l], out->cells_lookup[l] + n.tracklets[l + 1], ITSU_UNUSED_INDEX);
    }
  }
  if (ctx->stage >= kNeighbours) {
    for (int l = 0; l < ITSU_NEIGHBOUR_LAYERS; ++l) {
      if ((st = copy_range(ctx, out->neighbour_offsets[l], ctx->nb_off + s.cs[l + 1], (int64_t)n.cells[l + 1] + 1)) != ITSU_OK) return st;
      if ((st = copy_range(ctx, out->neighbours[l], ctx->nb + s.nbo[l + 1], n.neighbours[l])) != ITSU_OK) return st;
    }
  } else {
    for (int l = 0; l < ITSU_NEIGHBOUR_LAYERS; ++l) {  // no neighbours yet: empty rows
      if (out->neighbour_offsets[l]) std::fill(out->neighbour_offsets[l], out->neighbour_offsets[l] + n.cells[l + 1] + 1, 0);
    }
  }
  if (ctx->stage >= kRoads) {
    if ((st = copy_range(ctx, out->roads, ctx->roads + s.rs[0], n.roads)) != ITSU_OK) return st;
  }
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->stage >= kNeighbours) {
    for (int l = 0; l < ITSU_NEIGHBOUR_LAYERS; ++l) {  // rebase the CSR rows to this layer
      if (out->neighbour_offsets[l]) {
        for (int32_t k = 0; k <= n.cells[l + 1]; ++k) out->neighbour_offsets[l][k] -= s.nbo[l + 1];
      }
    }
  }
  return ITSU_OK;
}

itsu_status itsu_clusters_to_tracks(itsu_context *ctx, const itsu_cluster *const layers[ITSU_LAYERS],
                                    const int32_t counts[ITSU_LAYERS], const float vertex[3], itsu_road *roads,
                                    int32_t roads_capacity, int32_t *roads_count)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "null context");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  itsu_status st;
  if ((st = upload_vertex(ctx, layers, counts, vertex)) != ITSU_OK) return st;
  if ((st = ensure_outputs_for(ctx, ctx->n_clusters)) != ITSU_OK) return st;
  if ((st = run_all(ctx)) != ITSU_OK) return st;
  const int64_t total = ctx->h_status->total[itsu::kRoads];
  if (roads_count) *roads_count = (int32_t)total;
  if (roads) {
    if (total > roads_capacity) return fail(ctx, ITSU_ERR_CAPACITY, "%lld roads do not fit the %d given", (long long)total, roads_capacity);
    if ((st = copy_range(ctx, roads, (const itsu_road *)ctx->roads, total)) != ITSU_OK) return st;
    ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return ITSU_OK;
}

static itsu_status set_batch(itsu_context *ctx, const itsu_batch *batch)
{
  if (!batch) return fail(ctx, ITSU_ERR_INVALID, "null batch");
  if (batch->n_events < 0 || batch->n_clusters < 0 || batch->n_clusters > INT32_MAX) {
    return fail(ctx, ITSU_ERR_INVALID, "bad batch size (%d events, %lld clusters)", batch->n_events, (long long)batch->n_clusters);
  }
  if (batch->n_events > 0 && (!batch->layer_offsets || !batch->vertices || (batch->n_clusters > 0 && !batch->clusters))) {
    return fail(ctx, ITSU_ERR_INVALID, "null batch pointer");
  }
  itsu_status st;
  if ((st = ensure_clusters(ctx, batch->n_clusters, batch->n_events)) != ITSU_OK) return st;
  if ((st = ensure_outputs_for(ctx, batch->n_clusters)) != ITSU_OK) return st;
  ctx->n_events = batch->n_events;
  ctx->n_clusters = batch->n_clusters;
  ctx->in_raw = batch->clusters;
  ctx->in_raw_in = nullptr;
  ctx->in_raw_track = nullptr;
  ctx->in_raw_off = nullptr;
  ctx->in_layer_off = batch->layer_offsets;
  ctx->in_vtx = batch->vertices;
  ctx->h_layer_off.resize((size_t)batch->n_events * ITSU_LAYERS + 1);
  if (batch->n_events > 0) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->h_layer_off.data(), batch->layer_offsets, sizeof(int32_t) * ctx->h_layer_off.size(),
                                   cudaMemcpyDeviceToHost, ctx->stream));
    ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->h_layer_off[0] != 0 || ctx->h_layer_off.back() != batch->n_clusters) {
      return fail(ctx, ITSU_ERR_INVALID, "layer offsets must start at 0 and end at n_clusters");
    }
    for (size_t k = 1; k < ctx->h_layer_off.size(); ++k) {
      if (ctx->h_layer_off[k] < ctx->h_layer_off[k - 1]) return fail(ctx, ITSU_ERR_INVALID, "layer offsets decrease at %zu", k);
    }
  }
  ctx->stage = kNone;
  return ITSU_OK;
}

itsu_status itsu_batch_run(itsu_context *ctx, const itsu_batch *batch)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "null context");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  itsu_status st;
  if ((st = set_batch(ctx, batch)) != ITSU_OK) return st;
  return run_all(ctx);
}

itsu_status itsu_batch_launch(itsu_context *ctx, const itsu_batch *batch)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "null context");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  itsu_status st;
  const bool same = batch && ctx->stage != kNone && !ctx->in_raw_off && !ctx->in_raw_in && !ctx->in_raw_track &&
                    batch->clusters == ctx->in_raw &&
                    batch->layer_offsets == ctx->in_layer_off &&
                    batch->vertices == ctx->in_vtx && batch->n_events == ctx->n_events && batch->n_clusters == ctx->n_clusters;
  if (!same && (st = set_batch(ctx, batch)) != ITSU_OK) return st;
  if ((st = launch_all(ctx)) != ITSU_OK) return st;
  ctx->stage = kRoads;
  return ITSU_OK;
}

itsu_status itsu_batch_status(itsu_context *ctx)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "null context");
  itsu_status st;
  if ((st = sync_status(ctx)) != ITSU_OK) return st;
  if ((st = check_invalid(ctx)) != ITSU_OK) return st;
  if (ctx->h_status->flags & itsu::kCapacityMask) {
    ctx->stage = kNone;
    return fail(ctx, ITSU_ERR_CAPACITY, "a result exceeded the arena; run itsu_batch_run once to size it");
  }
  return ITSU_OK;
}

itsu_status itsu_batch_roads_device(itsu_context *ctx, const itsu_road **roads, const int32_t **road_offsets)
{
  itsu_status st;
  if ((st = require_stage(ctx, kRoads, "itsu_batch_roads_device")) != ITSU_OK) return st;
  if (roads) *roads = ctx->roads;
  if (road_offsets) *road_offsets = ctx->road_seg;
  return ITSU_OK;
}

itsu_status itsu_memory_usage_get(itsu_context *ctx, itsu_memory_usage *out)
{
  if (!ctx || !out) return fail(ctx, ITSU_ERR_INVALID, "itsu_memory_usage_get: null argument");
  std::memset(out, 0, sizeof *out);
  out->device_bytes = ctx->arena_bytes + (ctx->twin ? ctx->twin->arena_bytes : 0);
  out->clusters_capacity = ctx->cap_clusters;
  out->events_capacity = ctx->cap_events;
  out->capacity[0] = ctx->cap_tracklets;
  out->capacity[1] = ctx->cap_cells;
  out->capacity[2] = ctx->cap_neighbours;
  out->capacity[3] = ctx->cap_roads;
  for (int k = 0; k < 4; ++k) out->used[k] = ctx->h_status ? ctx->h_status->total[k] : 0;
  out->cell_entries_capacity = ctx->cap_cell_entries;
  return ITSU_OK;
}

itsu_status itsu_batch_road_count(itsu_context *ctx, int64_t *n_roads)
{
  itsu_status st;
  if (!n_roads) return fail(ctx, ITSU_ERR_INVALID, "itsu_batch_road_count: null output");
  if ((st = require_stage(ctx, kRoads, "itsu_batch_road_count")) != ITSU_OK) return st;
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  int32_t end = 0;
  ITSU_CUDA(ctx, cudaMemcpyAsync(&end, ctx->road_seg + ctx->n_events, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *n_roads = end;
  return ITSU_OK;
}

itsu_status itsu_roads_report(itsu_context *ctx, const itsu_road *roads, const int32_t *run_offsets, const int32_t *run_event,
                              int32_t n_runs, const itsu_label *labels, const int32_t *label_offsets, int32_t n_events,
                              uint8_t *road_class, itsu_report_counts *counts)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "itsu_roads_report: null context");
  if (n_runs < 0 || n_events < 0) return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: negative run or event count");
  if ((roads == nullptr) != (run_offsets == nullptr)) {
    return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: give both roads and run offsets, or neither");
  }
  if (n_events > 0 && !label_offsets) return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: null label offsets");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  const bool resident = roads == nullptr;
  if (resident) {
    itsu_status st;
    if ((st = require_stage(ctx, kRoads, "itsu_roads_report")) != ITSU_OK) return st;
    if (n_runs != ctx->n_events) {
      return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: %d runs given, the last run has %d", n_runs, ctx->n_events);
    }
  } else {
    if (n_runs > 0 && run_offsets[0] != 0) return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: run offsets must start at 0");
    for (int32_t r = 0; r < n_runs; ++r) {
      if (run_offsets[r + 1] < run_offsets[r]) return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: run offsets decrease at %d", r);
    }
  }
  for (int32_t r = 0; run_event && r < n_runs; ++r) {
    if (run_event[r] < 0 || run_event[r] >= n_events || (r > 0 && run_event[r] < run_event[r - 1])) {
      return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: run %d has event %d (events must be in [0, %d) and non-decreasing)", r,
                  run_event[r], n_events);
    }
  }
  if (!run_event && n_runs > n_events) {
    return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: %d runs but %d events and no run-to-event map", n_runs, n_events);
  }
  if (n_events > 0 && label_offsets[0] != 0) return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: label offsets must start at 0");
  for (int32_t e = 0; e < n_events; ++e) {
    if (label_offsets[e + 1] < label_offsets[e]) return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: label offsets decrease at %d", e);
  }
  const int64_t n_labels = n_events > 0 ? label_offsets[n_events] : 0;
  if (n_labels > 0 && !labels) return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: null labels");
  std::vector<int32_t> label_event((size_t)n_labels);
  std::vector<int64_t> table_base((size_t)n_events + 1, 0);
  for (int32_t e = 0; e < n_events; ++e) {
    const int64_t n = label_offsets[e + 1] - label_offsets[e];
    int64_t size = 2;
    while (size < 2 * n) size <<= 1;  // power of two, at least twice the labels: probes end at an empty slot
    table_base[e + 1] = table_base[e] + size;
    for (int64_t i = label_offsets[e]; i < label_offsets[e + 1]; ++i) {
      if (labels[i].mc_id == INT32_MIN) return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: label %lld has mc id INT32_MIN", (long long)i);
      label_event[(size_t)i] = e;
    }
  }
  const int64_t table_size = table_base[(size_t)n_events];

  // device inputs: the roads and their run offsets (the context's own when resident)
  int64_t n_roads = 0;
  if (resident) {
    int32_t end = 0;
    ITSU_CUDA(ctx, cudaMemcpyAsync(&end, ctx->road_seg + n_runs, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    n_roads = end;
  } else {
    n_roads = n_runs > 0 ? run_offsets[n_runs] : 0;
    if (n_roads > 0 && !roads) return fail(ctx, ITSU_ERR_INVALID, "itsu_roads_report: null roads");
  }
  // one scratch allocation for everything, freed before returning
  auto align = [](size_t n) { return (n + 255) / 256 * 256; };
  const size_t o_roads = 0;
  const size_t o_run = o_roads + (resident ? 0 : align(sizeof(itsu_road) * (size_t)n_roads));
  const size_t o_rev = o_run + (resident ? 0 : align(sizeof(int32_t) * ((size_t)n_runs + 1)));
  const size_t o_lab = o_rev + align(sizeof(int32_t) * (size_t)n_runs);
  const size_t o_lev = o_lab + align(sizeof(itsu_label) * (size_t)n_labels);
  const size_t o_tb = o_lev + align(sizeof(int32_t) * (size_t)n_labels);
  const size_t o_keys = o_tb + align(sizeof(int64_t) * ((size_t)n_events + 1));
  const size_t o_fl = o_keys + align(sizeof(int32_t) * (size_t)table_size);
  const size_t o_fr = o_fl + align(sizeof(int32_t) * (size_t)table_size);
  const size_t o_rs = o_fr + align(sizeof(int64_t) * (size_t)table_size);
  const size_t o_re = o_rs + align(sizeof(int64_t) * (size_t)n_roads);
  const size_t o_cls = o_re + align(sizeof(int32_t) * (size_t)n_roads);
  const size_t o_cnt = o_cls + align((size_t)n_roads);
  const size_t total = o_cnt + align(sizeof(itsu_report_counts) * (size_t)n_events);
  // the scratch stays with the context (grown when a call needs more)
  if ((int64_t)total > ctx->cap_report_scratch) {
    ITSU_CUDA(ctx, alloc(ctx, ctx->report_scratch, grow_to((int64_t)total)));
    ctx->cap_report_scratch = grow_to((int64_t)total);
  }
  unsigned char *buf = ctx->report_scratch;
  itsu::ReportArgs r{};
  r.roads = resident ? ctx->roads : reinterpret_cast<itsu_road *>(buf + o_roads);
  r.n_roads = n_roads;
  r.run_offsets = resident ? ctx->road_seg : reinterpret_cast<int32_t *>(buf + o_run);
  r.run_event = run_event ? reinterpret_cast<int32_t *>(buf + o_rev) : nullptr;
  r.n_runs = n_runs;
  r.n_events = n_events;
  r.labels = reinterpret_cast<itsu_label *>(buf + o_lab);
  r.label_event = reinterpret_cast<int32_t *>(buf + o_lev);
  r.n_labels = n_labels;
  r.table_base = reinterpret_cast<int64_t *>(buf + o_tb);
  r.table_size = table_size;
  r.keys = reinterpret_cast<int32_t *>(buf + o_keys);
  r.first_label = reinterpret_cast<int32_t *>(buf + o_fl);
  r.first_road = reinterpret_cast<int64_t *>(buf + o_fr);
  r.road_slot = reinterpret_cast<int64_t *>(buf + o_rs);
  r.road_event = reinterpret_cast<int32_t *>(buf + o_re);
  r.road_class = buf + o_cls;
  r.counts = reinterpret_cast<itsu_report_counts *>(buf + o_cnt);
  cudaStream_t s = ctx->stream;
  if (!resident && n_roads > 0) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(buf + o_roads, roads, sizeof(itsu_road) * (size_t)n_roads, cudaMemcpyHostToDevice, s));
  }
  if (!resident) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(buf + o_run, run_offsets, sizeof(int32_t) * ((size_t)n_runs + 1), cudaMemcpyHostToDevice, s));
  }
  if (run_event && n_runs > 0) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(buf + o_rev, run_event, sizeof(int32_t) * (size_t)n_runs, cudaMemcpyHostToDevice, s));
  }
  if (n_labels > 0) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(buf + o_lab, labels, sizeof(itsu_label) * (size_t)n_labels, cudaMemcpyHostToDevice, s));
    ITSU_CUDA(ctx, cudaMemcpyAsync(buf + o_lev, label_event.data(), sizeof(int32_t) * (size_t)n_labels, cudaMemcpyHostToDevice, s));
  }
  ITSU_CUDA(ctx, cudaMemcpyAsync(buf + o_tb, table_base.data(), sizeof(int64_t) * ((size_t)n_events + 1), cudaMemcpyHostToDevice, s));
  itsu::launch_report(r, s, ctx->num_sms);
  ITSU_CUDA(ctx, cudaGetLastError());
  if (road_class && n_roads > 0) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(road_class, r.road_class, (size_t)n_roads, cudaMemcpyDeviceToHost, s));
  }
  if (counts && n_events > 0) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(counts, r.counts, sizeof(itsu_report_counts) * (size_t)n_events, cudaMemcpyDeviceToHost, s));
  }
  ITSU_CUDA(ctx, cudaStreamSynchronize(s));
  return ITSU_OK;
}

}  // extern "C"

namespace {

constexpr int kMaxChunks = 16;
constexpr int64_t kChunkClusters = 1500000;  // default clusters per streamed chunk (about 34 central Pb-Pb-like events)

template <typename T>
itsu_status grow_buffer(itsu_context *ctx, T *&p, int64_t &cap, int64_t need)
{
  if (need > cap) {
    const int64_t c = grow_to(need);
    ITSU_CUDA(ctx, alloc(ctx, p, c));
    cap = c;
  }
  return ITSU_OK;
}

// The streamed path's second arena: a context on the same device with its own stream, the
// parent's flags (less ITSU_FLAG_STREAM_HOST) and initial capacities. Created on first use.
itsu_status ensure_twin(itsu_context *ctx)
{
  if (ctx->twin) return ITSU_OK;
  itsu_config c;
  itsu_config_default(&c);
  c.device = ctx->device;
  c.flags = ctx->flags & ~ITSU_FLAG_STREAM_HOST;
  c.max_tracklets = ctx->init_tracklets;
  c.max_cells = ctx->init_cells;
  c.max_neighbours = ctx->init_neighbours;
  c.max_roads = ctx->init_roads;
  itsu_context *t = nullptr;
  const itsu_status st = itsu_context_create(&c, &t);
  if (st != ITSU_OK) return fail(ctx, st, "streamed run: second arena: %s", g_thread_error.c_str());
  ctx->twin = t;
  return ITSU_OK;
}

// itsu_batch_run_host with ITSU_FLAG_STREAM_HOST: consecutive chunks of events, each one's
// upload (copy stream) overlapping the work on the ones before, and each one's roads downloaded
// (download stream) while later ones work. Chunks alternate between the context's arena and
// stream and a second arena with its own stream, so two chunks are in flight and one's small
// tail kernels overlap the next one's work; their roads are appended to the batch-wide output in
// chunk order. The first chunk is smaller, so that the device starts sooner. Sets *done to false,
// with nothing reported, when the batch is too small to split or a chunk outgrew its arena: the
// caller then runs the batch in one pass (which grows the arena).
// The host's raw clusters in one of the record formats: 36-byte itsu_cluster, 24-byte
// itsu_cluster_in or 16-byte itsu_cluster_track.
struct HostClusters {
  const itsu_cluster *full = nullptr;
  const itsu_cluster_in *compact = nullptr;
  const itsu_cluster_track *track = nullptr;
  bool any() const { return full || compact || track; }
};

// Uploads host clusters [a, b) to the context's raw buffer of their format (asynchronous on s).
itsu_status upload_clusters(itsu_context *ctx, const HostClusters &h, int64_t a, int64_t b, cudaStream_t s)
{
  if (b <= a) return ITSU_OK;
  if (h.track) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->raw_track + a, h.track + a, sizeof(itsu_cluster_track) * (b - a), cudaMemcpyHostToDevice, s));
  } else if (h.compact) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->raw_in + a, h.compact + a, sizeof(itsu_cluster_in) * (b - a), cudaMemcpyHostToDevice, s));
  } else {
    ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->raw + a, h.full + a, sizeof(itsu_cluster) * (b - a), cudaMemcpyHostToDevice, s));
  }
  return ITSU_OK;
}

// A run's inputs start at cluster a of the context's raw buffer of the format.
void point_inputs_at(itsu_context *x, const itsu_context *owner, const HostClusters &h, int64_t a)
{
  x->in_raw = h.full ? owner->raw + a : nullptr;
  x->in_raw_in = h.compact ? owner->raw_in + a : nullptr;
  x->in_raw_track = h.track ? owner->raw_track + a : nullptr;
}

itsu_status run_host_streamed(itsu_context *ctx, const HostClusters &clusters, const int32_t *layer_offsets, const float *vertices,
                              int32_t n_events, int64_t n_clusters, itsu_road *roads, int64_t roads_capacity,
                              int32_t *road_offsets, bool *done)
{
  *done = false;
  const int64_t per_chunk = ctx->chunk_clusters > 0 ? ctx->chunk_clusters : kChunkClusters;
  const int k_chunks = (int)std::min<int64_t>(std::min<int64_t>(kMaxChunks - 1, n_events), (n_clusters + per_chunk - 1) / per_chunk);
  if (k_chunks < 2) return ITSU_OK;
  // chunk boundaries (events): cluster shares 0.4 : 1 : 1 : ... (the first one small)
  constexpr double kFirst = 0.4;
  std::vector<int32_t> ev(k_chunks + 1, 0);
  ev[k_chunks] = n_events;
  for (int c = 1, e = 0; c < k_chunks; ++c) {
    const int64_t target = (int64_t)((double)n_clusters * (kFirst + (c - 1)) / (kFirst + (k_chunks - 1)));
    while (e < n_events && layer_offsets[(int64_t)e * ITSU_LAYERS] < target) ++e;
    ev[c] = std::max(e, ev[c - 1] + 1);
  }
  for (int c = 1; c <= k_chunks; ++c) {
    if (ev[c] <= ev[c - 1]) return ITSU_OK;  // degenerate split: one pass instead
  }
  int64_t max_chunk = 0;
  int32_t max_chunk_events = 0;
  for (int c = 0; c < k_chunks; ++c) {
    max_chunk = std::max<int64_t>(max_chunk, layer_offsets[(int64_t)ev[c + 1] * ITSU_LAYERS] - layer_offsets[(int64_t)ev[c] * ITSU_LAYERS]);
    max_chunk_events = std::max(max_chunk_events, ev[c + 1] - ev[c]);
  }
  itsu_status st;
  if ((st = ensure_clusters(ctx, n_clusters, n_events)) != ITSU_OK) return st;
  if ((st = ensure_outputs_for(ctx, max_chunk)) != ITSU_OK) return st;
  // the second arena (not for a fixed-size arena: that one stays as the caller configured it)
  itsu_context *twin = nullptr;
  if (!(ctx->flags & ITSU_FLAG_NO_GROW)) {
    if ((st = ensure_twin(ctx)) != ITSU_OK) return st;
    twin = ctx->twin;
    if ((st = ensure_clusters(twin, max_chunk, max_chunk_events)) != ITSU_OK) return fail(ctx, st, "%s", twin->error.c_str());
    if ((st = ensure_outputs_for(twin, max_chunk)) != ITSU_OK) return fail(ctx, st, "%s", twin->error.c_str());
    for (int b = 0; b < kBands; ++b) twin->tunes[b] = ctx->tunes[b];
    twin->override_tune = ctx->override_tune;
    twin->tuning = ctx->tuning;
  }
  if ((st = grow_buffer(ctx, ctx->chunk_off, ctx->cap_chunk_off, (int64_t)n_events * ITSU_LAYERS + k_chunks)) != ITSU_OK) return st;
  if ((st = grow_buffer(ctx, ctx->roads_all, ctx->cap_roads_all, std::max<int64_t>(ctx->cap_roads, n_clusters / 2 + 4096))) != ITSU_OK) {
    return st;
  }
  if ((st = grow_buffer(ctx, ctx->road_off_all, ctx->cap_road_off_all, (int64_t)n_events + 1)) != ITSU_OK) return st;
  if (!ctx->chunk_status) ITSU_CUDA(ctx, cudaMalloc((void **)&ctx->chunk_status, sizeof(DevStatus) * kMaxChunks));
  if (!ctx->h_chunk_status) ITSU_CUDA(ctx, cudaMallocHost((void **)&ctx->h_chunk_status, sizeof(DevStatus) * kMaxChunks));
  if (!ctx->h_road_end) ITSU_CUDA(ctx, cudaMallocHost((void **)&ctx->h_road_end, sizeof(int32_t) * kMaxChunks));
  if (!ctx->copy_stream) ITSU_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  if (!ctx->d2h_stream) ITSU_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->d2h_stream, cudaStreamNonBlocking));
  for (int c = 0; c < kMaxChunks; ++c) {
    if (!ctx->chunk_ready[c]) ITSU_CUDA(ctx, cudaEventCreateWithFlags(&ctx->chunk_ready[c], cudaEventDisableTiming));
    if (!ctx->chunk_done[c]) ITSU_CUDA(ctx, cudaEventCreateWithFlags(&ctx->chunk_done[c], cudaEventDisableTiming));
  }
  // each chunk's layer offsets, rebased (chunk c at 7 ev[c] + c), staged in pinned memory so that
  // their upload is asynchronous
  const int64_t n_off = (int64_t)n_events * ITSU_LAYERS + k_chunks;
  if (n_off > ctx->cap_h_chunk_off) {
    if (ctx->h_chunk_off) cudaFreeHost(ctx->h_chunk_off);
    ctx->h_chunk_off = nullptr;
    ctx->cap_h_chunk_off = 0;
    ITSU_CUDA(ctx, cudaMallocHost((void **)&ctx->h_chunk_off, sizeof(int32_t) * grow_to(n_off)));
    ctx->cap_h_chunk_off = grow_to(n_off);
  }
  // the previous call finished with a synchronisation: the staging buffers are free to refill
  for (int c = 0; c < k_chunks; ++c) {
    const int32_t base = layer_offsets[(int64_t)ev[c] * ITSU_LAYERS];
    for (int64_t k = (int64_t)ev[c] * ITSU_LAYERS; k <= (int64_t)ev[c + 1] * ITSU_LAYERS; ++k) {
      ctx->h_chunk_off[k + c] = layer_offsets[k] - base;
    }
  }
  // All uploads go on the copy stream, the small ones first: host-to-device copies share the copy
  // engine in submission order, so a small copy queued behind the clusters would hold up the
  // first chunk's work. The copy, download and second-arena streams first wait for any earlier
  // work of the context and for the zeroed road offsets.
  ITSU_CUDA(ctx, cudaMemsetAsync(ctx->road_off_all, 0, sizeof(int32_t) * ((int64_t)n_events + 1), ctx->stream));
  cudaEvent_t start = ctx->chunk_ready[kMaxChunks - 1];
  ITSU_CUDA(ctx, cudaEventRecord(start, ctx->stream));
  ITSU_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, start, 0));
  ITSU_CUDA(ctx, cudaStreamWaitEvent(ctx->d2h_stream, start, 0));
  if (twin) ITSU_CUDA(ctx, cudaStreamWaitEvent(twin->stream, start, 0));
  ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->chunk_off, ctx->h_chunk_off, sizeof(int32_t) * n_off, cudaMemcpyHostToDevice, ctx->copy_stream));
  ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->vtx, vertices, sizeof(float) * 3 * (int64_t)n_events, cudaMemcpyHostToDevice, ctx->copy_stream));
  for (int c = 0; c < k_chunks; ++c) {
    const int64_t a = layer_offsets[(int64_t)ev[c] * ITSU_LAYERS], b = layer_offsets[(int64_t)ev[c + 1] * ITSU_LAYERS];
    if ((st = upload_clusters(ctx, clusters, a, b, ctx->copy_stream)) != ITSU_OK) return st;
    ITSU_CUDA(ctx, cudaEventRecord(ctx->chunk_ready[c], ctx->copy_stream));
  }

  // The work, all chunks enqueued at once: per chunk (on its arena's stream, after its upload),
  // the whole sequence, then (after the previous chunk's append, which wrote this chunk's first
  // road index) its roads appended to the batch-wide output and its road end and status sent
  // back. The two arenas alternate; a stream runs its chunks in order, so an arena is reused only
  // after its previous chunk's append.
  for (int c = 0; c < k_chunks; ++c) {
    itsu_context *x = (twin && (c & 1)) ? twin : ctx;
    const int64_t a = layer_offsets[(int64_t)ev[c] * ITSU_LAYERS], b = layer_offsets[(int64_t)ev[c + 1] * ITSU_LAYERS];
    ITSU_CUDA(ctx, cudaStreamWaitEvent(x->stream, ctx->chunk_ready[c], 0));
    x->n_events = ev[c + 1] - ev[c];
    x->n_clusters = b - a;
    point_inputs_at(x, ctx, clusters, a);
    x->in_raw_off = nullptr;
    x->in_layer_off = ctx->chunk_off + (int64_t)ev[c] * ITSU_LAYERS + c;
    x->in_vtx = ctx->vtx + 3 * (int64_t)ev[c];
    Arena arena = arena_of(x);
    arena.mlp = ctx->prefilter ? ctx->d_mlp : nullptr;  // the context's models serve both arenas
    arena.gate = ctx->gate ? ctx->d_gate : nullptr;
    Launch l = launch_of(x);
    std::vector<int64_t> bounds;  // the chunk's event groups (read while its launches are enqueued)
    const int group = current_tune(x).group;
    group_bounds(ctx->h_chunk_off + (int64_t)ev[c] * ITSU_LAYERS + c, x->n_events, x->n_clusters, group, bounds);
    attach_groups(l, bounds, group);
    enqueue_run(arena, l);
    if (c > 0 && twin) ITSU_CUDA(ctx, cudaStreamWaitEvent(x->stream, ctx->chunk_done[c - 1], 0));
    itsu::launch_append_roads(arena, l, ctx->roads_all, ctx->road_off_all, ev[c], ctx->cap_roads_all, ctx->chunk_status + c);
    ITSU_CUDA(ctx, cudaGetLastError());
    ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->h_chunk_status + c, ctx->chunk_status + c, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                   x->stream));
    ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->h_road_end + c, ctx->road_off_all + ev[c + 1], sizeof(int32_t), cudaMemcpyDeviceToHost,
                                   x->stream));
    ITSU_CUDA(ctx, cudaEventRecord(ctx->chunk_done[c], x->stream));
  }

  // Each finished chunk's status is checked, in chunk order, and its roads go to the host on the
  // download stream while later chunks work. A chunk that outgrew its arena ends the streaming
  // (the chunks after it ran, but their roads are not downloaded) and the batch runs in one pass.
  int64_t downloaded = 0;
  bool fallback = false;
  int fail_chunk = -1;
  st = ITSU_OK;
  for (int c = 0; c < k_chunks && st == ITSU_OK && !fallback; ++c) {
    const cudaError_t err = cudaEventSynchronize(ctx->chunk_done[c]);
    if (err != cudaSuccess) {
      st = fail(ctx, ITSU_ERR_CUDA, "streamed run: chunk %d: %s", c, cudaGetErrorString(err));
      break;
    }
    const DevStatus &s = ctx->h_chunk_status[c];
    if (s.flags & itsu::kFlagInvalid) {
      if (s.invalid_event != INT32_MAX) {
        st = fail(ctx, ITSU_ERR_INVALID, "primary vertex of event %d is not finite or beyond 1e6 cm", ev[c] + s.invalid_event);
      } else {
        st = fail(ctx, ITSU_ERR_INVALID, "cluster %lld is malformed: a coordinate is not finite or beyond 1e6 cm, or it sits on the beam line at the vertex z (r == 0 and z == vertex z)",
                  (long long)layer_offsets[(int64_t)ev[c] * ITSU_LAYERS] + s.invalid_index);
      }
      break;
    }
    if (s.flags & itsu::kCapacityMask) {
      fallback = true;  // one pass instead, which grows the arena
      fail_chunk = c;
      break;
    }
    const int64_t end = ctx->h_road_end[c];
    if (roads && end > roads_capacity) {
      st = fail(ctx, ITSU_ERR_CAPACITY, "%lld roads do not fit the %lld given", (long long)end, (long long)roads_capacity);
      break;
    }
    if (roads && end > downloaded) {
      const cudaError_t e1 = cudaStreamWaitEvent(ctx->d2h_stream, ctx->chunk_done[c], 0);
      const cudaError_t e2 = e1 != cudaSuccess ? e1
                                               : cudaMemcpyAsync(roads + downloaded, ctx->roads_all + downloaded,
                                                                 sizeof(itsu_road) * (end - downloaded), cudaMemcpyDeviceToHost,
                                                                 ctx->d2h_stream);
      if (e2 != cudaSuccess) {
        st = fail(ctx, ITSU_ERR_CUDA, "streamed run: road download: %s", cudaGetErrorString(e2));
        break;
      }
    }
    downloaded = end;
  }
  for (itsu_context *x : {ctx, twin}) {
    if (!x) continue;
    x->stage = kNone;  // the arenas hold only their last chunk's intermediate results
    x->n_events = 0;
    x->n_clusters = 0;
  }
  if (st == ITSU_OK && !fallback && road_offsets) {
    const cudaError_t e1 = cudaStreamWaitEvent(ctx->d2h_stream, ctx->chunk_done[k_chunks - 1], 0);
    const cudaError_t e2 = e1 != cudaSuccess ? e1
                                             : cudaMemcpyAsync(road_offsets, ctx->road_off_all, sizeof(int32_t) * ((int64_t)n_events + 1),
                                                               cudaMemcpyDeviceToHost, ctx->d2h_stream);
    if (e2 != cudaSuccess) st = fail(ctx, ITSU_ERR_CUDA, "streamed run: offsets download: %s", cudaGetErrorString(e2));
  }
  // whatever happened, nothing of this call is left in flight
  const cudaError_t e1 = cudaStreamSynchronize(ctx->stream);
  const cudaError_t e2 = cudaStreamSynchronize(ctx->d2h_stream);
  const cudaError_t e3 = cudaStreamSynchronize(ctx->copy_stream);
  const cudaError_t e4 = twin ? cudaStreamSynchronize(twin->stream) : cudaSuccess;
  if (st != ITSU_OK) return st;
  ITSU_CUDA(ctx, e1);
  ITSU_CUDA(ctx, e2);
  ITSU_CUDA(ctx, e3);
  ITSU_CUDA(ctx, e4);
  if (fail_chunk >= 0 && !(ctx->flags & ITSU_FLAG_NO_GROW)) {
    // the arena that overflowed grows to the counted totals of the stage that overflowed, so that
    // later calls stream again (one stage per call when several are short)
    itsu_context *x = (twin && (fail_chunk & 1)) ? twin : ctx;
    const DevStatus &s = ctx->h_chunk_status[fail_chunk];
    itsu_status g = ITSU_OK;
    if (g == ITSU_OK && (s.flags & itsu::kFlagCapTracklets)) g = ensure_tracklets(x, s.total[itsu::kTracklets]);
    if (g == ITSU_OK && (s.flags & itsu::kFlagCapScratch)) g = ensure_cell_entries(x, s.cell_entries + cell_entry_slack(x));
    if (g == ITSU_OK && (s.flags & itsu::kFlagCapCells)) g = ensure_cells(x, s.total[itsu::kCells]);
    if (g == ITSU_OK && (s.flags & itsu::kFlagCapNeighbours)) g = ensure_neighbours(x, s.total[itsu::kNeighbours]);
    if (g == ITSU_OK && (s.flags & itsu::kFlagCapRoads)) g = ensure_roads(x, s.total[itsu::kRoads]);
    if (g != ITSU_OK) return x == ctx ? g : fail(ctx, g, "%s", x->error.c_str());
  }
  *done = !fallback;
  return ITSU_OK;
}

itsu_status batch_run_host(itsu_context *ctx, const HostClusters &clusters, const int32_t *layer_offsets, const float *vertices,
                           int32_t n_events, itsu_road *roads, int64_t roads_capacity, int32_t *road_offsets)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "null context");
  if (n_events < 0 || (n_events > 0 && (!layer_offsets || !vertices))) return fail(ctx, ITSU_ERR_INVALID, "bad batch arguments");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  const int64_t n_clusters = n_events > 0 ? layer_offsets[(int64_t)n_events * ITSU_LAYERS] : 0;
  if (n_clusters > 0 && !clusters.any()) return fail(ctx, ITSU_ERR_INVALID, "null clusters");
  if (layer_offsets && layer_offsets[0] != 0) return fail(ctx, ITSU_ERR_INVALID, "layer offsets must start at 0");
  for (int64_t k = 1; n_events > 0 && k <= (int64_t)n_events * ITSU_LAYERS; ++k) {
    if (layer_offsets[k] < layer_offsets[k - 1]) return fail(ctx, ITSU_ERR_INVALID, "layer offsets decrease at %lld", (long long)k);
  }
  itsu_status st;
  if ((st = ensure_clusters(ctx, n_clusters, n_events)) != ITSU_OK) return st;
  if (clusters.compact && (st = grow_buffer(ctx, ctx->raw_in, ctx->cap_raw_in, n_clusters)) != ITSU_OK) return st;
  if (clusters.track && (st = grow_buffer(ctx, ctx->raw_track, ctx->cap_raw_track, n_clusters)) != ITSU_OK) return st;
  if (ctx->flags & ITSU_FLAG_STREAM_HOST) {
    bool done = false;
    if ((st = run_host_streamed(ctx, clusters, layer_offsets, vertices, n_events, n_clusters, roads, roads_capacity, road_offsets,
                                &done)) != ITSU_OK) {
      return st;
    }
    if (done) return ITSU_OK;
  }
  if ((st = upload_clusters(ctx, clusters, 0, n_clusters, ctx->stream)) != ITSU_OK) return st;
  ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->layer_off, layer_offsets, sizeof(int32_t) * ((int64_t)n_events * ITSU_LAYERS + 1),
                                 cudaMemcpyHostToDevice, ctx->stream));
  ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->vtx, vertices, sizeof(float) * 3 * (int64_t)n_events, cudaMemcpyHostToDevice, ctx->stream));
  if ((st = ensure_outputs_for(ctx, n_clusters)) != ITSU_OK) return st;
  ctx->n_events = n_events;
  ctx->n_clusters = n_clusters;
  point_inputs_at(ctx, ctx, clusters, 0);
  ctx->in_raw_off = nullptr;
  ctx->in_layer_off = ctx->layer_off;
  ctx->in_vtx = ctx->vtx;
  ctx->h_layer_off.assign(layer_offsets, layer_offsets + (int64_t)n_events * ITSU_LAYERS + 1);
  if ((st = run_all(ctx)) != ITSU_OK) return st;
  const int64_t total = ctx->h_status->total[itsu::kRoads];
  if (road_offsets) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(road_offsets, ctx->road_seg, sizeof(int32_t) * ((int64_t)n_events + 1), cudaMemcpyDeviceToHost,
                                   ctx->stream));
  }
  if (roads) {
    if (total > roads_capacity) return fail(ctx, ITSU_ERR_CAPACITY, "%lld roads do not fit the %lld given", (long long)total, (long long)roads_capacity);
    if ((st = copy_range(ctx, roads, (const itsu_road *)ctx->roads, total)) != ITSU_OK) return st;
  }
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ITSU_OK;
}

}  // namespace

extern "C" {

itsu_status itsu_batch_run_host(itsu_context *ctx, const itsu_cluster *clusters, const int32_t *layer_offsets,
                                const float *vertices, int32_t n_events, itsu_road *roads, int64_t roads_capacity,
                                int32_t *road_offsets)
{
  HostClusters h;
  h.full = clusters;
  return batch_run_host(ctx, h, layer_offsets, vertices, n_events, roads, roads_capacity, road_offsets);
}

itsu_status itsu_batch_run_host_compact(itsu_context *ctx, const itsu_cluster_in *clusters, const int32_t *layer_offsets,
                                        const float *vertices, int32_t n_events, itsu_road *roads, int64_t roads_capacity,
                                        int32_t *road_offsets)
{
  HostClusters h;
  h.compact = clusters;
  return batch_run_host(ctx, h, layer_offsets, vertices, n_events, roads, roads_capacity, road_offsets);
}

itsu_status itsu_batch_run_host_tracks(itsu_context *ctx, const itsu_cluster_track *clusters, const int32_t *layer_offsets,
                                       const float *vertices, int32_t n_events, itsu_road *roads, int64_t roads_capacity,
                                       int32_t *road_offsets)
{
  HostClusters h;
  h.track = clusters;
  return batch_run_host(ctx, h, layer_offsets, vertices, n_events, roads, roads_capacity, road_offsets);
}

itsu_status itsu_frames_run_host(itsu_context *ctx, const itsu_frames *frames, itsu_road *roads, int64_t roads_capacity,
                                 int32_t *road_offsets)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "null context");
  if (!frames || frames->n_frames < 0 || frames->n_vertices < 0) return fail(ctx, ITSU_ERR_INVALID, "bad frames");
  const int32_t nf = frames->n_frames, nv = frames->n_vertices;
  if ((nf > 0 && !frames->frame_offsets) || (nv > 0 && (!frames->vertices || !frames->vertex_frame))) {
    return fail(ctx, ITSU_ERR_INVALID, "null frames pointer");
  }
  const int32_t *fo = frames->frame_offsets;
  const int64_t frame_clusters = nf > 0 ? fo[(int64_t)nf * ITSU_LAYERS] : 0;
  if (nf > 0 && fo[0] != 0) return fail(ctx, ITSU_ERR_INVALID, "frame offsets must start at 0");
  for (int64_t k = 1; k <= (int64_t)nf * ITSU_LAYERS; ++k) {
    if (fo[k] < fo[k - 1]) return fail(ctx, ITSU_ERR_INVALID, "frame offsets decrease at %lld", (long long)k);
  }
  if (frame_clusters > 0 && !frames->clusters) return fail(ctx, ITSU_ERR_INVALID, "null clusters");
  // one run per vertex over its frame's clusters: output layout per run, raw input shared
  std::vector<int32_t> run_off((size_t)nv * ITSU_LAYERS + 1, 0), raw_off((size_t)nv * ITSU_LAYERS, 0);
  int64_t total = 0;
  for (int32_t v = 0; v < nv; ++v) {
    const int32_t f = frames->vertex_frame[v];
    if (f < 0 || f >= nf) return fail(ctx, ITSU_ERR_INVALID, "vertex %d names frame %d of %d", v, f, nf);
    for (int l = 0; l < ITSU_LAYERS; ++l) {
      const int64_t k = (int64_t)v * ITSU_LAYERS + l;
      raw_off[k] = fo[(int64_t)f * ITSU_LAYERS + l];
      run_off[k] = (int32_t)total;
      total += fo[(int64_t)f * ITSU_LAYERS + l + 1] - fo[(int64_t)f * ITSU_LAYERS + l];
      if (total > INT32_MAX) return fail(ctx, ITSU_ERR_INVALID, "too many clusters over all vertices");
    }
  }
  run_off[(size_t)nv * ITSU_LAYERS] = (int32_t)total;
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  itsu_status st;
  if ((st = ensure_clusters(ctx, std::max(total, frame_clusters), nv)) != ITSU_OK) return st;
  if ((st = ensure_outputs_for(ctx, total)) != ITSU_OK) return st;
  if (frame_clusters > 0) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->raw, frames->clusters, sizeof(itsu_cluster) * frame_clusters, cudaMemcpyHostToDevice,
                                   ctx->stream));
  }
  ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->layer_off, run_off.data(), sizeof(int32_t) * run_off.size(), cudaMemcpyHostToDevice, ctx->stream));
  if (nv > 0) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->raw_off, raw_off.data(), sizeof(int32_t) * raw_off.size(), cudaMemcpyHostToDevice, ctx->stream));
    ITSU_CUDA(ctx, cudaMemcpyAsync(ctx->vtx, frames->vertices, sizeof(float) * 3 * (int64_t)nv, cudaMemcpyHostToDevice, ctx->stream));
  }
  ctx->n_events = nv;
  ctx->n_clusters = total;
  ctx->in_raw = ctx->raw;
  ctx->in_raw_in = nullptr;
  ctx->in_raw_track = nullptr;
  ctx->in_raw_off = ctx->raw_off;
  ctx->in_layer_off = ctx->layer_off;
  ctx->in_vtx = ctx->vtx;
  ctx->h_layer_off = run_off;
  if ((st = run_all(ctx)) != ITSU_OK) return st;
  const int64_t n_roads = ctx->h_status->total[itsu::kRoads];
  if (road_offsets) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(road_offsets, ctx->road_seg, sizeof(int32_t) * ((int64_t)nv + 1), cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (roads) {
    if (n_roads > roads_capacity) return fail(ctx, ITSU_ERR_CAPACITY, "%lld roads do not fit the %lld given", (long long)n_roads, (long long)roads_capacity);
    if ((st = copy_range(ctx, roads, (const itsu_road *)ctx->roads, n_roads)) != ITSU_OK) return st;
  }
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ITSU_OK;
}

itsu_status itsu_relaunch(itsu_context *ctx)
{
  itsu_status st;
  if ((st = require_stage(ctx, kRoads, "itsu_relaunch")) != ITSU_OK) return st;
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  return launch_all(ctx);
}

int32_t itsu_kernels_per_run(void) { return itsu::kernels_per_run(); }

itsu_status itsu_atan2f_device(itsu_context *ctx, const float *y, const float *x, float *out, int64_t n)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "itsu_atan2f_device: null context");
  if (n < 0 || (n > 0 && (!y || !x || !out))) return fail(ctx, ITSU_ERR_INVALID, "itsu_atan2f_device: bad arguments");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  itsu::launch_atan2f(y, x, out, n, ctx->num_sms, ctx->stream);
  ITSU_CUDA(ctx, cudaGetLastError());
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ITSU_OK;
}

int32_t itsu_multiplicity_band(int64_t n_clusters, int32_t n_events) { return band_of(n_clusters, n_events); }

itsu_status itsu_autotune(itsu_context *ctx, int32_t repeats, itsu_tune *best)
{
  itsu_status st;
  if ((st = require_stage(ctx, kRoads, "itsu_autotune")) != ITSU_OK) return st;
  if (repeats < 1) return fail(ctx, ITSU_ERR_INVALID, "repeats must be positive");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  int n = 0;
  const itsu::KernelStep *steps = itsu::pipeline_steps(&n);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ITSU_CUDA(ctx, cudaEventCreate(&e0));
  ITSU_CUDA(ctx, cudaEventCreate(&e1));
  Tune winner;
  winner.ms = 1e30f;
  const int blocks[] = {64, 128, 256, 512}, per_sm[] = {4, 8, 16}, prunes[] = {1, 2, 0}, groups[] = {0, 8, 16, 32};
  ctx->tuning = true;
  cudaError_t err = cudaSuccess;
  for (int b : blocks) {
    for (int m : per_sm) {
      for (int p : prunes) {
       for (int g : groups) {
        if (g > 0 && (p != 1 || g >= ctx->n_events)) continue;  // groups only with the plain pruning, below the batch
        ctx->override_tune = Tune{b, m, p, 0.0f, true, g};
        const Arena a = arena_of(ctx);
        const Launch l = whole_run_launch(ctx);
        float best_ms = 1e30f;
        for (int r = 0; r <= repeats && err == cudaSuccess; ++r) {  // the first pass warms up
          cudaEventRecord(e0, ctx->stream);
          for (int k = 0; k < n; ++k) steps[k].launch(a, l);
          cudaEventRecord(e1, ctx->stream);
          err = cudaStreamSynchronize(ctx->stream);
          float ms = 0;
          if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
          if (r > 0) best_ms = std::min(best_ms, ms);
        }
        if (err != cudaSuccess) break;
        if ((st = sync_status(ctx)) != ITSU_OK) break;
        if (ctx->h_status->flags == 0 && best_ms < winner.ms) {
          winner = ctx->override_tune;
          winner.ms = best_ms;
        }
       }
      }
    }
  }
  ctx->tuning = false;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ITSU_CUDA(ctx, err);
  if (st != ITSU_OK) return st;
  if (winner.ms >= 1e30f) return fail(ctx, ITSU_ERR_CAPACITY, "no candidate launch shape completed");
  const int band = band_of(ctx->n_clusters, ctx->n_events);
  ctx->tunes[band] = winner;
  drop_graph(ctx);
  // leave the arena holding this shape's results of the last run
  if ((st = run_all(ctx)) != ITSU_OK) return st;
  if (best) {
    best->band = band;
    best->threads_per_block = winner.block;
    best->blocks_per_sm = winner.blocks_per_sm;
    best->prune = winner.prune;
    best->ms = winner.ms;
    best->events_per_group = winner.group;
  }
  return ITSU_OK;
}

itsu_status itsu_get_tune(itsu_context *ctx, int32_t band, itsu_tune *out)
{
  if (!ctx || !out) return fail(ctx, ITSU_ERR_INVALID, "null argument");
  if (band < 0 || band >= kBands) return fail(ctx, ITSU_ERR_INVALID, "band %d out of range", band);
  const Tune &t = ctx->tunes[band];
  const Tune d;
  out->band = band;
  out->threads_per_block = t.set ? t.block : d.block;
  out->blocks_per_sm = t.set ? t.blocks_per_sm : d.blocks_per_sm;
  out->prune = t.set ? t.prune : d.prune;
  out->ms = t.set ? t.ms : 0.0f;
  out->events_per_group = t.set ? t.group : d.group;
  return ITSU_OK;
}

itsu_status itsu_set_tune(itsu_context *ctx, const itsu_tune *in)
{
  if (!ctx || !in) return fail(ctx, ITSU_ERR_INVALID, "null argument");
  if (in->band < 0 || in->band >= kBands) return fail(ctx, ITSU_ERR_INVALID, "band %d out of range", in->band);
  if (in->threads_per_block < 64 || in->threads_per_block > 512 || in->threads_per_block % 32 != 0 || in->blocks_per_sm < 1 ||
      in->blocks_per_sm > 32) {
    return fail(ctx, ITSU_ERR_INVALID, "launch shape %d threads x %d blocks/SM out of range", in->threads_per_block,
                in->blocks_per_sm);
  }
  if (in->events_per_group < 0) return fail(ctx, ITSU_ERR_INVALID, "events per group %d is negative", in->events_per_group);
  if (in->prune < 0 || in->prune > 2) return fail(ctx, ITSU_ERR_INVALID, "prune %d: 0, 1 or 2", in->prune);
  ctx->tunes[in->band] = Tune{in->threads_per_block, in->blocks_per_sm, in->prune, in->ms, true, in->events_per_group};
  drop_graph(ctx);
  return ITSU_OK;
}

itsu_status itsu_batch_profile(itsu_context *ctx, int32_t repeats, itsu_kernel_time *times, int32_t capacity, int32_t *count)
{
  itsu_status st;
  if ((st = require_stage(ctx, kRoads, "itsu_batch_profile")) != ITSU_OK) return st;
  if (repeats < 1 || !times || capacity < 0) return fail(ctx, ITSU_ERR_INVALID, "bad profile arguments");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  int n_all = 0;
  const itsu::KernelStep *all = itsu::pipeline_steps(&n_all);
  const Arena a = arena_of(ctx);
  const Launch l = whole_run_launch(ctx);
  std::vector<itsu::KernelStep> steps;  // the steps that launch a kernel in this context's form
  for (int k = 0; k < n_all; ++k) {
    const int only = all[k].learned_only;
    if (only == 0 || (only == itsu::kPairPrefilterStep && ctx->prefilter) || (only == itsu::kGateStep && ctx->gate) ||
        (only == itsu::kGroupedStep && l.n_groups > 0) || (only == itsu::kUngroupedStep && l.n_groups == 0)) {
      steps.push_back(all[k]);
    }
  }
  const int n = (int)steps.size();
  std::vector<cudaEvent_t> ev(n + 1, nullptr);
  std::vector<double> total(n, 0.0);
  for (auto &e : ev) {
    ITSU_CUDA(ctx, cudaEventCreate(&e));
  }
  cudaError_t err = cudaSuccess;
  for (int r = 0; r < repeats && err == cudaSuccess; ++r) {
    cudaEventRecord(ev[0], ctx->stream);
    for (int k = 0; k < n; ++k) {
      steps[k].launch(a, l);
      cudaEventRecord(ev[k + 1], ctx->stream);
    }
    err = cudaStreamSynchronize(ctx->stream);
    for (int k = 0; k < n && err == cudaSuccess; ++k) {
      float ms = 0.0f;
      err = cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
      total[k] += ms;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  ITSU_CUDA(ctx, err);
  if ((st = sync_status(ctx)) != ITSU_OK) return st;
  if (ctx->h_status->flags) return fail(ctx, ITSU_ERR_CAPACITY, "profile run did not complete (flags %d)", ctx->h_status->flags);
  const int m = std::min(n, (int)capacity);
  for (int k = 0; k < m; ++k) {
    std::memset(times[k].name, 0, sizeof times[k].name);
    std::strncpy(times[k].name, steps[k].name, sizeof times[k].name - 1);
    times[k].ms = (float)(total[k] / repeats);
    times[k].launches = repeats;
  }
  if (count) *count = n;
  return ITSU_OK;
}

}  // extern "C"

// ---- learned prefilter ----

namespace {

uint64_t host_splitmix64(uint64_t &state)
{
  uint64_t z = (state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// binary32 -> bfloat16, round to nearest even (NaN stays a quiet NaN)
uint16_t host_bf16(float f)
{
  uint32_t u;
  std::memcpy(&u, &f, sizeof u);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

uint64_t fnv1a64(const unsigned char *p, size_t n, uint64_t h = 0xcbf29ce484222325ull)
{
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 0x100000001b3ull;
  }
  return h;
}

// The two learned networks: the pair prefilter (itsu_prefilter_model) and the tracklet gate
// (itsu_gate_model) share their checkpoint format, training loop and host calls; NetOf<Model>
// names what differs.
template <class Model>
struct NetOf;

template <>
struct NetOf<itsu_prefilter_model> {
  using Model = itsu_prefilter_model;
  using Device = itsu::MlpDevice;
  static constexpr int kHidden = ITSU_MLP_HIDDEN;
  static constexpr int kParams = ITSU_MLP_PARAMS;
  static constexpr char kMagic[8] = {'I', 'T', 'S', 'U', 'M', 'L', 'P', '1'};
  static constexpr const char *kName = "prefilter";
  static Model *&master(itsu_context *c) { return c->d_master; }
  static Device *&device(itsu_context *c) { return c->d_mlp; }
  static bool &has(itsu_context *c) { return c->has_model; }
  static bool &enabled(itsu_context *c) { return c->prefilter; }
  static size_t device_bytes() { return itsu::mlp_device_bytes(); }
};

template <>
struct NetOf<itsu_gate_model> {
  using Model = itsu_gate_model;
  using Device = itsu::GateDevice;
  static constexpr int kHidden = ITSU_GATE_HIDDEN;
  static constexpr int kParams = ITSU_GATE_PARAMS;
  static constexpr char kMagic[8] = {'I', 'T', 'S', 'U', 'G', 'A', 'T', '4'};
  static constexpr const char *kName = "gate";
  static Model *&master(itsu_context *c) { return c->d_gate_master; }
  static Device *&device(itsu_context *c) { return c->d_gate; }
  static bool &has(itsu_context *c) { return c->has_gate; }
  static bool &enabled(itsu_context *c) { return c->gate; }
  static size_t device_bytes() { return itsu::gate_device_bytes(); }
};

constexpr uint32_t kCheckpointVersion = 1;

template <class Model>
constexpr uint32_t bf16_count()
{
  constexpr int H = NetOf<Model>::kHidden;
  return H * ITSU_MLP_INPUTS + H * H + H;
}

struct CheckpointHeader {
  char magic[8];
  uint32_t version, n_params, model_bytes, n_bf16;
};

// The BF16 copies of w1, w2, w3 in that order.
template <class Model>
std::vector<uint16_t> bf16_weights(const Model &m)
{
  constexpr int H = NetOf<Model>::kHidden;
  std::vector<uint16_t> out;
  out.reserve(bf16_count<Model>());
  for (int o = 0; o < H; ++o)
    for (int i = 0; i < ITSU_MLP_INPUTS; ++i) out.push_back(host_bf16(m.w1[o][i]));
  for (int o = 0; o < H; ++o)
    for (int i = 0; i < H; ++i) out.push_back(host_bf16(m.w2[o][i]));
  for (int i = 0; i < H; ++i) out.push_back(host_bf16(m.w3[i]));
  return out;
}

template <typename T>
struct DeviceScratch {  // a temporary device allocation freed on scope exit
  T *p = nullptr;
  ~DeviceScratch() { if (p) cudaFree(p); }
};

template <class Model>
itsu_status require_net(itsu_context *ctx, const char *what)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "%s: null context", what);
  if (!NetOf<Model>::has(ctx)) return fail(ctx, ITSU_ERR_STATE, "%s: no %s model set", what, NetOf<Model>::kName);
  return ITSU_OK;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

template <class Model>
void net_init(Model *model, uint64_t seed)
{
  constexpr int H = NetOf<Model>::kHidden;
  if (!model) return;
  std::memset(model, 0, sizeof *model);
  uint64_t state = seed;
  auto uniform = [&](float limit) {
    const double u = (double)(host_splitmix64(state) >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
    return (float)((2.0 * u - 1.0) * limit);
  };
  // Glorot-uniform limits sqrt(6 / (fan_in + fan_out))
  const float l1 = (float)std::sqrt(6.0 / (ITSU_MLP_INPUTS + H));
  const float l2 = (float)std::sqrt(6.0 / (2 * H));
  const float l3 = (float)std::sqrt(6.0 / (H + 1));
  for (int o = 0; o < H; ++o)
    for (int i = 0; i < ITSU_MLP_INPUTS; ++i) model->w1[o][i] = uniform(l1);
  for (int o = 0; o < H; ++o)
    for (int i = 0; i < H; ++i) model->w2[o][i] = uniform(l2);
  for (int i = 0; i < H; ++i) model->w3[i] = uniform(l3);
  for (int i = 0; i < ITSU_MLP_INPUTS; ++i) model->inv_std[i] = 1.0f;
  model->logit_threshold = 0.0f;
  if constexpr (std::is_same<Model, itsu_gate_model>::value) {
    for (int l = 0; l < ITSU_TRACKLET_LAYERS; ++l) {  // no first stage
      model->dphi_window[l] = 3.14159265358979323846f;
      model->dz_window[l] = HUGE_VALF;
    }
    model->mlp_layers = (1 << ITSU_TRACKLET_LAYERS) - 1;
  }
}

template <class Model>
itsu_status net_save(const Model *model, const char *path, const char *what)
{
  if (!model || !path) return fail(nullptr, ITSU_ERR_INVALID, "%s: null argument", what);
  CheckpointHeader h;
  std::memcpy(h.magic, NetOf<Model>::kMagic, sizeof h.magic);
  h.version = kCheckpointVersion;
  h.n_params = NetOf<Model>::kParams;
  h.model_bytes = sizeof(Model);
  h.n_bf16 = bf16_count<Model>();
  const std::vector<uint16_t> bf = bf16_weights(*model);
  std::vector<unsigned char> buf(sizeof h + sizeof *model + sizeof(uint16_t) * bf.size());
  std::memcpy(buf.data(), &h, sizeof h);
  std::memcpy(buf.data() + sizeof h, model, sizeof *model);
  std::memcpy(buf.data() + sizeof h + sizeof *model, bf.data(), sizeof(uint16_t) * bf.size());
  const uint64_t sum = fnv1a64(buf.data(), buf.size());
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(nullptr, ITSU_ERR_INVALID, "%s: cannot open %s", what, path);
  const bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size() && std::fwrite(&sum, sizeof sum, 1, f) == 1;
  if (std::fclose(f) != 0 || !ok) return fail(nullptr, ITSU_ERR_INVALID, "%s: write to %s failed", what, path);
  return ITSU_OK;
}

template <class Model>
itsu_status net_load(const char *path, Model *model, const char *what)
{
  if (!model || !path) return fail(nullptr, ITSU_ERR_INVALID, "%s: null argument", what);
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(nullptr, ITSU_ERR_INVALID, "%s: cannot open %s", what, path);
  const size_t body = sizeof(CheckpointHeader) + sizeof(Model) + sizeof(uint16_t) * bf16_count<Model>();
  std::vector<unsigned char> buf(body + sizeof(uint64_t) + 1);
  const size_t got = std::fread(buf.data(), 1, buf.size(), f);
  std::fclose(f);
  if (got != body + sizeof(uint64_t)) {
    return fail(nullptr, ITSU_ERR_INVALID, "%s: %s has %zu bytes, a checkpoint has %zu", what, path, got, body + sizeof(uint64_t));
  }
  CheckpointHeader h;
  std::memcpy(&h, buf.data(), sizeof h);
  if (std::memcmp(h.magic, NetOf<Model>::kMagic, sizeof h.magic) != 0 || h.version != kCheckpointVersion ||
      h.n_params != (uint32_t)NetOf<Model>::kParams || h.model_bytes != sizeof(Model) || h.n_bf16 != bf16_count<Model>()) {
    return fail(nullptr, ITSU_ERR_INVALID, "%s: %s is not a version-%u %s checkpoint", what, path, kCheckpointVersion,
                NetOf<Model>::kName);
  }
  uint64_t sum;
  std::memcpy(&sum, buf.data() + body, sizeof sum);
  if (fnv1a64(buf.data(), body) != sum) return fail(nullptr, ITSU_ERR_INVALID, "%s: %s: checksum mismatch", what, path);
  Model m;
  std::memcpy(&m, buf.data() + sizeof h, sizeof m);
  const std::vector<uint16_t> bf = bf16_weights(m);
  if (std::memcmp(bf.data(), buf.data() + sizeof h + sizeof m, sizeof(uint16_t) * bf.size()) != 0) {
    return fail(nullptr, ITSU_ERR_INVALID, "%s: %s: BF16 weights do not match the FP32 master", what, path);
  }
  *model = m;
  return ITSU_OK;
}

template <class Model>
itsu_status net_set_model(itsu_context *ctx, const Model *model, const char *what)
{
  using N = NetOf<Model>;
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "%s: null context", what);
  if (!model) return fail(ctx, ITSU_ERR_INVALID, "%s: null model", what);
  if constexpr (std::is_same<Model, itsu_gate_model>::value) {
    for (int l = 0; l < ITSU_TRACKLET_LAYERS; ++l) {
      // NaN or negative: the window would drop every tracklet
      if (!(model->dphi_window[l] >= 0.0f) || !(model->dz_window[l] >= 0.0f)) {
        return fail(ctx, ITSU_ERR_INVALID, "%s: window of layer %d (dphi %g, dz %g) is not a window", what, l,
                    (double)model->dphi_window[l], (double)model->dz_window[l]);
      }
    }
    if (model->mlp_layers < 0 || model->mlp_layers >= (1 << ITSU_TRACKLET_LAYERS)) {
      return fail(ctx, ITSU_ERR_INVALID, "%s: mlp_layers 0x%x names layers beyond %d", what, (unsigned)model->mlp_layers,
                  ITSU_TRACKLET_LAYERS - 1);
    }
  }
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!N::master(ctx)) ITSU_CUDA(ctx, cudaMalloc((void **)&N::master(ctx), sizeof(Model)));
  if (!N::device(ctx)) ITSU_CUDA(ctx, cudaMalloc((void **)&N::device(ctx), N::device_bytes()));
  ITSU_CUDA(ctx, cudaMemcpyAsync(N::master(ctx), model, sizeof *model, cudaMemcpyHostToDevice, ctx->stream));
  itsu::launch_mlp_publish(N::master(ctx), N::device(ctx), ctx->stream);
  ITSU_CUDA(ctx, cudaGetLastError());
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  N::has(ctx) = true;
  return ITSU_OK;
}

template <class Model>
itsu_status net_get_model(itsu_context *ctx, Model *model, const char *what)
{
  itsu_status st;
  if ((st = require_net<Model>(ctx, what)) != ITSU_OK) return st;
  if (!model) return fail(ctx, ITSU_ERR_INVALID, "%s: null model", what);
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  ITSU_CUDA(ctx, cudaMemcpyAsync(model, NetOf<Model>::master(ctx), sizeof *model, cudaMemcpyDeviceToHost, ctx->stream));
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ITSU_OK;
}

template <class Model>
itsu_status net_enable(itsu_context *ctx, int32_t enable, const char *what)
{
  if (!ctx) return fail(nullptr, ITSU_ERR_INVALID, "%s: null context", what);
  if (enable && !NetOf<Model>::has(ctx)) return fail(ctx, ITSU_ERR_STATE, "%s: no %s model set", what, NetOf<Model>::kName);
  NetOf<Model>::enabled(ctx) = enable != 0;
  return ITSU_OK;
}

template <class Model>
itsu_status net_score(itsu_context *ctx, const float *features, int64_t n, float *logits, const char *what)
{
  itsu_status st;
  if ((st = require_net<Model>(ctx, what)) != ITSU_OK) return st;
  if (n < 0 || (n > 0 && (!features || !logits))) return fail(ctx, ITSU_ERR_INVALID, "%s: bad arguments", what);
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  itsu::launch_mlp_score(NetOf<Model>::device(ctx), features, n, logits, ctx->num_sms, ctx->stream);
  ITSU_CUDA(ctx, cudaGetLastError());
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ITSU_OK;
}

template <class Model>
itsu_status net_train(itsu_context *ctx, const float *features, const uint8_t *labels, int64_t n, const itsu_train_config *cfg,
                      float *losses, const char *what)
{
  using N = NetOf<Model>;
  itsu_status st;
  if ((st = require_net<Model>(ctx, what)) != ITSU_OK) return st;
  if (!cfg || !features || !labels || n <= 0) return fail(ctx, ITSU_ERR_INVALID, "%s: bad arguments", what);
  if (cfg->steps < 0 || cfg->batch <= 0 || cfg->batch % 32 != 0 || !(cfg->lr >= 0.0f) || !(cfg->lr_final >= 0.0f) ||
      !(cfg->beta1 >= 0.0f && cfg->beta1 < 1.0f) || !(cfg->beta2 >= 0.0f && cfg->beta2 < 1.0f) || !(cfg->eps > 0.0f)) {
    return fail(ctx, ITSU_ERR_INVALID, "%s: bad configuration", what);
  }
  if (!aligned16(features)) return fail(ctx, ITSU_ERR_INVALID, "%s: features must be 16-byte aligned", what);
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  const int blocks = itsu::mlp_gradient_blocks(cfg->batch);
  DeviceScratch<float> partials, m, v, loss;
  ITSU_CUDA(ctx, cudaMalloc((void **)&partials.p, sizeof(float) * blocks * N::kParams));
  ITSU_CUDA(ctx, cudaMalloc((void **)&m.p, sizeof(float) * N::kParams));
  ITSU_CUDA(ctx, cudaMalloc((void **)&v.p, sizeof(float) * N::kParams));
  ITSU_CUDA(ctx, cudaMalloc((void **)&loss.p, sizeof(float) * std::max<int64_t>(cfg->steps, 1)));
  ITSU_CUDA(ctx, cudaMemsetAsync(m.p, 0, sizeof(float) * N::kParams, ctx->stream));
  ITSU_CUDA(ctx, cudaMemsetAsync(v.p, 0, sizeof(float) * N::kParams, ctx->stream));
  ITSU_CUDA(ctx, cudaMemsetAsync(loss.p, 0, sizeof(float) * std::max<int64_t>(cfg->steps, 1), ctx->stream));
  double b1t = 1.0, b2t = 1.0;
  for (int64_t step = 0; step < cfg->steps; ++step) {
    // cosine decay from lr to lr_final
    const double frac = cfg->steps > 1 ? (double)step / (double)(cfg->steps - 1) : 0.0;
    const float lr = (float)(cfg->lr_final + 0.5 * (cfg->lr - cfg->lr_final) * (1.0 + std::cos(3.14159265358979323846 * frac)));
    b1t *= cfg->beta1;
    b2t *= cfg->beta2;
    itsu::launch_mlp_gradient(N::device(ctx), features, labels, n, cfg->batch, false, cfg->seed, step, cfg->pos_weight, partials.p,
                              loss.p + step, ctx->stream);
    itsu::launch_mlp_adam(N::master(ctx), partials.p, blocks, m.p, v.p, lr, cfg->beta1, cfg->beta2, cfg->eps, cfg->weight_decay,
                          (float)(1.0 - b1t), (float)(1.0 - b2t), N::device(ctx), ctx->stream);
    if ((step & 1023) == 0) ITSU_CUDA(ctx, cudaGetLastError());
  }
  ITSU_CUDA(ctx, cudaGetLastError());
  if (losses && cfg->steps > 0) {
    ITSU_CUDA(ctx, cudaMemcpyAsync(losses, loss.p, sizeof(float) * cfg->steps, cudaMemcpyDeviceToHost, ctx->stream));
  }
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ITSU_OK;
}

template <class Model>
itsu_status net_gradient(itsu_context *ctx, const float *features, const uint8_t *labels, int64_t n, float pos_weight, float *grad,
                         float *loss_out, const char *what)
{
  using N = NetOf<Model>;
  itsu_status st;
  if ((st = require_net<Model>(ctx, what)) != ITSU_OK) return st;
  if (!features || !labels || !grad || n <= 0 || n > INT32_MAX - 31) return fail(ctx, ITSU_ERR_INVALID, "%s: bad arguments", what);
  if (!aligned16(features)) return fail(ctx, ITSU_ERR_INVALID, "%s: features must be 16-byte aligned", what);
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  const int32_t batch = (int32_t)n;
  const int blocks = itsu::mlp_gradient_blocks(batch);
  DeviceScratch<float> partials, loss;
  ITSU_CUDA(ctx, cudaMalloc((void **)&partials.p, sizeof(float) * blocks * N::kParams));
  ITSU_CUDA(ctx, cudaMalloc((void **)&loss.p, sizeof(float)));
  ITSU_CUDA(ctx, cudaMemsetAsync(loss.p, 0, sizeof(float), ctx->stream));
  itsu::launch_mlp_gradient(N::device(ctx), features, labels, n, batch, true, 0, 0, pos_weight, partials.p, loss.p, ctx->stream);
  ITSU_CUDA(ctx, cudaGetLastError());
  std::vector<float> h((size_t)blocks * N::kParams);
  float l = 0.0f;
  ITSU_CUDA(ctx, cudaMemcpyAsync(h.data(), partials.p, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
  ITSU_CUDA(ctx, cudaMemcpyAsync(&l, loss.p, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < N::kParams; ++i) {
    double sum = 0.0;
    for (int b = 0; b < blocks; ++b) sum += h[(size_t)b * N::kParams + i];
    grad[i] = (float)sum;
  }
  if (loss_out) *loss_out = l;
  return ITSU_OK;
}

}  // namespace

extern "C" {

static_assert(sizeof(itsu_prefilter_model) == sizeof(float) * (ITSU_MLP_PARAMS + 2 * ITSU_MLP_INPUTS + 1), "model layout");
static_assert(ITSU_MLP_PARAMS == itsu::kMlpParams, "parameter count");
static_assert(ITSU_GATE_PARAMS == itsu::kGateParams && ITSU_GATE_HIDDEN == itsu::kGateHidden, "gate parameter count");

void itsu_prefilter_init(itsu_prefilter_model *model, uint64_t seed) { net_init(model, seed); }
void itsu_gate_init(itsu_gate_model *model, uint64_t seed) { net_init(model, seed); }

void itsu_train_config_default(itsu_train_config *cfg)
{
  if (!cfg) return;
  std::memset(cfg, 0, sizeof *cfg);
  cfg->steps = 20000;
  cfg->batch = 8192;
  cfg->lr = 2e-3f;
  cfg->lr_final = 1e-4f;
  cfg->beta1 = 0.9f;
  cfg->beta2 = 0.999f;
  cfg->eps = 1e-8f;
  cfg->weight_decay = 0.0f;
  cfg->pos_weight = 1.0f;
  cfg->seed = 1;
}

itsu_status itsu_prefilter_save(const itsu_prefilter_model *model, const char *path) { return net_save(model, path, "itsu_prefilter_save"); }
itsu_status itsu_gate_save(const itsu_gate_model *model, const char *path) { return net_save(model, path, "itsu_gate_save"); }
itsu_status itsu_prefilter_load(const char *path, itsu_prefilter_model *model) { return net_load(path, model, "itsu_prefilter_load"); }
itsu_status itsu_gate_load(const char *path, itsu_gate_model *model) { return net_load(path, model, "itsu_gate_load"); }

itsu_status itsu_prefilter_set_model(itsu_context *ctx, const itsu_prefilter_model *model)
{
  return net_set_model(ctx, model, "itsu_prefilter_set_model");
}
itsu_status itsu_gate_set_model(itsu_context *ctx, const itsu_gate_model *model) { return net_set_model(ctx, model, "itsu_gate_set_model"); }
itsu_status itsu_prefilter_get_model(itsu_context *ctx, itsu_prefilter_model *model)
{
  return net_get_model(ctx, model, "itsu_prefilter_get_model");
}
itsu_status itsu_gate_get_model(itsu_context *ctx, itsu_gate_model *model) { return net_get_model(ctx, model, "itsu_gate_get_model"); }
itsu_status itsu_prefilter_enable(itsu_context *ctx, int32_t enable)
{
  return net_enable<itsu_prefilter_model>(ctx, enable, "itsu_prefilter_enable");
}
itsu_status itsu_gate_enable(itsu_context *ctx, int32_t enable) { return net_enable<itsu_gate_model>(ctx, enable, "itsu_gate_enable"); }

itsu_status itsu_prefilter_export(itsu_context *ctx, itsu_prefilter_samples *samples)
{
  itsu_status st;
  if ((st = require_stage(ctx, kRoads, "itsu_prefilter_export")) != ITSU_OK) return st;
  if (!samples) return fail(ctx, ITSU_ERR_INVALID, "itsu_prefilter_export: null samples");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  if ((st = sync_status(ctx)) != ITSU_OK) return st;
  const int64_t n_cells = ctx->h_status->total[itsu::kCells], n_roads = ctx->h_status->total[itsu::kRoads];
  samples->n_cells = n_cells;
  samples->n_roads = n_roads;
  if ((samples->features || samples->labels) && samples->capacity < n_cells) {
    return fail(ctx, ITSU_ERR_CAPACITY, "itsu_prefilter_export: %lld cells, room for %lld", (long long)n_cells,
                (long long)samples->capacity);
  }
  if ((samples->road_cells || samples->road_keys || samples->road_fake) && samples->road_capacity < n_roads) {
    return fail(ctx, ITSU_ERR_CAPACITY, "itsu_prefilter_export: %lld roads, room for %lld", (long long)n_roads,
                (long long)samples->road_capacity);
  }
  if (samples->features && !aligned16(samples->features)) {
    return fail(ctx, ITSU_ERR_INVALID, "itsu_prefilter_export: features must be 16-byte aligned");
  }
  itsu::launch_prefilter_export(arena_of(ctx), *samples, ctx->num_sms, ctx->stream);
  ITSU_CUDA(ctx, cudaGetLastError());
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ITSU_OK;
}

itsu_status itsu_gate_export(itsu_context *ctx, itsu_gate_samples *samples)
{
  itsu_status st;
  if ((st = require_stage(ctx, kRoads, "itsu_gate_export")) != ITSU_OK) return st;
  if (!samples) return fail(ctx, ITSU_ERR_INVALID, "itsu_gate_export: null samples");
  ITSU_CUDA(ctx, cudaSetDevice(ctx->device));
  if ((st = sync_status(ctx)) != ITSU_OK) return st;
  const int64_t n = ctx->h_status->total[itsu::kTracklets], n_roads = ctx->h_status->total[itsu::kRoads];
  samples->n_tracklets = n;
  samples->n_roads = n_roads;
  if ((samples->features || samples->labels) && samples->capacity < n) {
    return fail(ctx, ITSU_ERR_CAPACITY, "itsu_gate_export: %lld tracklets, room for %lld", (long long)n, (long long)samples->capacity);
  }
  if (samples->road_tracklets && samples->road_capacity < n_roads) {
    return fail(ctx, ITSU_ERR_CAPACITY, "itsu_gate_export: %lld roads, room for %lld", (long long)n_roads,
                (long long)samples->road_capacity);
  }
  if (samples->features && !aligned16(samples->features)) {
    return fail(ctx, ITSU_ERR_INVALID, "itsu_gate_export: features must be 16-byte aligned");
  }
  itsu::launch_gate_export(arena_of(ctx), *samples, ctx->num_sms, ctx->stream);
  ITSU_CUDA(ctx, cudaGetLastError());
  ITSU_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ITSU_OK;
}

itsu_status itsu_prefilter_score(itsu_context *ctx, const float *features, int64_t n, float *logits)
{
  return net_score<itsu_prefilter_model>(ctx, features, n, logits, "itsu_prefilter_score");
}
itsu_status itsu_gate_score(itsu_context *ctx, const float *features, int64_t n, float *logits)
{
  return net_score<itsu_gate_model>(ctx, features, n, logits, "itsu_gate_score");
}

itsu_status itsu_prefilter_train(itsu_context *ctx, const float *features, const uint8_t *labels, int64_t n,
                                 const itsu_train_config *cfg, float *losses)
{
  return net_train<itsu_prefilter_model>(ctx, features, labels, n, cfg, losses, "itsu_prefilter_train");
}
itsu_status itsu_gate_train(itsu_context *ctx, const float *features, const uint8_t *labels, int64_t n, const itsu_train_config *cfg,
                            float *losses)
{
  return net_train<itsu_gate_model>(ctx, features, labels, n, cfg, losses, "itsu_gate_train");
}

itsu_status itsu_prefilter_gradient(itsu_context *ctx, const float *features, const uint8_t *labels, int64_t n,
                                    float pos_weight, float *grad, float *loss_out)
{
  return net_gradient<itsu_prefilter_model>(ctx, features, labels, n, pos_weight, grad, loss_out, "itsu_prefilter_gradient");
}
itsu_status itsu_gate_gradient(itsu_context *ctx, const float *features, const uint8_t *labels, int64_t n, float pos_weight,
                               float *grad, float *loss_out)
{
  return net_gradient<itsu_gate_model>(ctx, features, labels, n, pos_weight, grad, loss_out, "itsu_gate_gradient");
}

}  // extern "C"
