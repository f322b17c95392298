// itsu_internal.h - device arena layout and kernel launchers shared by the C ABI layer.
//
// All results of a run live in flat, event-major device arrays; the single-vertex entry points
// are a batch of one event. Layout (E events, NC clusters, T tracklets, C cells):
//   layer_off[E*7+1]   cluster segment (event e, layer L) = [layer_off[7e+L], layer_off[7e+L+1])
//   sorted/xyzr/phi    clusters of each segment, stably sorted by index-table bin
//   index_tables       E*6 tables of 401 ints (table of layer L+1 at (6e+L)*401)
//   trk_count/trk_off  tracklets per inner cluster and their exclusive scan (NC+1)
//   trk_seg[E*6+1]     tracklet segment (e, L) = [trk_seg[6e+L], trk_seg[6e+L+1])
//   cell_count/off     cells per first tracklet and their scan (T+1); cell_seg[E*5+1]
//   nb_count/off       neighbours per next-layer cell and their scan (C+1): CSR over cells
//   road_count/off     roads per root cell and their scan (C+1); road_seg[E+1]
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "itsu.h"

namespace itsu {

template <int H>
struct MlpDeviceT;                   // a learned network as the device keeps it (itsu_mlp.cuh)
using MlpDevice = MlpDeviceT<64>;    // the tracklet-pair prefilter (8 -> 64 -> 64 -> 1, GELU)
using GateDevice = MlpDeviceT<16>;   // the tracklet gate (8 -> 16 -> 16 -> 1, ReLU)

enum : int32_t {
  kFlagInvalid = 1,
  kFlagCapTracklets = 2,
  kFlagCapCells = 4,
  kFlagCapNeighbours = 8,
  kFlagCapRoads = 16,
  kFlagCountOverflow = 32,
  kFlagCapScratch = 64,  // the cell entries of the count pass exceed their scratch
  kFlagLaunchShape = 128,  // a per-item pass was given a block size that is not whole warps (nothing ran)
  kFlagTimeout = 256,      // a bounded device wait gave up (the run's results are not used)
};
constexpr int kTrackletSlotsPerCluster = 48;  // outer clusters the tracklet count pass keeps per inner cluster
// Any of these stops every later kernel of the run (they check the mask first).
constexpr int32_t kCapacityMask = kFlagCapTracklets | kFlagCapCells | kFlagCapNeighbours | kFlagCapRoads |
                                  kFlagCountOverflow | kFlagCapScratch | kFlagLaunchShape | kFlagTimeout;
constexpr int kCellChunk = 64;  // cell entries a warp of the cell count pass reserves at a time

// Totals and requirements of a run, written by the device.
struct DevStatus {
  int32_t flags;
  int32_t invalid_index;  // first offending flat cluster index, INT32_MAX if none
  int32_t invalid_event;  // first event with a malformed vertex, INT32_MAX if none
  int32_t pad_;
  int64_t total[4];       // tracklets, cells, neighbours, roads
  int64_t cell_entries;   // cell entries reserved by the cell count pass (may exceed the scratch)
  int64_t crowded;        // tracklets the cell count pass listed in cell_crowded
  int64_t trk_crowded;    // inner clusters the tracklet count pass listed in clu_crowded
};
// The three list counters are reset together before each count pass (one 24-byte memset).
static_assert(offsetof(DevStatus, crowded) == offsetof(DevStatus, cell_entries) + 8 &&
                  offsetof(DevStatus, trk_crowded) == offsetof(DevStatus, cell_entries) + 16,
              "status counters");

// A cell as the count pass finds it: its first tracklet (flat) and the outgoing-tracklet bit it
// came from, and everything the cell record needs: its segment (5 e + L), its three clusters
// (local to layers L, L+1, L+2), its two tracklets (local to tracklet layers L and L+1), and what
// its geometry gave. The write pass scatters each entry whose bit survived to cell_off[t1] + (the
// rank of its bit among the tracklet's set bits) with no other gather; t1 < 0 marks an unused
// slot. The learned prefilter scores entries in place (the DCA, one of its features, goes to a
// separate array in that form only).
struct __align__(16) CellEntry {
  int32_t t1;
  int32_t bit;
  int32_t seg;
  int32_t c1;
  int32_t c2, c3;
  int32_t t1_local, t2_local;
  float nx, ny, nz, curvature;
};
static_assert(sizeof(CellEntry) == 48, "cell entry layout");

enum TotalIndex { kTracklets = 0, kCells = 1, kNeighbours = 2, kRoads = 3 };

struct Arena {
  int32_t n_events;
  int32_t pad_;
  int64_t n_clusters;
  // inputs (raw clusters in one of three record formats: raw_track set means the 16-byte one,
  // raw_in the 24-byte one, else raw)
  const itsu_cluster *raw;
  const itsu_cluster_in *raw_in;
  const itsu_cluster_track *raw_track;
  const int32_t *raw_off;  // per (run, layer): start of its raw clusters; null = same as layer_off
  const int32_t *layer_off;
  const float *vtx;
  // clustering
  itsu_cluster *sorted;
  float4 *xyzr;
  float *phi;
  itsu_cluster *tmp;
  int32_t *index_tables;
  int32_t *clu_seg;  // per sorted cluster: its segment 7e + L (null: not wanted)
  int4 *clu_aux;     // per sorted cluster: id, alpha bits, MC id, bin (the clustering scatters them here)
  int32_t *clu_crowded;  // inner clusters with more than kTrackletSlotsPerCluster tracklets (count pass list)
  // candidate-pruning index (null: not built): per bin, the bin's clusters sorted by (z, index),
  // each with its r and phi for the cut;
  // per (event, layer) the r range of its clusters and whether all its bins are regular
  float4 *zs;  // (z, r, phi, sorted index as int bits)
  float2 *seg_rrange;
  int32_t *seg_regular;  // per segment: 0 if not regular, else the pass-mask words its largest bin needs
  int32_t prune_tracklets;  // use the index: 0 no, 1 yes, 2 yes, from a shared-memory copy (tuning knob; results are identical)
  // tracklets
  int32_t *trk_count;
  int32_t *trk_slots;  // slot n of inner cluster i at n * slot_stride + i: the outer clusters of its first tracklets
  int64_t slot_stride;
  int32_t *trk_off;
  int32_t *trk_lookup;
  int32_t *trk_seg;
  itsu_tracklet *tracklets;
  float2 *trk_slope;  // per tracklet its (tanL, phi) again, packed: the cell pass's precut reads only these
  int32_t *trk_seg_id;
  int4 *cell_seginfo;  // per tracklet segment, two records: {first cluster of L (-1: no cells), of L+1, of L+2,
                       // first tracklet of L}, {first tracklet of L+1, vertex x, y, z (float bits)}
  // cells
  int32_t *cell_count;
  unsigned long long *cell_mask;  // per first tracklet: which outgoing tracklets make cells
  int32_t *cell_off;
  int32_t *cell_lookup;
  int32_t *cell_crowded;  // tracklets whose outer cluster has more than 64 outgoing tracklets
  int32_t *cell_seg;
  itsu_cell *cells;
  int32_t *cell_seg_id;
  CellEntry *cell_entries;  // scratch of the cell count pass
  float *cell_dca;  // per entry, its DCA (written in the learned form only: a prefilter feature)
  int64_t cap_cell_entries;
  // neighbours, levels, roads
  int32_t *nb_count;
  int32_t *nb_off;
  int32_t *nb_fill;
  unsigned long long *nb_mask;  // per cell of layers 0-3: its candidates that pass the cut (up to 64)
  int32_t *nb;
  int64_t *paths;  // per cell: its chain count and level (chain_word)
  int32_t *road_count;
  int32_t *road_off;
  int32_t *road_seg;
  itsu_road *roads;
  // learned prefilter of the cell stage (null: the plain path)
  const MlpDevice *mlp;
  // learned gate of the tracklet stage (null: the plain path)
  const GateDevice *gate;
  // scan scratch and status
  int64_t *scan_partials;
  DevStatus *status;
  // capacities of the growable outputs
  int64_t cap_tracklets, cap_cells, cap_neighbours, cap_roads;
};

// Launch geometry shared by the grid-stride kernels.
struct Launch {
  cudaStream_t stream;
  int num_sms;
  int block;          // threads per block of the per-item kernels (64..512, a multiple of 32)
  int blocks_per_sm;  // grid of the grid-stride kernels, in blocks per SM
  // Event groups of a whole run (0 groups: none): the tracklet write and cell count passes run
  // group after group, group g over events [g * group_events, ...) and inner clusters
  // [groups[g], groups[g + 1]) (a host array of n_groups + 1 entries, read while launching).
  int n_groups = 0;
  int group_events = 0;
  const int64_t *groups = nullptr;
};

// Stage launchers (asynchronous on l.stream).
void launch_status_init(const Arena &a, const Launch &l);
void launch_atan2f(const float *y, const float *x, float *out, int64_t n, int num_sms, cudaStream_t stream);
void launch_cluster_sort(const Arena &a, const Launch &l);
void launch_tracklets_count(const Arena &a, const Launch &l);
void launch_tracklets_write(const Arena &a, const Launch &l);
void launch_cells_count(const Arena &a, const Launch &l);
void launch_cells_write(const Arena &a, const Launch &l);
void launch_neighbours_count(const Arena &a, const Launch &l);
void launch_neighbours_write(const Arena &a, const Launch &l);
void launch_roads_count(const Arena &a, const Launch &l);
void launch_roads_write(const Arena &a, const Launch &l);

// Streamed host runs: append the last run's roads and road offsets at event e0 of the batch-wide
// output, and snapshot its status.
void launch_append_roads(const Arena &a, const Launch &l, itsu_road *dst, int32_t *dst_off, int32_t e0, int64_t cap,
                         DevStatus *snap);

// The road report (itsu_report.cu): device buffers of one itsu_roads_report call.
struct ReportArgs {
  const itsu_road *roads;      // n_roads, run-major
  int64_t n_roads;
  const int32_t *run_offsets;  // n_runs + 1
  const int32_t *run_event;    // n_runs (null: run r is event r)
  int32_t n_runs;
  int32_t n_events;
  const itsu_label *labels;    // n_labels, event-major
  const int32_t *label_event;  // the event of each label
  int64_t n_labels;
  const int64_t *table_base;   // n_events + 1: event e's table at [table_base[e], table_base[e+1]), a power of two
  int64_t table_size;
  int32_t *keys;               // per slot: the Monte Carlo id (INT32_MIN: empty)
  int32_t *first_label;        // per slot: its first label entry
  int64_t *first_road;         // per slot: its first non-fake road
  int64_t *road_slot;          // per road: its label's slot, -1 if the label is not in the map
  int32_t *road_event;         // per road: its event
  uint8_t *road_class;         // per road: ITSU_ROAD_*
  itsu_report_counts *counts;  // per event
};
void launch_report(const ReportArgs &r, cudaStream_t stream, int num_sms);

// Every kernel of a run, in launch order, with its name (the instrumentation API times them
// one by one). The stage launchers above enqueue consecutive ranges of this table.
// KernelStep::learned_only: the forms a step launches in (0: every run)
enum : int { kPairPrefilterStep = 1, kGateStep = 2, kGroupedStep = 3, kUngroupedStep = 4 };
struct KernelStep {
  const char *name;
  void (*launch)(const Arena &, const Launch &);
  int learned_only;  // 0, or the only form that launches it: a learned network's (kPairPrefilterStep, kGateStep),
                     // runs with event groups (kGroupedStep) or without (kUngroupedStep)
};
const KernelStep *pipeline_steps(int *count);
int kernels_per_run();  // kernels one plain run launches (the learned form adds the learned_only steps)

// Learned networks (itsu_prefilter.cu), all asynchronous on `stream`; each call has an
// overload for the pair prefilter (itsu_prefilter_model, MlpDevice) and one for the tracklet gate
// (itsu_gate_model, GateDevice).
// The FP32 master parameters -> the device model (BF16 weights).
void launch_mlp_publish(const itsu_prefilter_model *master, MlpDevice *model, cudaStream_t stream);
void launch_mlp_publish(const itsu_gate_model *master, GateDevice *model, cudaStream_t stream);
// One training sample per cell of the last run: its pair features and whether a found road uses
// it; per road, its 5 cells as sample rows and its key (event, 7 layer-local cluster indices).
void launch_prefilter_export(const Arena &a, const itsu_prefilter_samples &out, int num_sms, cudaStream_t stream);
// One training sample per tracklet of the last run: its gate features and whether a found road
// uses it.
void launch_gate_export(const Arena &a, const itsu_gate_samples &out, int num_sms, cudaStream_t stream);
void launch_mlp_score(const MlpDevice *model, const float *features, int64_t n, float *logits, int num_sms, cudaStream_t stream);
void launch_mlp_score(const GateDevice *model, const float *features, int64_t n, float *logits, int num_sms, cudaStream_t stream);
// Mean-loss gradient of one minibatch: each block writes its partial sum of the gradient to
// grad_partials[block][params] (mlp_gradient_blocks(batch) blocks) and adds the batch loss
// to *loss. With sequential set the batch is samples 0..batch-1; otherwise `batch` samples drawn
// with replacement from n by (seed, step). features: 16-byte aligned rows of 8 floats.
void launch_mlp_gradient(const MlpDevice *model, const float *features, const uint8_t *labels, int64_t n, int32_t batch,
                         bool sequential, uint64_t seed, int64_t step, float pos_weight, float *grad_partials, float *loss,
                         cudaStream_t stream);
void launch_mlp_gradient(const GateDevice *model, const float *features, const uint8_t *labels, int64_t n, int32_t batch,
                         bool sequential, uint64_t seed, int64_t step, float pos_weight, float *grad_partials, float *loss,
                         cudaStream_t stream);
int mlp_gradient_blocks(int32_t batch);
int mlp_max_gradient_blocks();
// One Adam step on the master parameters from the summed partials, then publishes the device model.
void launch_mlp_adam(itsu_prefilter_model *master, const float *grad_partials, int blocks, float *m, float *v, float lr,
                     float beta1, float beta2, float eps, float weight_decay, float bias1, float bias2, MlpDevice *model,
                     cudaStream_t stream);
void launch_mlp_adam(itsu_gate_model *master, const float *grad_partials, int blocks, float *m, float *v, float lr, float beta1,
                     float beta2, float eps, float weight_decay, float bias1, float bias2, GateDevice *model, cudaStream_t stream);
size_t mlp_device_bytes();
size_t gate_device_bytes();

// Sets the calling thread's last error message (returned by itsu_last_error(NULL)).
void set_thread_error(const char *message);

}  // namespace itsu
