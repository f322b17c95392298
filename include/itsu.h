/*
 * itsu.h - C ABI of the B200 ITS cellular-automaton track finder.
 *
 * This is the drop-in boundary for the hot path of the reference tracker: clustering into the
 * phi-z index table, tracklets, cells, neighbours / CA levels, roads and their Monte Carlo
 * labels. Plain pointers and sizes only. Every entry point returns an itsu_status; on failure
 * itsu_last_error() holds a one-line reason. The C++ facade in
 * tracking-itsu_b200/host/ maps statuses to std::runtime_error the way the reference does
 * (src/CA/gpu/cuda/Tracker.cu:326-335).
 *
 * Record layouts are the reference's, byte for byte:
 *   itsu_cluster  = Cluster   (include/ITSReconstruction/CA/Cluster.h:36-44)   36 bytes
 *   itsu_tracklet = Tracklet  (include/ITSReconstruction/CA/Tracklet.h:33-36)  16 bytes
 *   itsu_cell     = Cell      (include/ITSReconstruction/CA/Cell.h:47-54)      40 bytes
 *   itsu_road     = Road      (include/ITSReconstruction/CA/Road.h:47-50)      32 bytes
 * Indices inside records are local to their layer, as in the reference: a tracklet's cluster
 * indices index the SORTED clusters of layers L and L+1, a cell's tracklet indices index the
 * tracklets of layers L and L+1, a road's cell_ids[L] indexes the cells of layer L.
 */
#ifndef ITSU_H
#define ITSU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ITSU_LAYERS 7            /* Constants::ITS::LayersNumber (Constants.h:38) */
#define ITSU_TRACKLET_LAYERS 6   /* Constants::ITS::TrackletsPerRoad (Constants.h:39) */
#define ITSU_CELL_LAYERS 5       /* Constants::ITS::CellsPerRoad (Constants.h:40) */
#define ITSU_NEIGHBOUR_LAYERS 4  /* CellsPerRoad - 1 */
#define ITSU_Z_BINS 20           /* Constants::IndexTable::ZBins (Constants.h:77) */
#define ITSU_PHI_BINS 20         /* Constants::IndexTable::PhiBins (Constants.h:78) */
#define ITSU_INDEX_TABLE_SIZE 401 /* ZBins * PhiBins + 1 */
#define ITSU_UNUSED_INDEX (-1)   /* Constants::ITS::UnusedIndex (Constants.h:41) */

typedef struct itsu_cluster {
  float x, y, z;   /* global coordinates, cm */
  float phi;       /* azimuth about the primary vertex, [0, 2pi] (filled by clustering) */
  float r;         /* transverse distance to the primary vertex (filled by clustering) */
  int32_t cluster_id;
  float alpha;     /* sensor angle, carried through */
  int32_t mc_id;   /* Monte Carlo particle id, -1 for noise */
  int32_t bin;     /* phi-z index table bin (filled by clustering) */
} itsu_cluster;

/* A cluster as the caller delivers it, before clustering: the arguments of the reference's raw
 * constructor Cluster(clusterId, x, y, z, alpha, monteCarloId) (Cluster.cxx:27-33) without the
 * fields clustering computes (phi, r, bin), in 24 bytes instead of 36: the host-facing calls that
 * take it upload a third fewer bytes. */
typedef struct itsu_cluster_in {
  float x, y, z;
  int32_t cluster_id;
  float alpha;
  int32_t mc_id;
} itsu_cluster_in;

/* A cluster as a caller that wants only roads and their Monte Carlo labels delivers it: what the
 * tracking and the label vote read (coordinates and MC id), in 16 bytes. The sorted clusters of a
 * run fed these records carry the cluster's index in its layer's input order as cluster_id and 0
 * as alpha; every other output is the same as from the full records. */
typedef struct itsu_cluster_track {
  float x, y, z;
  int32_t mc_id;
} itsu_cluster_track;

typedef struct itsu_tracklet {
  int32_t first_cluster;  /* sorted index in layer L */
  int32_t second_cluster; /* sorted index in layer L+1 */
  float tan_lambda;
  float phi;
} itsu_tracklet;

typedef struct itsu_cell {
  int32_t first_cluster, second_cluster, third_cluster; /* layers L, L+1, L+2 */
  int32_t first_tracklet, second_tracklet;              /* tracklet layers L, L+1 */
  float nx, ny, nz;                                     /* unit normal of the circle plane */
  float curvature;
  int32_t level;                                        /* CA level, 1 + longest chain below */
} itsu_cell;

typedef struct itsu_road {
  int32_t cell_ids[ITSU_CELL_LAYERS]; /* cell index per cell layer, -1 if unused */
  int32_t size;
  int32_t label;   /* Moore-vote Monte Carlo label */
  uint8_t is_fake; /* C++ bool in the reference layout */
  uint8_t pad_[3];
} itsu_road;

typedef enum itsu_status {
  ITSU_OK = 0,
  ITSU_ERR_INVALID = 1,  /* malformed input or argument (rejected before any kernel runs) */
  ITSU_ERR_CAPACITY = 2, /* a result did not fit and the arena could not grow */
  ITSU_ERR_TIMEOUT = 3,  /* a bounded device wait gave up */
  ITSU_ERR_CUDA = 4,     /* a CUDA runtime call failed */
  ITSU_ERR_NOMEM = 5,    /* device or host allocation failed */
  ITSU_ERR_STATE = 6     /* call out of order (e.g. stage before initialize) */
} itsu_status;

/* Flags of itsu_config.flags */
#define ITSU_FLAG_NO_GROW 1u /* report ITSU_ERR_CAPACITY instead of growing and re-running */
/* itsu_batch_run_host streams: the batch runs as consecutive chunks of events, each chunk's
 * upload overlapping the work on the one before; only the roads and road offsets are kept
 * (the per-event results API then reports ITSU_ERR_STATE until the next run). */
#define ITSU_FLAG_STREAM_HOST 2u

typedef struct itsu_config {
  int32_t device;          /* CUDA device ordinal */
  uint32_t flags;
  int64_t max_clusters;    /* initial arena capacities; 0 = defaults. The arena grows on demand */
  int64_t max_tracklets;   /* unless ITSU_FLAG_NO_GROW is set. */
  int64_t max_cells;
  int64_t max_neighbours;
  int64_t max_roads;
  int32_t max_events;
  int32_t stream_chunk_clusters; /* ITSU_FLAG_STREAM_HOST: clusters per chunk (0 = 1,500,000) */
} itsu_config;

/* Per-vertex result sizes. */
typedef struct itsu_counts {
  int32_t clusters[ITSU_LAYERS];
  int32_t tracklets[ITSU_TRACKLET_LAYERS];
  int32_t cells[ITSU_CELL_LAYERS];
  int32_t neighbours[ITSU_NEIGHBOUR_LAYERS]; /* links between cell layers L and L+1 */
  int32_t roads;
} itsu_counts;

/* Host destinations for itsu_copy_results; any pointer may be NULL to skip that output.
 * Sizes follow itsu_counts:
 *   clusters[L]          N_L sorted clusters
 *   index_tables[L-1]    401 ints for layers L = 1..6 (PrimaryVertexContext::getIndexTables)
 *   tracklets[L]         T_L
 *   tracklets_lookup[L]  N_{L+1} ints for L = 0..4 (getTrackletsLookupTable): first tracklet of
 *                        layer L+1 whose first cluster is that cluster of layer L+1, else -1
 *   cells[L]             C_L (level filled in by neighbour finding)
 *   cells_lookup[L]      T_{L+1} ints for L = 0..3 (getCellsLookupTable): first cell of layer
 *                        L+1 built on that tracklet of layer L+1, else -1
 *   neighbour_offsets[L] C_{L+1} + 1 ints: CSR row starts over the cells of layer L+1
 *   neighbours[L]        counts.neighbours[L] ints: cells of layer L, ascending in each row
 *                        (getCellsNeighbours()[L][c] as a CSR)
 *   roads                counts.roads roads in the reference's emission order */
typedef struct itsu_results {
  itsu_cluster *clusters[ITSU_LAYERS];
  int32_t *index_tables[ITSU_TRACKLET_LAYERS];
  itsu_tracklet *tracklets[ITSU_TRACKLET_LAYERS];
  int32_t *tracklets_lookup[ITSU_CELL_LAYERS];
  itsu_cell *cells[ITSU_CELL_LAYERS];
  int32_t *cells_lookup[ITSU_NEIGHBOUR_LAYERS];
  int32_t *neighbour_offsets[ITSU_NEIGHBOUR_LAYERS];
  int32_t *neighbours[ITSU_NEIGHBOUR_LAYERS];
  itsu_road *roads;
} itsu_results;

/* Device-resident batch of events (one primary vertex each). */
typedef struct itsu_batch {
  const itsu_cluster *clusters;  /* device: raw clusters, event-major then layer-major */
  const int32_t *layer_offsets;  /* device: n_events*7 + 1 offsets into clusters */
  const float *vertices;         /* device: n_events*3 (x, y, z) */
  int32_t n_events;
  int32_t reserved_;
  int64_t n_clusters;            /* == layer_offsets[n_events*7] */
} itsu_batch;

typedef struct itsu_context itsu_context;

/* ---- library and context ---- */
const char *itsu_version(void);
const char *itsu_status_string(itsu_status status);
/* Last error message of the context (or of the thread when ctx is NULL). */
const char *itsu_last_error(const itsu_context *ctx);
void itsu_config_default(itsu_config *cfg);
itsu_status itsu_context_create(const itsu_config *cfg, itsu_context **out);
void itsu_context_destroy(itsu_context *ctx);
/* All work of the context is ordered on this stream (a cudaStream_t; NULL = a private stream). */
itsu_status itsu_context_set_stream(itsu_context *ctx, void *cuda_stream);
void *itsu_context_stream(const itsu_context *ctx);

/* ---- one primary vertex, stage by stage: the reference's per-vertex seam ----
 * Replaces PrimaryVertexContext::initialize(const Event&, int)
 *   (include/ITSReconstruction/CA/PrimaryVertexContext.h:51, src/CA/PrimaryVertexContext.cxx:31-142):
 * per-vertex cluster transform, stable sort by bin and the 6 index tables, on the device.
 * layers[L] points to counts[L] raw clusters in host memory. */
itsu_status itsu_pvc_initialize(itsu_context *ctx, const itsu_cluster *const layers[ITSU_LAYERS],
                                const int32_t counts[ITSU_LAYERS], const float vertex[3]);
/* Replaces TrackerTraits<IsGPU>::computeLayerTracklets(PrimaryVertexContext&)
 *   (include/ITSReconstruction/CA/Tracker.h:43,81; src/CA/Tracker.cxx:45-117;
 *    GPU form src/CA/gpu/cuda/Tracker.cu:285-367). */
itsu_status itsu_compute_layer_tracklets(itsu_context *ctx);
/* Replaces TrackerTraits<IsGPU>::computeLayerCells(PrimaryVertexContext&)
 *   (Tracker.h:44,82; Tracker.cxx:120-235; GPU form Tracker.cu:369-473). */
itsu_status itsu_compute_layer_cells(itsu_context *ctx);
/* Replaces Tracker<IsGPU>::findCellsNeighbours() (Tracker.h:69, Tracker.cxx:417-474). */
itsu_status itsu_find_cells_neighbours(itsu_context *ctx);
/* Replaces Tracker<IsGPU>::findTracks() + traverseCellsTree() (Tracker.h:70-71, Tracker.cxx:477-571). */
itsu_status itsu_find_tracks(itsu_context *ctx);
/* Replaces Tracker<IsGPU>::computeMontecarloLabels() (Tracker.h:72, Tracker.cxx:574-652). */
itsu_status itsu_compute_montecarlo_labels(itsu_context *ctx);

/* Sizes and host copies of the last run (event index e of a batch; 0 for the per-vertex API).
 * Replaces the PrimaryVertexContext getters (PrimaryVertexContext.h:52-77). */
itsu_status itsu_get_counts(itsu_context *ctx, int32_t event, itsu_counts *out);
itsu_status itsu_copy_results(itsu_context *ctx, int32_t event, const itsu_results *out);

/* Whole path for one vertex (Tracker<IsGPU>::clustersToTracks body for one vertex,
 * Tracker.cxx:251-262): host clusters in, roads out. roads may be NULL to query the count. */
itsu_status itsu_clusters_to_tracks(itsu_context *ctx, const itsu_cluster *const layers[ITSU_LAYERS],
                                    const int32_t counts[ITSU_LAYERS], const float vertex[3],
                                    itsu_road *roads, int32_t roads_capacity, int32_t *roads_count);

/* ---- batches: many events of uneven multiplicity in one pass of every stage ---- */
/* Runs every stage for every event of the batch and waits; grows the arena and re-runs
 * when a result overflowed (unless ITSU_FLAG_NO_GROW). */
itsu_status itsu_batch_run(itsu_context *ctx, const itsu_batch *batch);
/* Host in / host out: copies the batch to the device, runs it, and copies back the roads
 * (event-major) and road_offsets[n_events+1]. roads may be NULL to query the total. With
 * ITSU_FLAG_STREAM_HOST the batch runs as chunks of events whose copies overlap the work on
 * earlier chunks, two chunks in flight on two arenas (the context allocates its second arena
 * and stream on first use; pinned host buffers make the copies asynchronous). */
itsu_status itsu_batch_run_host(itsu_context *ctx, const itsu_cluster *clusters, const int32_t *layer_offsets,
                                const float *vertices, int32_t n_events, itsu_road *roads, int64_t roads_capacity,
                                int32_t *road_offsets);
/* itsu_batch_run_host with 24-byte input records (itsu_cluster_in): the same runs and results,
 * streamed the same way under ITSU_FLAG_STREAM_HOST. */
itsu_status itsu_batch_run_host_compact(itsu_context *ctx, const itsu_cluster_in *clusters, const int32_t *layer_offsets,
                                        const float *vertices, int32_t n_events, itsu_road *roads, int64_t roads_capacity,
                                        int32_t *road_offsets);
/* itsu_batch_run_host with 16-byte input records (itsu_cluster_track): the same roads, labels and
 * fake flags, streamed the same way under ITSU_FLAG_STREAM_HOST (two thirds of the compact upload). */
itsu_status itsu_batch_run_host_tracks(itsu_context *ctx, const itsu_cluster_track *clusters, const int32_t *layer_offsets,
                                       const float *vertices, int32_t n_events, itsu_road *roads, int64_t roads_capacity,
                                       int32_t *road_offsets);
/* Launches every stage of the batch on the context stream without waiting (CUDA-graph
 * replay after the first call with the same shape); itsu_batch_status waits and reports. */
itsu_status itsu_batch_launch(itsu_context *ctx, const itsu_batch *batch);
itsu_status itsu_batch_status(itsu_context *ctx);
/* Device pointer to the roads of the last batch (event-major) and to road_offsets[n_events+1]. */
itsu_status itsu_batch_roads_device(itsu_context *ctx, const itsu_road **roads, const int32_t **road_offsets);
/* Number of roads of the last batch or frames run (all its runs), read from the device. */
itsu_status itsu_batch_road_count(itsu_context *ctx, int64_t *n_roads);

/* ---- pile-up frames: several primary vertices over the same clusters ----
 * The reference tracks every vertex of an event over all of the event's clusters, running the
 * whole per-vertex sequence once per vertex (Tracker<IsGPU>::clustersToTracks, Tracker.cxx:251-262;
 * the pile-up merger of benchmarks/scripts/root/generatePileUpData.cxx builds such events).
 * Here each frame's clusters are uploaded once and every vertex becomes one run of the batch:
 * run v tracks vertex v over frame vertex_frame[v]. Host in / host out; per-run results through
 * itsu_get_counts / itsu_copy_results with event = v. */
typedef struct itsu_frames {
  const itsu_cluster *clusters; /* host: raw clusters, frame-major then layer-major */
  const int32_t *frame_offsets; /* host: n_frames*7 + 1 offsets into clusters */
  const float *vertices;        /* host: n_vertices*3 */
  const int32_t *vertex_frame;  /* host: n_vertices frame indices */
  int32_t n_frames;
  int32_t n_vertices;
} itsu_frames;
itsu_status itsu_frames_run_host(itsu_context *ctx, const itsu_frames *frames, itsu_road *roads, int64_t roads_capacity,
                                 int32_t *road_offsets);

/* Replays the whole sequence of the last run (any entry point) on the inputs already in device
 * memory, without waiting; itsu_batch_status waits and reports. */
itsu_status itsu_relaunch(itsu_context *ctx);

/* ---- road report: correct, duplicate and fake roads of each event ----
 * IOUtils::writeRoadsReport (src/CA/IOUtils.cxx:125-170) over the roads of every vertex of an event
 * and the event's labels map (IOUtils::loadLabels, IOUtils.cxx:80-123, keeps the particles with
 * |pdg| == 211 and 7 clusters). A road whose label is not in the map is not reported; one whose
 * label is in it is fake if the road is fake; otherwise it is correct when it is the first
 * non-fake road of its label in the event (vertex order, then road order) and a duplicate after
 * that. The classification runs on the device; the callers write the text streams
 * (host/itsu_ioutils.hpp IOUtils::writeRoadsReport, itsu/io.py write_roads_report). */
typedef struct itsu_label { /* Label (include/ITSReconstruction/CA/Label.h:27-40), same layout */
  int32_t mc_id;
  float pt, phi, eta;
  int32_t pdg;
  int32_t n_clusters;
} itsu_label;
#define ITSU_ROAD_UNREPORTED 0u
#define ITSU_ROAD_CORRECT 1u
#define ITSU_ROAD_DUPLICATE 2u
#define ITSU_ROAD_FAKE 3u
typedef struct itsu_report_counts {
  int32_t labels;    /* distinct Monte Carlo ids in the event's labels map */
  int32_t correct;   /* = labels found: the efficiency is correct / labels */
  int32_t duplicate;
  int32_t fake;
} itsu_report_counts;
/* roads, run_offsets: host, the roads of n_runs runs (vertices), run r's at
 * [run_offsets[r], run_offsets[r+1]); both NULL: the device-resident roads of the context's last
 * batch or frames run (n_runs must be its run count; not after a streamed host run, which keeps
 * no per-run results). run_event: host, the event of each run, non-decreasing (NULL: run r is
 * event r). labels, label_offsets: host, event e's labels map at [label_offsets[e],
 * label_offsets[e+1]) (a repeated mc id keeps its first entry, as std::unordered_map::emplace;
 * INT32_MIN is not a valid mc id). Outputs (host, each may be NULL): road_class[n_roads] (the
 * ITSU_ROAD_* class of each road) and counts[n_events]. */
itsu_status itsu_roads_report(itsu_context *ctx, const itsu_road *roads, const int32_t *run_offsets, const int32_t *run_event,
                              int32_t n_runs, const itsu_label *labels, const int32_t *label_offsets, int32_t n_events,
                              uint8_t *road_class, itsu_report_counts *counts);

/* ---- launch-shape autotuner for batches (no counterpart in the reference) ----
 * Runs are grouped in multiplicity bands: band = floor(log2(mean clusters per event)). For the
 * band of the last run, itsu_autotune times every candidate launch shape (threads per block of
 * the per-item kernels 64/128/256/512, resident blocks per SM of the grid-stride kernels 4/8/16,
 * the tracklet candidate index off/on/staged, event groups of 0/8/16/32 events) on the inputs
 * already resident, `repeats` times each, and
 * keeps the fastest for that band; later runs in the band use it. Results never depend on the
 * launch shape. itsu_get_tune / itsu_set_tune read and restore a band's entry (to persist a
 * tuned table). */
typedef struct itsu_tune {
  int32_t band;
  int32_t threads_per_block;
  int32_t blocks_per_sm;
  int32_t prune;  /* tracklet candidate pruning index off (0), on (1), or on and read from a
                     shared-memory copy of each block's rows made by one bulk copy (2) */
  float ms;       /* best time of one run of the tuned inputs, 0 if untuned */
  int32_t events_per_group; /* whole runs: the tracklet write and cell count passes run event group by
                               event group, so that a group's tracklets are still in L2 when its
                               cells gather them (0: all events at once) */
} itsu_tune;
int32_t itsu_multiplicity_band(int64_t n_clusters, int32_t n_events);
itsu_status itsu_autotune(itsu_context *ctx, int32_t repeats, itsu_tune *best);
itsu_status itsu_get_tune(itsu_context *ctx, int32_t band, itsu_tune *out);
itsu_status itsu_set_tune(itsu_context *ctx, const itsu_tune *in);

/* ---- instrumentation (no counterpart in the reference beyond its clock() stage timers,
 *      src/CA/Tracker.cxx:655-684) ---- */
typedef struct itsu_kernel_time {
  char name[40];
  float ms;      /* mean duration over the repeats, CUDA events on the context stream */
  int32_t launches;
} itsu_kernel_time;

/* Number of kernels one plain whole-path or batch run launches (the learned-prefilter form
 * launches one more, its scoring kernel). */
int32_t itsu_kernels_per_run(void);
/* The device's correctly rounded atan2 (include/itsu_atan2f.h, the azimuth of every cluster and
 * tracklet) on n device-resident argument pairs, out[i] = atan2(y[i], x[i]), on the context's
 * stream, synchronously: a self-check of the device build against the host's definition. */
itsu_status itsu_atan2f_device(itsu_context *ctx, const float *y, const float *x, float *out, int64_t n);
/* Re-runs the last batch `repeats` times with every kernel launched on its own and bracketed by
 * CUDA events on the context stream; fills up to `capacity` entries in launch order and sets
 * *count to the number of kernels of the context's form. Call after itsu_batch_run (or
 * itsu_batch_run_host) has sized the arena for that batch. */
itsu_status itsu_batch_profile(itsu_context *ctx, int32_t repeats, itsu_kernel_time *times, int32_t capacity,
                               int32_t *count);

/* ---- learned tracklet-pair prefilter (no counterpart in the reference) ----
 * A small MLP (8 -> 64 -> 64 -> 1, GELU, sigmoid output; BF16 weights and activations, FP32
 * accumulation) scores, inside the cell stage (the seam of TrackerTraits::computeLayerCells,
 * src/CA/Tracker.cxx:120-235), each tracklet pair that passes the exact cell cuts; a pair whose
 * logit is below the model's threshold does not become a cell. Its features, per pair: dphi, dz
 * and dtanL of the cell cuts (Tracker.cxx:161-171), the signed curvature of each tracklet's
 * circle through the primary vertex, the pair's DCA (Tracker.cxx:203-210), the inner layer
 * index and the first cluster's radius. The plain path is unchanged and stays the yardstick: a
 * learned run's cells are a subset of the plain run's, so its roads are plain roads. Training
 * labels come from plain runs (1 = the cell is on a found road). */
#define ITSU_MLP_INPUTS 8
#define ITSU_MLP_HIDDEN 64
/* trainable parameters: w1, b1, w2, b2, w3, b3, contiguous at the start of itsu_prefilter_model */
#define ITSU_MLP_PARAMS (ITSU_MLP_HIDDEN * ITSU_MLP_INPUTS + ITSU_MLP_HIDDEN + ITSU_MLP_HIDDEN * ITSU_MLP_HIDDEN + \
                         ITSU_MLP_HIDDEN + ITSU_MLP_HIDDEN + 1)
/* The FP32 master copy of a model; the device computes with BF16 copies of w1, w2, w3. */
typedef struct itsu_prefilter_model {
  float w1[ITSU_MLP_HIDDEN][ITSU_MLP_INPUTS]; /* [out][in] */
  float b1[ITSU_MLP_HIDDEN];
  float w2[ITSU_MLP_HIDDEN][ITSU_MLP_HIDDEN]; /* [out][in] */
  float b2[ITSU_MLP_HIDDEN];
  float w3[ITSU_MLP_HIDDEN];
  float b3;
  float mean[ITSU_MLP_INPUTS];    /* the network sees (feature - mean) * inv_std */
  float inv_std[ITSU_MLP_INPUTS];
  float logit_threshold;          /* a pair is kept unless its logit is below this */
} itsu_prefilter_model;

/* Device buffers that itsu_prefilter_export fills; every array may be NULL (then not written). */
typedef struct itsu_prefilter_samples {
  float *features;       /* [capacity][8]: the pair features of each cell of the last run */
  uint8_t *labels;       /* [capacity]: 1 if a found road uses the cell */
  int64_t capacity;      /* rows available; the export fails with ITSU_ERR_CAPACITY below n_cells */
  int32_t *road_cells;   /* [road_capacity][5]: each road's cells as sample rows, layers 0..4 */
  int32_t *road_keys;    /* [road_capacity][8]: each road's event and the layer-local sorted indices
                            of its 7 clusters, layers 0..6 */
  uint8_t *road_fake;    /* [road_capacity]: the road's fake flag (Moore vote, Tracker.cxx:574-652) */
  int64_t road_capacity;
  int64_t n_cells;       /* out: cells of the last run (rows in event, layer, cell order) */
  int64_t n_roads;       /* out: roads of the last run (in road order) */
} itsu_prefilter_samples;

typedef struct itsu_train_config {
  int64_t steps;          /* Adam steps */
  int32_t batch;          /* samples per step, a multiple of 32, drawn with replacement */
  int32_t reserved_;
  float lr;               /* peak learning rate; cosine decay to lr_final over the steps */
  float lr_final;
  float beta1, beta2, eps;
  float weight_decay;     /* decoupled, on the weight matrices only */
  float pos_weight;       /* loss weight of label-1 samples */
  uint64_t seed;          /* minibatch sampling */
} itsu_train_config;

/* Deterministic fresh model (host only): scaled-uniform weights from seed, zero biases, identity
 * standardisation, threshold 0 (probability 0.5). */
void itsu_prefilter_init(itsu_prefilter_model *model, uint64_t seed);
void itsu_train_config_default(itsu_train_config *cfg);
/* Checkpoint file: magic, sizes, the FP32 master model, the BF16 copies of its weights and a
 * 64-bit FNV-1a checksum. Loading verifies all of them (ITSU_ERR_INVALID on any mismatch). */
itsu_status itsu_prefilter_save(const itsu_prefilter_model *model, const char *path);
itsu_status itsu_prefilter_load(const char *path, itsu_prefilter_model *model);
/* The context's model (used by the learned form, the scorer and training). */
itsu_status itsu_prefilter_set_model(itsu_context *ctx, const itsu_prefilter_model *model);
itsu_status itsu_prefilter_get_model(itsu_context *ctx, itsu_prefilter_model *model);
/* Learned form on (1) or off (0) for later whole-path, batch and frames runs. Needs a model. */
itsu_status itsu_prefilter_enable(itsu_context *ctx, int32_t enable);
/* Training samples and road keys of the last whole-path / batch / frames run (after its roads). */
itsu_status itsu_prefilter_export(itsu_context *ctx, itsu_prefilter_samples *samples);
/* Logits of n feature rows (device pointers), with the same kernel code as the learned form. */
itsu_status itsu_prefilter_score(itsu_context *ctx, const float *features, int64_t n, float *logits);
/* Trains the context's model in place: cfg->steps Adam steps of binary cross-entropy on
 * minibatches of the n device samples (rows with non-finite features must be left out by the
 * caller). losses (host, may be NULL) receives each step's minibatch loss. */
itsu_status itsu_prefilter_train(itsu_context *ctx, const float *features, const uint8_t *labels, int64_t n,
                                 const itsu_train_config *cfg, float *losses);
/* Mean loss and its gradient over all n device samples at the current model (host outputs:
 * grad[ITSU_MLP_PARAMS] in itsu_prefilter_model order). */
itsu_status itsu_prefilter_gradient(itsu_context *ctx, const float *features, const uint8_t *labels, int64_t n,
                                    float pos_weight, float *grad, float *loss);

/* ---- learned tracklet gate (no counterpart in the reference) ----
 * The learned form's upstream stage: a smaller MLP (8 -> 16 -> 16 -> 1, ReLU, sigmoid output;
 * BF16 weights and activations, FP32 accumulation) scores every tracklet the tracklet stage finds
 * (the seam of TrackerTraits::computeLayerTracklets, src/CA/Tracker.cxx:45-117) before the
 * tracklets are written, and a tracklet whose logit is below the gate's threshold is not kept: the
 * cell stage then enumerates only pairs of kept tracklets (Tracker.cxx:133-158), where the plain
 * path spends most of its time. Its features, per tracklet: |dphi| and dphi of its clusters'
 * azimuths about the vertex, the tracklet cut's dz (Tracker.cxx:93-95) and |dz|, the signed
 * curvature of the circle through the vertex and its two clusters, the inner layer, the inner
 * cluster's radius and its slope from the vertex. The gate is a cascade: learned per-layer
 * windows on |dphi| and |dz| first (dphi_window, dz_window below), the network on the tracklets
 * inside them (of the layers in mlp_layers). Training labels come from plain runs (1 = the
 * tracklet is part of a found road). A learned run's tracklets, and so its cells and roads, are
 * subsets of the plain run's. Inner clusters with more than 48 tracklets inside the windows keep
 * all of them, unscored by the network.
 * The gate and the pair prefilter are enabled separately; the learned form is either or both. */
#define ITSU_GATE_HIDDEN 16
#define ITSU_GATE_PARAMS (ITSU_GATE_HIDDEN * ITSU_MLP_INPUTS + ITSU_GATE_HIDDEN + ITSU_GATE_HIDDEN * ITSU_GATE_HIDDEN + \
                          ITSU_GATE_HIDDEN + ITSU_GATE_HIDDEN + 1)
/* Same field order as itsu_prefilter_model, at the gate's width. */
typedef struct itsu_gate_model {
  float w1[ITSU_GATE_HIDDEN][ITSU_MLP_INPUTS]; /* [out][in] */
  float b1[ITSU_GATE_HIDDEN];
  float w2[ITSU_GATE_HIDDEN][ITSU_GATE_HIDDEN]; /* [out][in] */
  float b2[ITSU_GATE_HIDDEN];
  float w3[ITSU_GATE_HIDDEN];
  float b3;
  float mean[ITSU_MLP_INPUTS];
  float inv_std[ITSU_MLP_INPUTS];
  float logit_threshold;          /* a tracklet is kept unless its logit is below this */
  /* The cascade's first stage, learned from the training tracklets on found roads: per inner
   * layer, the largest |dphi| (the gate's feature 0) and |dz| (feature 2) a kept tracklet may
   * have. The tracklet count pass applies both to every tracklet it finds and walks only the phi
   * rows and z ranges they can reach; the network scores the tracklets inside them. pi and
   * infinity: no first stage. */
  float dphi_window[ITSU_TRACKLET_LAYERS];
  float dz_window[ITSU_TRACKLET_LAYERS];
  /* The layers the network scores: bit l set, inner layer l's tracklets inside the windows are
   * scored; clear, the windows alone decide for that layer. 0x3f: every layer. */
  int32_t mlp_layers;
} itsu_gate_model;

/* Device buffers that itsu_gate_export fills; every array may be NULL (then not written). */
typedef struct itsu_gate_samples {
  float *features;   /* [capacity][8]: the gate features of each tracklet of the last run */
  uint8_t *labels;   /* [capacity]: 1 if a found road uses the tracklet */
  int64_t capacity;  /* rows available; the export fails with ITSU_ERR_CAPACITY below n_tracklets */
  int32_t *road_tracklets; /* [road_capacity][6]: each road's tracklets as sample rows, layers 0..5 */
  int64_t road_capacity;
  int64_t n_tracklets; /* out: tracklets of the last run (rows in event, layer, tracklet order) */
  int64_t n_roads;     /* out: roads of the last run */
} itsu_gate_samples;

/* The gate's counterparts of the itsu_prefilter_* calls above, with the same semantics. */
void itsu_gate_init(itsu_gate_model *model, uint64_t seed);
itsu_status itsu_gate_save(const itsu_gate_model *model, const char *path);
itsu_status itsu_gate_load(const char *path, itsu_gate_model *model);
itsu_status itsu_gate_set_model(itsu_context *ctx, const itsu_gate_model *model);
itsu_status itsu_gate_get_model(itsu_context *ctx, itsu_gate_model *model);
itsu_status itsu_gate_enable(itsu_context *ctx, int32_t enable);
itsu_status itsu_gate_export(itsu_context *ctx, itsu_gate_samples *samples);
itsu_status itsu_gate_score(itsu_context *ctx, const float *features, int64_t n, float *logits);
itsu_status itsu_gate_train(itsu_context *ctx, const float *features, const uint8_t *labels, int64_t n,
                            const itsu_train_config *cfg, float *losses);
itsu_status itsu_gate_gradient(itsu_context *ctx, const float *features, const uint8_t *labels, int64_t n,
                               float pos_weight, float *grad, float *loss);

/* ---- arena occupancy ----
 * The reference preallocates each vertex's tracklet and cell vectors from coefficients of the
 * cluster counts (Constants::Memory, Constants.h:87-92; PrimaryVertexContext.cxx:59-73, 125-131)
 * and its memory benchmark prints capacity against use per vertex
 * (Tracker::clustersToTracksMemoryBenchmark, Tracker.cxx:304-363; itsu/io.py MemoryModel writes
 * that file from per-run counts). Here the count passes size the arena exactly (it grows to the
 * counted totals, across multiplicity bands); this reports what the arena holds against what the
 * last run used. */
typedef struct itsu_memory_usage {
  int64_t device_bytes;          /* arena buffers of the context and of its streamed second arena */
  int64_t clusters_capacity;     /* clusters and events the arena holds */
  int64_t events_capacity;
  int64_t capacity[4];           /* tracklets, cells, neighbours, roads the arena holds */
  int64_t used[4];               /* the last synchronised run's totals (0 before any) */
  int64_t cell_entries_capacity; /* the cell count pass's entry scratch */
} itsu_memory_usage;
itsu_status itsu_memory_usage_get(itsu_context *ctx, itsu_memory_usage *out);

/* ---- clustering without any allocation ----
 * No counterpart in the reference: its GPU backend allocates per call (gpu/Vector.h:97-122).
 * For callers that cannot call cudaMalloc (a process whose memory pool owns the device's memory,
 * or a latency-critical loop that cannot afford an allocation's implicit synchronisation), this
 * runs the clustering stage of one primary vertex (PrimaryVertexContext::initialize,
 * src/CA/PrimaryVertexContext.cxx:31-142) using only the caller's device buffers and a scratch
 * array of fixed size compiled into the library; it allocates nothing.
 *   clusters       device: n_clusters raw clusters, layer-major
 *   layer_offsets  device: 8 offsets, layer L = [layer_offsets[L], layer_offsets[L+1])
 *   vertex         device: x, y, z of the primary vertex
 *   sorted         device out: n_clusters clusters, per layer sorted stably by bin
 *   index_tables   device out: 6 x 401 ints (tables of layers 1..6)
 * At most ITSU_NOALLOC_MAX_CLUSTERS clusters (ITSU_ERR_CAPACITY beyond). Runs on cuda_stream on
 * the current device and waits for it, so no call can be captured into a CUDA graph; the first
 * call on a device looks up the scratch array's address, which is cached for the life of the
 * library: do not call this on a device after a cudaDeviceReset of it. All calls share the
 * scratch array: calls that overlap on the GPU race. Errors are reported through
 * itsu_last_error(NULL). */
#define ITSU_NOALLOC_MAX_CLUSTERS 65536
itsu_status itsu_pvc_initialize_noalloc(const itsu_cluster *clusters, const int32_t *layer_offsets, const float *vertex,
                                        int64_t n_clusters, itsu_cluster *sorted, int32_t *index_tables, void *cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* ITSU_H */
