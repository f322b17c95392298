/*
 * itsu_oracle.h - CPU restatement of the reference tracker's hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA path is compared against; the product
 * library never links, loads or calls it. It restates, in plain C, the reference CPU Tracker
 * (src/CA/PrimaryVertexContext.cxx, src/CA/Tracker.cxx and the headers they use) with the
 * harness patches that make the reference well defined:
 *   P1 the inclusive candidate loop stops at the last cluster of the layer
 *      (Tracker.cxx:88 reads one element past the end otherwise);
 *   P2 the cells lookup table of layer L has one entry per tracklet of layer L
 *      (PrimaryVertexContext.cxx:70-73 sizes it from a memory coefficient instead);
 *   P3 clusters are sorted stably by bin, so ties keep input order (PrimaryVertexContext.cxx:52
 *      uses the unstable std::sort);
 *   P4 azimuths use the correctly rounded itsu_atan2f (include/itsu_atan2f.h).
 * It is pinned against the reference itself, compiled from its own sources with the same
 * patches (oracle/build_ref.sh), on seeded events and on the committed golden fixtures.
 */
#ifndef ITSU_ORACLE_H
#define ITSU_ORACLE_H

#include "../include/itsu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_result oracle_result;

/* Output kinds for oracle_size / oracle_data. */
enum {
  ORACLE_CLUSTERS = 0,         /* layer 0..6: sorted itsu_cluster */
  ORACLE_INDEX_TABLE = 1,      /* layer 0..5 (table of layer L+1): 401 int32 */
  ORACLE_TRACKLETS = 2,        /* layer 0..5: itsu_tracklet */
  ORACLE_TRACKLETS_LOOKUP = 3, /* layer 0..4: int32 per cluster of layer L+1 */
  ORACLE_CELLS = 4,            /* layer 0..4: itsu_cell */
  ORACLE_CELLS_LOOKUP = 5,     /* layer 0..3: int32 per tracklet of layer L+1 */
  ORACLE_NEIGHBOUR_OFFSETS = 6,/* layer 0..3: C_{L+1} + 1 int32 */
  ORACLE_NEIGHBOURS = 7,       /* layer 0..3: int32 */
  ORACLE_ROADS = 8             /* layer 0: itsu_road */
};

/* Runs the whole per-vertex path: initialize, tracklets, cells, neighbours, tracks, labels.
 * layers[L] holds counts[L] raw clusters. Returns NULL on allocation failure. */
oracle_result *oracle_run_vertex(const itsu_cluster *const layers[ITSU_LAYERS], const int32_t counts[ITSU_LAYERS],
                                 const float vertex[3]);
int64_t oracle_size(const oracle_result *res, int kind, int layer);
const void *oracle_data(const oracle_result *res, int kind, int layer);
void oracle_free(oracle_result *res);

/* Single-function hooks for unit tests. */
float oracle_atan2f(float y, float x);
void oracle_transform_cluster(int layer, const float vertex[3], const itsu_cluster *raw, itsu_cluster *out);

/* Timing helper for the CPU baseline: runs n_events events (one vertex each, batch layout of
 * itsu_batch in host memory) and returns the total number of roads. */
int64_t oracle_run_batch(const itsu_cluster *clusters, const int32_t *layer_offsets, const float *vertices,
                         int32_t n_events);

/* IOUtils::writeRoadsReport (IOUtils.cxx:125-170), its classification: same arguments and
 * outputs as itsu_roads_report with host roads (road_class and counts may be NULL). Returns 0, or
 * -1 on allocation failure. */
int oracle_roads_report(const itsu_road *roads, const int32_t *run_offsets, const int32_t *run_event, int32_t n_runs,
                        const itsu_label *labels, const int32_t *label_offsets, int32_t n_events, uint8_t *road_class,
                        itsu_report_counts *counts);

#ifdef __cplusplus
}
#endif

#endif
