// TrackerB200.cxx - the B200 backend of the reference tracker, behind its own seam.
//
// This translation unit is compiled together with the reference's sources (src/CA/*.cxx, their
// headers in include/) and linked against libitsu_b200.so. It supplies what the reference's
// backend seam asks of a device backend:
//   TrackerTraits<IsGPU>::computeLayerTracklets / computeLayerCells
//       (include/ITSReconstruction/CA/Tracker.h:39-48, 81-82; CPU bodies src/CA/Tracker.cxx:43-236,
//       CUDA bodies src/CA/gpu/cuda/Tracker.cu:285-473)
//   the backend step of PrimaryVertexContext::initialize
//       (src/CA/PrimaryVertexContext.cxx:87-141; CUDA mode: gpu/PrimaryVertexContext.h:39-42)
//
// The build defines TRACKINGITSU_B200 and keeps the reference's CPU data structures on the host
// (TRACKINGITSU_GPU_MODE stays false, so the tracker is Tracker<false> and its per-vertex context
// has the CPU members: index tables, tracklets and their lookup tables). Two edits to the
// reference select this backend, each guarded by TRACKINGITSU_B200:
//   Tracker.cxx:43                the CPU bodies of the two trait stages are left out (these
//                                 definitions replace them)
//   PrimaryVertexContext.cxx:141  at the end of the CPU branch of initialize, b200Initialize
//                                 (below) runs the clustering on the device
//
// Data flow per vertex, as the reference's CUDA mode leaves it (src/CA/gpu/cuda/Tracker.cu:
// 455-472): after computeLayerCells the cells and the cells lookup tables are in host memory for
// the reference's own findCellsNeighbours / findTracks / computeMontecarloLabels, which run on the
// host unchanged. The device's sorted clusters and index tables replace the host's after
// initialize (computeMontecarloLabels reads the clusters, Tracker.cxx:604-631; the memory benchmark
// their sizes, Tracker.cxx:317), and the tracklets and their lookup tables are copied into the CPU
// members after computeLayerTracklets (the memory benchmark reads them, Tracker.cxx:322-338).
//
// Errors become std::runtime_error with the library's message, as the reference's CUDA backend
// throws on CUDA errors (Tracker.cu:326-335). Each host thread drives its own device context
// (one arena and stream, created on first use on the device named by ITSU_DEVICE, default 0), as
// the reference runs one Tracker per thread.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "ITSReconstruction/CA/Event.h"
#include "ITSReconstruction/CA/PrimaryVertexContext.h"
#include "ITSReconstruction/CA/Tracker.h"
#include "itsu.h"

#if !defined(TRACKINGITSU_B200) || TRACKINGITSU_GPU_MODE
#error "TrackerB200.cxx is the TRACKINGITSU_B200 backend of a build with the CPU data structures"
#endif

namespace o2
{
namespace ITS
{
namespace CA
{
namespace
{

static_assert(sizeof(Cluster) == sizeof(itsu_cluster), "Cluster and itsu_cluster share their layout");
static_assert(sizeof(Tracklet) == sizeof(itsu_tracklet), "Tracklet and itsu_tracklet share their layout");

struct ContextDeleter {
  void operator()(itsu_context* ctx) const { itsu_context_destroy(ctx); }
};

void check(itsu_status st, itsu_context* ctx)
{
  if (st != ITSU_OK) {
    throw std::runtime_error(std::string("B200 backend: ") + itsu_status_string(st) + ": " + itsu_last_error(ctx));
  }
}

// The calling thread's device context.
itsu_context* b200()
{
  thread_local std::unique_ptr<itsu_context, ContextDeleter> ctx;
  if (!ctx) {
    itsu_config cfg;
    itsu_config_default(&cfg);
    if (const char* dev = std::getenv("ITSU_DEVICE")) {
      cfg.device = std::atoi(dev);
    }
    itsu_context* c = nullptr;
    check(itsu_context_create(&cfg, &c), nullptr);
    ctx.reset(c);
  }
  return ctx.get();
}

itsu_counts counts()
{
  itsu_counts n;
  check(itsu_get_counts(b200(), 0, &n), b200());
  return n;
}

}  // namespace

// The backend step of PrimaryVertexContext::initialize (called at the end of its CPU branch,
// PrimaryVertexContext.cxx:87-141): the vertex's clusters are transformed, stably sorted by bin
// and indexed on the device (itsu_pvc_initialize); the device's sorted clusters and index tables
// then replace the host's, so the host sees exactly what the device stages work on.
void b200Initialize(PrimaryVertexContext& pvc, const Event& event, int vertex)
{
  itsu_context* ctx = b200();
  const itsu_cluster* layers[ITSU_LAYERS];
  int32_t sizes[ITSU_LAYERS];
  for (int l = 0; l < ITSU_LAYERS; ++l) {
    const std::vector<Cluster>& raw = event.getLayer(l).getClusters();
    layers[l] = reinterpret_cast<const itsu_cluster*>(raw.data());
    sizes[l] = static_cast<int32_t>(raw.size());
  }
  const float3& pv = event.getPrimaryVertex(vertex);
  const float v[3] = { pv.x, pv.y, pv.z };
  check(itsu_pvc_initialize(ctx, layers, sizes, v), ctx);

  itsu_results r;
  std::memset(&r, 0, sizeof r);
  for (int l = 0; l < ITSU_LAYERS; ++l) {
    // the reference filled these vectors with the host's sorted clusters already: same sizes
    std::vector<Cluster>& clusters = pvc.getClusters()[l];
    if (static_cast<int32_t>(clusters.size()) != sizes[l]) {
      throw std::runtime_error("B200 backend: the host clusters of a layer do not match the event's");
    }
    r.clusters[l] = reinterpret_cast<itsu_cluster*>(clusters.data());
  }
  for (int l = 0; l < ITSU_TRACKLET_LAYERS; ++l) {
    r.index_tables[l] = pvc.getIndexTables()[l].data();
  }
  check(itsu_copy_results(ctx, 0, &r), ctx);
}

// TrackerTraits::computeLayerTracklets (CPU body Tracker.cxx:45-117): the tracklets of every layer
// on the device, then copied into the context's host tracklets and tracklets lookup tables.
template<>
void TrackerTraits<false>::computeLayerTracklets(PrimaryVertexContext& pvc)
{
  itsu_context* ctx = b200();
  check(itsu_compute_layer_tracklets(ctx), ctx);
  const itsu_counts n = counts();
  std::vector<std::vector<itsu_tracklet>> staging(ITSU_TRACKLET_LAYERS);
  itsu_results r;
  std::memset(&r, 0, sizeof r);
  for (int l = 0; l < ITSU_TRACKLET_LAYERS; ++l) {
    staging[l].resize(n.tracklets[l]);
    r.tracklets[l] = staging[l].data();
  }
  for (int l = 0; l < ITSU_CELL_LAYERS; ++l) {
    std::vector<int>& lookup = pvc.getTrackletsLookupTable()[l];
    lookup.assign(n.clusters[l + 1], Constants::ITS::UnusedIndex);
    r.tracklets_lookup[l] = lookup.data();
  }
  check(itsu_copy_results(ctx, 0, &r), ctx);
  for (int l = 0; l < ITSU_TRACKLET_LAYERS; ++l) {
    // Tracklet's members are const and its value constructor recomputes the slope and azimuth on
    // the host: each record is default-constructed in place and takes the device's bytes
    // (the layouts are identical and the type is trivially copyable). Appended one by one, as the
    // reference does, so the vector's capacity grows as the reference's (its memory benchmark
    // prints it, Tracker.cxx:304-363).
    std::vector<Tracklet>& tracklets = pvc.getTracklets()[l];
    tracklets.clear();
    for (const itsu_tracklet& t : staging[l]) {
      tracklets.emplace_back();
      std::memcpy(static_cast<void*>(&tracklets.back()), &t, sizeof t);
    }
  }
}

// TrackerTraits::computeLayerCells (CPU body Tracker.cxx:120-235): the cells of every layer on the
// device, then the cells and cells lookup tables in host memory for the host's neighbour finding.
template<>
void TrackerTraits<false>::computeLayerCells(PrimaryVertexContext& pvc)
{
  itsu_context* ctx = b200();
  check(itsu_compute_layer_cells(ctx), ctx);
  const itsu_counts n = counts();
  std::vector<std::vector<itsu_cell>> staging(ITSU_CELL_LAYERS);
  std::vector<std::vector<int32_t>> lookup(ITSU_NEIGHBOUR_LAYERS);
  itsu_results r;
  std::memset(&r, 0, sizeof r);
  for (int l = 0; l < ITSU_CELL_LAYERS; ++l) {
    staging[l].resize(n.cells[l]);
    r.cells[l] = staging[l].data();
  }
  for (int l = 0; l < ITSU_NEIGHBOUR_LAYERS; ++l) {
    lookup[l].resize(n.tracklets[l + 1]);
    r.cells_lookup[l] = lookup[l].data();
  }
  check(itsu_copy_results(ctx, 0, &r), ctx);
  for (int l = 0; l < ITSU_CELL_LAYERS; ++l) {
    std::vector<Cell>& cells = pvc.getCells()[l];
    cells.clear();
    for (const itsu_cell& c : staging[l]) {
      cells.emplace_back(c.first_cluster, c.second_cluster, c.third_cluster, c.first_tracklet, c.second_tracklet,
                         float3{ c.nx, c.ny, c.nz }, c.curvature);
    }
  }
  for (int l = 0; l < ITSU_NEIGHBOUR_LAYERS; ++l) {
    // initialize sized the table from a memory coefficient (PrimaryVertexContext.cxx:68-73); it
    // holds at least one entry per tracklet of layer l + 1, the rest stay unused
    std::vector<int>& table = pvc.getCellsLookupTable()[l];
    if (table.size() < lookup[l].size()) {
      table.resize(lookup[l].size(), Constants::ITS::UnusedIndex);
    }
    std::fill(table.begin(), table.end(), Constants::ITS::UnusedIndex);
    std::copy(lookup[l].begin(), lookup[l].end(), table.begin());
  }
}

}  // namespace CA
}  // namespace ITS
}  // namespace o2
