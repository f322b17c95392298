// itsu_ca.hpp - C++ facade of the B200 track finder with the reference tracker's interface.
//
// Same class names, member names, argument meaning and error behaviour as the reference's
// o2::ITS::CA API for this path (include/ITSReconstruction/CA/{Cluster,Tracklet,Cell,Road,Layer,
// Event,PrimaryVertexContext,Tracker}.h), implemented on the C ABI of include/itsu.h:
//   Tracker<true>::clustersToTracks(const Event&)  -> std::vector<std::vector<Road>>, one per vertex
//   PrimaryVertexContext::initialize(const Event&, int) and the getters of every result
//   TrackerTraits<true>::computeLayerTracklets / computeLayerCells(PrimaryVertexContext&)
// Records keep the reference layouts (static_asserts below). Failures throw std::runtime_error
// with the library's message, as the reference's GPU backend does (Tracker.cu:326-335).
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "itsu.h"

namespace itsu {
namespace ca {

constexpr int LayersNumber = ITSU_LAYERS;
constexpr int TrackletsPerRoad = ITSU_TRACKLET_LAYERS;
constexpr int CellsPerRoad = ITSU_CELL_LAYERS;
constexpr int UnusedIndex = ITSU_UNUSED_INDEX;
constexpr int IndexTableSize = ITSU_INDEX_TABLE_SIZE;

struct float3 {
  float x, y, z;
};

// Cluster.h:30-45
struct Cluster final {
  Cluster() = default;
  Cluster(int clusterId, int /*layerIndex*/, float x, float y, float z, float alpha, int monteCarloId)
      : xCoordinate{x}, yCoordinate{y}, zCoordinate{z}, phiCoordinate{0}, rCoordinate{0}, clusterId{clusterId},
        alphaAngle{alpha}, monteCarloId{monteCarloId}, indexTableBinIndex{0}
  {
  }
  float xCoordinate = 0, yCoordinate = 0, zCoordinate = 0, phiCoordinate = 0, rCoordinate = 0;
  int clusterId = 0;
  float alphaAngle = 0;
  int monteCarloId = 0;
  int indexTableBinIndex = 0;
};
static_assert(sizeof(Cluster) == sizeof(itsu_cluster) && sizeof(Cluster) == 36, "Cluster layout");

// Tracklet.h:27-37
struct Tracklet final {
  int firstClusterIndex = 0;
  int secondClusterIndex = 0;
  float tanLambda = 0;
  float phiCoordinate = 0;
};
static_assert(sizeof(Tracklet) == sizeof(itsu_tracklet) && sizeof(Tracklet) == 16, "Tracklet layout");

// Cell.h:30-55
class Cell final {
 public:
  int getFirstClusterIndex() const { return c_.first_cluster; }
  int getSecondClusterIndex() const { return c_.second_cluster; }
  int getThirdClusterIndex() const { return c_.third_cluster; }
  int getFirstTrackletIndex() const { return c_.first_tracklet; }
  int getSecondTrackletIndex() const { return c_.second_tracklet; }
  int getLevel() const { return c_.level; }
  float getCurvature() const { return c_.curvature; }
  float3 getNormalVectorCoordinates() const { return float3{c_.nx, c_.ny, c_.nz}; }
  void setLevel(int level) { c_.level = level; }

 private:
  itsu_cell c_{};
};
static_assert(sizeof(Cell) == 40, "Cell layout");

// Road.h:29-51
class Road final {
 public:
  Road() { resetRoad(); }
  Road(int cellLayer, int cellId) : Road() { addCell(cellLayer, cellId); }
  int getRoadSize() const { return r_.size; }
  int getLabel() const { return r_.label; }
  void setLabel(int label) { r_.label = label; }
  bool isFakeRoad() const { return r_.is_fake != 0; }
  void setFakeRoad(bool fake) { r_.is_fake = fake ? 1 : 0; }
  int &operator[](const int &i) { return r_.cell_ids[i]; }
  int operator[](const int &i) const { return r_.cell_ids[i]; }
  void resetRoad()
  {
    for (int &c : r_.cell_ids) c = UnusedIndex;
    r_.size = 0;
  }
  void addCell(int cellLayer, int cellId)
  {
    if (r_.cell_ids[cellLayer] == UnusedIndex) ++r_.size;
    r_.cell_ids[cellLayer] = cellId;
  }

 private:
  itsu_road r_{};
};
static_assert(sizeof(Road) == sizeof(itsu_road) && sizeof(Road) == 32, "Road layout");

// Label.h:27-41 and its stream format (Label.cxx:32-37)
constexpr int PionCode = 211;  // Constants::PDGCodes::PionCode
struct Label final {
  int monteCarloId;
  float transverseMomentum;
  float phiCoordinate;
  float pseudorapidity;
  int pdgCode;
  int numberOfClusters;
};
static_assert(sizeof(Label) == sizeof(itsu_label) && sizeof(Label) == 24, "Label layout");
inline std::ostream &operator<<(std::ostream &out, const Label &l)
{
  return out << l.monteCarloId << "\t" << l.transverseMomentum << "\t" << l.phiCoordinate << "\t" << l.pseudorapidity << "\t"
             << l.pdgCode << "\t" << l.numberOfClusters;
}

// Layer.h:30-46
class Layer final {
 public:
  Layer() = default;
  explicit Layer(int layerIndex) : mLayerIndex{layerIndex} {}
  int getLayerIndex() const { return mLayerIndex; }
  const std::vector<Cluster> &getClusters() const { return mClusters; }
  const Cluster &getCluster(int i) const { return mClusters[i]; }
  int getClustersSize() const { return static_cast<int>(mClusters.size()); }
  void addCluster(int clusterId, float x, float y, float z, float alpha, int monteCarlo)
  {
    mClusters.emplace_back(clusterId, mLayerIndex, x, y, z, alpha, monteCarlo);
  }

 private:
  int mLayerIndex = UnusedIndex;
  std::vector<Cluster> mClusters;
};

// Event.h:31-50
class Event final {
 public:
  explicit Event(int eventId) : mEventId{eventId}
  {
    for (int l = 0; l < LayersNumber; ++l) mLayers[l] = Layer(l);
  }
  int getEventId() const { return mEventId; }
  const float3 &getPrimaryVertex(int i) const { return mPrimaryVertices[i]; }
  const Layer &getLayer(int l) const { return mLayers[l]; }
  int getPrimaryVerticesNum() const { return static_cast<int>(mPrimaryVertices.size()); }
  void addPrimaryVertex(float x, float y, float z) { mPrimaryVertices.push_back(float3{x, y, z}); }
  void pushClusterToLayer(int layer, int clusterId, float x, float y, float z, float alpha, int monteCarlo)
  {
    mLayers[layer].addCluster(clusterId, x, y, z, alpha, monteCarlo);
  }
  int getTotalClusters() const
  {
    int n = 0;
    for (const Layer &l : mLayers) n += l.getClustersSize();
    return n;
  }

 private:
  int mEventId;
  std::vector<float3> mPrimaryVertices;
  std::array<Layer, LayersNumber> mLayers;
};

inline void check(itsu_status st, const itsu_context *ctx)
{
  if (st != ITSU_OK) {
    throw std::runtime_error(std::string("itsu: ") + itsu_status_string(st) + ": " + itsu_last_error(ctx));
  }
}

// One device context (arena + stream); shared by a Tracker and its PrimaryVertexContext.
class DeviceContext {
 public:
  explicit DeviceContext(int device = 0)
  {
    itsu_config cfg;
    itsu_config_default(&cfg);
    cfg.device = device;
    itsu_context *ctx = nullptr;
    check(itsu_context_create(&cfg, &ctx), nullptr);
    ctx_.reset(ctx);
  }
  itsu_context *get() const { return ctx_.get(); }

 private:
  struct Destroy {
    void operator()(itsu_context *c) const { itsu_context_destroy(c); }
  };
  std::unique_ptr<itsu_context, Destroy> ctx_;
};

// PrimaryVertexContext.h:42-99, device-backed: initialize() runs the clustering stage on the
// device; the getters return host copies of the device results of the stages run so far.
class PrimaryVertexContext final {
 public:
  explicit PrimaryVertexContext(std::shared_ptr<DeviceContext> device = std::make_shared<DeviceContext>())
      : mDevice{std::move(device)}
  {
  }
  PrimaryVertexContext(const PrimaryVertexContext &) = delete;
  PrimaryVertexContext &operator=(const PrimaryVertexContext &) = delete;

  void initialize(const Event &event, int primaryVertexIndex)
  {
    mPrimaryVertex = event.getPrimaryVertex(primaryVertexIndex);
    const itsu_cluster *layers[LayersNumber];
    int32_t counts[LayersNumber];
    for (int l = 0; l < LayersNumber; ++l) {
      const auto &c = event.getLayer(l).getClusters();
      layers[l] = reinterpret_cast<const itsu_cluster *>(c.data());
      counts[l] = static_cast<int32_t>(c.size());
    }
    const float v[3] = {mPrimaryVertex.x, mPrimaryVertex.y, mPrimaryVertex.z};
    check(itsu_pvc_initialize(ctx(), layers, counts, v), ctx());
    mFetched = false;
  }

  const float3 &getPrimaryVertex() const { return mPrimaryVertex; }
  std::array<std::vector<Cluster>, LayersNumber> &getClusters() { fetch(); return mClusters; }
  std::array<std::array<int, IndexTableSize>, TrackletsPerRoad> &getIndexTables() { fetch(); return mIndexTables; }
  std::array<std::vector<Tracklet>, TrackletsPerRoad> &getTracklets() { fetch(); return mTracklets; }
  std::array<std::vector<int>, CellsPerRoad> &getTrackletsLookupTable() { fetch(); return mTrackletsLookupTable; }
  std::array<std::vector<Cell>, CellsPerRoad> &getCells() { fetch(); return mCells; }
  std::array<std::vector<int>, CellsPerRoad - 1> &getCellsLookupTable() { fetch(); return mCellsLookupTable; }
  std::array<std::vector<std::vector<int>>, CellsPerRoad - 1> &getCellsNeighbours() { fetch(); return mCellsNeighbours; }
  std::vector<Road> &getRoads() { fetch(); return mRoads; }

  itsu_context *ctx() const { return mDevice->get(); }
  void invalidate() { mFetched = false; }

 private:
  void fetch()
  {
    if (mFetched) return;
    itsu_counts n;
    check(itsu_get_counts(ctx(), 0, &n), ctx());
    itsu_results r;
    std::memset(&r, 0, sizeof r);
    std::array<std::vector<int32_t>, CellsPerRoad - 1> offsets, flat;
    for (int l = 0; l < LayersNumber; ++l) {
      mClusters[l].resize(n.clusters[l]);
      r.clusters[l] = reinterpret_cast<itsu_cluster *>(mClusters[l].data());
    }
    for (int l = 0; l < TrackletsPerRoad; ++l) {
      r.index_tables[l] = mIndexTables[l].data();
      mTracklets[l].resize(n.tracklets[l]);
      r.tracklets[l] = reinterpret_cast<itsu_tracklet *>(mTracklets[l].data());
    }
    for (int l = 0; l < CellsPerRoad; ++l) {
      mTrackletsLookupTable[l].resize(n.clusters[l + 1]);
      r.tracklets_lookup[l] = mTrackletsLookupTable[l].data();
      mCells[l].resize(n.cells[l]);
      r.cells[l] = reinterpret_cast<itsu_cell *>(mCells[l].data());
    }
    for (int l = 0; l < CellsPerRoad - 1; ++l) {
      mCellsLookupTable[l].resize(n.tracklets[l + 1]);
      r.cells_lookup[l] = mCellsLookupTable[l].data();
      offsets[l].resize(n.cells[l + 1] + 1);
      flat[l].resize(n.neighbours[l]);
      r.neighbour_offsets[l] = offsets[l].data();
      r.neighbours[l] = flat[l].data();
    }
    mRoads.resize(n.roads);
    r.roads = reinterpret_cast<itsu_road *>(mRoads.data());
    check(itsu_copy_results(ctx(), 0, &r), ctx());
    for (int l = 0; l < CellsPerRoad - 1; ++l) {
      mCellsNeighbours[l].assign(n.cells[l + 1], {});
      for (int32_t c = 0; c < n.cells[l + 1]; ++c) {
        mCellsNeighbours[l][c].assign(flat[l].begin() + offsets[l][c], flat[l].begin() + offsets[l][c + 1]);
      }
    }
    mFetched = true;
  }

  std::shared_ptr<DeviceContext> mDevice;
  float3 mPrimaryVertex{0, 0, 0};
  bool mFetched = false;
  std::array<std::vector<Cluster>, LayersNumber> mClusters;
  std::array<std::array<int, IndexTableSize>, TrackletsPerRoad> mIndexTables{};
  std::array<std::vector<Tracklet>, TrackletsPerRoad> mTracklets;
  std::array<std::vector<int>, CellsPerRoad> mTrackletsLookupTable;
  std::array<std::vector<Cell>, CellsPerRoad> mCells;
  std::array<std::vector<int>, CellsPerRoad - 1> mCellsLookupTable;
  std::array<std::vector<std::vector<int>>, CellsPerRoad - 1> mCellsNeighbours;
  std::vector<Road> mRoads;
};

// Tracker.h:39-48: the backend seam. The device specialisation runs each stage on the B200.
template <bool IsGPU>
class TrackerTraits;

template <>
class TrackerTraits<true> {
 public:
  void computeLayerTracklets(PrimaryVertexContext &pvc)
  {
    check(itsu_compute_layer_tracklets(pvc.ctx()), pvc.ctx());
    pvc.invalidate();
  }
  void computeLayerCells(PrimaryVertexContext &pvc)
  {
    check(itsu_compute_layer_cells(pvc.ctx()), pvc.ctx());
    pvc.invalidate();
  }

 protected:
  ~TrackerTraits() = default;
};

// Tracker.h:50-79 with IsGPU = true: neighbours, roads and labels run on the device too.
template <bool IsGPU>
class Tracker : private TrackerTraits<IsGPU> {
  using Trait = TrackerTraits<IsGPU>;

 public:
  explicit Tracker(int device = 0) : mPrimaryVertexContext{std::make_shared<DeviceContext>(device)} {}
  Tracker(const Tracker &) = delete;
  Tracker &operator=(const Tracker &) = delete;

  // Tracker.cxx:245-265
  std::vector<std::vector<Road>> clustersToTracks(const Event &event)
  {
    std::vector<std::vector<Road>> roads;
    roads.reserve(event.getPrimaryVerticesNum());
    for (int iv = 0; iv < event.getPrimaryVerticesNum(); ++iv) {
      mPrimaryVertexContext.initialize(event, iv);
      computeTracklets();
      computeCells();
      findCellsNeighbours();
      findTracks();
      computeMontecarloLabels();
      roads.emplace_back(mPrimaryVertexContext.getRoads());
    }
    return roads;
  }

  PrimaryVertexContext &getPrimaryVertexContext() { return mPrimaryVertexContext; }

 protected:
  void computeTracklets() { Trait::computeLayerTracklets(mPrimaryVertexContext); }
  void computeCells() { Trait::computeLayerCells(mPrimaryVertexContext); }
  void findCellsNeighbours()
  {
    check(itsu_find_cells_neighbours(mPrimaryVertexContext.ctx()), mPrimaryVertexContext.ctx());
    mPrimaryVertexContext.invalidate();
  }
  void findTracks()
  {
    check(itsu_find_tracks(mPrimaryVertexContext.ctx()), mPrimaryVertexContext.ctx());
    mPrimaryVertexContext.invalidate();
  }
  void computeMontecarloLabels()
  {
    check(itsu_compute_montecarlo_labels(mPrimaryVertexContext.ctx()), mPrimaryVertexContext.ctx());
  }

 private:
  PrimaryVertexContext mPrimaryVertexContext;
};

}  // namespace ca
}  // namespace itsu
