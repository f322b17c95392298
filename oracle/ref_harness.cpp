// ref_harness.cpp - drives the reference CPU Tracker and dumps every intermediate result.
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/build_ref.sh together with the reference's own
// (patched) sources into oracle/_ref/. Events are read with the reference's own text loader
// (IOUtils::loadEventData, IOUtils.cxx:38-78).
//
//   ref_cr dump <events.txt> <out.bin>   run every vertex stage by stage, write all results
//   ref_cr time <events.txt> <repeats>   time Tracker::clustersToTracks per event (steady_clock,
//                                        one warm-up event first, as main.cpp:74-75) -> JSON line
//   ref_cr timebin <events.bin> <repeats> [first count]   the same on binary events
//   ref_cr report <events.txt> <labels.txt> <outdir>   main.cpp's benchmark data: every event
//                                        through clustersToTracks, then IOUtils::writeRoadsReport
//                                        into outdir/{Correct,Duplicate,Fake}Roads.txt; prints the
//                                        time spent in writeRoadsReport (JSON line)
//   ref_cr labels <labels.txt> <n_events> <out.txt>   IOUtils::loadLabels, each map's entries
//                                        (ascending id) one per line, "-1" after each map
//   ref_cr events <events.txt> <out.txt>   IOUtils::loadEventData, every vertex and cluster
//   ref_cr memory <events.txt> <out.txt>   main.cpp's MEMORY_BENCHMARK run: one warm-up event,
//                                        then Tracker::clustersToTracksMemoryBenchmark per event
//
// The dump needs the tracker's private per-vertex context and its protected stages, so the
// reference headers are included with private/protected opened up (standard headers first, so
// only the tracker's classes are affected).
#include <algorithm>
#include <array>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <ostream>
#include <sstream>
#include <string>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#define private public
#define protected public
#include "ITSReconstruction/CA/IOUtils.h"
#include "ITSReconstruction/CA/Tracker.h"
#undef private
#undef protected

#if defined(ITSU_REF_CR)
extern "C" float itsu_ref_cr_atan2f(float y, float x);
#endif

using namespace o2::ITS::CA;

namespace
{

void put_i32(std::FILE *f, int32_t v) { std::fwrite(&v, 4, 1, f); }
void put_f32(std::FILE *f, float v) { std::fwrite(&v, 4, 1, f); }

void dump_vertex(std::FILE *f, int event, int vertex, PrimaryVertexContext &pvc)
{
  put_i32(f, event);
  put_i32(f, vertex);
  put_f32(f, pvc.getPrimaryVertex().x);
  put_f32(f, pvc.getPrimaryVertex().y);
  put_f32(f, pvc.getPrimaryVertex().z);
  for (int l = 0; l < Constants::ITS::LayersNumber; ++l) {
    const auto &cl = pvc.getClusters()[l];
    put_i32(f, static_cast<int32_t>(cl.size()));
    for (const Cluster &c : cl) {
      put_f32(f, c.xCoordinate);
      put_f32(f, c.yCoordinate);
      put_f32(f, c.zCoordinate);
      put_f32(f, c.phiCoordinate);
      put_f32(f, c.rCoordinate);
      put_i32(f, c.clusterId);
      put_f32(f, c.alphaAngle);
      put_i32(f, c.monteCarloId);
      put_i32(f, c.indexTableBinIndex);
    }
  }
  for (int l = 0; l < Constants::ITS::TrackletsPerRoad; ++l) {
    for (int b = 0; b <= Constants::IndexTable::ZBins * Constants::IndexTable::PhiBins; ++b) {
      put_i32(f, pvc.getIndexTables()[l][b]);
    }
  }
  for (int l = 0; l < Constants::ITS::TrackletsPerRoad; ++l) {
    const auto &tr = pvc.getTracklets()[l];
    put_i32(f, static_cast<int32_t>(tr.size()));
    for (const Tracklet &t : tr) {
      put_i32(f, t.firstClusterIndex);
      put_i32(f, t.secondClusterIndex);
      put_f32(f, t.tanLambda);
      put_f32(f, t.phiCoordinate);
    }
  }
  for (int l = 0; l < Constants::ITS::CellsPerRoad; ++l) {
    const auto &lt = pvc.getTrackletsLookupTable()[l];
    put_i32(f, static_cast<int32_t>(lt.size()));
    for (int v : lt) put_i32(f, v);
  }
  for (int l = 0; l < Constants::ITS::CellsPerRoad; ++l) {
    const auto &cells = pvc.getCells()[l];
    put_i32(f, static_cast<int32_t>(cells.size()));
    for (const Cell &c : cells) {
      put_i32(f, c.getFirstClusterIndex());
      put_i32(f, c.getSecondClusterIndex());
      put_i32(f, c.getThirdClusterIndex());
      put_i32(f, c.getFirstTrackletIndex());
      put_i32(f, c.getSecondTrackletIndex());
      put_f32(f, c.getNormalVectorCoordinates().x);
      put_f32(f, c.getNormalVectorCoordinates().y);
      put_f32(f, c.getNormalVectorCoordinates().z);
      put_f32(f, c.getCurvature());
      put_i32(f, c.getLevel());
    }
  }
  for (int l = 0; l < Constants::ITS::CellsPerRoad - 1; ++l) {
    const auto &lt = pvc.getCellsLookupTable()[l];
    put_i32(f, static_cast<int32_t>(lt.size()));
    for (int v : lt) put_i32(f, v);
  }
  for (int l = 0; l < Constants::ITS::CellsPerRoad - 1; ++l) {
    const auto &nb = pvc.getCellsNeighbours()[l];
    put_i32(f, static_cast<int32_t>(nb.size()));
    for (const auto &list : nb) {
      put_i32(f, static_cast<int32_t>(list.size()));
      for (int v : list) put_i32(f, v);
    }
  }
  auto &roads = pvc.getRoads();
  put_i32(f, static_cast<int32_t>(roads.size()));
  for (Road &r : roads) {
    for (int k = 0; k < Constants::ITS::CellsPerRoad; ++k) put_i32(f, r[k]);
    put_i32(f, r.getRoadSize());
    put_i32(f, r.getLabel());
    put_i32(f, r.isFakeRoad() ? 1 : 0);
  }
}

int run_dump(const std::string &events_file, const std::string &out_file)
{
  std::vector<Event> events = IOUtils::loadEventData(events_file);
  std::FILE *f = std::fopen(out_file.c_str(), "wb");
  if (!f) {
    std::perror("fopen");
    return 1;
  }
  int32_t records = 0;
  for (const Event &e : events) records += e.getPrimaryVerticesNum();
  std::fwrite("ITSUREF1", 1, 8, f);
  put_i32(f, records);
  Tracker<false> tracker{};
  for (size_t ie = 0; ie < events.size(); ++ie) {
    const Event &event = events[ie];
    for (int iv = 0; iv < event.getPrimaryVerticesNum(); ++iv) {
      // The body of Tracker::clustersToTracks for one vertex (Tracker.cxx:253-259).
      tracker.mPrimaryVertexContext.initialize(event, iv);
      tracker.computeTracklets();
      tracker.computeCells();
      tracker.findCellsNeighbours();
      tracker.findTracks();
      tracker.computeMontecarloLabels();
      dump_vertex(f, static_cast<int>(ie), iv, tracker.mPrimaryVertexContext);
    }
  }
  std::fclose(f);
  return 0;
}

// Binary events (test infrastructure format "ITSUEVT1"): int32 n_events, then per event
// int32 n_vertices, float xyz per vertex, int32 counts[7], and per cluster float x, y, z, alpha
// and int32 mc, layer by layer. Events are built through the reference's public Event API with
// the running cluster ids IOUtils::loadEventData assigns (IOUtils.cxx:63,71).
std::vector<Event> load_binary_events(const std::string &file, int first, int count)
{
  std::vector<Event> events;
  std::FILE *f = std::fopen(file.c_str(), "rb");
  if (!f) {
    std::perror("fopen");
    return events;
  }
  char magic[8];
  int32_t n = 0;
  if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "ITSUEVT1", 8) != 0 || std::fread(&n, 4, 1, f) != 1) {
    std::fclose(f);
    std::fprintf(stderr, "not an ITSUEVT1 file\n");
    return events;
  }
  const int last = count < 0 ? n : std::min(n, first + count);
  for (int e = 0; e < last; ++e) {
    int32_t nv = 0, counts[7];
    if (std::fread(&nv, 4, 1, f) != 1) break;
    std::vector<float> v(3 * static_cast<size_t>(nv));
    std::fread(v.data(), 4, v.size(), f);
    std::fread(counts, 4, 7, f);
    const bool keep = e >= first;
    if (keep) events.emplace_back(static_cast<int>(events.size()));
    int cluster_id = 0;
    for (int iv = 0; iv < nv && keep; ++iv) events.back().addPrimaryVertex(v[3 * iv], v[3 * iv + 1], v[3 * iv + 2]);
    for (int l = 0; l < 7; ++l) {
      for (int32_t k = 0; k < counts[l]; ++k) {
        float xyza[4];
        int32_t mc;
        std::fread(xyza, 4, 4, f);
        std::fread(&mc, 4, 1, f);
        if (keep) events.back().pushClusterToLayer(l, cluster_id, xyza[0], xyza[1], xyza[2], xyza[3], mc);
        ++cluster_id;
      }
    }
  }
  std::fclose(f);
  return events;
}

int run_time_events(std::vector<Event> &events, int repeats);

int run_time(const std::string &events_file, int repeats)
{
  std::vector<Event> events = IOUtils::loadEventData(events_file);
  return run_time_events(events, repeats);
}

int run_time_events(std::vector<Event> &events, int repeats)
{
  if (events.empty()) {
    std::printf("{\"events\": 0}\n");
    return 0;
  }
  Tracker<false> tracker{};
  tracker.clustersToTracks(events[0]); // warm-up, as main.cpp:74-75
  long long roads = 0, vertices = 0, clusters = 0;
  auto t0 = std::chrono::steady_clock::now();
  for (int rep = 0; rep < repeats; ++rep) {
    for (const Event &event : events) {
      std::vector<std::vector<Road>> r = tracker.clustersToTracks(event);
      for (const auto &v : r) roads += static_cast<long long>(v.size());
      vertices += event.getPrimaryVerticesNum();
      clusters += event.getTotalClusters();
    }
  }
  auto t1 = std::chrono::steady_clock::now();
  const double seconds = std::chrono::duration<double>(t1 - t0).count();
  std::printf("{\"events\": %lld, \"vertices\": %lld, \"clusters\": %lld, \"roads\": %lld, \"seconds\": %.9f}\n",
              static_cast<long long>(events.size()) * repeats, vertices, clusters, roads, seconds);
  return 0;
}

int run_report(const char *events_path, const char *labels_path, const std::string &outdir)
{
  std::vector<Event> events = IOUtils::loadEventData(events_path);
  std::vector<std::unordered_map<int, Label>> labels = IOUtils::loadLabels(static_cast<int>(events.size()), labels_path);
  std::ofstream correct(outdir + "/CorrectRoads.txt"), duplicate(outdir + "/DuplicateRoads.txt"),
      fake(outdir + "/FakeRoads.txt");
  Tracker<false> tracker{};
  double seconds = 0;
  long long n_roads = 0;
  const std::unordered_map<int, Label> none{};
  for (size_t e = 0; e < events.size(); ++e) {
    std::vector<std::vector<Road>> roads = tracker.clustersToTracks(events[e]);
    for (const auto &v : roads) n_roads += static_cast<long long>(v.size());
    const auto t0 = std::chrono::steady_clock::now();
    IOUtils::writeRoadsReport(correct, duplicate, fake, roads, e < labels.size() ? labels[e] : none);
    const auto t1 = std::chrono::steady_clock::now();
    seconds += std::chrono::duration<double>(t1 - t0).count();
  }
  std::printf("{\"events\": %lld, \"roads\": %lld, \"report_seconds\": %.9f}\n", static_cast<long long>(events.size()),
              n_roads, seconds);
  return 0;
}

int run_labels(const char *labels_path, int n_events, const char *out_path)
{
  std::vector<std::unordered_map<int, Label>> labels = IOUtils::loadLabels(n_events, labels_path);
  std::FILE *f = std::fopen(out_path, "w");
  if (!f) return 3;
  for (const auto &m : labels) {
    std::vector<int> ids;
    for (const auto &kv : m) ids.push_back(kv.first);
    std::sort(ids.begin(), ids.end());
    for (int id : ids) {
      const Label &l = m.at(id);
      std::fprintf(f, "%d %.9g %.9g %.9g %d %d\n", l.monteCarloId, l.transverseMomentum, l.phiCoordinate, l.pseudorapidity,
                   l.pdgCode, l.numberOfClusters);
    }
    std::fprintf(f, "-1\n");
  }
  std::fclose(f);
  return 0;
}

int run_events(const char *events_path, const char *out_path)
{
  std::vector<Event> events = IOUtils::loadEventData(events_path);
  std::FILE *f = std::fopen(out_path, "w");
  if (!f) return 3;
  for (const Event &ev : events) {
    std::fprintf(f, "event %d vertices %d\n", ev.getEventId(), ev.getPrimaryVerticesNum());
    for (int v = 0; v < ev.getPrimaryVerticesNum(); ++v) {
      const float3 &p = ev.getPrimaryVertex(v);
      std::fprintf(f, "v %.9g %.9g %.9g\n", p.x, p.y, p.z);
    }
    for (int l = 0; l < Constants::ITS::LayersNumber; ++l) {
      for (const Cluster &c : ev.getLayer(l).getClusters()) {
        std::fprintf(f, "c %d %d %.9g %.9g %.9g %.9g %d\n", l, c.clusterId, c.xCoordinate, c.yCoordinate, c.zCoordinate,
                     c.alphaAngle, c.monteCarloId);
      }
    }
  }
  std::fclose(f);
  return 0;
}

int run_memory(const char *events_path, const char *out_path)
{
  std::vector<Event> events = IOUtils::loadEventData(events_path);
  std::ofstream out(out_path);
  Tracker<false> tracker{};
  if (!events.empty()) tracker.clustersToTracks(events[0]);  // main.cpp:74-75
  for (size_t e = 0; e < events.size(); ++e) {
    tracker.clustersToTracksMemoryBenchmark(events[e], out);
  }
  return 0;
}

} // namespace

int main(int argc, char **argv)
{
#if defined(ITSU_REF_CR)
  // The override must be in effect for the reference's calls (same symbol resolution). These
  // arguments are ones where the C library's atan2f is not correctly rounded.
  volatile float ya = -4.0587134f, xa = 3.7113914f, yb = 1.96216f, xb = 4.643577f;
  if (atan2f(ya, xa) != itsu_ref_cr_atan2f(ya, xa) || atan2f(yb, xb) != itsu_ref_cr_atan2f(yb, xb)) {
    std::fprintf(stderr, "ref_harness: atan2f override is not active\n");
    return 4;
  }
#endif
  if (argc < 4) {
    std::fprintf(stderr,
                 "usage: %s dump <events.txt> <out.bin> | time <events.txt> <repeats> |"
                 " timebin <events.bin> <repeats> [first count] | report <events.txt> <labels.txt> <outdir> |"
                 " labels <labels.txt> <n_events> <out.txt> | events <events.txt> <out.txt> | memory <events.txt> <out.txt>\n",
                 argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  if (mode == "dump") return run_dump(argv[2], argv[3]);
  if (mode == "time") return run_time(argv[2], std::atoi(argv[3]));
  if (mode == "report" && argc > 4) return run_report(argv[2], argv[3], argv[4]);
  if (mode == "labels" && argc > 4) return run_labels(argv[2], std::atoi(argv[3]), argv[4]);
  if (mode == "events") return run_events(argv[2], argv[3]);
  if (mode == "memory") return run_memory(argv[2], argv[3]);
  if (mode == "timebin") {
    const int first = argc > 5 ? std::atoi(argv[4]) : 0;
    const int count = argc > 5 ? std::atoi(argv[5]) : -1;
    std::vector<Event> events = load_binary_events(argv[2], first, count);
    return run_time_events(events, std::atoi(argv[3]));
  }
  std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
  return 2;
}
