// itsu_tracker_main.cpp - the reference driver (main.cpp:27-154) on the device tracker.
//
//   itsu_tracker_main <events.txt> [labels.txt] [--roads roads.bin]
// Loads the events, runs Tracker<true>::clustersToTracks on each (after one warm-up event, as
// main.cpp:74-75) and prints per-event roads and times. With a labels file, as main.cpp:50-61
// and 131-135, it writes the road report of every event (IOUtils::writeRoadsReport, classified
// on the device) to CorrectRoads.txt, DuplicateRoads.txt and FakeRoads.txt in the events file's
// folder. --roads writes every vertex's roads (int32 count, then 32-byte Road records) for
// comparison with the reference.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>
#include <string>

#include "itsu_ca.hpp"
#include "itsu_ioutils.hpp"

using itsu::ca::Event;
using itsu::ca::Road;
using itsu::ca::Tracker;

static std::string directory_of(const std::string &path)
{
  const size_t pos = path.find_last_of("\\/");
  return pos == std::string::npos ? "" : path.substr(0, pos + 1);
}

int main(int argc, char **argv)
{
  const char *events_path = nullptr, *labels_path = nullptr, *roads_path = nullptr;
  for (int i = 1; i < argc; ++i) {
    if (std::strcmp(argv[i], "--roads") == 0 && i + 1 < argc) {
      roads_path = argv[++i];
    } else if (!events_path) {
      events_path = argv[i];
    } else if (!labels_path) {
      labels_path = argv[i];
    }
  }
  if (!events_path) {
    std::fprintf(stderr, "Please, provide a data file.\n");
    return 1;
  }
  try {
    std::vector<Event> events = itsu::ca::IOUtils::loadEventData(events_path);
    std::vector<std::unordered_map<int, itsu::ca::Label>> labels;
    std::ofstream correct, duplicate, fake;
    if (labels_path) {
      labels = itsu::ca::IOUtils::loadLabels(static_cast<int>(events.size()), labels_path);
      const std::string dir = directory_of(events_path);
      correct.open(dir + "CorrectRoads.txt");
      duplicate.open(dir + "DuplicateRoads.txt");
      fake.open(dir + "FakeRoads.txt");
    }
    std::FILE *out = roads_path ? std::fopen(roads_path, "wb") : nullptr;
    Tracker<true> tracker{};
    if (!events.empty()) tracker.clustersToTracks(events[0]);  // warm-up
    double total_ms = 0;
    int vertices = 0;
    const std::unordered_map<int, itsu::ca::Label> no_labels;
    for (size_t ie = 0; ie < events.size(); ++ie) {
      const auto t0 = std::chrono::steady_clock::now();
      std::vector<std::vector<Road>> roads = tracker.clustersToTracks(events[ie]);
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      total_ms += ms;
      for (size_t iv = 0; iv < roads.size(); ++iv) {
        std::printf("Found %zu roads for vertex %zu\n", roads[iv].size(), iv + 1);
        if (out) {
          const int32_t n = static_cast<int32_t>(roads[iv].size());
          std::fwrite(&n, 4, 1, out);
          std::fwrite(roads[iv].data(), sizeof(Road), roads[iv].size(), out);
        }
        ++vertices;
      }
      std::printf("Event %zu processed in: %.3fms\n", ie + 1, ms);
      if (labels_path) {
        itsu::ca::IOUtils::writeRoadsReport(tracker.getPrimaryVertexContext().ctx(), correct, duplicate, fake, roads,
                                            ie < labels.size() ? labels[ie] : no_labels);
      }
    }
    if (out) std::fclose(out);
    std::printf("Avg time: %.3fms\n", vertices ? total_ms / vertices : 0.0);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 3;
  }
  return 0;
}
