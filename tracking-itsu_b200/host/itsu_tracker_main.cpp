// itsu_tracker_main.cpp - the reference driver (main.cpp:27-154) on the device tracker.
//
//   itsu_tracker_main <events.txt> [roads.bin]
// Loads the events, runs Tracker<true>::clustersToTracks on each (after one warm-up event, as
// main.cpp:74-75), prints per-event roads and times, and optionally writes every vertex's roads
// (int32 count, then 32-byte Road records) for comparison with the reference.
#include <chrono>
#include <cstdio>
#include <exception>

#include "itsu_ca.hpp"
#include "itsu_ioutils.hpp"

using itsu::ca::Event;
using itsu::ca::Road;
using itsu::ca::Tracker;

int main(int argc, char **argv)
{
  if (argc < 2) {
    std::fprintf(stderr, "Please, provide a data file.\n");
    return 1;
  }
  try {
    std::vector<Event> events = itsu::ca::IOUtils::loadEventData(argv[1]);
    std::FILE *out = argc > 2 ? std::fopen(argv[2], "wb") : nullptr;
    Tracker<true> tracker{};
    if (!events.empty()) tracker.clustersToTracks(events[0]);  // warm-up
    double total_ms = 0;
    int vertices = 0;
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
    }
    if (out) std::fclose(out);
    std::printf("Avg time: %.3fms\n", vertices ? total_ms / vertices : 0.0);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 3;
  }
  return 0;
}
