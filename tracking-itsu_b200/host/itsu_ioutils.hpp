// itsu_ioutils.hpp - file I/O of the facade, same formats and semantics as the reference's
// IOUtils (src/CA/IOUtils.cxx) and Label (src/CA/Label.cxx):
//   loadEventData     IOUtils.cxx:38-78: a "-1 x y z" line adds a primary vertex (opening a new
//                     event unless it follows another vertex line); a cluster line is
//                     "layer x y z _ _ _ alpha mc"; cluster ids run per event in file order
//   loadLabels        IOUtils.cxx:80-123: a header line, then "mc pT phi eta pdg nClusters" lines
//                     kept when |pdg| == 211 and nClusters == 7; "-1" ends an event's map
//   writeRoadsReport  IOUtils.cxx:125-170: the road classes come from the device
//                     (itsu_roads_report); the streams get the same lines as the reference's
#pragma once

#include <cstdlib>
#include <fstream>
#include <ostream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "itsu_ca.hpp"

namespace itsu {
namespace ca {
namespace IOUtils {

inline std::vector<Event> loadEventData(const std::string &fileName)
{
  std::vector<Event> events;
  std::ifstream in(fileName);
  std::string line, unused;
  int layerId = 0, monteCarlo = 0, clusterId = -1;
  float x = 0, y = 0, z = 0, alpha = 0;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    if (!(ls >> layerId >> x >> y >> z)) continue;
    if (layerId == -1) {
      if (clusterId != 0) events.emplace_back(static_cast<int>(events.size()));
      events.back().addPrimaryVertex(x, y, z);
      clusterId = 0;
    } else if (ls >> unused >> unused >> unused >> alpha >> monteCarlo) {
      events.back().pushClusterToLayer(layerId, clusterId, x, y, z, alpha, monteCarlo);
      ++clusterId;
    }
  }
  return events;
}

inline std::vector<std::unordered_map<int, Label>> loadLabels(const int eventsNum, const std::string &fileName)
{
  std::vector<std::unordered_map<int, Label>> maps;
  std::unordered_map<int, Label> current;
  maps.reserve(eventsNum > 0 ? eventsNum : 0);
  std::ifstream in(fileName);
  std::string line;
  std::getline(in, line);  // header
  int mc = 0, pdg = 0, ncl = 0;
  float pt = 0, phi = 0, eta = 0;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    if (!(ls >> mc)) continue;
    if (mc == -1) {
      maps.emplace_back(current);
      current.clear();
    } else if ((ls >> pt >> phi >> eta >> pdg >> ncl) && std::abs(pdg) == PionCode && ncl == 7) {
      current.emplace(mc, Label{mc, pt, phi, eta, pdg, ncl});
    }
  }
  maps.emplace_back(current);
  return maps;
}

// One event's roads (one vector per vertex) against its labels map, on the given context.
inline void writeRoadsReport(itsu_context *ctx, std::ofstream &correctRoadsOutputStream, std::ofstream &duplicateRoadsOutputStream,
                             std::ofstream &fakeRoadsOutputStream, const std::vector<std::vector<Road>> &roads,
                             const std::unordered_map<int, Label> &labelsMap)
{
  std::vector<itsu_road> flat;
  std::vector<int32_t> runOffsets{0}, runEvent;
  for (const std::vector<Road> &vertexRoads : roads) {
    const itsu_road *r = reinterpret_cast<const itsu_road *>(vertexRoads.data());
    flat.insert(flat.end(), r, r + vertexRoads.size());
    runOffsets.push_back(static_cast<int32_t>(flat.size()));
    runEvent.push_back(0);
  }
  std::vector<itsu_label> labels;
  labels.reserve(labelsMap.size());
  for (const auto &kv : labelsMap) {
    const Label &l = kv.second;
    labels.push_back(itsu_label{l.monteCarloId, l.transverseMomentum, l.phiCoordinate, l.pseudorapidity, l.pdgCode,
                                l.numberOfClusters});
  }
  const int32_t labelOffsets[2] = {0, static_cast<int32_t>(labels.size())};
  std::vector<uint8_t> classes(flat.size() + 1);
  itsu_road none{};
  check(itsu_roads_report(ctx, flat.empty() ? &none : flat.data(), runOffsets.data(), runEvent.data(),
                          static_cast<int32_t>(roads.size()), labels.data(), labelOffsets, 1, classes.data(), nullptr),
        ctx);
  correctRoadsOutputStream << -1 << std::endl;
  fakeRoadsOutputStream << -1 << std::endl;
  for (size_t i = 0; i < flat.size(); ++i) {
    if (classes[i] == ITSU_ROAD_UNREPORTED) continue;
    const Label &label = labelsMap.at(flat[i].label);
    std::ofstream &out = classes[i] == ITSU_ROAD_FAKE ? fakeRoadsOutputStream
                         : classes[i] == ITSU_ROAD_CORRECT ? correctRoadsOutputStream
                                                           : duplicateRoadsOutputStream;
    out << label << std::endl;
  }
}

// The reference's signature: the classification runs on a context of device 0 kept by the calling
// thread (created on first use).
inline void writeRoadsReport(std::ofstream &correctRoadsOutputStream, std::ofstream &duplicateRoadsOutputStream,
                             std::ofstream &fakeRoadsOutputStream, const std::vector<std::vector<Road>> &roads,
                             const std::unordered_map<int, Label> &labelsMap)
{
  thread_local DeviceContext device{0};
  writeRoadsReport(device.get(), correctRoadsOutputStream, duplicateRoadsOutputStream, fakeRoadsOutputStream, roads, labelsMap);
}

}  // namespace IOUtils
}  // namespace ca
}  // namespace itsu
