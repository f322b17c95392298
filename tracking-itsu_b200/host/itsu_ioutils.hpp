// itsu_ioutils.hpp - event file reader of the facade, same format and semantics as the
// reference's IOUtils::loadEventData (src/CA/IOUtils.cxx:38-78): a "-1 x y z" line adds a
// primary vertex (opening a new event unless it follows another vertex line); a cluster line is
// "layer x y z _ _ _ alpha mc"; cluster ids run per event in file order.
#pragma once

#include <fstream>
#include <sstream>
#include <string>
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

}  // namespace IOUtils
}  // namespace ca
}  // namespace itsu
