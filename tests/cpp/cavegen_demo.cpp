// cavegen_demo.cpp -- test program: the reference's cave generator mains (test3DCaveGen.cpp,
// test2DCaveGen.cpp) written against the C++ facade.
//
// usage: cavegen_demo <cavegenconfig> 3d|2d|gen
// Prints the path written, the region count and the largest region's size, and the
// neighbour counts of the first on cell.
#include <cstdio>
#include <string>

#include "nanomap_b200/nanomap.hpp"

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  try {
    nanomap::mapgen::CaveGen generator(argv[1]);
    const std::string mode = argv[2];
    if (mode == "3d") {
      generator.populateMap();
      generator.smoothMap();
      generator.setFloorAndCeil();
      generator.getRegions();
      generator.keepLargestRegion();
      generator.invertAndSave();
    } else if (mode == "2d") {
      generator.populateMap2D();
      generator.smoothMapXY();
      generator.getRegions();
      generator.keepLargestRegion();
      generator.invertAndSave();
    } else {
      generator.gen();
    }
    std::printf("%s %lld %lld\n", generator.writtenPath().c_str(),
                (long long)generator.regionCount(), (long long)generator.largestRegion());
  } catch (const nanomap::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
