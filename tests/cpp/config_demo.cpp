// config_demo.cpp -- test program: the facade's Config and Agent accessors, host only.
//
// usage: config_demo <config>
// Prints the config's derived sizes and agent 0's sensors and observation rays before and
// after resetAgent(), one "key value" pair per line.
#include <cstdio>

#include "nanomap_b200/nanomap.hpp"

int main(int argc, char** argv) {
  if (argc != 2) return 2;
  try {
    nanomap::config::Config cfg(argv[1]);
    std::printf("leafVolume %d\n", cfg.leafVolume());
    std::printf("maxPCLSize %d\n", cfg.maxPCLSize());
    std::printf("frustumPCLSize %d\n", cfg.frustumPCLSize());
    std::printf("laserPCLSize %d\n", cfg.laserPCLSize());
    std::printf("frustumLeafBufferSize %d\n", cfg.frustumLeafBufferSize());
    std::printf("laserVoxelBufferSize %d\n", cfg.laserVoxelBufferSize());
    std::printf("processType %d\n", cfg.processType());
    std::printf("exploreType %d\n", cfg.exploreType());
    std::printf("simType %d\n", cfg.simType());
    std::printf("serialUpdate %d\n", cfg.serialUpdate() ? 1 : 0);
    nanomap::agent::Agent agent(cfg, 0);
    std::printf("agentId %d\n", agent.getId());
    std::printf("sensors %zu\n", agent.sensorNames().size());
    std::printf("observationRays %zu\n", agent.observationRays().size());
    const auto norms = agent.observationNorms();
    std::printf("observationNorms %zu %g %g\n", norms.size(), norms.empty() ? 0.0 : norms[0][0],
                norms.empty() ? 0.0 : norms[0][1]);
    agent.resetAgent();
    std::printf("sensorsAfterReset %zu\n", agent.sensorNames().size());
    std::printf("raysAfterReset %zu\n", agent.observationRays().size());
  } catch (const nanomap::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
