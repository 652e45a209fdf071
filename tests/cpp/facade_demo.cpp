// facade_demo.cpp -- test program: drives the C++ facade the way a NanoMap user does.
//
// usage: facade_demo <config> <frames.bin> <manager_map.bin> <sim_map.bin> <sim_poses.bin>
//                    [<collisions.bin>]
//   frames.bin: int32 n, width, height, step; n poses (7 floats: x y z qw qx qy qz);
//               n clouds of width*height records of `step` bytes (xyz at 0/4/8).
// Writes the maps' leaves (uint64 n, then origins, log-odds, active words) and the sensor
// poses the sim manager used (int32 count, then per view: int32 sensor index, 7 floats), and
// getAgentSimCollision for agent 0 over a 5x5x3 grid of position deltas (int32 count, then
// per delta: 3 floats and an int32 0/1).
#include <cstdint>
#include <cstdio>
#include <vector>

#include "nanomap_b200/nanomap.hpp"

static void dump(nanomap::map::Map& m, const char* path) {
  std::vector<int32_t> o;
  std::vector<float> v;
  std::vector<uint32_t> a;
  m.exportLeaves(o, v, a);
  FILE* f = std::fopen(path, "wb");
  const uint64_t n = o.size() / 3;
  std::fwrite(&n, 8, 1, f);
  std::fwrite(o.data(), 4, o.size(), f);
  std::fwrite(v.data(), 4, v.size(), f);
  std::fwrite(a.data(), 4, a.size(), f);
  std::fclose(f);
}

int main(int argc, char** argv) {
  if (argc != 6 && argc != 7) return 2;
  try {
    auto cfg = std::make_shared<nanomap::config::Config>(argv[1]);
    FILE* f = std::fopen(argv[2], "rb");
    int32_t hdr[4];
    if (!f || std::fread(hdr, 4, 4, f) != 4) return 3;
    const int n = hdr[0], w = hdr[1], h = hdr[2], step = hdr[3];
    std::vector<float> poses((size_t)n * 7);
    if (std::fread(poses.data(), 4, poses.size(), f) != poses.size()) return 3;
    std::vector<unsigned char> clouds((size_t)n * w * h * step);
    if (std::fread(clouds.data(), 1, clouds.size(), f) != clouds.size()) return 3;
    std::fclose(f);

    // Manager::insertPointCloud into a map built from the config (Manager.h:52-63)
    nanomap::manager::Manager mgr(cfg);
    auto map = std::make_shared<nanomap::map::Map>(cfg->mapDesc());
    const std::string cam = cfg->sensorData(0)->getName();
    for (int i = 0; i < n; ++i) {
      nanomap::Pose p;
      const float* q = &poses[(size_t)i * 7];
      p.position = nanomap::Vector3f(q[0], q[1], q[2]);
      p.orientation = nanomap::Quaternionf(q[3], q[4], q[5], q[6]);
      mgr.insertPointCloud(cam, w, h, step, clouds.data() + (size_t)i * w * h * step, p, map);
      mgr.insertPointCloud("no-such-sensor", w, h, step, clouds.data(), p, map);  // no-op
    }
    mgr.printUpdateTime(n);
    dump(*map, argv[3]);

    // SimManager: sim grid from the config's SimGrid file, agents from Agent: files
    nanomap::manager::SimManager sim(cfg);
    std::vector<std::pair<int, nanomap::Pose>> used;
    auto record = [&]() {
      auto a = sim.agent(0);
      const auto names = a->sensorNames();
      for (size_t j = 0; j < names.size(); ++j)
        for (size_t k = 0; k < cfg->sensorData().size(); ++k)
          if (cfg->sensorData()[k]->getName() == names[j]) used.push_back({(int)k, a->sensorPose((int)j)});
    };
    sim.updateAgentViews();
    record();
    nanomap::Pose moved = sim.agentPoses()[0];
    moved.position = nanomap::Vector3f(moved.position(0) + 0.7f, moved.position(1) - 0.4f, moved.position(2));
    moved.orientation = nanomap::Quaternionf(0.9659258f, 0.f, 0.f, 0.2588190f);
    sim.updateAgentPoses({moved});
    sim.updateAgentViews();
    record();
    dump(*sim.getMap(0), argv[4]);
    FILE* g = std::fopen(argv[5], "wb");
    const int32_t cnt = (int32_t)used.size();
    std::fwrite(&cnt, 4, 1, g);
    for (auto& u : used) {
      const nm_pose p = u.second.c();
      std::fwrite(&u.first, 4, 1, g);
      std::fwrite(p.position, 4, 3, g);
      std::fwrite(p.orientation, 4, 4, g);
    }
    std::fclose(g);
    if (argc == 7) {
      FILE* c = std::fopen(argv[6], "wb");
      const int32_t nd = 5 * 5 * 3;
      std::fwrite(&nd, 4, 1, c);
      for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j)
          for (int k = 0; k < 3; ++k) {
            const nanomap::Vector3f d(-2.0f + 1.0f * i, -2.0f + 1.0f * j, -0.5f + 0.5f * k);
            const int32_t free_ = sim.getAgentSimCollision(0, d) ? 1 : 0;
            std::fwrite(d.v, 4, 3, c);
            std::fwrite(&free_, 4, 1, c);
          }
      std::fclose(c);
    }
  } catch (const nanomap::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
