// nanomap.hpp -- C++ facade with NanoMap's class names and signatures over the C ABI.
//
// Header only; link libnanomap_b200.so.  Mirrors the reference's public API for the mapping
// and simulation path:
//   nanomap::Pose                               nanomap.h:20-28
//   nanomap::config::Config(std::string)        Config.h:42-91, Config.cpp:18-59
//   nanomap::map::Map(gridRes, probThresHit, probThresMiss)   OccupancyMap.h:35-61
//   nanomap::agent::Agent (updatePose, sensorPose, map)       Agent.h:49-210
//   nanomap::manager::Manager::insertPointCloud               Manager.h:46-72
//   nanomap::manager::SimManager::updateAgentViews([map])     SimManager.h:68-168
//   nanomap::mapgen::CaveGen(std::string) and its stages      CaveGen.h:32-68
// Eigen is not required: Vector3f / Quaternionf below keep Eigen's construction order
// (Quaternionf(w, x, y, z)) and accessors.  Failures of the library raise nanomap::Error
// (the reference reports nothing); an unknown sensor name in insertPointCloud is a no-op, as
// in the reference's name scan (Manager.h:55-57).
#pragma once

#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_set>
#include <vector>

#include "../nanomap_b200.h"

namespace nanomap {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

namespace detail {
inline void check(int rc) {
  if (rc != NM_OK) throw Error(rc, std::string("nanomap_b200: ") + nm_last_error());
}
inline int& device_index() {
  static int dev = 0;
  return dev;
}
// One library context per process (created on first use, on device_index()).
inline nm_context context() {
  static std::shared_ptr<nm_context_s> ctx;
  if (!ctx) {
    nm_context c = nullptr;
    check(nm_context_create(device_index(), &c));
    ctx.reset(c, [](nm_context p) { nm_context_destroy(p); });
  }
  return ctx.get();
}
inline float logit(double p) { return (float)(std::log(p) - std::log(1.0 - p)); }
}  // namespace detail

// Device used by every object created afterwards (default 0).
inline void setDevice(int device) { detail::device_index() = device; }

struct Vector3f {
  float v[3];
  Vector3f() : v{0.f, 0.f, 0.f} {}
  Vector3f(float x, float y, float z) : v{x, y, z} {}
  float& operator()(int i) { return v[i]; }
  float operator()(int i) const { return v[i]; }
  float x() const { return v[0]; }
  float y() const { return v[1]; }
  float z() const { return v[2]; }
  Vector3f operator+(const Vector3f& o) const { return {v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]}; }
};

struct Quaternionf {
  float w_, x_, y_, z_;
  Quaternionf() : w_(1.f), x_(0.f), y_(0.f), z_(0.f) {}
  Quaternionf(float w, float x, float y, float z) : w_(w), x_(x), y_(y), z_(z) {}
  float w() const { return w_; }
  float x() const { return x_; }
  float y() const { return y_; }
  float z() const { return z_; }
  Quaternionf normalized() const {
    const float n = std::sqrt(w_ * w_ + x_ * x_ + y_ * y_ + z_ * z_);
    return {w_ / n, x_ / n, y_ / n, z_ / n};
  }
  // Hamilton product, Eigen's operator* order (this applied after o).
  Quaternionf operator*(const Quaternionf& o) const {
    return {w_ * o.w_ - x_ * o.x_ - y_ * o.y_ - z_ * o.z_, w_ * o.x_ + x_ * o.w_ + y_ * o.z_ - z_ * o.y_,
            w_ * o.y_ - x_ * o.z_ + y_ * o.w_ + z_ * o.x_, w_ * o.z_ + x_ * o.y_ - y_ * o.x_ + z_ * o.w_};
  }
};

// nanomap.h:20-28: default orientation Quaternionf(0, 0, 0, 1), i.e. w = 0, z = 1.
struct Pose {
  Vector3f position;
  Quaternionf orientation;
  Pose() : position(0.f, 0.f, 0.f), orientation(0.f, 0.f, 0.f, 1.f) {}
  nm_pose c() const {
    nm_pose p;
    for (int i = 0; i < 3; ++i) p.position[i] = position(i);
    p.orientation[0] = orientation.w();
    p.orientation[1] = orientation.x();
    p.orientation[2] = orientation.y();
    p.orientation[3] = orientation.z();
    return p;
  }
};

namespace sensor {
// Parsed sensor description (the parts of FrustumData / LaserData the path uses).
class SensorData {
 public:
  SensorData(std::string name, const nm_sensor_desc& d) : name_(std::move(name)), desc_(d) {}
  std::string sensorName() const { return name_; }
  std::string getName() const { return name_; }
  int getId() const { return desc_.id; }
  int type() const { return desc_.type; }
  int hRes() const { return desc_.hres; }
  int vRes() const { return desc_.vres; }
  const nm_sensor_desc& desc() const { return desc_; }
  // The library-side sensor (created on first use).
  nm_sensor handle() {
    if (!handle_) {
      nm_sensor s = nullptr;
      detail::check(nm_sensor_create(detail::context(), &desc_, &s));
      handle_.reset(s, [](nm_sensor p) { nm_sensor_destroy(p); });
    }
    return handle_.get();
  }

 private:
  std::string name_;
  nm_sensor_desc desc_;
  std::shared_ptr<nm_sensor_s> handle_;
};
}  // namespace sensor

namespace config {
class Config {
 public:
  explicit Config(std::string configFile) : file_(std::move(configFile)) {
    nm_config c = nullptr;
    detail::check(nm_config_load(file_.c_str(), &c));
    cfg_.reset(c, [](nm_config p) { nm_config_destroy(p); });
    detail::check(nm_config_get_info(c, &info_));
    for (int i = 0; i < info_.n_sensors; ++i) {
      nm_sensor_desc d;
      char name[256];
      detail::check(nm_config_sensor(c, i, &d, name, sizeof(name)));
      sensors_.push_back(std::make_shared<sensor::SensorData>(name, d));
    }
    leaf_volume_ = info_.leaf_edge * info_.leaf_edge * info_.leaf_edge;
    for (const auto& sd : sensors_) {
      const nm_sensor_desc& d = sd->desc();
      const int pcl = d.hres * d.vres;
      max_pcl_ = std::max(max_pcl_, pcl);
      if (d.type == NM_SENSOR_FRUSTUM) {
        frustum_pcl_ = std::max(frustum_pcl_, pcl);
        const double leaf = (double)info_.mapping_res * info_.leaf_edge;
        const int n = leaf > 0.0 ? (int)std::ceil(2.0 * d.max_range / leaf) + 2 : 0;
        frustum_leaf_buffer_ = std::max(frustum_leaf_buffer_, n * n * n);
      } else if (d.type == NM_SENSOR_LASER) {
        laser_pcl_ = std::max(laser_pcl_, pcl);
      }
    }
  }
  std::vector<std::shared_ptr<sensor::SensorData>>& sensorData() { return sensors_; }
  std::shared_ptr<sensor::SensorData> sensorData(int index, bool searchById = false) {
    if (searchById) {
      for (auto& s : sensors_)
        if (s->getId() == index) return s;
      return nullptr;
    }
    return (index >= 0 && index < (int)sensors_.size()) ? sensors_[index] : nullptr;
  }
  std::shared_ptr<sensor::SensorData> sensorData(const std::string& name) {
    for (auto& s : sensors_)
      if (s->getName() == name) return s;
    return nullptr;
  }
  float& mappingRes() { return info_.mapping_res; }
  float& gridRes() { return info_.grid_res; }
  int& leafEdge() { return info_.leaf_edge; }
  int& filterType() { return info_.filter_type; }
  int& updateType() { return info_.update_type; }
  int& processType() { return info_.process_type; }
  int& precisionType() { return info_.precision_type; }
  int& publishSensor() { return info_.publish_sensor; }
  float& probHitThres() { return info_.prob_hit_thres; }
  float& probMissThres() { return info_.prob_miss_thres; }
  float& frustumAllocationFactor() { return info_.frustum_allocation_factor; }
  // Keys the reference's reader never reads (Config.cpp:60-113): they keep their defaults.
  int& exploreType() { return explore_type_; }
  int& simType() { return sim_type_; }
  bool& serialUpdate() { return serial_update_; }
  float& laserAllocationFactor() { return laser_allocation_factor_; }
  // Derived as in Config::init (Config.cpp:24-58): leaf volume and the largest point cloud of
  // all, of the frustum and of the laser sensors.  frustumLeafBufferSize is an upper bound of
  // the leaves any rotation of a frustum sensor covers, the leaf box of its range sphere (the
  // reference searches 5.8 M rotations for the exact worst case; this library bounds each
  // frame's leaves from its pose instead).  laserVoxelBufferSize is left at 0, as the
  // reference leaves it unset.
  int& leafVolume() { return leaf_volume_; }
  int& maxPCLSize() { return max_pcl_; }
  int& frustumPCLSize() { return frustum_pcl_; }
  int& laserPCLSize() { return laser_pcl_; }
  int& frustumLeafBufferSize() { return frustum_leaf_buffer_; }
  int& laserVoxelBufferSize() { return laser_voxel_buffer_; }
  std::string& config() { return file_; }
  std::string simGrid() const { return info_.sim_grid; }
  int agentCount() const { return info_.n_agents; }
  nm_config handle() const { return cfg_.get(); }
  nm_map_desc mapDesc() const {
    nm_map_desc d;
    detail::check(nm_config_map_desc(cfg_.get(), &d));
    return d;
  }

 private:
  std::string file_;
  std::shared_ptr<nm_config_s> cfg_;
  nm_config_info info_{};
  std::vector<std::shared_ptr<sensor::SensorData>> sensors_;
  int explore_type_ = 0, sim_type_ = 0;
  bool serial_update_ = false;
  float laser_allocation_factor_ = 0.f;
  int leaf_volume_ = 0, max_pcl_ = 0, frustum_pcl_ = 0, laser_pcl_ = 0;
  int frustum_leaf_buffer_ = 0, laser_voxel_buffer_ = 0;
};
}  // namespace config

namespace map {
// OccupancyMap.h:35-52: thresholds logit(probThres*), clamps logit(0.12) / logit(0.97).  The
// map lives on the device; exportLeaves() copies it out.
class Map {
 public:
  Map() : Map(0.1f, 0.5f, 0.5f) {}
  Map(float gridRes, float probThresHit, float probThresMiss, float mappingRes = 0,
      float plannerRes = 0, int nodeEdge = 0) {
    (void)mappingRes;
    (void)plannerRes;
    (void)nodeEdge;
    std::memset(&desc_, 0, sizeof(desc_));
    desc_.res = gridRes;
    desc_.leaf_edge = 8;
    desc_.thres_hit = detail::logit(probThresHit);
    desc_.thres_miss = detail::logit(probThresMiss);
    desc_.clamp_min = detail::logit(0.12);
    desc_.clamp_max = detail::logit(0.97);
    desc_.clamp_mode = NM_CLAMP_ALWAYS;
    desc_.update_mode = NM_UPDATE_LABEL;
    desc_.rounding = NM_ROUND_DOWN;
    desc_.max_agents = 1;
  }
  explicit Map(const nm_map_desc& d) : desc_(d) {}
  float occupiedClampingThreshold() const { return desc_.clamp_max; }
  float emptyClampingThreshold() const { return desc_.clamp_min; }
  float logOddsHitThreshold() const { return desc_.thres_hit; }
  float logOddsMissThreshold() const { return desc_.thres_miss; }
  float gridRes() const { return desc_.res; }
  nm_map_desc& desc() { return desc_; }
  nm_map handle() {
    if (!handle_) {
      nm_map m = nullptr;
      detail::check(nm_map_create(detail::context(), &desc_, &m));
      handle_.reset(m, [](nm_map p) { nm_map_destroy(p); });
    }
    return handle_.get();
  }
  // Leaves: origins (3 per leaf), log-odds (512 per leaf), active words (16 per leaf).
  void exportLeaves(std::vector<int32_t>& origins, std::vector<float>& values,
                    std::vector<uint32_t>& active) {
    uint64_t n = 0;
    detail::check(nm_map_export(handle(), nullptr, nullptr, nullptr, 0, &n));
    origins.resize(n * 3);
    values.resize(n * 512);
    active.resize(n * 16);
    if (n) detail::check(nm_map_export(handle(), origins.data(), values.data(), active.data(), n, &n));
  }
  nm_stats stats() {
    nm_stats s;
    detail::check(nm_map_stats(handle(), &s));
    return s;
  }

 private:
  nm_map_desc desc_;
  std::shared_ptr<nm_map_s> handle_;
};
}  // namespace map

namespace agent {
class Agent {
 public:
  // Agent `index` of the config (Agent.h:49-135): fixed spawn position, the reference's fixed
  // body rotation (columns (0,-1,0), (1,0,0), (0,0,1)), sensors with mount poses.
  Agent(config::Config& cfg, int index, std::shared_ptr<map::Map> map = nullptr) : id_(index) {
    nm_agent_info a;
    detail::check(nm_config_agent(cfg.handle(), index, &a));
    if (a.spawn_random)
      throw Error(NM_ERR_UNSUPPORTED,
                  "nanomap_b200: random agent spawns are not supported; give the agent a spawn pose");
    pose_.position = Vector3f(a.position[0], a.position[1], a.position[2]);
    pose_.orientation = Quaternionf(std::sqrt(0.5f), 0.f, 0.f, -std::sqrt(0.5f));
    num_obs_ = a.num_obs;
    len_obs_ = a.len_obs;
    collision_dist_ = a.collision_dist;
    if (num_obs_ >= 2) {
      std::vector<float> d(3 * (size_t)num_obs_);
      detail::check(nm_observation_sphere(num_obs_, d.data()));
      for (int i = 0; i < num_obs_; ++i)
        obs_rays_.push_back(Vector3f(d[3 * i], d[3 * i + 1], d[3 * i + 2]));
    }
    for (int j = 0; j < a.n_sensors; ++j) {
      char name[256];
      nm_pose o;
      detail::check(nm_config_agent_sensor(cfg.handle(), index, j, name, sizeof(name), &o));
      Pose p;
      p.position = Vector3f(o.position[0], o.position[1], o.position[2]);
      p.orientation = Quaternionf(o.orientation[0], o.orientation[1], o.orientation[2], o.orientation[3]);
      names_.push_back(name);
      origins_.push_back(p);
    }
    poses_ = origins_;
    map_ = map ? map : std::make_shared<map::Map>(cfg.mapDesc());
    updatePose(pose_);
  }
  // Agent.h:136-145: sensor position = agent position (the mount offset is not applied),
  // sensor orientation = agent orientation * mount orientation.
  void updatePose(Pose pose) {
    pose_ = pose;
    for (size_t i = 0; i < origins_.size(); ++i) {
      poses_[i].position = pose_.position;
      poses_[i].orientation = pose_.orientation * origins_[i].orientation;
    }
  }
  Pose pose() const { return pose_; }
  Pose sensorPose(int index) const { return poses_[index]; }
  std::vector<Pose> sensorPoses() const { return poses_; }
  std::vector<Pose> sensorOrigins() const { return origins_; }
  std::vector<std::string> sensorNames() const { return names_; }
  std::shared_ptr<map::Map> map() { return map_; }
  bool spawnRandom() const { return false; }
  // Observation sphere (Agent.h:147-192): unit ray directions, collision distance (m) and
  // observation length (m) from the agent file's Observations: line.
  const std::vector<Vector3f>& observationRays() const { return obs_rays_; }
  float collisionDist() const { return collision_dist_; }
  float observationLength() const { return len_obs_; }
  // Agent.h:181-192: (collision distance, observation length) for each observation ray.
  std::vector<std::array<float, 2>> observationNorms() const {
    return std::vector<std::array<float, 2>>(obs_rays_.size(), {collision_dist_, len_obs_});
  }
  // Agent.h:198-207
  void clearSensors() {
    poses_.clear();
    names_.clear();
    origins_.clear();
  }
  void clearObservationRays() { obs_rays_.clear(); }
  void resetAgent() {
    clearSensors();
    clearObservationRays();
  }
  // The reference never sets its agent id and name; here the id is the config index.
  int getId() const { return id_; }
  std::string getName() const { return std::string(); }

 private:
  int id_ = 0;
  int num_obs_ = 0;
  float len_obs_ = 0.f, collision_dist_ = 0.f;
  std::vector<Vector3f> obs_rays_;
  Pose pose_;
  std::vector<std::string> names_;
  std::vector<Pose> origins_, poses_;
  std::shared_ptr<map::Map> map_;
};
}  // namespace agent

namespace manager {

using Map = nanomap::map::Map;

class Manager {
 public:
  explicit Manager(std::shared_ptr<config::Config> config) : config_(std::move(config)) {}

  void insertPointCloud(std::string sensorName, int pcl_width, int pcl_height, int pcl_step,
                        unsigned char* cloud, const nanomap::Pose& pose, std::shared_ptr<Map> map) {
    for (auto& s : config_->sensorData()) {
      if (s->sensorName() != sensorName) continue;
      const auto t0 = std::chrono::high_resolution_clock::now();
      const nm_pose p = pose.c();
      detail::check(nm_map_insert_points(map->handle(), s->handle(), &p, cloud, pcl_width, pcl_height,
                                         pcl_step, NM_INPUT_HOST | NM_SYNC, nullptr));
      const auto t1 = std::chrono::high_resolution_clock::now();
      gpu_ms_ += std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
  }
  void printUpdateTime(int count) {
    std::cout << "gpu update time per loop:" << gpu_ms_ / count << std::endl;
    std::cout << "map update time per loop:" << 0.0 << std::endl;
  }
  void closeHandler() {}
  std::shared_ptr<config::Config> config() { return config_; }

 private:
  std::shared_ptr<config::Config> config_;
  double gpu_ms_ = 0.0;
};

class SimManager {
 public:
  // Loads the sim grid named by the config's SimGrid: key (a .vdb grid or an NMSIMv1 voxel
  // list) and the agents.
  explicit SimManager(std::shared_ptr<config::Config> config) : config_(std::move(config)) {
    nm_simmap sm = nullptr;
    detail::check(nm_simmap_load(detail::context(), config_->simGrid().c_str(), &sm));
    sim_.reset(sm, [](nm_simmap p) { nm_simmap_destroy(p); });
    load_agents();
  }
  // With a sim map built by the caller (nm_simmap_create_primitives / _voxels).
  SimManager(std::shared_ptr<config::Config> config, nm_simmap sim) : config_(std::move(config)) {
    sim_.reset(sim, [](nm_simmap) {});
    load_agents();
  }

  void updateAgentPoses(std::vector<Pose> poses) {
    for (size_t i = 0; i < poses.size() && i < agents_.size(); ++i) agents_[i]->updatePose(poses[i]);
  }
  std::vector<Pose> agentPoses() {
    std::vector<Pose> out;
    for (auto& a : agents_) out.push_back(a->pose());
    return out;
  }
  // Every agent's sensors render from the sim map and map into the agent's own map.
  void updateAgentViews() {
    for (auto& a : agents_) view(*a, a->map());
  }
  // Every agent maps into one shared map (SimManager.h:114-127).
  void updateAgentViews(std::shared_ptr<Map> map_ptr) {
    for (auto& a : agents_) view(*a, map_ptr);
  }
  std::shared_ptr<Map> getMap(int index) { return agents_[index]->map(); }
  // SimManager.h:141-168: true when agent `index` can move by positionDelta, i.e. none of its
  // observation rays, cast from the new position, meets an active sim voxel closer than the
  // agent's collision distance (exact to the voxel; the reference tests leaf-node spans).
  bool getAgentSimCollision(int index, Vector3f positionDelta) {
    const agent::Agent& a = *agents_[index];
    const auto& rays = a.observationRays();
    if (rays.empty()) return true;
    const Vector3f eye = a.pose().position + positionDelta;
    std::vector<float> o(3 * rays.size()), d(3 * rays.size()), dist(rays.size());
    for (size_t i = 0; i < rays.size(); ++i)
      for (int k = 0; k < 3; ++k) {
        o[3 * i + k] = eye(k);
        d[3 * i + k] = rays[i](k);
      }
    detail::check(nm_sim_cast_rays(sim_.get(), o.data(), d.data(), (int64_t)rays.size(),
                                   a.collisionDist(), dist.data(),
                                   NM_INPUT_HOST | NM_OUTPUT_HOST, nullptr));
    for (float x : dist)
      if (x > 0.f && x < a.collisionDist()) return false;
    return true;
  }
  std::shared_ptr<agent::Agent> agent(int index) { return agents_[index]; }
  nm_simmap simMap() { return sim_.get(); }
  void closeHandler() {}
  // empty in the reference (SimManager.h:137-139)
  void step() {}
  void updateObservations() {}

 private:
  void load_agents() {
    for (int i = 0; i < config_->agentCount(); ++i)
      agents_.push_back(std::make_shared<agent::Agent>(*config_, i));
  }
  // SimHandler::processPointCloud per sensor (SimHandler.cpp:234-280): render and insert in
  // one launch, without a range-image buffer.
  void view(agent::Agent& a, std::shared_ptr<Map> map) {
    const auto names = a.sensorNames();
    for (size_t j = 0; j < names.size(); ++j) {
      auto s = config_->sensorData(names[j]);
      if (!s) continue;
      const nm_pose p = a.sensorPose((int)j).c();
      detail::check(nm_sim_insert(sim_.get(), map->handle(), s->handle(), &p, 0.0f, 0.0f, 0,
                                  nullptr, 0, nullptr));
    }
  }

  std::shared_ptr<config::Config> config_;
  std::shared_ptr<nm_simmap_s> sim_;
  std::vector<std::shared_ptr<agent::Agent>> agents_;
};

}  // namespace manager

namespace mapgen {

// nanomap::mapgen::CaveGen (CaveGen.h:32-68) over nm_cave_*: the same stages in the same
// order give the same cave for the same #cavegenconfig file (the fill reproduces the
// reference's srand/rand draws without changing the caller's rand() state).  The cells stay
// on the device; invertAndSave / Save write file_out (ending in ".vdb": the active band as the
// float grid "grid" of a .vdb file, as the reference writes it; otherwise an NMSIMv1 voxel
// list; writtenPath() names it) for SimManager's sim grid loader, and simMap() hands the cave
// to a SimManager without a file.
class CaveGen {
 public:
  explicit CaveGen(std::string config) { loadConfig(std::move(config)); }

  // CaveGen::gen (CaveGen.cpp:337-342)
  void gen() {
    populateMap();
    smoothMap();
    getRegions();
    invertAndSave();
  }
  void populateMap() { detail::check(nm_cave_populate(cave_.get(), 0)); }
  void populateMap2D() { detail::check(nm_cave_populate(cave_.get(), NM_CAVE_2D)); }
  void smoothMap() { detail::check(nm_cave_smooth(cave_.get(), 0)); }
  void smoothMapXY() { detail::check(nm_cave_smooth(cave_.get(), NM_CAVE_2D)); }
  void setFloorAndCeil() { detail::check(nm_cave_floor_ceil(cave_.get())); }
  void getRegions() { detail::check(nm_cave_regions(cave_.get(), &regions_, &largest_)); }
  void keepLargestRegion() { detail::check(nm_cave_keep_largest(cave_.get())); }
  void addNoise() {}  // empty in the reference (CaveGen.cpp:254-256)
  // level-set band with topologyToLevelSet's defaults (half width 3, closing 1)
  void invertAndSave() { save(1); }
  // the on cells' leaves, voxelised
  void Save() { save(0); }
  void loadConfig(std::string file_in) {
    detail::check(nm_cave_config_load(file_in.c_str(), &desc_));
    nm_cave c = nullptr;
    detail::check(nm_cave_create(detail::context(), &desc_, &c));
    cave_.reset(c, [](nm_cave p) { nm_cave_destroy(p); });
  }
  // CaveGen::getActiveNeighbourCount / get2DNeighbourCount (CaveGen.cpp:258-292): on cells
  // among the 26 (8 in the floor plane) lattice neighbours of voxel (x, y, z) / (x, y).
  int getActiveNeighbourCount(int x, int y, int z) {
    const auto on = onCells();
    int n = 0;
    for (int dx = -8; dx <= 8; dx += 8)
      for (int dy = -8; dy <= 8; dy += 8)
        for (int dz = -8; dz <= 8; dz += 8)
          if ((dx || dy || dz) && on.count(key(x + dx, y + dy, z + dz))) ++n;
    return n;
  }
  int get2DNeighbourCount(int x, int y) {
    int32_t half[3];
    detail::check(nm_cave_dims(cave_.get(), half, nullptr));
    const auto on = onCells();
    int n = 0;
    for (int dx = -8; dx <= 8; dx += 8)
      for (int dy = -8; dy <= 8; dy += 8)
        if ((dx || dy) && on.count(key(x + dx, y + dy, -half[2]))) ++n;
    return n;
  }

  // additions
  nm_simmap simMap(bool shell = true) {
    nm_simmap sm = nullptr;
    detail::check(nm_cave_simmap(cave_.get(), shell ? 1 : 0, 3, 1, &sm));
    return sm;  // the caller destroys it (nm_simmap_destroy)
  }
  const std::string& writtenPath() const { return written_; }
  int64_t regionCount() const { return regions_; }
  int64_t largestRegion() const { return largest_; }
  const nm_cave_desc& desc() const { return desc_; }

 private:
  static uint64_t key(int x, int y, int z) {
    return ((uint64_t)(uint32_t)(x + (1 << 20)) << 42) | ((uint64_t)(uint32_t)(y + (1 << 20)) << 21) |
           (uint64_t)(uint32_t)(z + (1 << 20));
  }
  std::unordered_set<uint64_t> onCells() {
    int64_t n = 0;
    detail::check(nm_cave_cells(cave_.get(), nullptr, 0, &n));
    std::vector<int32_t> xyz((size_t)n * 3 + 3);
    detail::check(nm_cave_cells(cave_.get(), xyz.data(), n, &n));
    std::unordered_set<uint64_t> on;
    for (int64_t q = 0; q < n; ++q) on.insert(key(xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]));
    return on;
  }
  void save(int shell) {
    char written[512] = {0};
    detail::check(nm_cave_save(cave_.get(), shell, 3, 1, desc_.file_out, written));
    written_ = written;
  }

  nm_cave_desc desc_{};
  std::shared_ptr<nm_cave_s> cave_;
  int64_t regions_ = 0, largest_ = 0;
  std::string written_;
};

}  // namespace mapgen
}  // namespace nanomap
