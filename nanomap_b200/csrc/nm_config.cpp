// nm_config.cpp -- parser of NanoMap's text configuration files.
//
// Formats (whitespace-separated tokens, as read with operator>> by the reference):
//   main config    "#config" ... "#endconfig"          (Config.cpp:60-113, 119-169)
//   frustum sensor "#frustumconfig" ... "#endconfig"   (Config.cpp:226-264)
//   laser sensor   "#laserconfig" ... "#endconfig"     (Config.cpp:185-225)
//   agent          "#agentconfig" ... "#endconfig"     (Agent.h:63-125)
//   cave generator "#cavegenconfig" ... "seed <s>"    (CaveGen.cpp:358-401)
// Every key the reference reads is accepted with the same meaning.  Optional keys extend the
// formats: main config ClampMin:, ClampMax:, UpdateMode: (label|accumulate), ClampOrder:
// (always|crossing), Rounding: (down|nearest), PublishSensor: (the key the shipped config
// writes; the reference only reads PublishType:); sensor configs HFOV: (frustum), LogOddsHit:,
// LogOddsMiss:.  Unknown keys are skipped token by token, as the reference does.  Relative
// file names are tried as given and then relative to the including file's directory.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <functional>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "nanomap_b200.h"
#include "nm_objects.h"

using nm::fail;

namespace {

struct SensorEntry {
  std::string name;
  nm_sensor_desc desc;
};

struct AgentEntry {
  std::string file;
  int spawn_random = 0;
  float position[3] = {0, 0, 0};
  int num_obs = 0;
  float len_obs = 0.f, collision_dist = 0.f;
  std::vector<std::string> sensor_names;
  std::vector<nm_pose> sensor_origins;
};

}  // namespace

struct nm_config_s {
  nm_config_info info{};
  std::string sim_grid;
  std::vector<SensorEntry> sensors;
  std::vector<AgentEntry> agents;
};

namespace {

std::string dir_of(const std::string& p) {
  const size_t k = p.find_last_of('/');
  return k == std::string::npos ? std::string() : p.substr(0, k + 1);
}

bool open_near(const std::string& file, const std::string& base_dir, std::ifstream& in,
               std::string* resolved) {
  in.open(file);
  if (in.good()) {
    *resolved = file;
    return true;
  }
  if (!base_dir.empty() && (file.empty() || file[0] != '/')) {
    in.clear();
    in.open(base_dir + file);
    if (in.good()) {
      *resolved = base_dir + file;
      return true;
    }
  }
  return false;
}

float logit(double p) { return (float)(std::log(p) - std::log(1.0 - p)); }

int parse_sensor(const std::string& file, const std::string& base, SensorEntry* out) {
  std::ifstream in;
  std::string path;
  if (!open_near(file, base, in, &path)) return fail(NM_ERR_IO, "cannot open sensor config '%s'", file.c_str());
  std::string tok;
  in >> tok;
  nm_sensor_desc& d = out->desc;
  std::memset(&d, 0, sizeof(d));
  d.frame_transform[0] = d.frame_transform[4] = d.frame_transform[8] = 1.0f;
  bool laser;
  if (tok == "#laserconfig") {
    laser = true;
  } else if (tok == "#frustumconfig") {
    laser = false;
  } else {
    return fail(NM_ERR_IO, "%s: first token is '%s', expected #frustumconfig or #laserconfig",
                path.c_str(), tok.c_str());
  }
  d.type = laser ? NM_SENSOR_LASER : NM_SENSOR_FRUSTUM;
  float ahres = 0.f, avres = 0.f;
  bool have_lh = false, have_lm = false, ended = false;
  while (in >> tok) {
    if (tok == "Name:") in >> out->name;
    else if (tok == "Id:") in >> d.id;
    else if (tok == "HRes:") in >> d.hres;
    else if (tok == "VRes:") in >> d.vres;
    else if (tok == "AngularHRes:") in >> ahres;
    else if (tok == "AngularVRes:") in >> avres;
    else if (tok == "HFOV:") in >> d.hfov_deg;
    else if (tok == "VFOV:") in >> d.vfov_deg;
    else if (tok == "Rate:") in >> d.rate;
    else if (tok == "MaxRange:") in >> d.max_range;
    else if (tok == "MinRange:") in >> d.min_range;
    else if (tok == "ProbHit:") in >> d.prob_hit;
    else if (tok == "ProbMiss:") in >> d.prob_miss;
    else if (tok == "LogOddsHit:") { in >> d.log_odds_hit; have_lh = true; }
    else if (tok == "LogOddsMiss:") { in >> d.log_odds_miss; have_lm = true; }
    else if (tok == "FrameTransform:") {
      for (int i = 0; i < 9; ++i) in >> d.frame_transform[i];  // column by column (Config.cpp:210-216)
    } else if (tok == "#endconfig") {
      ended = true;
      break;
    }
    if (in.fail()) return fail(NM_ERR_IO, "%s: bad value after '%s'", path.c_str(), tok.c_str());
  }
  if (!ended) return fail(NM_ERR_IO, "%s: missing #endconfig", path.c_str());
  if (laser) {
    if (!(ahres > 0.f) || !(avres > 0.f))
      return fail(NM_ERR_IO, "%s: AngularHRes and AngularVRes must be positive", path.c_str());
    d.hres = (int)(d.hfov_deg / ahres + 1);  // LaserData.h:260-261
    d.vres = (int)(d.vfov_deg / avres + 1);
  }
  if (have_lh != have_lm)
    return fail(NM_ERR_IO, "%s: LogOddsHit and LogOddsMiss must be given together", path.c_str());
  d.explicit_log_odds = have_lh ? 1 : 0;
  if (out->name.empty()) return fail(NM_ERR_IO, "%s: sensor has no Name", path.c_str());
  return NM_OK;
}

int parse_agent(const std::string& file, const std::string& base, AgentEntry* a) {
  std::ifstream in;
  std::string path;
  if (!open_near(file, base, in, &path)) return fail(NM_ERR_IO, "cannot open agent config '%s'", file.c_str());
  a->file = path;
  std::string tok;
  in >> tok;
  if (tok != "#agentconfig")
    return fail(NM_ERR_IO, "%s: first token is '%s', expected #agentconfig", path.c_str(), tok.c_str());
  bool ended = false;
  while (in >> tok) {
    if (tok == "Spawn:") {
      std::string type_key, type;
      in >> type_key >> type;  // "Type:" fixed|Random (Agent.h:73-76)
      if (type == "Random") {
        a->spawn_random = 1;
      } else {
        std::string k;
        float q[4];
        in >> k >> a->position[0] >> a->position[1] >> a->position[2];
        in >> k >> q[0] >> q[1] >> q[2] >> q[3];  // read and ignored (Agent.h:92-102)
      }
    } else if (tok == "Observations:") {
      std::string k;
      in >> k >> a->num_obs >> k >> a->len_obs >> k >> a->collision_dist;
    } else if (tok == "Sensor:") {
      std::string k, name;
      nm_pose p;
      in >> k >> name >> k >> p.position[0] >> p.position[1] >> p.position[2];
      in >> k >> p.orientation[0] >> p.orientation[1] >> p.orientation[2] >> p.orientation[3];  // w x y z
      a->sensor_names.push_back(name);
      a->sensor_origins.push_back(p);
    } else if (tok == "#endconfig") {
      ended = true;
      break;
    }
    if (in.fail()) return fail(NM_ERR_IO, "%s: bad value after '%s'", path.c_str(), tok.c_str());
  }
  if (!ended) return fail(NM_ERR_IO, "%s: missing #endconfig", path.c_str());
  return NM_OK;
}

}  // namespace

extern "C" {

int nm_config_load(const char* path, nm_config* out) {
  if (!path || !out) return fail(NM_ERR_ARG, "null argument");
  *out = nullptr;
  std::ifstream in(path);
  if (!in.good()) return fail(NM_ERR_IO, "cannot open config '%s'", path);
  std::unique_ptr<nm_config_s> c(new nm_config_s());
  nm_config_info& I = c->info;
  // Defaults: the values of the reference's shipped config/config.txt, and the reference's
  // fixed clamps logit(0.12) / logit(0.97) (OccupancyMap.h:41-42).
  I.mapping_res = 0.1f;
  I.grid_res = 0.1f;
  I.prob_hit_thres = 0.5f;
  I.prob_miss_thres = 0.5f;
  I.leaf_edge = 8;
  I.frustum_allocation_factor = 0.4f;
  I.filter_type = 0;
  I.update_type = 0;
  I.precision_type = 0;
  I.publish_sensor = 0;
  I.clamp_min = logit(0.12);
  I.clamp_max = logit(0.97);
  I.update_mode = NM_UPDATE_LABEL;
  I.clamp_mode = NM_CLAMP_ALWAYS;
  I.rounding = NM_ROUND_DOWN;
  std::string tok;
  in >> tok;
  if (tok != "#config")
    return fail(NM_ERR_IO, "%s: first token is '%s', expected #config", path, tok.c_str());
  std::vector<std::string> sensor_files, agent_files;
  bool ended = false;
  while (in >> tok) {
    if (tok == "MappingRes:") in >> I.mapping_res;
    else if (tok == "ProbHitThres:") in >> I.prob_hit_thres;
    else if (tok == "ProbMissThres:") in >> I.prob_miss_thres;
    else if (tok == "GridRes:") in >> I.grid_res;
    else if (tok == "NodeEdge:") in >> I.leaf_edge;
    else if (tok == "FrustumAllocationFactor:") in >> I.frustum_allocation_factor;
    else if (tok == "FilterType:") in >> I.filter_type;
    else if (tok == "UpdateType:") in >> I.update_type;
    else if (tok == "PrecisionType:") in >> I.precision_type;
    else if (tok == "PublishType:" || tok == "PublishSensor:") in >> I.publish_sensor;
    else if (tok == "ClampMin:") in >> I.clamp_min;
    else if (tok == "ClampMax:") in >> I.clamp_max;
    else if (tok == "UpdateMode:") {
      std::string v;
      in >> v;
      if (v == "label") I.update_mode = NM_UPDATE_LABEL;
      else if (v == "accumulate") I.update_mode = NM_UPDATE_ACCUMULATE;
      else return fail(NM_ERR_IO, "%s: UpdateMode '%s' (label|accumulate)", path, v.c_str());
    } else if (tok == "ClampOrder:") {
      std::string v;
      in >> v;
      if (v == "always") I.clamp_mode = NM_CLAMP_ALWAYS;
      else if (v == "crossing") I.clamp_mode = NM_CLAMP_ON_CROSSING;
      else return fail(NM_ERR_IO, "%s: ClampOrder '%s' (always|crossing)", path, v.c_str());
    } else if (tok == "Rounding:") {
      std::string v;
      in >> v;
      if (v == "down") I.rounding = NM_ROUND_DOWN;
      else if (v == "nearest") I.rounding = NM_ROUND_NEAREST;
      else return fail(NM_ERR_IO, "%s: Rounding '%s' (down|nearest)", path, v.c_str());
    } else if (tok == "SimGrid:") in >> c->sim_grid;
    else if (tok == "Sensor:") {
      std::string f;
      in >> f;
      sensor_files.push_back(f);
    } else if (tok == "Agent:") {
      std::string f;
      in >> f;
      agent_files.push_back(f);
    } else if (tok == "#endconfig") {
      ended = true;
      break;
    }
    if (in.fail()) return fail(NM_ERR_IO, "%s: bad value after '%s'", path, tok.c_str());
  }
  if (!ended) return fail(NM_ERR_IO, "%s: missing #endconfig", path);
  const std::string base = dir_of(path);
  for (const auto& f : sensor_files) {
    SensorEntry e;
    const int rc = parse_sensor(f, base, &e);
    if (rc != NM_OK) return rc;
    c->sensors.push_back(e);
  }
  for (const auto& f : agent_files) {
    AgentEntry a;
    const int rc = parse_agent(f, base, &a);
    if (rc != NM_OK) return rc;
    c->agents.push_back(a);
  }
  // processType = 1 when any frustum sensor exists (Config.cpp:55-57)
  I.process_type = 0;
  for (const auto& e : c->sensors)
    if (e.desc.type == NM_SENSOR_FRUSTUM) I.process_type = 1;
  I.n_sensors = (int32_t)c->sensors.size();
  I.n_agents = (int32_t)c->agents.size();
  std::snprintf(I.sim_grid, sizeof(I.sim_grid), "%s", c->sim_grid.c_str());
  if (!c->sim_grid.empty() && c->sim_grid[0] != '/' && !base.empty()) {
    std::ifstream t(c->sim_grid);
    if (!t.good()) std::snprintf(I.sim_grid, sizeof(I.sim_grid), "%s%s", base.c_str(), c->sim_grid.c_str());
  }
  *out = c.release();
  return NM_OK;
}

int nm_config_destroy(nm_config c) {
  delete c;
  return NM_OK;
}

int nm_config_get_info(nm_config c, nm_config_info* out) {
  if (!c || !out) return fail(NM_ERR_ARG, "null argument");
  *out = c->info;
  return NM_OK;
}

int nm_config_sensor(nm_config c, int32_t i, nm_sensor_desc* desc, char* name, int32_t name_cap) {
  if (!c || !desc) return fail(NM_ERR_ARG, "null argument");
  if (i < 0 || i >= (int32_t)c->sensors.size()) return fail(NM_ERR_ARG, "sensor index %d out of range", i);
  *desc = c->sensors[i].desc;
  if (name && name_cap > 0) std::snprintf(name, (size_t)name_cap, "%s", c->sensors[i].name.c_str());
  return NM_OK;
}

int nm_config_agent(nm_config c, int32_t i, nm_agent_info* out) {
  if (!c || !out) return fail(NM_ERR_ARG, "null argument");
  if (i < 0 || i >= (int32_t)c->agents.size()) return fail(NM_ERR_ARG, "agent index %d out of range", i);
  const AgentEntry& a = c->agents[i];
  std::memset(out, 0, sizeof(*out));
  out->spawn_random = a.spawn_random;
  for (int k = 0; k < 3; ++k) out->position[k] = a.position[k];
  out->num_obs = a.num_obs;
  out->len_obs = a.len_obs;
  out->collision_dist = a.collision_dist;
  out->n_sensors = (int32_t)a.sensor_names.size();
  return NM_OK;
}

int nm_config_agent_sensor(nm_config c, int32_t agent, int32_t j, char* name, int32_t name_cap,
                           nm_pose* origin) {
  if (!c || !origin) return fail(NM_ERR_ARG, "null argument");
  if (agent < 0 || agent >= (int32_t)c->agents.size()) return fail(NM_ERR_ARG, "agent index %d out of range", agent);
  const AgentEntry& a = c->agents[agent];
  if (j < 0 || j >= (int32_t)a.sensor_names.size()) return fail(NM_ERR_ARG, "agent sensor %d out of range", j);
  if (name && name_cap > 0) std::snprintf(name, (size_t)name_cap, "%s", a.sensor_names[j].c_str());
  *origin = a.sensor_origins[j];
  return NM_OK;
}

int nm_config_map_desc(nm_config c, nm_map_desc* out) {
  if (!c || !out) return fail(NM_ERR_ARG, "null argument");
  const nm_config_info& I = c->info;
  std::memset(out, 0, sizeof(*out));
  out->res = I.mapping_res;
  out->leaf_edge = I.leaf_edge;
  // OccupancyMap.h:30-31: thresholds are logit(ProbHitThres) / logit(ProbMissThres)
  out->thres_hit = logit(I.prob_hit_thres);
  out->thres_miss = logit(I.prob_miss_thres);
  out->clamp_min = I.clamp_min;
  out->clamp_max = I.clamp_max;
  out->clamp_mode = I.clamp_mode;
  out->update_mode = I.update_mode;
  out->rounding = I.rounding;
  out->max_agents = 1;
  return NM_OK;
}

// CaveGen::loadConfig (CaveGen.cpp:358-401): keys are read in any order until "seed <s>";
// random_seed 1 seeds from the clock, anything else from the seed string.  The seed is the
// reference's: std::hash of the string (or of time(0)) stored in an int, i.e. its low 32 bits,
// which srand receives.  A missing random_seed key counts as 0 (the reference leaves it
// unset).
int nm_cave_config_load(const char* path, nm_cave_desc* out) {
  if (!path || !out) return fail(NM_ERR_ARG, "null argument");
  std::memset(out, 0, sizeof(*out));
  std::ifstream in(path, std::ios::in | std::ios::binary);
  if (!in) return fail(NM_ERR_IO, "cannot open cave config '%s'", path);
  std::string line;
  in >> line;
  if (line != "#cavegenconfig")
    return fail(NM_ERR_IO, "%s: first token is [%s] instead of [#cavegenconfig]", path,
                line.c_str());
  std::string file_out, seed;
  int random_seed = 0;
  bool done = false;
  while (in.good() && !done) {
    if (!(in >> line)) break;
    if (line == "file_out") {
      in >> file_out;
    } else if (line == "map_size") {
      in >> out->map_size[0] >> out->map_size[1] >> out->map_size[2];
    } else if (line == "grid_res") {
      in >> out->grid_res;
    } else if (line == "fill_percentage") {
      in >> out->fill_percentage;
    } else if (line == "smoothing_count") {
      in >> out->smoothing_count;
    } else if (line == "active") {
      in >> out->active_max >> out->active_min;
    } else if (line == "random_seed") {
      in >> random_seed;
    } else if (line == "seed") {
      in >> seed;
      done = true;
    }
  }
  if (file_out.size() >= sizeof(out->file_out))
    return fail(NM_ERR_IO, "%s: file_out is longer than %zu bytes", path,
                sizeof(out->file_out) - 1);
  std::snprintf(out->file_out, sizeof(out->file_out), "%s", file_out.c_str());
  out->time_seed = (random_seed == 1) ? 1 : 0;
  const size_t h = out->time_seed ? std::hash<std::time_t>{}(std::time(nullptr))
                                  : std::hash<std::string>{}(seed);
  out->seed = (uint32_t)h;
  if (!(out->grid_res > 0.0))
    return fail(NM_ERR_IO, "%s: grid_res missing or not positive", path);
  return NM_OK;
}

}  // extern "C"
