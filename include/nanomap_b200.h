/*
 * nanomap_b200.h -- C ABI of the B200-native NanoMap mapping and simulation path.
 *
 * Plain C types only: opaque handles, pointers and sizes.  Every call returns an int status
 * (NM_OK or an NM_ERR_* code); nm_last_error() gives the message of the calling thread's
 * last failure.  All device memory belongs to the library; inputs are borrowed for the call;
 * outputs go to caller buffers.  `stream` arguments are cudaStream_t values passed as void*
 * (NULL = the context's own stream).  A context is used from one host thread at a time.
 * The work given to one map is ordered: use one stream per map, or order the streams (an
 * event), since a frame's kernels share the map's tables, counters and claim-order buffers.
 * Calls return once their work is enqueued unless NM_SYNC is given; host input must then
 * stay unchanged until the stream has passed the call.
 * No call changes the caller's floating-point environment.
 *
 * Reference interfaces each entry point replaces are cited as path:line within the
 * NanoMap source tree.
 */
#ifndef NANOMAP_B200_H_
#define NANOMAP_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NM_ABI_VERSION 1

/* status codes */
#define NM_OK 0
#define NM_ERR_ARG 1         /* bad argument (null, size, range) */
#define NM_ERR_CAPACITY 2    /* a fixed-capacity device structure overflowed */
#define NM_ERR_CUDA 3        /* a CUDA runtime call failed */
#define NM_ERR_TIMEOUT 4     /* a bounded device-side wait gave up */
#define NM_ERR_STATE 5       /* call not valid in the object's current state */
#define NM_ERR_IO 6          /* file could not be read or parsed */
#define NM_ERR_UNSUPPORTED 7 /* input format or option this library does not handle */

/* sensor types (SharedParameters::_type, SharedParameters.h:197) */
#define NM_SENSOR_FRUSTUM 0
#define NM_SENSOR_LASER 1

/* map update modes */
#define NM_UPDATE_LABEL 0      /* one update per voxel per frame; hit overrides miss */
#define NM_UPDATE_ACCUMULATE 1 /* per-ray sums (Handler.cpp:47-56, 77-82), from exact counts */

/* clamp order (Handler.cpp:98-110 vs SimHandler.cpp:98-110) */
#define NM_CLAMP_ALWAYS 0
#define NM_CLAMP_ON_CROSSING 1

/* rounding of the per-point host-path arithmetic (the reference sets FE_DOWNWARD in
 * SensorData::updatePose, SensorData.h:42, and never restores it) */
#define NM_ROUND_NEAREST 0
#define NM_ROUND_DOWN 1

/* flags for insert / render / tick calls */
#define NM_INPUT_HOST 0x1u       /* input pointer is host memory, copied inside the call */
#define NM_DEFER_INTEGRATE 0x2u  /* label only; nm_map_integrate applies the labels later */
#define NM_SYNC 0x4u             /* wait for completion; report device-side errors now */
#define NM_OUTPUT_HOST 0x8u      /* output pointer is host memory */
/* Voxel filter of an insert (SensorBucket filter type 1, filterCloud.cu:463-553): the points
 * are binned by the voxel holding their end point and one ray is traced per occupied voxel,
 * to the mean position of its points (voxelFilter + rayFromFilter, filterCloud.cu:84-133,
 * 279-318) or, with NM_FILTER_CENTRE, to the voxel centre (the integer-buffer variants
 * rayFromFilterSimple / rayFromFilterSimpleQuad, filterCloud.cu:360-434). */
#define NM_FILTER_MEAN 0x10u
#define NM_FILTER_CENTRE 0x20u

typedef struct nm_context_s* nm_context;
typedef struct nm_sensor_s* nm_sensor;
typedef struct nm_map_s* nm_map;
typedef struct nm_simmap_s* nm_simmap;
typedef struct nm_tick_plan_s* nm_tick_plan;
typedef struct nm_config_s* nm_config;

/* nanomap::Pose (nanomap.h:20-28): position (m) and unit quaternion (w, x, y, z). */
typedef struct {
  float position[3];
  float orientation[4];
} nm_pose;

/* Sensor parameters (FrustumData.h:261-288, LaserData.h:255-284, Config.cpp:172-267). */
typedef struct {
  int32_t type;              /* NM_SENSOR_FRUSTUM or NM_SENSOR_LASER */
  int32_t id;
  int32_t hres, vres;        /* pixels (frustum) or columns/rows (laser) */
  float hfov_deg;            /* frustum: <= 0 derives it from the aspect ratio (Sensor.h:158-161) */
  float vfov_deg;
  float min_range, max_range;
  float prob_hit, prob_miss; /* used when explicit_log_odds == 0 (Sensor.h:183-184) */
  float log_odds_hit, log_odds_miss;
  int32_t explicit_log_odds;
  int32_t rate;
  float frame_transform[9];  /* column-major: entries 0..2 are column 0 (Config.cpp:210-216) */
} nm_sensor_desc;

/* Map parameters (OccupancyMap.h:35-52 plus the explicit-constant extension). */
typedef struct {
  float res;                 /* voxel edge, metres */
  int32_t leaf_edge;         /* must be 8 (NodeEdge) */
  float thres_hit, thres_miss;   /* log-odds thresholds of the active flag */
  float clamp_min, clamp_max;    /* log-odds clamps */
  int32_t clamp_mode;        /* NM_CLAMP_* */
  int32_t update_mode;       /* NM_UPDATE_* */
  int32_t rounding;          /* NM_ROUND_* */
  uint32_t initial_leaf_capacity; /* 0 = default; the table grows on demand */
  int32_t max_agents;        /* label planes kept for batched ticks (>= 1) */
} nm_map_desc;

/* Cumulative counters of a map, reset by nm_map_reset. */
typedef struct {
  uint64_t frames;
  uint64_t rays;           /* points that produced a traversal */
  uint64_t visits;         /* label events: voxels left by a step plus end voxels */
  uint64_t unique_voxels;  /* voxels integrated (one per voxel per frame) */
  uint64_t touched_leaves; /* leaves integrated, summed over frames */
  uint64_t leaf_count;     /* leaves currently allocated */
  uint64_t leaf_capacity;  /* current hash-table capacity */
  uint32_t error_flags;    /* sticky device error bits, cleared by nm_map_stats */
  uint32_t grow_count;     /* table growths so far */
  uint64_t depth_visits;   /* voxels visited by expected-depth renders, adjoints, refinement */
} nm_stats;

/* One frame of a batched tick. */
typedef struct {
  nm_sensor sensor;
  nm_pose pose;
  const float* ranges;     /* device range image, hres*vres floats (metres; <=0/NaN = none) */
  int32_t agent;           /* label plane, 0 .. max_agents-1; planes integrate in order */
  int32_t pad;
} nm_frame;

/* Main config values (Config.cpp:60-113 plus the optional extension keys). */
typedef struct {
  float mapping_res, grid_res;
  float prob_hit_thres, prob_miss_thres;
  float frustum_allocation_factor;
  float clamp_min, clamp_max;
  int32_t leaf_edge, filter_type, update_type, precision_type, publish_sensor, process_type;
  int32_t update_mode, clamp_mode, rounding;
  int32_t n_sensors, n_agents;
  char sim_grid[512];
} nm_config_info;

/* One agent config (Agent.h:49-135). */
typedef struct {
  int32_t spawn_random;
  float position[3];
  int32_t num_obs;
  float len_obs, collision_dist;
  int32_t n_sensors;
} nm_agent_info;

/* ---- library -------------------------------------------------------------------------- */
int nm_abi_version(void);
const char* nm_last_error(void);

/* ---- configuration files (replaces nanomap::config::Config, Config.cpp:18-267) ---------- */
/* Parses a main config and the sensor / agent configs it names (paths as given, else
 * relative to the main config's directory).  Host only; no device needed. */
int nm_config_load(const char* path, nm_config* out);
int nm_config_destroy(nm_config c);
int nm_config_get_info(nm_config c, nm_config_info* out);
int nm_config_sensor(nm_config c, int32_t i, nm_sensor_desc* desc, char* name, int32_t name_cap);
int nm_config_agent(nm_config c, int32_t i, nm_agent_info* out);
int nm_config_agent_sensor(nm_config c, int32_t agent, int32_t j, char* name, int32_t name_cap,
                           nm_pose* origin);
/* Map parameters a config implies (thresholds logit(ProbHitThres/ProbMissThres), clamps). */
int nm_config_map_desc(nm_config c, nm_map_desc* out);

/* ---- context (replaces Handler's stream pair, Handler.cpp:17-25, and closeHandler) ------ */
int nm_context_create(int32_t device, nm_context* out);
int nm_context_destroy(nm_context ctx);
int nm_context_sync(nm_context ctx);
/* Device buffers for callers without their own CUDA allocator (e.g. range images). */
int nm_alloc_device(nm_context ctx, size_t bytes, void** out);
int nm_free_device(void* p);

/* ---- sensors (replaces FrustumData / LaserData and gpu::Sensor, Sensor.h:147-211) ----- */
int nm_sensor_create(nm_context ctx, const nm_sensor_desc* desc, nm_sensor* out);
int nm_sensor_destroy(nm_sensor s);
/* Frustum constants the kernels use: hw, hh, 2hw, 2hh, 1/W, 1/H. */
int nm_sensor_params(nm_sensor s, float out[6]);

/* ---- maps (replaces nanomap::map::Map, OccupancyMap.h:35-61) --------------------------- */
int nm_map_create(nm_context ctx, const nm_map_desc* desc, nm_map* out);
int nm_map_destroy(nm_map m);
int nm_map_reset(nm_map m);
int nm_map_stats(nm_map m, nm_stats* out);

/* Non-blocking status read for pipelined use: enqueues on `stream` (after the work already on
 * it) a copy of the map's status words into host_status[0..1]: the allocated leaf count and
 * the sticky device error bits (1: leaf-table probe limit reached, 2: a bounded wait gave up;
 * cleared by nm_map_stats).  host_status should be page-locked (the copy is then
 * asynchronous); it is valid once the stream has passed this point, e.g. after an event
 * recorded behind it has completed.  A caller feeding frames without NM_SYNC reads each
 * frame's status this way while the next frame's host input is already being copied. */
int nm_map_status_async(nm_map m, uint32_t* host_status, void* stream);

/* Insert one xyz point cloud: `width*height` records of `step` bytes, float x, y, z at byte
 * offsets 0, 4, 8, in the sensor frame.  Replaces Manager::insertPointCloud (Manager.h:52-63)
 * -> Handler::processPointCloud (Handler.cpp:237-284) -> filterCloud (filterCloud.cu:476)
 * + frustumCastCloud (frustumCastCloud.cu:311) + the host map update (Handler.cpp:134-182). */
int nm_map_insert_points(nm_map m, nm_sensor s, const nm_pose* pose, const void* cloud,
                         int32_t width, int32_t height, int32_t step, uint32_t flags,
                         void* stream);

/* Insert one range image (hres*vres floats, radial metres, <=0 or NaN = no return); the
 * sensor's pixel model turns each range into a sensor-frame point on the device. */
int nm_map_insert_ranges(nm_map m, nm_sensor s, const nm_pose* pose, const float* ranges,
                         uint32_t flags, void* stream);

/* The voxel filter alone: the rays an NM_FILTER_MEAN (or NM_FILTER_CENTRE) insert of this
 * input would trace, as `points` (3 floats per voxel: the ray's end point as a world-frame
 * offset from the sensor position, metres) and `counts` (input points per voxel), in voxel
 * order (x, then y, then z of the end voxel).  step > 0: `input` is an xyz cloud as in
 * nm_map_insert_points; step == 0: `input` is a range image of the sensor (width and height
 * ignored).  NM_INPUT_HOST marks host input; outputs are host memory; the call waits.
 * *n receives the voxel count; at most max_points are written. */
int nm_map_filter_points(nm_map m, nm_sensor s, const nm_pose* pose, const void* input,
                         int32_t width, int32_t height, int32_t step, uint32_t flags,
                         float* points, uint32_t* counts, uint64_t max_points, uint64_t* n);

/* Launch shape of the traversal: tile of tile_w x tile_h pixels per work item (area 64, 128
 * or a multiple of 256 up to 4096; a CTA has min(area, 256) threads) and shared-memory
 * leaf-table entries per CTA (power of two, 16..512).  Results do not depend on it; the autotuner picks it.  No reference
 * counterpart (the reference launches fixed 8x8 / 512-thread grids, filterCloud.cu:482). */
int nm_map_set_launch(nm_map m, int32_t tile_w, int32_t tile_h, int32_t leaf_table_entries);

/* Apply labels left by NM_DEFER_INTEGRATE inserts. */
int nm_map_integrate(nm_map m, void* stream);

/* Batched tick: every frame of `frames` is labelled in one persistent launch, then all label
 * planes are integrated in agent order.  Replaces SimManager::updateAgentViews
 * (SimManager.h:100-127), which runs agents one after another. */
int nm_map_tick(nm_map m, const nm_frame* frames, int32_t n_frames, uint32_t flags,
                void* stream);

/* Tick plans: a batched tick over fixed slots (sensor, device range buffer, agent plane),
 * replayed as a CUDA graph each tick: upload of the per-frame constants derived from the
 * slots' poses, one launch rendering (and noising) every slot from `sim` when it is given,
 * one persistent traversal over all slots, and one integration of all planes in agent order.
 * At most 32 slots.  nm_tick_plan_run with NM_DEFER_INTEGRATE replays a graph without the
 * integration: every slot's labels stay in its agent plane (nm_map_export_labels reads them)
 * until nm_map_integrate applies them.  Replaces the per-agent loop of
 * SimManager::updateAgentViews(map) (SimManager.h:114-127). */
int nm_tick_plan_create(nm_map m, nm_simmap sim, const nm_frame* slots, int32_t n_slots,
                        nm_tick_plan* out);
int nm_tick_plan_destroy(nm_tick_plan p);
int nm_tick_plan_set_pose(nm_tick_plan p, int32_t slot, const nm_pose* pose);
/* Range noise of rendered slots: sigma = sigma_coef * r^2, drop probability; seeded per tick. */
int nm_tick_plan_set_noise(nm_tick_plan p, float sigma_coef, float drop_prob, uint64_t seed);
int nm_tick_plan_set_launch(nm_tick_plan p, int32_t tile_w, int32_t tile_h, int32_t entries);
int nm_tick_plan_run(nm_tick_plan p, uint32_t flags, void* stream);
/* Autotuner: times candidate traversal shapes on a scratch map with the plan's slots and
 * poses: the tile (rays per warp: one ray per thread for tiles of up to 256 pixels, two or four
 * for 512 and 1024), the shared leaf-table entries; applies the fastest to the plan, and
 * appends it to cache_path (reused on later calls with the same device and slot shapes).
 * best = tile_w, tile_h, entries. */
int nm_tick_plan_autotune(nm_tick_plan p, const char* cache_path, int32_t best[3], float* best_us);

/* Leaves of the map (any order): origins (3 ints per leaf, voxel units), 512 log-odds per
 * leaf (x-major, z fastest: index x*64 + y*8 + z), 16 active-mask words per leaf.  Any output
 * pointer may be NULL.  *n receives the leaf count; at most max_leaves are written. */
int nm_map_export(nm_map m, int32_t* origins, float* values, uint32_t* active,
                  uint64_t max_leaves, uint64_t* n);

/* Labels left by the last NM_DEFER_INTEGRATE insert or tick for one agent plane: leaf
 * origins and 32 words per leaf (words 0..15 hit bits, 16..31 miss bits, bit l%32 of word
 * l/32 for voxel index l).  Only leaves with a label are written. */
int nm_map_export_labels(nm_map m, int32_t agent, int32_t* origins, uint32_t* words,
                         uint64_t max_leaves, uint64_t* n);

/* The per-frame constants the host path derives from a pose: rotation (row-major,
 * world-from-sensor), index-space eye, max_time = max_range / res. */
int nm_map_frame_params(nm_map m, nm_sensor s, const nm_pose* pose, float rotation[9],
                        double eye[3], float* max_time);

/* Host-only form of the above for a sensor description (no context, no device): also returns
 * the frustum pixel model (hw, hh, 2hw, 2hh, 1/W, 1/H).  Replaces the host derivations of
 * SensorData::updatePose / gpu::Sensor::updateShared (SensorData.h:40-83, Sensor.h:172-211). */
int nm_frame_params(const nm_sensor_desc* desc, const nm_pose* pose, float res, int32_t rounding,
                    float rotation[9], double eye[3], float* max_time, float pixel_model[6]);

/* Labels of one range image without any device allocation (no counterpart in the reference;
 * an addition for callers that cannot allocate device memory while they run, such as
 * real-time loops that forbid allocation after start-up, or hosts whose memory pool owns the
 * device).  Same traversal and labels as nm_map_insert_ranges + NM_DEFER_INTEGRATE on a map
 * of resolution `res` (positive, finite) and rounding `rounding`, but the working memory is
 * a fixed static device array of about 9 MiB.  Inputs and outputs are device memory owned by
 * the caller: `ranges` (hres*vres floats), `origins` (3 ints per leaf), `words` (32 label
 * words per leaf, as nm_map_export_labels), `status` (2 uints: labelled leaf count, error
 * bits).  Limits: at most 8388608 pixels per frame (larger frames are rejected with
 * NM_ERR_ARG) and at most 32768 labelled leaves per call (more is reported as
 * NM_ERR_CAPACITY under NM_SYNC, else as bit 16 of status[1]); a frame with more labelled
 * leaves than `max_leaves` writes the first `max_leaves` and reports NM_ERR_CAPACITY (bit 8),
 * with the full count in status[0].  The array is loaded with the library's module on each
 * GPU when that module is first used there (lazy loading, CUDA's default), so the first call
 * on each device is the start-up warm-up: it makes the array resident and looks up its device
 * address.  Make it before the phase that must not allocate and before any stream capture;
 * the array then stays resident until the process exits.  Every call shares the array and
 * first clears it; calls that overlap on the GPU race on it. */
int nm_label_frame_static(nm_sensor s, const nm_pose* pose, const float* ranges, float res,
                          int32_t rounding, int32_t* origins, uint32_t* words,
                          uint32_t max_leaves, uint32_t* status, uint32_t flags, void* stream);

/* ---- soft expected-depth rendering, its adjoint, scan-to-map pose refinement ------------
 * No reference counterpart: an addition beside the unchanged mapping path, reading the
 * device map in place.  Per pixel ray (the sensor's pixel model, double precision): voxel DDA
 * from the voxel holding the sensor over [0, max_range / res].  Occupancy
 * o = sigmoid(scale * log-odds + bias) (log-odds 0 where the map has no leaf) is the
 * probability that the ray ends within one voxel length of a voxel: a segment of length D_k in
 * voxel k ends it with probability 1 - (1 - o_k)^D_k (density softplus(scale * L + bias)); the
 * voxel holding the sensor is empty.  The expected depth, with the remaining probability at
 * max range, is res times the integral of the transmittance, accumulated in FP32 (metres).  It
 * is continuous in the pose. */

/* Sensor pose with double precision: position (m) and world-from-sensor rotation (row-major,
 * the sensor's frame transform included). */
typedef struct {
  double position[3];
  double rotation[9];
} nm_ray_pose;

/* rotation = rot(q / |q|) * frame_transform, evaluated in double and not rounded to float. */
int nm_ray_pose_from_pose(nm_sensor s, const nm_pose* pose, nm_ray_pose* out);

/* The map's log-odds in slot layout (capacity * 512 floats, device to device); *n_floats
 * receives the size.  `values` arguments below take this layout (NULL = the map's own). */
int nm_map_values_copy(nm_map m, float* dst, uint64_t max_floats, uint64_t* n_floats,
                       void* stream);
/* Leaf origin (voxel units, 3 ints) of every slot, INT32_MIN for empty slots (host output). */
int nm_map_slot_origins(nm_map m, int32_t* origins, uint64_t max_slots, uint64_t* n_slots);

/* Expected depth of every pixel (hres*vres floats, device).  `values` holds n_floats floats
 * (at least the map's capacity * 512; NULL = the map's own log-odds). */
int nm_depth_render(nm_map m, nm_sensor s, const nm_ray_pose* pose, const float* values,
                    uint64_t n_floats, float scale, float bias, float* depth, void* stream);

/* Adjoint: for upstream gradients grad_depth (hres*vres floats, device), adds
 * sum_pixels grad_depth * dD/dlog-odds into grad_values (slot layout, device, n_floats
 * floats like `values`; may be NULL)
 * and writes sum_pixels grad_depth * dD/dxi to grad_pose (host; may be NULL) for the
 * world-frame pose increment xi = (rho, phi): position + rho, rotation exp([phi]x) R.
 * The traversal is replayed, not stored (memory independent of ray length): twice per pixel,
 * or once when `depth` (device, hres*vres floats; may be NULL) holds nm_depth_render's output
 * for the same pose, values, scale and bias, which then stands in for the first replay. */
int nm_depth_backward(nm_map m, nm_sensor s, const nm_ray_pose* pose, const float* values,
                      uint64_t n_floats, float scale, float bias, const float* grad_depth,
                      const float* depth, float* grad_values, double grad_pose[6],
                      void* stream);

/* Scan-to-map pose refinement: `steps` Adam steps (learning rates lr_position in metres,
 * lr_rotation in radians, decayed to zero over the steps by a cosine schedule) on the mean
 * L1 distance between the expected depth and `target`, each residual truncated at
 * max_residual metres when that is positive (0 = plain L1)
 * (hres*vres floats, device; <= 0 or NaN = no return), each step re-linearised at the
 * current pose.  `pose` is updated in place; losses (host, steps + 1 floats, may be NULL)
 * receives the loss before each step and after the last. */
int nm_pose_refine(nm_map m, nm_sensor s, nm_ray_pose* pose, const float* target, float scale,
                   float bias, float max_residual, int32_t steps, float lr_position,
                   float lr_rotation, float* losses);

/* Options of scan-to-map refinement.  surface_offset (0..1) places the predicted surface that
 * fraction of a voxel past the face the ray enters the voxel it ends in (0 = at the face, as
 * nm_pose_refine; 0.5 = at the middle of the voxel, the unbiased choice against a target
 * rendered from a different voxel grid, whose surfaces lie 0 or 1 voxel past that face).
 * edge_threshold (m, 0 = off) leaves out target pixels on silhouettes: a 4-neighbour without
 * a return or with a range that differs by more than the threshold. */
typedef struct nm_refine_desc {
  float scale, bias;       /* occupancy = sigmoid(scale * log-odds + bias) */
  float max_residual;      /* truncation of the L1 residual (m; 0 = plain L1) */
  int32_t steps;
  float lr_position;       /* m */
  float lr_rotation;       /* rad */
  float surface_offset;
  float edge_threshold;
} nm_refine_desc;

/* nm_pose_refine with the options above. */
int nm_pose_refine_desc(nm_map m, nm_sensor s, nm_ray_pose* pose, const float* target,
                        const nm_refine_desc* desc, float* losses);

/* ---- simulation map (replaces the NanoVDB sim grid, SimHandler.cpp:13-24) -------------- */
/* Voxelise primitives into a sparse device map: boxes are 6 doubles (min xyz, max xyz, m);
 * cylinders are 5 doubles (cx, cy, radius, z0, z1, m).  A voxel is active when its centre is
 * inside a primitive.  Only voxels in [vox_min, vox_max) are considered. */
int nm_simmap_create_primitives(nm_context ctx, float res, const int32_t vox_min[3],
                                const int32_t vox_max[3], const double* boxes, int32_t n_boxes,
                                const double* cylinders, int32_t n_cylinders, nm_simmap* out);
/* From a list of active voxel coordinates (3 ints each, host memory). */
int nm_simmap_create_voxels(nm_context ctx, float res, const int32_t* ijk, int64_t n,
                            nm_simmap* out);
/* From a file.  Replaces SimManager::loadSimGrid / loadGridFromFile (SimManager.h:171-213).
 * A path ending in ".vdb" is an OpenVDB file: the active voxels of its grid named "grid" (the
 * file's first grid when none is), read by nm_vdb_active_voxels; the voxel size must be
 * uniform and the translation a whole number of voxels.  Any other path is a voxel list:
 * 8-byte magic "NMSIMv1", float res (m), int64 count, then count triplets of int32 voxel
 * coordinates (little endian). */
int nm_simmap_load(nm_context ctx, const char* path, nm_simmap* out);
/* Active voxels of a grid in an OpenVDB .vdb file (no GPU used): file format versions
 * 222-224 (OpenVDB 3 onwards), trees 5-4-3 of float (also saved as half) or double values,
 * values stored raw, zip or blosc (only the tree topology is read: leaf value masks and
 * active tiles, the latter expanded to their voxels; no decompression), transforms that are a
 * scale and a translation.  `grid` names the grid (NULL: "grid", else the file's first grid).
 * voxel_size and translation (3 doubles each, may be NULL) map index to world:
 * world = index * voxel_size + translation, voxel (i, j, k) covering index [i, i + 1) etc.
 * With ijk NULL only *n is set; else up to max_voxels triplets are written (more active
 * voxels than that: NM_ERR_CAPACITY, *n the count).  Grids of more than 2^28 active voxels
 * are refused (NM_ERR_CAPACITY). */
int nm_vdb_active_voxels(const char* path, const char* grid, double voxel_size[3],
                         double translation[3], int32_t* ijk, int64_t max_voxels, int64_t* n);
/* Writes n active voxels (3 int32 each) as a float grid named `grid` (NULL: "grid") of an
 * OpenVDB-layout file (format version 224, tree 5-4-3, uniform scale voxel_size, values 0
 * stored raw with active-mask compression, grid class "unknown"), the layout
 * nm_vdb_active_voxels reads. */
int nm_vdb_write_active_voxels(const char* path, const char* grid, double voxel_size,
                               const int32_t* ijk, int64_t n);
int nm_simmap_destroy(nm_simmap sm);
/* active bounding box (min xyz, max xyz, inclusive), active voxel count, leaf count */
int nm_simmap_info(nm_simmap sm, int32_t bbox[6], uint64_t* active_voxels, uint64_t* leaves);
/* leaf origins and 16 mask words per leaf (any order) */
int nm_simmap_export(nm_simmap sm, int32_t* origins, uint32_t* words, uint64_t max_leaves,
                     uint64_t* n);
/* Simulated range image of one sensor at one pose (replaces generateCloud,
 * generateCloud.cu:84-94).  Output: hres*vres floats, radial metres, 0 = no return. */
int nm_sim_render(nm_simmap sm, nm_sensor s, const nm_pose* pose, float* ranges,
                  uint32_t flags, void* stream);

/* nm_sim_render and nm_ranges_add_noise in one launch (same ranges bit for bit): the range
 * noise of the simulated sensors, sigma = sigma_coef * r^2 and drop probability drop_prob,
 * counter-based per pixel from `seed`. */
int nm_sim_render_noisy(nm_simmap sm, nm_sensor s, const nm_pose* pose, float* ranges,
                        float sigma_coef, float drop_prob, uint64_t seed, uint32_t flags,
                        void* stream);

/* SimHandler::processPointCloud for one sensor (SimHandler.cpp:234-280: generateCloud, then
 * the insertion): the simulated range image of `s` at `pose` over the sim map, with the
 * simulated sensors' range noise as nm_sim_render_noisy applies it (sigma_coef = drop_prob = 0
 * for none), inserted into `m`.  In label mode one launch does both: each tile of pixels is
 * rendered into on-chip memory and walked from there.  The ranges and the map are those of
 * nm_sim_render_noisy followed by nm_map_insert_ranges.  `ranges` (device, hres*vres floats,
 * or host with NM_OUTPUT_HOST; may be NULL) receives the image.  Flags: NM_DEFER_INTEGRATE,
 * NM_SYNC, NM_OUTPUT_HOST and the voxel-filter flags (which render first, then insert). */
int nm_sim_insert(nm_simmap sm, nm_map m, nm_sensor s, const nm_pose* pose, float sigma_coef,
                  float drop_prob, uint64_t seed, float* ranges, uint32_t flags, void* stream);

/* Ray casts against the sim map for agent observation and collision rays
 * (SimManager::getAgentSimCollision, SimManager.h:141-168): n rays from `origins` (metres,
 * 3 floats each) along `directions` (3 floats each, any length, normalised here); distances
 * (metres) to the first active voxel entered within max_range, 0 when none (the voxel holding
 * the origin is not tested).  NM_INPUT_HOST / NM_OUTPUT_HOST mark host arrays.  The reference
 * intersects leaf-node spans (openvdb::tools::VolumeRayIntersector); this cast is exact to
 * the voxel. */
int nm_sim_cast_rays(nm_simmap sm, const float* origins, const float* directions, int64_t n,
                     float max_range, float* distances, uint32_t flags, void* stream);

/* The n unit observation directions of an agent (host output, 3 floats each): the spiral
 * sphere of Agent::generateObservationSphere (Agent.h:147-192), n >= 2. */
int nm_observation_sphere(int32_t n, float* directions);

/* Sensor noise on a device range image: r += N(0, (sigma_coef * r^2)^2), then each pixel
 * is set to 0 with probability drop_prob.  Counter-based generator keyed by `seed`. */
int nm_ranges_add_noise(nm_context ctx, float* ranges, int64_t n, float sigma_coef,
                        float drop_prob, uint64_t seed, void* stream);

/* ---- procedural cave generator (replaces nanomap::mapgen::CaveGen, CaveGen.h:32-68) ----
 * The cave lives on a lattice of cells 8 voxels apart (CaveGen's LEAF_SIZE): with
 * D = ceil(ceil(map_size / grid_res) / 2) voxels per half axis, cell (i, j, k) sits at voxel
 * (-Dx + 8 + 8i, -Dy + 8 + 8j, -Dz + 8k) for k < nz, plus one ceiling plane k = nz at
 * z = +Dz (setFloorAndCeil).  Each cell stands for the 8^3-voxel leaf that holds it. */
typedef struct nm_cave_s* nm_cave;

/* #cavegenconfig file (CaveGen::loadConfig, CaveGen.cpp:358-401). */
typedef struct {
  double map_size[3];      /* map_size (m) */
  double grid_res;         /* grid_res (m) */
  int32_t fill_percentage; /* fill_percentage: a cell starts on when rand() % 100 is below it */
  int32_t smoothing_count; /* smoothing_count */
  int32_t active_max;      /* active <max> <min>: on when more than max of the neighbours are */
  int32_t active_min;      /* on, off when fewer than min are, unchanged otherwise */
  int32_t time_seed;       /* random_seed 1: seeded from the clock */
  uint32_t seed;           /* the value given to srand: std::hash of the seed string, or of
                              the time, truncated to 32 bits as CaveGen's int _seed does */
  char file_out[256];      /* file_out */
} nm_cave_desc;

#define NM_CAVE_2D 0x1u          /* columns: populateMap2D / smoothMapXY */
#define NM_CAVE_COUNTER_RNG 0x2u /* fill from a counter-based generator on the device instead
                                    of the C library's srand/rand sequence on the host */

int nm_cave_config_load(const char* path, nm_cave_desc* out);
int nm_cave_create(nm_context ctx, const nm_cave_desc* desc, nm_cave* out);
int nm_cave_destroy(nm_cave c);
/* half sizes D (voxels) and lattice size (cells along x, y; z planes below the ceiling) */
int nm_cave_dims(nm_cave c, int32_t half[3], int32_t cells[3]);
/* CaveGen::populateMap (CaveGen.cpp:13-47), or populateMap2D (:49-84) with NM_CAVE_2D: the
 * cells are cleared and filled again. */
int nm_cave_populate(nm_cave c, uint32_t flags);
/* smoothing_count steps of CaveGen::smoothMap (:95-129: 26 neighbours), or smoothMapXY
 * (:130-176: 8 neighbours in the floor plane, written to whole columns) with NM_CAVE_2D. */
int nm_cave_smooth(nm_cave c, uint32_t flags);
/* CaveGen::setFloorAndCeil (:86-94). */
int nm_cave_floor_ceil(nm_cave c);
/* CaveGen::getRegions (:178-240): 6-connected regions of on cells; their number and the
 * size of the largest (either pointer may be NULL). */
int nm_cave_regions(nm_cave c, int64_t* n_regions, int64_t* largest);
/* CaveGen::keepLargestRegion (:242-252): only the largest region stays on; ties go to the
 * region met first in OpenVDB's value order, as in the reference. */
int nm_cave_keep_largest(nm_cave c);
/* on cells as voxel coordinates (3 ints each, host), in OpenVDB value order */
int nm_cave_cells(nm_cave c, int32_t* xyz, int64_t max_cells, int64_t* n);
/* The cave as a sim map.  shell = 0: every voxel of the on cells' leaves (CaveGen::Save,
 * :326-335); shell = 1: the narrow band of tools::topologyToLevelSet as invertAndSave calls
 * it (:294-324): with the leaves' voxels T and face-neighbour morphology,
 * M = erode^closing(dilate^closing(T)) and the active band is
 * dilate^half_width(M) minus erode^half_width(M) (half_width 3, closing 1 in the reference). */
int nm_cave_simmap(nm_cave c, int32_t shell, int32_t half_width, int32_t closing,
                   nm_simmap* out);
/* nm_cave_simmap written to `path`, the reference's file_out (CaveGen.cpp:299-325): a path
 * ending in ".vdb" gets the band's active voxels as the float grid "grid" of a .vdb file
 * (nm_vdb_write_active_voxels; the reference writes the same active set as a level set), any
 * other path an NMSIMv1 voxel list; both are what nm_simmap_load reads.  The name written is
 * copied to written_path (may be NULL, 512 bytes). */
int nm_cave_save(nm_cave c, int32_t shell, int32_t half_width, int32_t closing,
                 const char* path, char* written_path);

#ifdef __cplusplus
}
#endif

#endif /* NANOMAP_B200_H_ */
