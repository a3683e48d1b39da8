// Internal context of the MID-Fusion B200 library (not part of the C ABI).
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/midfusion_b200.h"
#include "mf_common.cuh"

namespace mf {

constexpr int MAX_INSTANCES = 32;
constexpr int MAX_PYR = 4;

// Instance ids of one stage, passed to kernels by value.
struct IdList {
  int n;
  int v[32];
};

// Per-instance quantities derived on the device from the device-resident poses
// before each stage (so a stage never waits on the host for a pose).
struct InstFrame {
  M4 T_w_o, inv_T_w_o;
  // allocation (apps/kfusion/src/cpp/kfusion/alloc_impl.hpp:121-191)
  M4 kPose;            // T_w_c * inverse(K)
  F3 o_cam;            // camera centre in the volume frame
  float inv_voxel;     // 1 / voxelSize
  float band;          // 2 mu
  int num_steps;
  unsigned long long reserved;
  // integration (lib/functors/projective_functor.hpp:43-166)
  M4 Tcw;              // inverse(T_w_c) * T_w_o
  M4 KTcw;             // K * Tcw
  F3 delta, cam_delta;
  // raycast (apps/kfusion/src/cpp/rendering/rendering.cpp:37-45)
  F3 o_origin;
  int label;
  M4 view;             // T_w_c * inverse(K)
  int pad[3];
};

struct Instance {
  int size;
  float dim;
  int label;
  Volume vol;          // device pointers, host copy
  size_t reserved;     // reference allocation-list capacity
  // semantic class (Object::class_id_, semanticfusion_, fused_time_)
  int class_id = 0;
  int fused_time = 0;
  std::vector<float> sem;
  bool pose_saved = false;   // Object::pose_saved_: later poses append
};

// One GN problem (camera or object) tracked on the device.
struct TrackState;

// Launch shapes chosen by the autotuner (mf_tune.cu): an index into each
// tuned kernel's candidate table, 0 = the default shape.  `gen` changes with
// every choice so that captured frame graphs are rebuilt.
constexpr int MAX_TUNE_VARIANTS = MF_TUNE_MAX_VARIANTS;
struct Tune {
  int ray = 0;        // raycast_objects_kernel (ray_variants, mf_raycast.cu)
  int integrate = 0;  // integrate_blocks_kernel (int_variants, mf_volume.cu)
  unsigned gen = 0;
};

struct Context {
  mf_config cfg;
  int W = 0, H = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  std::string last_error;

  Pool pool{};                      // host copy of device pointers
  std::vector<Instance> inst;
  Volume* d_vols = nullptr;         // device copy of every instance's Volume
  float* d_Two = nullptr;           // MAX_INSTANCES x 16 volume poses
  float* d_Twc = nullptr;           // 16, camera pose
  InstFrame* d_frames = nullptr;    // MAX_INSTANCES
  int* d_status = nullptr;          // OR of Status flags
  unsigned long long* d_reserved = nullptr;  // MAX_INSTANCES reference list capacities
  int* d_inst_label = nullptr;      // MAX_INSTANCES instance labels
  int* d_scratch_i = nullptr;       // small device scratch (export slot lists)
  void* d_export = nullptr;         // export staging (grown on demand)
  size_t export_bytes = 0;
  int* d_visit = nullptr;           // integration visit list
  int* d_visit_count = nullptr;
  int* d_visit_side = nullptr;      // the side stream's visit list (overlapped frames)
  int* d_visit_count_side = nullptr;
  bool visit_side_used = false;     // the last batched frame used it

  // frame inputs
  float* d_depth = nullptr;         // W*H metres
  uint8_t* d_rgb8 = nullptr;        // W*H*3
  F3* d_rgb = nullptr;              // W*H in [0, 1]
  float* d_grey = nullptr;          // W*H
  float* d_masks = nullptr;         // MAX_INSTANCES x W*H generalized masks
  uint16_t* d_labels = nullptr;     // W*H ground-truth instance labels

  // raycast outputs (composite model maps)
  F3* d_vertex = nullptr;
  F3* d_normal = nullptr;
  int* d_label = nullptr;
  // phased raycast: per instance and pixel, the unbounded hit (x, y, z, t) and
  // (crossing sample t, foreground at the hit); max_instances x W*H each
  F4* d_rayhit = nullptr;
  float2* d_raytf = nullptr;
  int8_t* d_mc_tris = nullptr;      // marching-cubes triangulation table (mf_mesh)

  // staging
  float* h_pinned = nullptr;        // small pinned host staging area
  size_t h_pinned_bytes = 0;

  float ray_epsilon = 0.f;          // ray iterator direction epsilon (first volume)
  void* graphs = nullptr;           // captured frame graphs (mf_pipeline.cu)
  bool use_graphs = true;
  bool gn_persistent = false;       // batched GN: one cooperative launch per level
  // batched frames: the background's allocation and integration run on a
  // low-priority side stream while the objects are tracked (overlap_ctas:
  // CTAs of that integration launch, < 0 the launch shape's own grid;
  // 0 = in order on the main stream)
  int overlap_ctas = -1;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_start = nullptr, ev_pre = nullptr, ev_obj = nullptr, ev_gen = nullptr,
              ev_fork = nullptr, ev_join = nullptr;
  TrackState* track = nullptr;
  Tune tune;                        // autotuned launch shapes
  // mf_process_frame_motion: frames it has processed, and two planes of
  // result rows (2 x W*H int8 each) for the mask refinement
  int motion_frames = 0;
  int8_t* d_motion_rows = nullptr;
  // mf_frame_stage / mf_process_staged: two device slots of frame inputs,
  // uploaded on their own stream (all created with the first staged frame);
  // ev_staged[s]: slot s's upload is done; ev_consumed[s]: the frame processed
  // from slot s has copied it out (the next upload into s may start)
  cudaStream_t upload = nullptr;
  float* stg_depth[2] = {};
  uint8_t* stg_rgb8[2] = {};
  uint16_t* stg_labels[2] = {};
  bool stg_labels_set[2] = {};
  bool stg_pending[2] = {};
  cudaEvent_t ev_staged[2] = {}, ev_consumed[2] = {};
  uint8_t* d_render = nullptr;      // W*H*4 render scratch for host destinations
  void* d_render_small = nullptr;   // colour / pointer tables of a render
  size_t render_small_bytes = 0;
};

#define MF_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t e__ = (call);                                                  \
    if (e__ != cudaSuccess) {                                                  \
      ctx->last_error = std::string(#call) + ": " + cudaGetErrorString(e__);   \
      return MF_E_CUDA;                                                        \
    }                                                                          \
  } while (0)

// kernels / stages implemented in the .cu files
int stage_prepare(Context* ctx, const IdList& ids);
int stage_alloc(Context* ctx, const IdList& ids);
int stage_integrate(Context* ctx, const IdList& ids, int ctas = 0);
int stage_raycast(Context* ctx, const IdList& ids, float epsilon);
bool raycast_is_phased(const Context* ctx);
int stage_raycast_hits(Context* ctx, const IdList& ids, int base, float epsilon);
int stage_raycast_fold(Context* ctx, const IdList& ids, float epsilon);
// The same raycast into other map buffers.
int stage_raycast_to(Context* ctx, const IdList& ids, float epsilon, F3* vertex, F3* normal,
                     int* label);
int alloc_keys(Context* ctx, int id, const uint64_t* keys, int n);
int export_blocks(Context* ctx, int id, uint64_t* keys, int32_t* coords, uint8_t* active,
                  void* voxels, int cap, int* n);
int export_nodes(Context* ctx, int id, uint64_t* keys, uint32_t* side, uint8_t* cmask,
                 void* values, int cap, int* n);
int interp_points(Context* ctx, int id, const float* pos, int n, int field, float* out);
int root_children(Context* ctx, int id, uint8_t* mask);
int track_init(Context* ctx);
void track_free(Context* ctx);
// clear_mask false: the ICP outlier mask planes are left to track_camera_mask,
// which writes them whole
int track_preprocess(Context* ctx, bool clear_mask = true);
int track_set_ref(Context* ctx);
int track_camera(Context* ctx, uint32_t moving, int retrack = 0);
int track_objects(Context* ctx, const IdList& ids);
// the same in phases, for a frame that runs the pose-independent parts on
// another stream: track_camera = pre + mask + gn; track_objects = pre + gn
int track_camera_pre(Context* ctx, int retrack = 0);
int track_camera_mask(Context* ctx, uint32_t moving);
int track_camera_gn(Context* ctx);
int track_objects_pre(Context* ctx, const IdList& ids);
int track_objects_gn(Context* ctx, const IdList& ids);
int track_info(Context* ctx, int slot, int* iters, double* sums, double* T64);
int track_eval(Context* ctx, int slot, int L, const float* pose16, double* sums);
int track_eval_static(Context* ctx, int slot, int L, const float* pose16, double* sums);
int gn_step_check(Context* ctx, int n, const double* state, const double* sums, double* out_dev,
                  double* out_host);
int camera_cost(Context* ctx, const float* T_live16, int want_grad, double* out8, float* d_grad);
int motion_residuals(Context* ctx, float threshold, float moved, float* ratio,
                     uint32_t* moving);
int motion_download(Context* ctx, int8_t* res, float* err, float* lvert, int32_t* llabel);
int track_results(Context* ctx, int slot, int8_t* d_out, float* d_err, float* pose_eval);
int object_residuals(Context* ctx, int i, float threshold, int8_t* d_rows, float* T_virtual);
int mesh_set_table(Context* ctx, const int* table);
int raycast_records(Context* ctx, const IdList& ids, mf_ray_record* d_records,
                    mf_ray_origin* d_origins);
int raycast_fold(Context* ctx, const mf_ray_record* d_records, const mf_ray_origin* d_origins);
int motion_planes(Context* ctx, const int8_t** res, const float** err);
// headless renders (mf_render.cu; the shaded volume render in mf_raycast.cu)
// formats (mf_io.cu)
int frame_upload_raw(Context* ctx, const uint16_t* depth_mm, const uint8_t* rgb, int in_w,
                     int in_h);
void pose_quaternion(const float* T, float* q);
int tum_line(int frame, const float* T_translation, const float* T_rotation, char* buf, int cap);
// mesh export (mf_mesh.cu)
int mesh_volume(Context* ctx, int id, int float_bounds, float* tris, long long cap,
                long long* n_tris);
int write_vtk_mesh(const char* path, const float* tris, long long n);
// object management (mf_objects.cu)
int ensure_export(Context* ctx, size_t bytes);
int spawn_object(Context* ctx, const uint8_t* mask, float* T_w_o, float* volume_size,
                 int* volume_resol);
int set_semantics(Context* ctx, int id, int class_id, const float* probs, int n);
int fuse_semantics(Context* ctx, int id, int class_id, const float* probs, int n,
                   int recog_times);
int render_target(Context* ctx, void* out, size_t bytes, void** target);
int render_finish(Context* ctx, void* out, void* target, size_t bytes);
int render_stage_small(Context* ctx, const void* src, size_t bytes, void** dst);
int render_volume(Context* ctx, const float* T_w_c, int render_color, float largestep,
                  const float* ambient, const uint8_t* colors, int n_colors, uint8_t* out);
int render_image(Context* ctx, int which, uint8_t* out);
int render_track(Context* ctx, int mode, const int8_t* d_res, const float* d_err, uint8_t* out);
int render_mask(Context* ctx, int mode, const int32_t* d_labels, const uint8_t* colors,
                int n_colors, const int8_t* const* d_rows, int n_rows, uint8_t* out);
int refine_mask_use_motion(Context* ctx, int id, const int8_t* d_res, int use_icp, int use_rgb);
int stage_raycast_adjoint(Context* ctx, const IdList& ids, const double* gV, const double* gN,
                          float* d_grad);
int track_download_level(Context* ctx, int L, int which, float* out);
void track_save_prev_camera(Context* ctx);
bool track_has_ref(Context* ctx);
int track_parity(Context* ctx);
void track_set_parity(Context* ctx, int parity);
int launch_generalize(Context* ctx);
int process_frame(Context* ctx, bool labels);
int process_frame_motion(Context* ctx, float residual_threshold, float moved_threshold,
                         uint32_t* moving_labels);
int profile_integrate(Context* ctx, int reps, double* us, double* bytes);
int profile_gn(Context* ctx, int reps, double* us, double* bytes);
int profile_raycast(Context* ctx, int reps, double* us, double* bytes);
void pipeline_free(Context* ctx);
// launch-shape candidates (autotuner)
int ray_variant_count();
void ray_variant_describe(int v, char* buf, int cap);
int int_variant_count();
void int_variant_describe(int v, char* buf, int cap);
// integrate_blocks_kernel alone, on `pool` (the live pool or a scratch copy),
// over the visit list of the last stage_integrate / visit_list
int launch_integrate_blocks(Context* ctx, const Pool& pool, int variant, int ctas = 0);
int build_visit_list(Context* ctx, uint32_t inst_mask);
// the autotuner (mf_tune.cu)
int tune_variant_count(int stage);
int autotune(Context* ctx, int reps, float* ray_us, float* int_us);
int tune_set(Context* ctx, int stage, int variant);
size_t graph_kernel_nodes(Context* ctx);
int volume_create(Context* ctx, Instance& in);
void volume_free(Instance& in);

}  // namespace mf
