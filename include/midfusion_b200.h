/* MID-Fusion per-frame dense hot path on NVIDIA B200 (sm_100a): C ABI.
 *
 * Plain C types only: a caller written in C, C++ (the reference's Kfusion
 * pipeline), Python (ctypes) or any FFI binds these directly.  Each entry point
 * names the reference interface it replaces (paths relative to the reference
 * project root).
 *
 * Conventions
 *  - Every function returns MF_OK (0) or a negative MF_E_* code;
 *    mf_last_error() gives a one-line description of the last failure.
 *  - Matrices are 4x4 float, row-major (the reference's Matrix4:
 *    utils/math_utils.h:47-49).  Intrinsics k = {fx, fy, cx, cy}.
 *  - Host pointers are borrowed for the duration of the call; device state is
 *    owned by the context.  All work is queued on the context's stream; calls
 *    that return host data synchronise that stream.
 *  - One context per host thread (the reference is not re-entrant either).
 */
#ifndef MIDFUSION_B200_H
#define MIDFUSION_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MF_OK 0
#define MF_E_ARG (-1)          /* invalid argument or size */
#define MF_E_CUDA (-2)         /* CUDA runtime error (see mf_last_error) */
#define MF_E_POOL_FULL (-3)    /* voxel-block pool exhausted */
#define MF_E_NOT_FOUND (-4)    /* unknown instance id */
#define MF_E_STATE (-5)        /* call made in the wrong order */
#define MF_E_TIMEOUT (-6)      /* a bounded device wait gave up */

/* Device status flags accumulated since the last mf_status() call. */
#define MF_STATUS_POOL_FULL 1
#define MF_STATUS_ALLOC_OVERFLOW 2  /* more keys than the reference's list holds */
#define MF_STATUS_RAY_GUARD 4
#define MF_STATUS_GN_FALLBACK 8     /* a 6x6 system used the truncated eigen solve */
#define MF_STATUS_ADJOINT 16        /* mf_camera_cost skipped the TSDF adjoint of a ray */
#define MF_STATUS_GN_TIMEOUT 32     /* a grid barrier of the persistent GN launch gave up */

/* Robust kernels of Tracking::calc_robust_weight,
 * apps/kfusion/src/cpp/tracking/tracking.cpp:1504-1532 (enum RobustW,
 * tracking/tracking.h:19-24). */
#define MF_ROBUST_NONE 0
#define MF_ROBUST_HUBER 1
#define MF_ROBUST_TUKEY 2
#define MF_ROBUST_CAUCHY 3

typedef struct mf_config {
  int width, height;          /* computationSize */
  float k[4];                 /* fx, fy, cx, cy */
  float mu;                   /* TSDF truncation, default_parameters.h:26 (0.1) */
  float near_plane, far_plane;/* constant_parameters.h:20-21 (0.1, 4.0) */
  int max_weight;             /* sdf_update maxweight, object.cpp:165 (100) */
  int pyramid_levels;         /* default_parameters.h:22-23 (3) */
  int gn_iterations[4];       /* {10, 5, 4} */
  int robust_kernel;          /* MF_ROBUST_* (reference default Cauchy) */
  int use_icp, use_rgb;       /* Tracking(using_ICP, using_RGB) */
  long long pool_blocks;      /* capacity of the shared voxel-block pool */
  int max_instances;          /* <= 32 */
  int batched;                /* 1: one launch per stage for all instances */
} mf_config;

typedef struct mf_context mf_context;

/* Fill `cfg` with the reference defaults for a width x height frame. */
int mf_config_default(mf_config* cfg, int width, int height);
int mf_create(const mf_config* cfg, mf_context** out);
int mf_destroy(mf_context* ctx);
const char* mf_last_error(const mf_context* ctx);
/* Pending device status flags (MF_STATUS_*), cleared by the call. */
int mf_status(mf_context* ctx, int* flags);
/* The cudaStream_t all work is queued on. */
int mf_get_stream(mf_context* ctx, void** stream);
int mf_synchronize(mf_context* ctx);

/* --- instances ---------------------------------------------------------
 * One octree volume per instance: the background (label 0) and every object.
 * Replaces Object::Object + Volume::init (object/object.cpp:13-40,
 * continuous/volume_template.hpp:63-67).  size: voxels per side (power of
 * two, 32..4096); dim: metres per side; T_w_o: volume corner pose. */
int mf_instance_add(mf_context* ctx, int size, float dim, const float T_w_o[16],
                    int label, int* id);
int mf_instance_count(mf_context* ctx, int* n);
int mf_instance_set_pose(mf_context* ctx, int id, const float T_w_o[16]);
int mf_instance_get_pose(mf_context* ctx, int id, float T_w_o[16]);
int mf_set_camera_pose(mf_context* ctx, const float T_w_c[16]);
int mf_get_camera_pose(mf_context* ctx, float T_w_c[16]);

/* --- frame input ------------------------------------------------------
 * depth: metres (floatDepth after mm2metersKernel, preprocessing.cpp:132-159);
 * rgb: uint8 x 3 per pixel; masks: one generalized float mask per instance in
 * instance order (instance_seg::generalize_label, segmentation.cpp:10-48), or
 * NULL to keep the previous masks.  Host pointers (copied to the device). */
int mf_frame_upload(mf_context* ctx, const float* depth, const uint8_t* rgb,
                    const float* masks, int n_masks);
/* Same with device pointers (no host copy). */
int mf_frame_set_device(mf_context* ctx, const float* d_depth, const uint8_t* d_rgb,
                        const float* d_masks, int n_masks);
/* Ground-truth uint16 instance labels (host) -> generalized masks on the
 * device for every instance (fg 1, 5x5-ellipse ring 0, elsewhere -1). */
int mf_frame_labels(mf_context* ctx, const uint16_t* labels);

/* --- allocation + integration -----------------------------------------
 * Object::integrate_volume_kernel (object/object.cpp:128-195) for each id:
 * buildVolumeAllocationList (kfusion/alloc_impl.hpp:121-191) +
 * Octree::alloc_update (lib/octree.hpp:761-786) + projective_functor with
 * sdf_update (lib/functors/projective_functor.hpp:139-156,
 * kfusion/mapping_impl.hpp:15-72), at the current camera pose. */
int mf_integrate(mf_context* ctx, const int* ids, int n);
/* Octree::alloc_update (lib/octree.hpp:761-786) on explicit keys. */
int mf_alloc_update(mf_context* ctx, int id, const uint64_t* keys, int n);

/* --- raycast ----------------------------------------------------------
 * raycastObjectList (rendering/rendering.cpp:9-181) over every instance at
 * the current camera pose: composite vertex/normal/label maps stay on the
 * device as the tracking model. */
int mf_raycast(mf_context* ctx);
/* --- instance-sharded raycast (no counterpart in the reference, which runs
 * on one host) ------------------------------------------------------------
 * The composite of raycastObjectList (rendering.cpp:9-181) split into a part
 * per instance, which the GPU that holds the instance's volume computes, and
 * an ordered per-pixel fold, which needs no volume: across GPUs, each rank
 * records its own instances, the records are gathered (e.g. an NCCL
 * all-gather), and every rank folds all of them into the same maps.
 * The reference bounds each instance's march by the nearest hit so far; a
 * record holds the march to the far plane and the parameter at which it
 * crossed the surface, and the fold applies the bound afterwards: the
 * bounded march finds that crossing exactly when it lies before the bound,
 * and otherwise returns the zero hit, whose values the origin record holds. */
typedef struct mf_ray_record {
  float hit[4];      /* (x, y, z, t) in the instance's frame; 0 without a crossing */
  float tc;          /* march parameter of the crossing sample; +inf: none */
  float fg;          /* foreground probability interpolated at the hit */
  float normal[3];   /* world normal normalize(R_wo grad(hit)) */
  int zero_grad;     /* 1: the gradient is zero (the reference writes only normal.x) */
  int pad[2];
} mf_ray_record;     /* 48 bytes */
typedef struct mf_ray_origin {
  float fg;          /* foreground probability at the volume origin (the zero hit) */
  float normal[3];   /* world normal at the zero hit */
  int zero_grad;
  int pad[3];
} mf_ray_origin;     /* 32 bytes */
/* Records of instances ids[0..n) at the current camera pose into device
 * memory: d_records[k * W * H + p] for instance ids[k] and pixel p, and
 * d_origins[k]. */
int mf_raycast_records(mf_context* ctx, const int* ids, int n, mf_ray_record* d_records,
                       mf_ray_origin* d_origins);
/* The composite maps from the records of EVERY instance of the context, in
 * instance order (d_records[i * W * H + p], d_origins[i], device memory), with
 * the context's instance poses and labels: the maps mf_raycast makes, bit for
 * bit.  They replace the context's model maps. */
int mf_raycast_fold(mf_context* ctx, const mf_ray_record* d_records,
                    const mf_ray_origin* d_origins);
/* Copy the composite maps to the host (any pointer may be NULL). */
int mf_download_raycast(mf_context* ctx, float* vertex, float* normal, int32_t* label);

/* --- tracking ---------------------------------------------------------
 * Tracking::set_params_frame (tracking/tracking.cpp:142-171): bilateral
 * filter of intensity and depth, robust half-sampled pyramid, vertex, normal,
 * gradient and ICP-covariance maps of the current frame. */
int mf_preprocess(mf_context* ctx);
/* Tracking::setRefImgFromCurr (tracking.cpp:1400-1413): the current frame's
 * intensity and vertex pyramids become the photometric reference. */
int mf_set_ref_from_current(mf_context* ctx);
/* Tracking::trackLiveFrame (tracking.cpp:208-357, mask variant :1750-1879)
 * against the composite model maps of the last mf_raycast: the camera pose is
 * updated in place on the device.  Pixels whose model label has its bit set in
 * `moving_labels` are excluded from ICP (the dynamic-object mask); 0 = none. */
int mf_track_camera(mf_context* ctx, uint32_t moving_labels);
/* The second trackLiveFrame of a frame with moving objects (kfusion.cpp:
 * 347-373): from the current (tracked) camera pose, against the reference pose
 * and model maps of this frame's mf_track_camera, with the pixels of the
 * `moving_labels` objects excluded from ICP.  MF_E_STATE without an
 * mf_track_camera since the last mf_set_ref_from_current. */
int mf_retrack_camera(mf_context* ctx, uint32_t moving_labels);
/* Tracking::trackEachObject (tracking.cpp:580-708) for each id (>= 1) against
 * its own model map; T_w_c1 is the camera pose before the last camera update
 * (mf_track_camera or mf_set_camera_pose), T_w_c2 the current one.  The volume
 * poses are updated on the device. */
int mf_track_objects(mf_context* ctx, const int* ids, int n);
/* Diagnostics of a GN problem (slot 0: camera, slot i: object i): iterations
 * per level (int[4]), last normal-equation sums per level (double[4][32]),
 * FP64 pose (double[16]); any pointer may be NULL. */
int mf_track_info(mf_context* ctx, int slot, int* iterations, double* sums, double* pose);
/* One evaluation of the normal equations (the 32 reduceKernel sums,
 * tracking.cpp:1191-1352) of a problem at `level` and at `pose` (NULL: its
 * current pose), without a GN step.  MF_E_STATE when the slot holds no
 * tracking problem yet (mf_track_camera sets up slot 0, mf_track_objects the
 * object slots). */
int mf_track_eval(mf_context* ctx, int slot, int level, const float* pose, double* sums);
/* No counterpart in the reference.  mf_track_eval without any device memory
 * allocation, for callers that must not allocate while they run: a real-time
 * tracking loop with a fixed memory budget, or a host that has handed the rest
 * of the device memory to other work.  Its scratch (FP64 per-CTA partials, the
 * 32 sums and a CTA ticket) is one static device array of 1 MiB + 512 B, so a
 * level may have at most 4096 x 768 pixels at level 0 and 4096 x 256 above
 * (larger levels return MF_E_ARG).  The pose is passed to the kernel by value
 * and the context's poses and sums are not modified.  Same results as
 * mf_track_eval, bit for bit.
 *  - The first call on a device looks up the scratch's device address; make
 *    it (for example once at start-up) before any stream capture.  The
 *    address is kept for the life of the process, which assumes the device's
 *    primary context is not reset (cudaDeviceReset) in between.
 *  - The slot must hold a tracking problem (set up by mf_track_camera /
 *    mf_track_objects); otherwise MF_E_STATE, as for mf_track_eval.
 *  - The context's device must be the current device.
 *  - The scratch is shared by every context on the device: calls that overlap
 *    in time (other threads, other contexts) race on it and give wrong sums.
 *    Calls from one thread are serialised, because the call synchronises. */
int mf_track_eval_static(mf_context* ctx, int slot, int level, const float* pose,
                         double* sums);
/* No counterpart in the reference: the camera-tracking cost and its adjoint.
 * Raycasts every instance at the current camera pose, which is the reference
 * pose T_w_r (the model maps are replaced), then evaluates at pyramid level 0
 *   E = sum_p rho(e_icp(p)) + rho(e_rgb(p))
 * with the camera rows of mf_track_camera (robust kernel of the config) for
 * the live frame of the last mf_preprocess at pose T_live, against the
 * reference frame of mf_set_ref_from_current.  out[0] = E; out[1..6] =
 * dE/d(twist) for T_live <- exp(twist) T_live, twist = (v, w), at twist = 0;
 * out[7] = the number of valid rows.  When d_grad_tsdf is not NULL (device
 * memory, one float per pool voxel, indexed like mf_pool_tsdf) dE/d(tsdf) is
 * ADDED to it: through the model vertex, the model normal and the rendered
 * photometric reference depth of every pixel.  Voxel colours do not enter E.
 * The camera GN problem's state is overwritten.  Synchronises. */
int mf_camera_cost(mf_context* ctx, const float T_live[16], double* out, float* d_grad_tsdf);
/* Diagnostic, no reference counterpart: one GN step (the decision logic of
 * tracking.cpp:287-335 / :657-686: cost test with step back, 6x6 solve,
 * convergence test, SE(3) update) on given inputs, once by the device step
 * that the batched GN runs (one warp per problem) and once by the host step of
 * the plain path; the two must agree bit for bit.  state: n x 36 doubles
 * (T[16], prevT[16], prev_err, kind 0 camera / 1 object, first iteration of a
 * level 0/1, level); sums: n x 32 (the reduceKernel layout).  out_device,
 * out_host: n x 68 doubles (T[16], prevT[16], prev_err, done, fallback to the
 * truncated solve, iterations at the level, float pose[16], its inverse[16]).
 * Allocates and synchronises. */
int mf_debug_gn_step(mf_context* ctx, int n, const double* state, const double* sums,
                     double* out_device, double* out_host);

/* --- motion segmentation ------------------------------------------------
 * Tracking::compute_residuals (tracking/tracking.cpp:1535-1747) with the
 * moving-object test of kfusion.cpp:287-338 (check_static_state,
 * rendering/rendering.cpp:907-947).  Call after mf_track_camera: T_w_l is the
 * current camera pose, T_w_r the pose the model maps of the last mf_raycast
 * were rendered at.  Raycasts every instance at T_w_l (objects at their
 * current poses) into a second set of maps (the model maps stay), then
 * computes per pixel of level 0 an ICP row (live vertex against the model
 * maps) and a photometric row (the rendered live depth, seen from T_w_r,
 * warped into the reference intensity) with result codes 1 (inlier), -1 no
 * data, -2 outside the image, -3 no model point, -4 over the distance or
 * residual threshold, -5 normal / occlusion test.
 * inlier_ratio[i] (optional, one per instance): for objects i >= 1 with
 * pixels in the live render, the share of those pixels whose rows are all
 * > -3; -1 for the background and for objects out of view.
 * moving_labels (optional): bit `label` set for each object with
 * 0.05 < ratio < moved_threshold (the reference's defaults: residual
 * threshold 1.5, kernels.h:95; moved threshold 0.9, config --obj-moved)
 * whose class (mf_instance_set_semantics) is not one of the never-moving
 * classes 63, 69, 70 (Object::static_object, object.cpp:326).
 * The bits can be passed to mf_track_camera.  Synchronises. */
int mf_motion_residuals(mf_context* ctx, float residual_threshold, float moved_threshold,
                        float* inlier_ratio, uint32_t* moving_labels);
/* Host copies of the last mf_motion_residuals (each pointer optional):
 * results int8[2][H][W] (ICP rows, then photometric rows), errors
 * float[2][H][W] (valid where the result is 1, else 0), the live render's
 * vertex float[H][W][3] and label int32[H][W].  Synchronises. */
int mf_motion_download(mf_context* ctx, int8_t* results, float* errors, float* live_vertex,
                       int32_t* live_label);
/* The result codes (device int8[2][H][W], ICP then photometric) of instance
 * id's tracking rows at level 0 from its last GN iteration: the camera
 * (id 0, mf_track_camera) or object id (mf_track_objects) -- what the
 * reference copies into Object::trackresult_ (kfusion.cpp:282-283, 397-405)
 * for Object::refine_mask_use_motion.  pose_eval (optional, host float[16]):
 * the pose those rows were evaluated at (the camera's T_w_l, or the object's
 * T_c2_o2 = inverse(T_w_c2) T_w_o2); given, the call synchronises, else it
 * is asynchronous on the context stream.  d_errors (optional, device
 * float[2][H][W]): TrackData::error of the rows with result 1, else 0. */
int mf_track_results(mf_context* ctx, int id, int8_t* d_results, float* d_errors,
                     float* pose_eval);
/* Replaces the object part of Kfusion::tracking's residual pass,
 * kfusion.cpp:446-466: after a moving object id >= 1 was tracked
 * (mf_track_objects) and the live raycast redone at its new pose
 * (mf_motion_residuals), its result rows recomputed by
 * Tracking::compute_residuals (tracking.cpp:1535-1747) at its virtual camera
 * pose T_w_o1 inverse(T_c2_o2) (tracking.cpp:696) against its own pixels of
 * the model maps and of the live raycast -- what the reference copies into
 * the object's trackresult_ for Object::refine_mask_use_motion.  Rows to
 * d_results (device int8[2][H][W]); the virtual pose (host float[16],
 * optional; given, the call synchronises). */
int mf_object_residuals(mf_context* ctx, int id, float threshold, int8_t* d_results,
                        float* T_virtual);
/* Object::refine_mask_use_motion (object/object.cpp:255-315, outliers not
 * absorbed into the background) on instance id's generalized mask of the
 * current frame: where the mask is >= 0, an ICP row of -4 or -6 or a
 * photometric row below -3 in d_results (device int8[2][H][W]) sets it to -1
 * (not integrated).  d_results NULL = the planes of the last
 * mf_motion_residuals.  Asynchronous on the context stream. */
int mf_refine_mask_use_motion(mf_context* ctx, int id, const int8_t* d_results);
/* Host copy (float[H][W]) of instance id's generalized mask of the current
 * frame, as uploaded and refined.  Synchronises. */
int mf_download_mask(mf_context* ctx, int id, float* out);

/* --- object spawning and semantics -------------------------------------
 * Kfusion::spawnNewObjectKernel (kfusion.cpp:1080-1150): the placement of a
 * new object's volume from the current depth frame and camera pose.  mask:
 * uint8[H][W] (host or device), nonzero on the new object's pixels.  Every
 * masked pixel's vertex (zero where the depth is 0) goes to the world frame;
 * their bounding box and mean (float sums in row-major order, as the
 * reference accumulates them) give volume_size = min(2.5 max(dx, dy, dz / 2),
 * 5) and T_w_o = identity with the translation mean - size / 2;
 * volume_resol = 256 / 512 / 1024 / 2048 for sizes below 0.64 / 1.28 / 2.56 /
 * 5.12 m (0 where the reference leaves it unset).  n_pixels (optional): the
 * masked pixel count.  The caller adds the instance (mf_instance_add) and
 * integrates it, as Kfusion::generate_new_objects does.  Synchronises. */
int mf_spawn_object(mf_context* ctx, const uint8_t* mask, float T_w_o[16], float* volume_size,
                    int* volume_resol, int* n_pixels);
/* Object::Object's semantic state (object.cpp:11-34): class id, the class
 * probabilities of the segmentation that created it (n_classes, 80 in the
 * reference) and a fused count of 1. */
int mf_instance_set_semantics(mf_context* ctx, int id, int class_id, const float* probs,
                              int n_classes);
/* Object::fuse_semantic_kernel / fuseSemanticLabel (object.cpp:197-252): for
 * class_id != 0, the running mean (probs * recog_times + fused * fused_time) /
 * (fused_time + recog_times) in float; the object's class becomes 1 + the
 * first index of the largest fused probability.  MF_E_ARG when n_classes
 * differs from the object's (the reference exits). */
int mf_fuse_semantics(mf_context* ctx, int id, int class_id, const float* probs, int n_classes,
                      int recog_times);
/* The object's class id, fused count and (up to cap) fused probabilities. */
int mf_instance_semantics(mf_context* ctx, int id, int* class_id, int* fused_time, float* probs,
                          int cap);

/* --- formats ------------------------------------------------------------
 * Kfusion::preprocessing's input stage (kfusion.cpp:210-217): a sensor frame
 * of in_width x in_height with uint16 millimetre depth and uchar3 colour (host
 * or device pointers, each optional), subsampled by the integer ratio
 * in_width / width (mm2metersKernel, preprocessing.cpp:132-159;
 * rgb2intensity :73-102) into the frame's metres, float colour and grey.
 * MF_E_ARG for sizes the reference rejects.  Synchronises. */
int mf_frame_upload_raw(mf_context* ctx, const uint16_t* depth_mm, const uint8_t* rgb,
                        int in_width, int in_height);
/* The SLAMBench .raw reader (RawDepthReader, interface.h:207-335): per frame
 * uint32 (w, h), uint16 depth[w*h] (mm), uint32 (w, h), uchar3 rgb[w*h].
 * mf_raw_read: frame -1 = the next one; MF_E_NOT_FOUND past the end; either
 * destination may be NULL.  Host code only: needs no device. */
typedef struct mf_raw mf_raw;
int mf_raw_open(const char* path, mf_raw** out, int* width, int* height, long long* n_frames);
int mf_raw_read(mf_raw* raw, long long frame, uint16_t* depth_mm, uint8_t* rgb);
int mf_raw_close(mf_raw* raw);
/* Kfusion::save_poses (kfusion.cpp:1591-1626): appends one TUM line
 * "frame tx ty tz qx qy qz qw" (tab-separated, %g) per instance to
 * <prefix>_camera (label 0) or <prefix>_<label>; the first call per instance
 * truncates the file.  As the reference does, every line carries the camera's
 * translation with the instance's own rotation. */
int mf_save_poses(mf_context* ctx, const char* prefix, int frame);
/* The quaternion (x, y, z, w) of a pose's rotation (getQuaternion,
 * preprocessing.cpp:312-320) and one TUM line of mf_save_poses; host code
 * only.  mf_tum_line returns the line length. */
int mf_pose_quaternion(const float T[16], float q[4]);
int mf_tum_line(int frame, const float T_translation[16], const float T_rotation[16], char* buf,
                int cap);

/* --- mesh export ----------------------------------------------------------
 * Marching cubes over instance id's octree: algorithms::marching_cube
 * (lib/algorithms/meshing.hpp:20-208) as Kfusion::dump_mesh calls it
 * (kfusion.cpp:1560-1588): cells whose eight corners all have weight > 0,
 * foreground probability > 0.5 and count > 3, inside = tsdf < 0, the
 * reference's edge intersections, triangles dropped when a vertex leaves
 * (0, (int)dim] -- the reference truncates the extent to an int, so volumes
 * under 1 m mesh to nothing; float_bounds = 1 bounds by the float extent
 * instead.  The triangulation table is generated from the cube's
 * geometry (gen_mc_tables.py): the same polygons as the reference's table,
 * possibly split along other diagonals; with the reference's own table
 * (mf_mesh_set_triangle_table) the triangles are the reference's, one for
 * one.  Triangles are 9 floats (three
 * vertices, metres, volume frame), blocks in Morton order and cells x-major
 * within a block.  tris may be host or device memory; with tris NULL or cap
 * below the count only n_tris is set.  Synchronises. */
int mf_mesh(mf_context* ctx, int id, int float_bounds, float* tris, long long cap,
            long long* n_tris);
/* The marching-cubes triangulation table mf_mesh uses for this context: 256
 * rows of 16 ints, each at most 5 edge triples (edges 0..11 as
 * lib/algorithms/meshing.hpp numbers them) ended by -1 -- the layout of the
 * reference's triTable (lib/algorithms/edge_tables.h), which a caller that has
 * it passes as &triTable[0][0] to get the reference's triangles.  NULL
 * restores the built-in table.  MF_E_ARG for a malformed row. */
int mf_mesh_set_triangle_table(mf_context* ctx, const int* table);
/* writeVtkMesh (commons.h:945-1011): legacy ASCII VTK polydata, three points
 * per triangle.  Host code only. */
int mf_write_vtk_mesh(const char* path, const float* tris, long long n);
/* Kfusion::dump_mesh: <prefix>_<label>.vtk for every instance (the
 * reference's int bound). */
int mf_dump_mesh(mf_context* ctx, const char* prefix);

/* --- headless renders ---------------------------------------------------
 * The reference's visualisation kernels (rendering/rendering.cpp) into
 * uchar4 images of W x H (mf_render_normal: uchar3).  `out` may be device
 * memory (written asynchronously on the context stream) or host memory
 * (rendered into a context scratch image and copied; the call synchronises).
 * Float-to-byte conversions keep the low byte of the 32-bit integer value,
 * as the reference does when built with gcc for x86-64.
 *
 * renderVolume_many_Kernel (rendering.cpp:489-646) as Kfusion::renderVolume
 * calls it (kfusion.cpp:1303-1309: near plane, 2 x far plane).  T_w_c: the
 * view pose to raycast every instance from, with that kernel's own
 * composite rules; NULL = shade the maps of the last mf_raycast (the
 * reference's doraycast == false).  render_color: shade with the
 * interpolated voxel colour, else with colors[label] (the background white).
 * largestep: the march step outside the band (the reference's benchmark
 * passes 0.75 mu).  ambient: float[3] or NULL for (0.1, 0.1, 0.1)
 * (constant_parameters.h:24).  colors: n_colors RGBA entries indexed by
 * instance label; labels outside the table render black. */
int mf_render_volume(mf_context* ctx, const float* T_w_c, int render_color, float largestep,
                     const float* ambient, const uint8_t* colors, int n_colors, uint8_t* out);
/* renderDepthKernel (rendering.cpp:366-393) of the current input depth with
 * the config's near and far planes. */
int mf_render_depth(mf_context* ctx, uint8_t* out);
/* renderIntensityKernel (rendering.cpp:648-664) of the current grey input. */
int mf_render_intensity(mf_context* ctx, uint8_t* out);
/* renderNormalKernel (rendering.cpp:346-364) of the model normal map (uchar3). */
int mf_render_normal(mf_context* ctx, uint8_t* out);
/* Track renders of result rows (device int8[2][H][W], errors float[2][H][W]
 * from mf_track_results; both NULL = the last mf_motion_residuals): mode 0
 * renderTrackKernel (rendering.cpp:395-432) of the ICP rows, 1
 * renderRGBTrackKernel (:434-487) of the photometric rows, 2
 * render_RGBD_TrackKernel (:183-237) of both. */
int mf_render_track(mf_context* ctx, int mode, const int8_t* d_results, const float* d_errors,
                    uint8_t* out);
/* Label renders of a label image (device int32[H][W]; NULL = the last
 * mf_raycast's): mode 0 renderInstanceMaskKernel (rendering.cpp:797-820;
 * pass colours indexed by class for renderClassMaskKernel :822-847), 1
 * renderMaskWithImageKernel (:679-723) over the current RGB input, 2
 * renderMaskMotionWithImageKernel (:725-795), which also reads each label's
 * result rows: d_rows[label] (a host array of n_rows device pointers, each
 * int8[2][H][W] or NULL), the Object::trackresult_ of that instance. */
int mf_render_mask(mf_context* ctx, int mode, const int32_t* d_labels, const uint8_t* colors,
                   int n_colors, const int8_t* const* d_rows, int n_rows, uint8_t* out);
/* The pool's TSDF values: a device pointer to pool capacity x 512 floats
 * (voxel v of pool slot s at s * 512 + v). */
int mf_pool_tsdf(mf_context* ctx, float** d_tsdf, long long* n);
/* Which block each used pool slot holds: 4 ints per slot (corner voxel x, y,
 * z and the instance id), for slots 0 .. *n - 1 (at most `cap` written). */
int mf_pool_slots(mf_context* ctx, int32_t* meta, long long cap, long long* n);
/* Pyramid planes of the current frame: which 0 depth, 1 intensity, 2 vertex,
 * 3 normal, 4 x-gradient, 5 y-gradient, 6 ICP covariance, 7 camera reference
 * vertex (float3 planes are 3 floats per pixel). */
int mf_download_pyramid(mf_context* ctx, int level, int which, float* out);

/* --- whole frame -------------------------------------------------------
 * One frame of Kfusion in the reference's order (mainQt.cpp:262-291,
 * benchmark.cpp:113-159): preprocessing; from the second frame on, camera
 * tracking against the last raycast (moving-object pixels excluded from ICP)
 * and trackEachObject for every object instance; generalized masks from the
 * uint16 ground-truth labels (NULL: keep the current masks); allocation +
 * integration of every instance; raycastObjectList; setRefImgFromCurr.
 * Host pointers (copied in; nothing is read back -- see mf_get_poses). */
int mf_process_frame(mf_context* ctx, const float* depth, const uint8_t* rgb,
                     const uint16_t* labels);
/* Same with device pointers. */
int mf_process_frame_device(mf_context* ctx, const float* d_depth, const uint8_t* d_rgb,
                            const uint16_t* d_labels);
/* No counterpart in the reference, which reads each frame on the host before
 * processing it.  A stream of frames with its uploads overlapped:
 * mf_frame_stage copies a frame's inputs (as mf_process_frame takes them;
 * labels may be NULL) from host memory into input slot `slot` (0 or 1) on
 * the context's upload stream and returns without waiting; mf_process_staged
 * then processes the frame in that slot exactly as mf_process_frame would.
 * Staging frame f + 1 into the other slot before mf_get_poses of frame f lets
 * its copy run while frame f is processed.  An upload into a slot waits, on
 * the device, until the frame processed from it has copied it out.  The host
 * buffers must be pinned for the copy to overlap, and must stay unchanged
 * until the frame has been processed (mf_get_poses after mf_process_staged).
 * MF_E_STATE: staging into a slot whose frame has not been processed, or
 * processing an empty slot.  The slots (2 x W*H*9 bytes) and the stream are
 * created by the first call. */
int mf_frame_stage(mf_context* ctx, int slot, const float* depth, const uint8_t* rgb,
                   const uint16_t* labels);
int mf_process_staged(mf_context* ctx, int slot);
/* The upload stream of mf_frame_stage (created on first use), as a
 * cudaStream_t, for callers that order their own work with it. */
int mf_upload_stream(mf_context* ctx, void** stream);
/* Kfusion::tracking with motion segmentation (apps/kfusion/src/cpp/
 * kfusion.cpp:265-466) and the integration that follows (:606-630), for one
 * frame from host buffers (labels required).  Host-driven (it synchronises
 * between stages), not a replayed graph:
 *  1. the camera is tracked against the whole model;
 *  2. mf_motion_residuals at the tracked pose gives every object's inlier
 *     ratio and the moving labels (residual_threshold: the reference's 1.5,
 *     kernels.h:95; moved_threshold: 0.9, --obj-moved);
 *  3. with moving objects the camera is tracked again with their pixels
 *     excluded, only the moving objects are tracked, and the motion residuals
 *     are computed again;
 *  4. from this entry point's third frame on, every instance's generalized
 *     mask is refined (mf_refine_mask_use_motion): the background and static
 *     objects with the camera's rows (those motion residuals when objects
 *     move, else the camera's last GN rows), a moving object with its rows
 *     recomputed at its virtual camera pose (mf_object_residuals,
 *     kfusion.cpp:446-466);
 *  5. every instance is integrated, the composite raycast replaces the model
 *     maps, and the frame becomes the photometric reference.
 * The first frame (no reference yet) is integrated and raycast untracked.
 * moving_labels receives the moving-label bits of step 2 (0 on the first
 * frame).  Objects of the never-moving classes (Object::static_object)
 * never move. */
int mf_process_frame_motion(mf_context* ctx, const float* depth, const uint8_t* rgb,
                            const uint16_t* labels, float residual_threshold,
                            float moved_threshold, uint32_t* moving_labels);
/* Camera pose (16 floats) and every instance's volume pose (16 floats each,
 * instance order); either pointer may be NULL.  Synchronises. */
int mf_get_poses(mf_context* ctx, float* T_w_c, float* T_w_o);
/* Work counters of the last frame: out[0] voxel blocks in the pool (at most
 * its capacity; a full pool is the MF_STATUS_POOL_FULL flag), out[1]
 * blocks visited by the last integration, out[2 + i] ray samples instance i
 * emitted into its allocation list, out[2 + n_instances] kernel launches in one
 * replay of the batched frame graph (0 before capture).  Synchronises. */
int mf_frame_stats(mf_context* ctx, long long* out, int n);
/* Kernel timing on the current frame (CUDA events on the context's stream,
 * `reps` launches each): out[0] us per camera GN evaluation at level 0 and
 * out[1] its algorithmic bytes; out[2] us per integration launch and out[3] its
 * algorithmic bytes (counted); out[4] us per raycast launch and out[5] its
 * algorithmic bytes (counted by a replay of the march: 8 B per voxel read,
 * 32 B per trilinear interpolation, 64 + 192 B per candidate hit's
 * foreground interpolation and gradient, 28 B of output per pixel).
 * Re-integrates the current frame, so call it only after the frames that
 * matter. */
int mf_profile(mf_context* ctx, int reps, double* out, int n);
/* Batched mode replays the frame as a CUDA graph once captured (default 1). */
int mf_set_graphs(mf_context* ctx, int enable);
/* No counterpart in the reference.  Batched GN runs every iteration of a
 * pyramid level in one cooperative launch per level and stage, with a grid
 * barrier between iterations and an early end once every problem has stopped
 * (1), or one launch per iteration, each chained to the previous one by
 * programmatic dependent launch (0, the default: faster on B200, where the
 * frame graph already removes the launch overhead and the grid barrier costs
 * more than a launch boundary).  Both give the same poses bit for bit.
 * Applies to frames captured after the call. */
int mf_set_gn_persistent(mf_context* ctx, int enable);
/* No counterpart in the reference.  Batched frames with objects: the
 * background's allocation and integration (which need only the camera pose)
 * run on a low-priority side stream while the objects are tracked on the
 * context's stream (highest priority); the objects' allocation and
 * integration follow.  ctas < 0 (the default): the integration launch shape's
 * own grid; ctas > 0: that many integration CTAs; 0: everything in order on
 * the context's stream.  The volumes and poses are the in-order frame's (pool
 * slots are handed out in another order).  Applies to frames captured after
 * the call. */
int mf_set_overlap(mf_context* ctx, int ctas);

/* --- launch-shape autotuner (no counterpart in the reference) ----------
 * Two kernels of the frame run in one of several launch shapes that change
 * their speed but not their results (each pixel / voxel is computed by one
 * thread from the same inputs in every shape):
 *   MF_TUNE_RAYCAST    the composite raycast (raycastObjectList): the pixel
 *                      tile of a 128-thread CTA and the register bound;
 *   MF_TUNE_INTEGRATE  the voxel-block integration (projective_functor::
 *                      update_block): 512-thread CTAs resident per SM.
 * Variant 0 of each is the default.  A context starts with the defaults. */
#define MF_TUNE_RAYCAST 0
#define MF_TUNE_INTEGRATE 1
#define MF_TUNE_MAX_VARIANTS 16
/* Number of candidate shapes of `stage` (no context, no device needed). */
int mf_tune_candidates(int stage, int* n);
/* One-line description of candidate `variant` of `stage` into buf. */
int mf_tune_describe(int stage, int variant, char* buf, int cap);
/* Times every candidate of both stages on the current frame (`reps` launches,
 * best of 3 trials, CUDA events) and keeps the fastest of each; the current
 * choice stays unless another is more than 1 % faster.  raycast_us and
 * integrate_us (MF_TUNE_MAX_VARIANTS floats each, may be NULL) receive the
 * microseconds per launch of every candidate.  Needs a processed frame (the
 * instances, the frame inputs and the map of the last mf_process_frame or
 * mf_integrate).  Leaves the map and the model maps unchanged: the raycasts
 * write scratch maps and the integrations update a scratch copy of the pool
 * slots in use (allocated for the call and freed before it returns).  The
 * next batched frame re-captures its graph with the chosen shapes.
 * Synchronises. */
int mf_autotune(mf_context* ctx, int reps, float* raycast_us, float* integrate_us);
/* The candidate in use for `stage`, or set it (a saved choice of an earlier
 * mf_autotune); an unknown stage or variant is MF_E_ARG. */
int mf_tune_get(mf_context* ctx, int stage, int* variant);
int mf_tune_set(mf_context* ctx, int stage, int variant);

/* --- inspection (parity checks, debugging) -----------------------------
 * Blocks: key (code | level), corner voxel, VoxelBlock::active_, and when
 * `voxels` is not NULL the 512 voxels in the reference's 40-byte AoS layout
 * (voxel_traits<SDF>::ComputeType).  Order is unspecified. */
int mf_block_count(mf_context* ctx, int id, int* n);
int mf_export_blocks(mf_context* ctx, int id, uint64_t* keys, int32_t* coords,
                     uint8_t* active, void* voxels, int cap, int* n);
/* Internal nodes (levels 1..block level - 1): key, side, children mask,
 * and Node::value_[8] (40-byte AoS) when `values` is not NULL. */
int mf_node_count(mf_context* ctx, int id, int* n);
int mf_export_nodes(mf_context* ctx, int id, uint64_t* keys, uint32_t* side,
                    uint8_t* children_mask, void* values, int cap, int* n);
int mf_root_children(mf_context* ctx, int id, uint8_t* mask);
/* Volume::interp (continuous/volume_template.hpp:97-104) at n points
 * (metres, volume frame); field 0 = tsdf, 1 = foreground probability,
 * 2, 3, 4 = colour r, g, b. */
int mf_interp(mf_context* ctx, int id, const float* pos, int n, int field, float* out);

#ifdef __cplusplus
}
#endif
#endif /* MIDFUSION_B200_H */
