// Whole-frame pipeline: the reference's Kfusion per-frame order
// (apps/kfusion/src/mainQt.cpp:262-291, apps/kfusion/src/benchmark.cpp:113-159):
//   preprocessing -> tracking (camera, then every moving object)
//   -> integration of every instance -> multi-instance raycast
//   -> the frame becomes the photometric reference.
// Batched mode queues the whole frame without a host round trip and replays
// it as a CUDA graph (one graph per parity of the double-buffered reference
// pyramid).  Plain mode runs one instance per launch and drives every GN
// iteration from the host.
#include <algorithm>
#include <cstring>
#include <utility>
#include <vector>
#include "mf_internal.h"

namespace mf {

struct FrameGraphs {
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  size_t kernel_nodes[2] = {0, 0};
  int n_instances = -1;
  bool labels = false;
  unsigned tune_gen = 0;   // launch shapes the graphs were captured with
};

static FrameGraphs& graphs(Context* ctx) {
  if (!ctx->graphs) ctx->graphs = new FrameGraphs;
  return *(FrameGraphs*)ctx->graphs;
}

void pipeline_free(Context* ctx) {
  if (ctx->d_motion_rows) cudaFree(ctx->d_motion_rows);
  ctx->d_motion_rows = nullptr;
  if (!ctx->graphs) return;
  FrameGraphs& g = *(FrameGraphs*)ctx->graphs;
  for (auto& e : g.exec)
    if (e) cudaGraphExecDestroy(e);
  delete (FrameGraphs*)ctx->graphs;
  ctx->graphs = nullptr;
}

// A batched frame with objects, in two branches of one graph.  The main
// stream (highest priority) runs the critical path: the pyramid, the camera's
// outlier mask and GN, the objects' GN, allocation, integration and raycast
// marches, and the composite's fold.  The side stream (lowest priority) runs
// what does not wait for it: first the tracking setup that needs no live
// frame and no tracked pose (the camera's and the objects' problems from the
// previous poses, their rendered references, the camera's outlier mask of the
// moving objects' pixels) and the integration masks while the pyramid is
// built; then, once the camera is tracked, the background's
// allocation, integration (own visit list, overlap_ctas CTAs or the launch
// shape's own grid) and raycast marches while the objects are tracked.
// Nothing one branch reads is written by the other before the event that
// orders them, so the frame equals the in-order frame bit for bit (pool
// slots are handed out in another order).  Every event is recorded and
// waited on whatever happens, so that a stream capture always ends joined.
static int frame_overlapped(Context* ctx, bool gen, const IdList& all, const IdList& objs,
                            uint32_t moving) {
  IdList bg;
  bg.n = 1;
  bg.v[0] = 0;
  const bool phased = raycast_is_phased(ctx);
  cudaStream_t main = ctx->stream, side = ctx->side;
  int rc = MF_OK;
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t x) { if (x != cudaSuccess && e == cudaSuccess) e = x; };
  ctx->visit_side_used = true;
  // side: the pose-independent tracking setup, then the masks
  ok(cudaEventRecord(ctx->ev_start, main));
  ok(cudaStreamWaitEvent(side, ctx->ev_start, 0));
  ctx->stream = side;
  // the camera's first (it is needed first): its problem, its rendered
  // reference, and the moving objects' pixels written whole into every level
  // of its outlier mask (the pyramid then leaves the mask planes alone)
  rc = track_camera_pre(ctx, 0);
  if (!rc) rc = track_camera_mask(ctx, moving);
  ok(cudaEventRecord(ctx->ev_pre, side));
  if (!rc) rc = track_objects_pre(ctx, objs);
  ok(cudaEventRecord(ctx->ev_obj, side));
  if (!rc && gen) rc = launch_generalize(ctx);
  ok(cudaEventRecord(ctx->ev_gen, side));
  ctx->stream = main;
  // main: the pyramid, then the camera's GN
  if (!rc) rc = track_preprocess(ctx, /*clear_mask=*/moving == 0);
  ok(cudaStreamWaitEvent(main, ctx->ev_pre, 0));
  if (!rc) rc = track_camera_gn(ctx);
  ok(cudaEventRecord(ctx->ev_fork, main));
  // side: the background, at the tracked camera pose
  ok(cudaStreamWaitEvent(side, ctx->ev_fork, 0));
  ctx->stream = side;
  std::swap(ctx->d_visit, ctx->d_visit_side);
  std::swap(ctx->d_visit_count, ctx->d_visit_count_side);
  if (!rc) rc = stage_prepare(ctx, bg);
  if (!rc) rc = stage_alloc(ctx, bg);
  if (!rc) rc = stage_integrate(ctx, bg, ctx->overlap_ctas > 0 ? ctx->overlap_ctas : 0);
  if (!rc && phased) rc = stage_raycast_hits(ctx, bg, 0, ctx->ray_epsilon);
  ok(cudaEventRecord(ctx->ev_join, side));
  std::swap(ctx->d_visit, ctx->d_visit_side);
  std::swap(ctx->d_visit_count, ctx->d_visit_count_side);
  ctx->stream = main;
  // main: the objects
  ok(cudaStreamWaitEvent(main, ctx->ev_obj, 0));
  if (!rc) rc = track_objects_gn(ctx, objs);
  ok(cudaStreamWaitEvent(main, ctx->ev_gen, 0));
  if (!rc) rc = stage_prepare(ctx, objs);
  if (!rc) rc = stage_alloc(ctx, objs);
  if (!rc) rc = stage_integrate(ctx, objs);
  if (!rc && phased) rc = stage_raycast_hits(ctx, objs, 1, ctx->ray_epsilon);
  ok(cudaStreamWaitEvent(main, ctx->ev_join, 0));
  if (rc) return rc;
  if (e != cudaSuccess) {
    ctx->last_error = std::string("overlapped frame: ") + cudaGetErrorString(e);
    return MF_E_CUDA;
  }
  if (int rc2 = phased ? stage_raycast_fold(ctx, all, ctx->ray_epsilon)
                       : stage_raycast(ctx, all, ctx->ray_epsilon))
    return rc2;
  return track_set_ref(ctx);
}

// Everything of one frame after the inputs are on the device.
static int frame_body(Context* ctx, bool track, bool labels) {
  const int n = (int)ctx->inst.size();
  ctx->visit_side_used = false;
  IdList all, objs;
  all.n = n;
  objs.n = 0;
  uint32_t moving = 0;
  for (int i = 0; i < n; ++i) {
    all.v[i] = i;
    if (i > 0) {
      objs.v[objs.n++] = i;
      if (ctx->inst[i].label >= 0 && ctx->inst[i].label < 32) moving |= 1u << ctx->inst[i].label;
    }
  }
  const bool gen = labels && n > 0;
  if (track && objs.n && ctx->cfg.batched && ctx->overlap_ctas != 0)
    return frame_overlapped(ctx, gen, all, objs, moving);
  if (gen)
    if (int rc = launch_generalize(ctx)) return rc;
  if (int rc = track_preprocess(ctx)) return rc;
  if (track) {
    if (int rc = track_camera(ctx, moving)) return rc;
    if (objs.n)
      if (int rc = track_objects(ctx, objs)) return rc;
  }
  if (ctx->cfg.batched) {
    if (int rc = stage_prepare(ctx, all)) return rc;
    if (int rc = stage_alloc(ctx, all)) return rc;
    if (int rc = stage_integrate(ctx, all)) return rc;
  } else {
    for (int i = 0; i < n; ++i) {
      IdList one;
      one.n = 1;
      one.v[0] = i;
      if (int rc = stage_prepare(ctx, one)) return rc;
      if (int rc = stage_alloc(ctx, one)) return rc;
      if (int rc = stage_integrate(ctx, one)) return rc;
    }
  }
  // the instance frames prepared for integration hold for the raycast: no
  // pose changes in between
  if (int rc = stage_raycast(ctx, all, ctx->ray_epsilon)) return rc;
  return track_set_ref(ctx);
}

int process_frame(Context* ctx, bool labels) {
  if (ctx->inst.empty()) return MF_E_STATE;
  if (int rc = track_init(ctx)) return rc;
  const bool track = track_has_ref(ctx);
  if (!ctx->cfg.batched || !track || !ctx->use_graphs) return frame_body(ctx, track, labels);
  FrameGraphs& g = graphs(ctx);
  if (g.n_instances != (int)ctx->inst.size() || g.labels != labels ||
      g.tune_gen != ctx->tune.gen) {
    for (auto& e : g.exec)
      if (e) { cudaGraphExecDestroy(e); e = nullptr; }
    g.n_instances = (int)ctx->inst.size();
    g.labels = labels;
    g.tune_gen = ctx->tune.gen;
  }
  const int parity = track_parity(ctx);
  if (!g.exec[parity]) {
    cudaGraph_t graph = nullptr;
    MF_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = frame_body(ctx, true, labels);
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (e != cudaSuccess) {
      ctx->last_error = std::string("graph capture: ") + cudaGetErrorString(e);
      return MF_E_CUDA;
    }
    // the capture flipped the reference parity on the host; flip it back: the
    // launch below performs that frame
    track_set_parity(ctx, parity);
    size_t n_nodes = 0;
    cudaGraphGetNodes(graph, nullptr, &n_nodes);
    std::vector<cudaGraphNode_t> nodes(n_nodes);
    cudaGraphGetNodes(graph, nodes.data(), &n_nodes);
    size_t kernels = 0;
    for (auto nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
    }
    g.kernel_nodes[parity] = kernels;
    // the kernel nodes keep the priorities of the streams they were captured
    // from (the overlapped background integration runs at the lowest)
    MF_CUDA(cudaGraphInstantiate(&g.exec[parity], graph, cudaGraphInstantiateFlagUseNodePriority));
    cudaGraphDestroy(graph);
  }
  MF_CUDA(cudaGraphLaunch(g.exec[parity], ctx->stream));
  track_set_parity(ctx, 1 - parity);
  return MF_OK;
}

// Kfusion::tracking with motion segmentation (kfusion.cpp:265-466), then the
// integration of kfusion.cpp:606-630 with motion-refined masks, the raycast
// and the new reference frame.  Host-driven: which objects move is decided on
// the host between the stages, as the reference decides it.
//  1. the camera is tracked against the whole model (no mask, :274-281);
//  2. motion residuals at the tracked pose (the model raycast with the
//     objects at their last poses), per-object inlier ratios and the moving
//     labels (:291-347);
//  3. with moving objects: the camera is tracked again with their pixels
//     excluded (:358-393), only the moving objects are tracked (:396-411),
//     and the motion residuals are computed again at the new pose (:418-441);
//  4. from the third frame on (frame > 1, :620), every instance's generalized
//     mask is refined with result rows (Object::refine_mask_use_motion): the
//     background and the static objects with the camera's rows (the motion
//     residuals of step 3 when objects move, else the rows of the camera's
//     last GN iteration, :282, :396-400), a moving object with its rows
//     recomputed at its virtual camera pose against its own maps (:446-466);
//  5. every instance is integrated with its mask, the composite raycast
//     replaces the model maps and the frame becomes the reference.
// The first frame (no reference yet) is integrated and raycast untracked.
int process_frame_motion(Context* ctx, float thr, float moved, uint32_t* moving_out) {
  if (ctx->inst.empty()) return MF_E_STATE;
  if (int rc = track_init(ctx)) return rc;
  const int frame = ctx->motion_frames++;
  *moving_out = 0;
  if (!track_has_ref(ctx)) return frame_body(ctx, false, true);
  const int n = (int)ctx->inst.size();
  const size_t WH = (size_t)ctx->W * ctx->H;
  if (!ctx->d_motion_rows) MF_CUDA(cudaMalloc(&ctx->d_motion_rows, 4 * WH));
  int8_t* cam_rows = ctx->d_motion_rows;
  int8_t* obj_rows = ctx->d_motion_rows + 2 * WH;
  if (int rc = launch_generalize(ctx)) return rc;
  if (int rc = track_preprocess(ctx)) return rc;
  if (int rc = track_camera(ctx, 0)) return rc;
  uint32_t moving = 0, again = 0;
  float ratio[MAX_INSTANCES];
  if (n > 1)
    if (int rc = motion_residuals(ctx, thr, moved, ratio, &moving)) return rc;
  IdList mov;
  mov.n = 0;
  bool is_moving[MAX_INSTANCES] = {};
  for (int i = 1; i < n; ++i) {
    const int l = ctx->inst[i].label;
    if (l >= 0 && l < 32 && ((moving >> l) & 1u)) {
      mov.v[mov.n++] = i;
      is_moving[i] = true;
    }
  }
  if (mov.n) {
    if (int rc = track_camera(ctx, moving, 1)) return rc;
    if (int rc = track_objects(ctx, mov)) return rc;
    if (int rc = motion_residuals(ctx, thr, moved, ratio, &again)) return rc;
  }
  if (frame > 1) {
    const int8_t* rows0 = nullptr;  // the last motion residuals
    if (!mov.n) {
      if (int rc = track_results(ctx, 0, cam_rows, nullptr, nullptr)) return rc;
      rows0 = cam_rows;
    }
    for (int i = 0; i < n; ++i) {
      const int8_t* rows = rows0;
      if (is_moving[i]) {
        if (int rc = object_residuals(ctx, i, thr, obj_rows, nullptr)) return rc;
        rows = obj_rows;
      }
      if (int rc = refine_mask_use_motion(ctx, i, rows, ctx->cfg.use_icp, ctx->cfg.use_rgb))
        return rc;
    }
  }
  IdList all;
  all.n = n;
  for (int i = 0; i < n; ++i) all.v[i] = i;
  if (ctx->cfg.batched) {
    if (int rc = stage_prepare(ctx, all)) return rc;
    if (int rc = stage_alloc(ctx, all)) return rc;
    if (int rc = stage_integrate(ctx, all)) return rc;
  } else {
    for (int i = 0; i < n; ++i) {
      IdList one;
      one.n = 1;
      one.v[0] = i;
      if (int rc = stage_prepare(ctx, one)) return rc;
      if (int rc = stage_alloc(ctx, one)) return rc;
      if (int rc = stage_integrate(ctx, one)) return rc;
    }
  }
  if (int rc = stage_raycast(ctx, all, ctx->ray_epsilon)) return rc;
  if (int rc = track_set_ref(ctx)) return rc;
  *moving_out = moving;
  return MF_OK;
}

size_t graph_kernel_nodes(Context* ctx) {
  if (!ctx->graphs) return 0;
  FrameGraphs& g = *(FrameGraphs*)ctx->graphs;
  return std::max(g.kernel_nodes[0], g.kernel_nodes[1]);
}

}  // namespace mf
