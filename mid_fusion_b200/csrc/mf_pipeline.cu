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
  if (!ctx->graphs) return;
  FrameGraphs& g = *(FrameGraphs*)ctx->graphs;
  for (auto& e : g.exec)
    if (e) cudaGraphExecDestroy(e);
  delete (FrameGraphs*)ctx->graphs;
  ctx->graphs = nullptr;
}

// Everything of one frame after the inputs are on the device.
static int frame_body(Context* ctx, bool track, bool labels) {
  const int n = (int)ctx->inst.size();
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
  if (labels && n > 0)
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
    MF_CUDA(cudaGraphInstantiate(&g.exec[parity], graph, 0));
    cudaGraphDestroy(graph);
  }
  MF_CUDA(cudaGraphLaunch(g.exec[parity], ctx->stream));
  track_set_parity(ctx, 1 - parity);
  return MF_OK;
}

size_t graph_kernel_nodes(Context* ctx) {
  if (!ctx->graphs) return 0;
  FrameGraphs& g = *(FrameGraphs*)ctx->graphs;
  return std::max(g.kernel_nodes[0], g.kernel_nodes[1]);
}

}  // namespace mf
