// CUDA-graph capture of a context's work.  A caller records a fixed sequence
// of evaluations (for example a batch's HMult -> relinearise -> rescale chain
// with its rotations and additions) once and replays it with one launch, so
// the per-kernel launch cost of the many small stages disappears.  No
// reference counterpart (the reference launches every kernel from the host).
//
// Between capture_begin and capture_end only asynchronous calls may be made
// on the context (evaluations, device copies); calls that synchronise
// (downloads, decode, key creation, aoa_ctx_sync) end the capture with an
// error.  Work sizes must already have been run once on the context, so
// that its workspaces exist and nothing is allocated while capturing.
#include "aoa_internal.h"

struct aoa_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  size_t nodes = 0;
};

using namespace aoa;

extern "C" {

int aoa_ctx_capture_begin(aoa_ctx* c) {
  if (!c) return fail(AOA_ERR_BAD_PARAM, "null context");
  return guarded([&] { AOA_CUDA(cudaStreamBeginCapture(c->c.stream, cudaStreamCaptureModeThreadLocal)); });
}

int aoa_ctx_capture_end(aoa_ctx* c, aoa_graph** out) {
  if (!c || !out) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] {
    aoa_graph* g = new aoa_graph();
    cudaError_t e = cudaStreamEndCapture(c->c.stream, &g->graph);
    if (e != cudaSuccess) {
      cudaGetLastError();
      delete g;
      throw AoaError(AOA_ERR_CUDA, std::string("capture failed: ") + cudaGetErrorString(e));
    }
    e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e != cudaSuccess) {
      cudaGetLastError();
      cudaGraphDestroy(g->graph);
      delete g;
      throw AoaError(AOA_ERR_CUDA, std::string("graph instantiation failed: ") + cudaGetErrorString(e));
    }
    AOA_CUDA(cudaGraphGetNodes(g->graph, nullptr, &g->nodes));
    *out = g;
  });
}

int aoa_graph_launch(aoa_ctx* c, aoa_graph* g) {
  if (!c || !g) return fail(AOA_ERR_BAD_PARAM, "null argument");
  return guarded([&] { AOA_CUDA(cudaGraphLaunch(g->exec, c->c.stream)); });
}

int aoa_graph_nodes(const aoa_graph* g, long* nodes) {
  if (!g || !nodes) return fail(AOA_ERR_BAD_PARAM, "null argument");
  *nodes = (long)g->nodes;
  return AOA_OK;
}

int aoa_graph_destroy(aoa_graph* g) {
  if (!g) return AOA_OK;
  int st = guarded([&] {
    if (g->exec) AOA_CUDA(cudaGraphExecDestroy(g->exec));
    if (g->graph) AOA_CUDA(cudaGraphDestroy(g->graph));
  });
  delete g;
  return st;
}

}  // extern "C"
