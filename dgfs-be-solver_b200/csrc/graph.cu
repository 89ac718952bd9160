// CUDA graphs at the C ABI: a caller that drives the library through its C
// entry points alone (frfs's PyCUDA backend, for one) captures a Runge-Kutta
// stage -- the dgfs_vhs_apply, dgfs_dg_updatebc, dgfs_dg_interp and
// dgfs_dg_rhs calls of frfs's StdTVDRK2DGFSStepper stage
// (frfs/integrators/std/steppers.py:157-221) -- once, and replays it every
// step with one launch.  The reference launches each kernel of a stage
// from Python every step.
#include <cuda_runtime.h>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"

struct dgfs_graph {
  cudaGraph_t graph;
  cudaGraphExec_t exec;
};

using dgfs::clear_error;
using dgfs::set_error;

extern "C" int dgfs_graph_begin(void* stream) {
  clear_error();
  if (!stream) return set_error(DGFS_ERR_INVALID, "capture needs a created stream, not the legacy default stream");
  const cudaError_t e = cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_graph_end(void* stream, dgfs_graph** out) {
  clear_error();
  if (!stream || !out) return set_error(DGFS_ERR_INVALID, "null argument");
  *out = nullptr;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture((cudaStream_t)stream, &g);
  if (e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    return set_error(DGFS_ERR_CUDA, "end capture (a call inside the capture failed or synchronised?): %s",
                     cudaGetErrorString(e != cudaSuccess ? e : cudaErrorStreamCaptureInvalidated));
  }
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return set_error(DGFS_ERR_CUDA, "instantiate graph: %s", cudaGetErrorString(e));
  }
  *out = new dgfs_graph{g, x};
  return DGFS_OK;
}

extern "C" int dgfs_graph_launch(dgfs_graph* g, void* stream) {
  clear_error();
  if (!g) return set_error(DGFS_ERR_INVALID, "null graph");
  const cudaError_t e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(DGFS_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
  return DGFS_OK;
}

extern "C" int dgfs_graph_destroy(dgfs_graph* g) {
  clear_error();
  if (!g) return DGFS_OK;
  cudaGraphExecDestroy(g->exec);
  cudaGraphDestroy(g->graph);
  delete g;
  return DGFS_OK;
}
