// CUDA-graph capture of a block's launch sequence (the batched form).
//
// dsb_graph_begin starts a stream capture; every launch the host then makes
// on that stream (the library's kernels, memsets) is recorded instead of
// run.  dsb_graph_end_launch ends the capture, turns the recorded graph into
// an executable one -- the first time by instantiating it, later by
// updating the previous executable graph in place (cudaGraphExecUpdate: the
// same topology with new arguments, which is what the next block's sequence
// is: its stream times move, its kernels and buffers stay) -- and launches
// it on the stream.  A sequence whose topology changed (a different number
// of launches) is instantiated afresh.
#include "dsb_common.cuh"

extern "C" {

int dsb_graph_begin(cudaStream_t stream) {
  if (!stream) return DSB_E_ARG;  // the legacy default stream cannot be captured
  return cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed) == cudaSuccess
             ? DSB_OK
             : DSB_E_CUDA;
}

int dsb_graph_end_launch(cudaStream_t stream, void** exec) {
  if (!stream || !exec) return DSB_E_ARG;
  cudaGraph_t graph = nullptr;
  if (cudaStreamEndCapture(stream, &graph) != cudaSuccess || !graph) {
    cudaGetLastError();
    return DSB_E_CUDA;
  }
  cudaGraphExec_t ge = static_cast<cudaGraphExec_t>(*exec);
  bool fresh = ge == nullptr;
  if (!fresh) {
    cudaGraphExecUpdateResultInfo info{};
    if (cudaGraphExecUpdate(ge, graph, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(ge);
      ge = nullptr;
      fresh = true;
    }
  }
  if (fresh && cudaGraphInstantiate(&ge, graph, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(graph);
    *exec = nullptr;
    return DSB_E_CUDA;
  }
  cudaGraphDestroy(graph);
  *exec = ge;
  return cudaGraphLaunch(ge, stream) == cudaSuccess ? DSB_OK : DSB_E_CUDA;
}

int dsb_graph_abort(cudaStream_t stream) {
  // ends a capture whose host side failed part-way; nothing is launched
  if (!stream) return DSB_E_ARG;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(stream, &graph);
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();
  return e == cudaSuccess ? DSB_OK : DSB_E_CUDA;
}

int dsb_graph_destroy(void* exec) {
  if (!exec) return DSB_OK;
  return cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(exec)) == cudaSuccess ? DSB_OK
                                                                                 : DSB_E_CUDA;
}

}  // extern "C"
