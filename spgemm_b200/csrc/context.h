// What a spgemm_handle_t points to: the engine and the batch plan that
// runs on it.
#pragma once

#include "batch.h"
#include "engine.h"

struct spgemm_context {
  sg::Engine eng;
  sg::Batch batch;
  sg::DevBuf coo_scratch, coo_scan;  // spgemm_coo_to_cm workspace
  // host-buffer entry points: C is copied back in pieces of about
  // copy_chunk bytes on copy_stream, each after the event that marks its
  // rows computed
  static constexpr int MAX_PIECES = 16;
  long long copy_chunk = 64ll << 20;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t piece_done[MAX_PIECES] = {};

  ~spgemm_context() {
    coo_scratch.release();
    coo_scan.release();
    for (cudaEvent_t& e : piece_done)
      if (e) cudaEventDestroy(e);
    if (copy_stream) cudaStreamDestroy(copy_stream);
  }
};
