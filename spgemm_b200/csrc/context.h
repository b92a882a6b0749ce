// What a spgemm_handle_t points to: the engine and the batch plan that
// runs on it.
#pragma once

#include "batch.h"
#include "engine.h"

struct spgemm_context {
  sg::Engine eng;
  sg::Batch batch;
  sg::DevBuf coo_scratch, coo_scan;  // spgemm_coo_to_cm workspace

  ~spgemm_context() {
    coo_scratch.release();
    coo_scan.release();
  }
};
