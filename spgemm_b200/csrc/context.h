// What a spgemm_handle_t points to: the engine and the batch plan that
// runs on it.
#pragma once

#include "batch.h"
#include "engine.h"

struct spgemm_context {
  sg::Engine eng;
  sg::Batch batch;
};
