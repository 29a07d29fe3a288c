// api_internal.h — host-side accessors shared between the library's
// translation units (not exported).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tsi.h"

struct TsiTapeView {
  const uint2 *code;
  uint32_t len, nregs, out_reg;
  int device;
  cudaStream_t stream;
};

// Device view of an uploaded tape.
tsi_status tsi_internal_tape_view(const tsi_tape *t, TsiTapeView *v);
// Sets the message tsi_last_error returns on this thread.
void tsi_internal_set_error(const char *msg);
// Context of a scene, and the most scenes one fused launch takes.
tsi_ctx *tsi_internal_scene_ctx(const tsi_scene *s);
uint32_t tsi_internal_max_scenes(const tsi_ctx *c);
