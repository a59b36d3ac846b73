// Host side of the output path shared by the context entry points
// (output.cu) and the member engine (engine.cu).
#pragma once

#include "context.cuh"

namespace nimbus_host
{

constexpr int kHistoryFields = 9;

// Enqueues one history frame on st: the cell-centre launch for the selected
// velocity components into staging (3 * cells floats, device), then the
// device-to-host copies into host_image: one for the staged velocities, one
// per selected scalar field.
// src: the nine device fields in NIMBUS_HISTORY_* order; ground: device
// [nx][ny] lower-face w or null.  Arguments are already validated.
nimbus_status enqueue_history(nimbus_cuda_context* ctx, cudaStream_t st, const float* const src[kHistoryFields],
                              unsigned fields, const double* ground, int nx, int ny, int nz, float* staging,
                              float* host_image);

}  // namespace nimbus_host
