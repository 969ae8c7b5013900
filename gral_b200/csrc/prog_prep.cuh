// prog_prep.cuh -- the flat-terrain set-up of one situation on the device (prog_prep.cu), shared
// by gral_prog_flat_init and the load that builds the initial fields on the device.
#pragma once

#include <cuda_runtime.h>

#include "gral_prog.h"

struct gral_ctx;

namespace gral {

// Checks of a flat-terrain set-up request (grid against the context's capacity, HOKART, met
// profile, near-wall options); GRAL_OK or the error code with the context's error text set.
int flat_check(gral_ctx *ctx, const gral_flat_grid *g, const float *hokart, const gral_met *met, bool have_advdom);

// MicroscaleFlat.cs:29-357 for one situation on ctx's stream: the host tables (profile per
// Obukhov length, wall-damping factors) into the context's set-up buffers, then zeroed device
// fields du, dv, dw (flat [NII+2][NJJ+2][NKK+2]) filled by the column and near-wall kernels.
// d_cutk, d_adv: device CUTK and ADVDOM (ADVDOM read for near_wall 1 only).  KKART, AHK and the
// KADVMAX reduction go to the context's set-up buffers; *d_kadv receives the device address of
// that reduction (max KKART of the building columns, at least 1).  With `timed`, ev[0] and ev[1]
// of the context bracket the kernels.  Asynchronous: no synchronisation.
int flat_fill(gral_ctx *ctx, const gral_flat_grid *g, const float *d_cutk, const uint8_t *d_adv, const float *dzk,
              const float *hokart, const gral_met *met, float *du, float *dv, float *dw, int **d_kadv, bool timed);

}  // namespace gral
