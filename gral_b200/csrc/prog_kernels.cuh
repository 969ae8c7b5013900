// prog_kernels.cuh -- host-side launchers of the solver kernels (implemented in prog_gs.cu and
// prog_kernels.cu).  Every launcher enqueues on the given stream and returns immediately.
#pragma once

#include <cuda_runtime.h>

#include "prog_common.cuh"

namespace gral {

// Boundary-condition event lists (PrognosticFlowfield.cs:595-696): for the W/E pass one list per
// row j of the columns i (ascending) that copy inflow; for the S/N pass one list per column i.
// Entry = index | (west_or_south << 16) | (east_or_north << 17).
struct BcLists {
    const int *we_ptr, *we_ev;   // we_ptr[j]..we_ptr[j+1]
    const int *sn_ptr, *sn_ev;   // sn_ptr[i]..sn_ptr[i+1]
};

// Full-height staging copies of the host fields of one situation: [NII+2][NJJ+2][NKK+2].
struct Staging {
    float *uk, *vk, *wk, *turb, *tdiss;
    size_t stride;   // floats between situations
};

int gs_num_variants();
int gs_block_threads(bool il, int variant);
cudaError_t gs_prepare(bool il, int ks, int model);
cudaError_t gs_occupancy(bool il, int kind, int model, int simd, int ks, int variant, int *blocks_per_sm);
// one Gauss-Seidel phase (kind = PH_PRESSURE, PH_U, PH_V, PH_W or PH_TKE) of the loaded model
void launch_gs(int kind, const KArgs &a, const SweepGeom &g, int grid, cudaStream_t st);
// strip schedule of the slab family's model-1 sweeps (kind = PH_PRESSURE, PH_U, PH_V, PH_W): a
// block per strip of strip_rows(variant) sweep rows, hand-offs inside a strip in shared memory
int strip_num_variants();
int strip_rows(int variant);
int strip_block_threads(int variant);
cudaError_t strip_occupancy(int kind, int variant, int *blocks_per_sm);
void launch_strip(int kind, const KArgs &a, const SweepGeom &g, int variant, int grid, cudaStream_t st);
// pressure, velocity correction, averages and model-1 U in one launch on the strip schedule:
// claims (per situation) alternate pressure strips and U strips, 2*strips+1 of them
cudaError_t fused_strip_occupancy(int *blocks_per_sm);
int fused_strip_claims(const SweepGeom &gp);
void launch_fused_strip(const KArgs &a, const FusedGeom &fg, int grid, cudaStream_t st);
// pressure + velocity correction + averages + model-1 U in one wavefront launch (slab family)
cudaError_t fused_occupancy(int *blocks_per_sm);
void launch_fused_pvau(const KArgs &a, const FusedGeom &fg, int grid, cudaStream_t st);

void launch_bc(const KArgs &a, const BcLists &bc, cudaStream_t st);
void launch_velcorr(const KArgs &a, cudaStream_t st);
void launch_average(const KArgs &a, cudaStream_t st);
void launch_bookkeeping(const KArgs &a, cudaStream_t st);

// set-up and tear-down of a batch (PrognosticFlowfield.cs:295-329, 410-579); varw = per
// (situation, column) vertical-variance term of the TURB initialisation (model != 1), or null
void launch_setup(const KArgs &a, const Staging &sg, int model, const float *varw, const float *z0_init,
                  cudaStream_t st);
void launch_gather(const KArgs &a, const Staging &sg, int model, cudaStream_t st);
void launch_scatter(const KArgs &a, const Staging &sg, int model, cudaStream_t st);
// for every situation with quantisation: whether ConvToInt(x*Frund)/Frund may use the reciprocal
// (SitDev::rcp_ok); bad = n ints of zeroed scratch
void launch_rcp_check(const KArgs &a, int *bad, cudaStream_t st);
// post-checks (PrognosticFlowfield.cs:1193-1243); counts[s*4 + 0..3] = UK, VK, WK, non-finite
void launch_postcheck(const KArgs &a, int *counts, cudaStream_t st);

// DiagnosticFlowfield.Calculate (DiagnosticFlowfield.cs:24-436) and the final vertical velocity of
// the columns outside the prognostic sub-domains (MicroscaleFlat.cs:389-462), on full-height
// fields: `a` describes them as a slab layout with KS = NKK+2 and a.dpm the diagnostic DPM.
cudaError_t diag_prepare(int ks);
cudaError_t diag_occupancy(int ks, int *blocks_per_sm);
void launch_diag_dtime(const KArgs &a, int kadvmax, float *dtime, cudaStream_t st);
void launch_diag_pressure(const KArgs &a, const SweepGeom &g, const DiagTabs &t, int grid, cudaStream_t st);
void launch_diag_velcorr(const KArgs &a, const DiagTabs &t, cudaStream_t st);
void launch_diag_wfinal(const KArgs &a, const DiagTabs &t, cudaStream_t st);

}  // namespace gral
