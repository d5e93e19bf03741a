// Internal interface between the fused-step dispatcher (step_fused.cu) and the
// TMA pipeline (step_tma.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/warp_fdtd_b200.h"

namespace wfb {

// Shared-memory layout of the TMA pipeline for one tile shape.
struct TmaLayout {
    int ty, tz, stages;
    int hz, ez, mz;        // row lengths (elements) of the H, E and material boxes
    int off_e, off_m;      // byte offsets of the E and material boxes in a stage
    int stage_bytes;       // bytes per stage (128-byte aligned pieces)
    unsigned tx_bytes;     // bytes the three TMA loads of a stage deliver
    int off_stages, off_enew, off_coef, off_mtab, smem_bytes;
};

TmaLayout tma_layout(int ty, int tz, int stages, int mat);
bool tma_eligible(const fdtd_step_args &a);
int launch_tma(const fdtd_step_args &a, cudaStream_t stream);
bool fz_eligible(const fdtd_step_args &a);
void fz_defaults(fdtd_step_args &a);
int fz_occupancy(const fdtd_step_args &a, int *blocks_per_sm);
int launch_fz(const fdtd_step_args &a, cudaStream_t stream);

}  // namespace wfb
