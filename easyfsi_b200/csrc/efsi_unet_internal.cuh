// Internal entry points of the U-Net used by the flexible PCG (efsi_fv.cu).
#pragma once

#include <cuda_runtime.h>

struct efsi_unet;

namespace efsi {

// Allocates the network's workspace for a level-0 volume (call before any
// stream capture of unet_run).
int unet_prepare(efsi_unet* U, int nx, int ny, int nz);

// One forward pass over a prepared volume: input [n][16] BF16; *out is set
// to the network's FP32 output [n][16] (channel 0 is the preconditioned
// residual).  Convolutions that give up on a wait set *error_word.  Launches
// only (no allocation, no synchronisation), so it can be captured.
int unet_run(efsi_unet* U, int nx, int ny, int nz, const void* input, int* error_word, const float** out,
             cudaStream_t s);

}  // namespace efsi
