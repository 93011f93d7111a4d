// serve_kernels.h -- launchers of the serving engine's interpreter kernel.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "serve_common.h"

extern "C" {
// grid one-warp CTAs of the interpreter of shape `shape` (kSrvShapes), each
// with max_slots * srv_slot_bytes(shape) of shared memory, serving the
// epoch's narrow (cls 0) or wide (cls 1) jobs
int nsat_launch_serve_epoch(const SrvEpoch* hdr, SrvJob* jobs, uint32_t max_slots, uint8_t* vals, int grid,
                            uint32_t cls, uint32_t shape, cudaStream_t stream);
// raises that kernel's shared-memory limit for max_slots and reports CTAs per SM
int nsat_serve_occupancy(uint32_t max_slots, uint32_t shape, int* ctas_per_sm);
}
