// static_kernels.h -- launchers of the nvcc-compiled (circuit independent) kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// Per-solve state of the doubling rounds, in device memory.
typedef struct {
    unsigned long long best[72];   // best[r]: lowest resolved start after round r (~0 = none)
    uint32_t final_round;          // round whose answer ended the loop early (0 = none)
    uint32_t pad;
} NsatJoinState;

int nsat_launch_join_round(int fmt, const void* src, void* dst, uint64_t N, uint32_t n,
                           uint32_t u, uint32_t r, uint32_t mode, NsatJoinState* st,
                           int sm_count, cudaStream_t stream);

// random 8-byte gathers from a table of 2^logn u64 (items reads); out holds
// blocks * 256 words
int nsat_launch_gather_probe(const uint64_t* table, uint32_t logn, uint64_t items, uint64_t* out, int blocks,
                             cudaStream_t stream);
int nsat_launch_lop3_probe(uint32_t* out, int blocks, int iters, uint64_t* clk,
                           cudaStream_t stream);

#ifdef __cplusplus
}
#endif
