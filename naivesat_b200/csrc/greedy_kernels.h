// greedy_kernels.h -- launchers of the partitioned greedysatostop kernels
// (greedy_kernels.cu).  All take a stream and return 0 or -4 (launch error).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

extern "C" {
// packed (bits-wide) entries -> u64 entries; count entries
int nsat_greedy_unpack(const uint64_t* packed, uint64_t count, uint32_t bits, uint64_t* out, int sms,
                       cudaStream_t st);
// u64 entries -> packed entries; count a multiple of 64
int nsat_greedy_pack(const uint64_t* in, uint64_t count, uint32_t bits, uint64_t* packed, int sms, cudaStream_t st);
// dest[i] = second[next - start2] where dest[i] has no STOP and its next lies in [start2, start2+count2)
int nsat_greedy_join(uint64_t* dest, uint64_t count, const uint64_t* second, uint64_t start2, uint64_t count2,
                     uint32_t n, int sms, cudaStream_t st);
// the same join reading `second` as packed (n+1)-bit entries
int nsat_greedy_join_packed(uint64_t* dest, uint64_t count, const uint64_t* second_packed, uint64_t start2,
                            uint64_t count2, uint32_t n, int sms, cudaStream_t st);
// atomicMin into *best of the unknown starts of [start, start+count) with STOP
int nsat_greedy_find(const uint64_t* dest, uint64_t start, uint64_t count, uint32_t n, uint32_t unknowns,
                     uint64_t* best, int sms, cudaStream_t st);
}
