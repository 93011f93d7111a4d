// internal.h -- library-internal entry points shared between translation units.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <functional>
#include <string>

#include "nsat.h"

#include <cuda_runtime.h>

#include "circuit.h"

namespace nsat {

// Device ordinal a context is bound to, its stream and SM count.
int ctx_device(const nsat_ctx* ctx);
cudaStream_t ctx_stream(const nsat_ctx* ctx);
int ctx_sm_count(const nsat_ctx* ctx);
bool ctx_no_optimize(const nsat_ctx* ctx);
// The options a context was created with.
nsat_opts ctx_opts(const nsat_ctx* ctx);
// Records a failure on the context (nsat_last_error) and returns `code`.
int ctx_fail(nsat_ctx* ctx, int code, const std::string& msg);
// Per-call device buffers (tables, partition images, work areas) from the
// context's stream-ordered pool: allocated and freed in order on the
// context's stream, and kept for reuse by the next call (up to a release
// threshold), so a repeated solve pays no cudaMalloc/cudaFree.  A buffer
// used on another stream needs the context's stream synchronised after the
// allocation.
cudaError_t ctx_alloc(nsat_ctx* ctx, void** p, size_t bytes);
void ctx_free(nsat_ctx* ctx, void* p);
// Returns the pool's unused memory to the device (after the context's
// stream finishes), for a caller about to size a buffer by free memory.
void ctx_trim(nsat_ctx* ctx);

// Circuit from the C ABI's flat description (not validated).
Circuit circuit_from_desc(const nsat_circuit_desc* d);

// nsat_qsat_solve with the last-CTA scratch area supplied by the caller
// instead of the context's cudaMalloc'd buffer; fails with NSAT_EUNSUPPORTED
// when a launch would need more than scratch_bytes.
int qsat_solve_with_scratch(nsat_ctx* ctx, nsat_circuit* c, const uint8_t* quants,
                            const nsat_qsat_opts* opts, nsat_qsat_result* res,
                            unsigned char* scratch, size_t scratch_bytes);

// The QSAT sub-problems under prefixes first .. first + count - 1 of
// prefix_bits fixed inputs, solved back to back through the launch ring when
// each is one launch (otherwise only count == 1 is accepted); on_block sees
// each result in prefix order and returns false to stop.
int qsat_solve_blocks(nsat_ctx* ctx, nsat_circuit* c, const uint8_t* quants, uint32_t prefix_bits,
                      uint64_t first, uint64_t count,
                      const std::function<bool(uint64_t, const nsat_qsat_result&)>& on_block);

// Next-state entries (next | STOP << n, u64) of states first_state ..
// first_state+count-1 (both multiples of 32) into device memory dev_out, on
// the context's stream (synchronous); any_stop reports a STOP among them.
int table_chunk_u64(nsat_ctx* ctx, nsat_circuit* c, uint64_t first_state, uint64_t count, uint64_t* dev_out,
                    uint32_t* any_stop, float* ms);

const Circuit& circuit_of(const nsat_circuit* c);

}  // namespace nsat
