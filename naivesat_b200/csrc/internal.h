// internal.h -- library-internal entry points shared between translation units.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "nsat.h"

namespace nsat {

// Device ordinal a context is bound to.
int ctx_device(const nsat_ctx* ctx);

// nsat_qsat_solve with the last-CTA scratch area supplied by the caller
// instead of the context's cudaMalloc'd buffer; fails with NSAT_EUNSUPPORTED
// when a launch would need more than scratch_bytes.
int qsat_solve_with_scratch(nsat_ctx* ctx, nsat_circuit* c, const uint8_t* quants,
                            const nsat_qsat_opts* opts, nsat_qsat_result* res,
                            unsigned char* scratch, size_t scratch_bytes);

}  // namespace nsat
