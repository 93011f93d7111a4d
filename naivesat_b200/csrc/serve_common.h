// serve_common.h -- records shared by the serving host code and the LOP3
// bytecode interpreter kernel (serve_kernels.cu).
#pragma once
#include <stdint.h>

// One instruction of a circuit program: a 3-input LUT over slots
//   slot[d] = lut(slot[a], slot[b], slot[c]) with truth table tt
// (bit (x<<2 | y<<1 | z) of tt is the value for a=x, b=y, c=z).
// Packed as a | b<<12 | c<<24 | d<<36 | tt<<48.
#define SRV_SLOT_BITS 12
#define SRV_MAX_SLOTS 256          // shared-memory slots per lane the interpreter supports
#define SRV_TILE_BITS 15           // assignments per warp tile (32 iterations x 1024)
#define SRV_MAX_NB 48              // enumeration bits a serving job may have

#define SRV_WARPS_PER_CTA 4

enum { SRV_SAT = 0, SRV_QSAT = 1, SRV_TABLE = 2 };

// Epoch header read by the kernel (so one captured graph serves every epoch).
struct SrvEpoch {
    uint32_t njobs;
    uint32_t pad[63];
};

// Device job record; 256 bytes.  Static fields are written at admission,
// the slice fields every epoch, the result fields by the kernels.
typedef unsigned long long srv_u64;   // the device atomics' 64-bit type

struct SrvJob {
    // static
    const srv_u64* prog;        // instructions
    const uint16_t* outs;        // output slots (bit 15 = negated), nout of them
    srv_u64* table;             // TABLE: 2^np u64 entries (next|STOP<<n | 1<<32)
    uint32_t ninstr;
    uint32_t nslots;
    uint32_t kind;               // SRV_SAT / SRV_QSAT / SRV_TABLE
    uint32_t nb;                 // enumeration bits (padding included)
    uint32_t nout;
    uint32_t m;                  // QSAT: unit level (inner bits below the first block)
    uint32_t q0all;              // QSAT: first quantifier is All
    uint32_t n;                  // TABLE: state bits
    srv_u64 allbits;            // QSAT: enumeration bit j has quantifier All
    int8_t in_slot[SRV_MAX_NB];  // enumeration bit -> input slot (-1: dummy)
    // per epoch
    srv_u64 tile_begin, tile_end;   // slice of tiles to evaluate
    uint32_t val_off;                // QSAT: offset of this slice's tile values in the epoch buffer
    uint32_t pad0;
    // claimed by the kernel
    srv_u64 claim;              // next tile (starts at tile_begin)
    // results
    srv_u64 count;              // SAT: satisfying assignments in evaluated tiles
    srv_u64 min_idx;            // SAT: lowest witness; QSAT (m < tile bits): lowest decisive unit
    uint32_t any;                // TABLE: some state has STOP
    uint32_t pad1;
    srv_u64 reserved[11];
};

static_assert(sizeof(SrvJob) == 256, "SrvJob layout");
