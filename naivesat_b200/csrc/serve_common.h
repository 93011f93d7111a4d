// serve_common.h -- records shared by the serving host code and the LOP3
// bytecode interpreter kernel (serve_kernels.cu).
#pragma once
#include <stdint.h>
#include <vector_types.h>

// Geometry of the interpreter: each lane evaluates SRV_WORDS 32-bit words
// per program pass (SRV_WORDS * 1024 assignments per warp), and a tile of
// 2^SRV_TILE_BITS assignments takes 32 / SRV_WORDS passes.  A slot of a warp
// is SRV_SLOT_BYTES of shared memory laid out [lane][word].
#ifndef SRV_WORDS
#define SRV_WORDS 4
#endif
#ifndef SRV_GROUP
#define SRV_GROUP 4               // instructions issued together (mutually independent)
#endif
#define SRV_LOG_WORDS (SRV_WORDS == 4 ? 2 : 1)
#define SRV_SLOT_BYTES (32 * SRV_WORDS * 4)
#define SRV_MAX_SLOTS 384          // slots per warp (384 x 512 B = 192 KB of shared memory)
#define SRV_TILE_BITS 15           // assignments per warp tile
#define SRV_MAX_NB 48              // enumeration bits a serving job may have

// One instruction: slot[d] = LUT(slot[a], slot[b], slot[c]), 16 bytes:
//   ab = a | b << 16, cd = c | d << 16   (slot indices)
//   tlo, thi: the truth table tt (bit x<<2 | y<<1 | z is the value for
//   a=x, b=y, c=z) spread so that bit k of tt is the sign bit of byte k of
//   the 8-byte pair {thi, tlo}; the kernel expands mask k (all ones or all
//   zeros) with one byte permute that replicates that sign bit.
// Programs are sequences of groups of SRV_GROUP instructions none of which
// reads another's result.
struct SrvIns {
    uint32_t ab, cd, tlo, thi;
};
static_assert(sizeof(SrvIns) == 16, "SrvIns layout");

enum { SRV_SAT = 0, SRV_QSAT = 1, SRV_TABLE = 2 };

// Epoch header read by the kernel (so one captured graph serves every epoch).
// Jobs [0, n_narrow) run in the launch sized for SRV_NARROW_SLOTS slots per
// warp, jobs [n_narrow, njobs) in the launch sized for the epoch's widest.
struct SrvEpoch {
    uint32_t njobs;
    uint32_t n_narrow;
    uint32_t hi_mul;        // 65536 and SRV_SLOT_BYTES, read at run time so the
    uint32_t slot_bytes;    // kernel's slot decode stays multiply-adds
    uint32_t pad[60];
};
#define SRV_NARROW_SLOTS 48

// Device job record; 256 bytes.  Static fields are written at admission,
// the slice fields every epoch, the result fields by the kernels.
typedef unsigned long long srv_u64;   // the device atomics' 64-bit type

struct SrvJob {
    // static
    const SrvIns* prog;          // ngroups * SRV_GROUP instructions
    const void* unused0;
    const uint16_t* outs;        // output slots (bit 15 = negated), nout of them
    srv_u64* table;             // TABLE: 2^np u64 entries (next|STOP<<n | 1<<32)
    uint32_t ngroups;
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
    srv_u64 reserved[10];
};

static_assert(sizeof(SrvJob) == 256, "SrvJob layout");
