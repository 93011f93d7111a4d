// serve_common.h -- records shared by the serving host code and the LOP3
// bytecode interpreter kernel (serve_kernels.cu).
#pragma once
#include <stdint.h>
#include <vector_types.h>

// Geometry of the interpreter.  A shape fixes the words each lane evaluates
// per program pass (W: W * 1024 assignments per warp), the size of the groups
// of mutually independent instructions the program is scheduled into (G: a
// group's operands are all loaded before any of its results is stored), and
// how a LUT with a run-time truth table is evaluated: a 7-lop3 mux tree over
// masks expanded from the table, or a jump on the warp-uniform table to one
// lop3 with that table as its immediate.  A tile of 2^SRV_TILE_BITS
// assignments takes 32 / W passes; a slot of a warp is 32 * W * 4 bytes of
// shared memory laid out [lane][word].  The server picks one shape (option,
// tuned and persisted per GPU, or the default) and builds its programs with
// that shape's group size.
struct SrvShape {
    uint32_t words;      // W: 2 or 4
    uint32_t group;      // G: 1, 2 or 4
    uint32_t dispatch;   // 0: mux tree, 1: jump on the truth table
};
#define SRV_NSHAPES 6
static const SrvShape kSrvShapes[SRV_NSHAPES] = {
    {4, 4, 0}, {4, 1, 1}, {4, 2, 1}, {4, 4, 1}, {2, 1, 1}, {2, 2, 1},
};
#define SRV_MAX_GROUP 4
#define SRV_MAX_SLOTS 384          // slots per warp (384 x 512 B = 192 KB of shared memory at W = 4)
#define SRV_TILE_BITS 15           // assignments per warp tile
#define SRV_MAX_NB 48              // enumeration bits a serving job may have
inline uint32_t srv_slot_bytes(uint32_t shape) { return 32u * kSrvShapes[shape].words * 4u; }

// One instruction: slot[d] = LUT(slot[a], slot[b], slot[c]), 16 bytes:
//   ab = a | b << 16, cd = c | d << 16   (slot indices)
//   tlo, thi: the truth table tt (bit x<<2 | y<<1 | z is the value for
//   a=x, b=y, c=z) spread so that bit k of tt is the sign bit of byte k of
//   the 8-byte pair {thi, tlo}; the kernel expands mask k (all ones or all
//   zeros) with one byte permute that replicates that sign bit.
// Programs are sequences of groups of G instructions (the shape's group
// size) none of which reads another's result.
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
    uint32_t hi_mul;        // 65536 and the shape's slot bytes, read at run time so
    uint32_t slot_bytes;    // the kernel's slot decode stays multiply-adds
    uint32_t pad[60];
};
#define SRV_NARROW_SLOTS 48

// A job's search cursor and results, in device memory from admission to
// release (one entry of the server's state array): the kernel claims tiles
// by advancing `claim` and accumulates the results here, so they persist
// across epochs without the host.  64 bytes.
typedef unsigned long long srv_u64;   // the device atomics' 64-bit type

struct SrvState {
    srv_u64 claim;              // next tile to hand out; only grows, never past the epoch's limit
    srv_u64 count;              // SAT: satisfying assignments in the tiles evaluated so far
    srv_u64 min_idx;            // SAT: lowest witness so far; QSAT (m < tile bits): lowest decisive unit
    uint32_t any;                // TABLE: some state has STOP
    uint32_t pad;
    srv_u64 reserved[4];
};
static_assert(sizeof(SrvState) == 64, "SrvState layout");

// Device job record of one epoch; 256 bytes.  Static fields are written at
// admission, the slice fields every epoch.
#define SRV_JOB_FIND_ALL 1u      // flags: a SAT job that counts every solution (no early stop)

struct SrvJob {
    // static
    const SrvIns* prog;          // ngroups * G instructions (G: the server shape's group size)
    SrvState* st;                // the job's persistent cursor and results
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
    // per epoch: tiles below tile_end are handed out first; once a warp finds
    // every job's slice used up it may go on to tile_hard (the next slice,
    // without a host round trip), unless the job has already been decided
    srv_u64 tile_begin, tile_end;   // the planned slice
    srv_u64 tile_hard;               // roll-over limit (== tile_end: none)
    uint32_t val_off;                // QSAT: offset of the slice's tile values in the epoch buffer
    uint32_t flags;                  // SRV_JOB_FIND_ALL
    srv_u64 reserved[13];
};

static_assert(sizeof(SrvJob) == 256, "SrvJob layout");
