// ws_bounds.cuh -- the bounds-checked build of the library (compiled with -DWS_BOUNDS_CHECK into
// libwarpsym_bc.so).
//
// The hot kernels test their shared- and global-memory indices against the extents of the
// buffers they address.  In the checked build an index out of range is recorded -- the first
// one per device module, as (check site << 32) | index -- and its access is skipped, so a
// wrong index never faults or traps; `ws_bounds_status` reads the record back.  In the normal
// build every check is the constant `true` and compiles away.  The checked build stands in for
// a memory checker: tests run small shapes through it and require the recorded word to stay
// zero and every result to equal the normal build's bit for bit.
#pragma once

#include <cstdint>

#ifndef WS_HD
#define WS_HD __host__ __device__ __forceinline__
#endif

namespace ws {

// Check sites (the upper half of a recorded violation).
enum BcSite : uint32_t {
  BC_NONE = 0,
  BC_FIT_TAPE_LEN = 1,   // fitness: a program's tape longer than its tape capacity
  BC_FIT_X = 2,          // fitness: a variable operand or accumulator load outside the X tile
  BC_FIT_SLOT = 3,       // fitness: a spill slot outside the warp's slots
  BC_SMALL_X = 5,        // small-data-set fitness: operand outside the staged rows
  BC_SMALL_SLOT = 6,     // small-data-set fitness: spill slot outside the lane's slots
  BC_SMALL_TAPE_LEN = 7,
  BC_COMPILE_NODES = 8,  // compiler: node count beyond its node array
  BC_ADJ_PARSE = 9,      // adjoint parse (both modes): operators, constant leaves, variables or
                         // scalars beyond the block's arrays, a variable index beyond V
  BC_SELFTEST = 99,      // ws_debug_bounds_selftest
};

// Host side: the word of host-compiled checks, and the registry of the device modules' words.
void bc_host_fail(uint32_t site, uint32_t idx);
using BcReader = unsigned long long (*)(bool reset);
int bc_register(BcReader reader);

#ifdef WS_BOUNDS_CHECK
// This device module's first violation (each .cu file is its own module).
static __device__ unsigned long long g_bc_word = 0ull;

WS_HD void bc_fail(uint32_t site, uint32_t idx) {
#ifdef __CUDA_ARCH__
  atomicCAS(&g_bc_word, 0ull, ((unsigned long long)site << 32) | (unsigned long long)idx);
#else
  bc_host_fail(site, idx);
#endif
}

namespace {
// Reads (and optionally clears) this module's word; registered once per module at load time.
unsigned long long bc_read_module(bool reset) {
  unsigned long long v = 0ull;
  if (cudaMemcpyFromSymbol(&v, g_bc_word, sizeof(v)) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0ull;
  }
  if (reset && v != 0ull) {
    const unsigned long long z = 0ull;
    (void)cudaMemcpyToSymbol(g_bc_word, &z, sizeof(z));
  }
  return v;
}
const int bc_registered_ = bc_register(&bc_read_module);
}  // namespace

// True when the condition holds; otherwise records (site, idx) and yields false, so that
// `if (WS_BC(i < n, SITE, i)) a[i] = ...;` skips the access.
#define WS_BC(cond, site, idx) \
  ((cond) ? true : (::ws::bc_fail((site), (uint32_t)(idx)), false))
#else
#define WS_BC(cond, site, idx) true
#endif

}  // namespace ws
