/* Host-C++ shim that lets the reference's CUDA C kernel sources compile with
 * g++ so they can be executed on the CPU as a checker (oracle/_ref).
 *
 * TEST INFRASTRUCTURE ONLY: nothing under oracle/ is part of the product.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it.
 *
 * Mapping:
 *   __device__, __global__            -> nothing (plain host functions)
 *   __forceinline__                   -> inline
 *   __constant__                      -> thread_local (each OpenMP thread, or a
 *                                        per-CZ parameter set, writes its own copy)
 *   threadIdx/blockIdx/blockDim       -> thread_local structs; the wrapper sets
 *                                        blockDim.x = 1, blockIdx.x = 0,
 *                                        threadIdx.x = unit index before each call
 *   atomicCAS on 64-bit words         -> __atomic_compare_exchange_n (seq_cst)
 *   __double_as_longlong and inverse  -> memcpy bit casts
 * The sources themselves are read in place from the reference checkout and are
 * never copied into this repository.
 */
#pragma once
#include <cmath>
#include <cstring>
#include <cstdint>
#include <algorithm>

using std::max;
using std::min;

#define __device__
#define __global__
#define __forceinline__ inline
#define __constant__ thread_local

struct icf_shim_dim3 { unsigned int x, y, z; };
static thread_local icf_shim_dim3 threadIdx = {0u, 0u, 0u};
static thread_local icf_shim_dim3 blockIdx = {0u, 0u, 0u};
static thread_local icf_shim_dim3 blockDim = {1u, 1u, 1u};

static inline unsigned long long atomicCAS(unsigned long long *addr,
                                           unsigned long long compare,
                                           unsigned long long val) {
  /* On success `compare` keeps the old value; on failure it receives the
   * current value. Either way it is what CUDA's atomicCAS returns. */
  __atomic_compare_exchange_n(addr, &compare, val, false, __ATOMIC_SEQ_CST,
                              __ATOMIC_SEQ_CST);
  return compare;
}

static inline long long __double_as_longlong(double d) {
  long long r;
  std::memcpy(&r, &d, sizeof r);
  return r;
}

static inline double __longlong_as_double(long long l) {
  double r;
  std::memcpy(&r, &l, sizeof r);
  return r;
}

static inline void icf_shim_set_thread(int idx) {
  threadIdx.x = (unsigned int)idx;
  blockIdx.x = 0u;
  blockDim.x = 1u;
}
