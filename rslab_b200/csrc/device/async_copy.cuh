// cp.async global -> shared copies with zero fill, and 16-byte vector loads
// of short shared-memory rows; used by the factor and solve kernels.
#pragma once

#include <cstdint>
#include <cstring>

#include "tcgen05.cuh"

namespace rsd {

// Copy BYTES (4, 8 or 16) from src to dst asynchronously; `valid` false
// writes zeros and reads nothing (src must still be a valid address).
template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES),
               "r"(valid ? BYTES : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// v[c] = p[c], c < NR, with 16-byte shared-memory loads when the row allows
// (p 16-byte aligned).
template <typename T, int NR>
__device__ __forceinline__ void lds_row(const T* p, T (&v)[NR]) {
  constexpr int B = (int)sizeof(T) * NR;
  if constexpr (B % 16 == 0) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    uint4 w[B / 16];
#pragma unroll
    for (int k = 0; k < B / 16; ++k) w[k] = q[k];
    memcpy(&v[0], &w[0], B);
  } else {
#pragma unroll
    for (int c = 0; c < NR; ++c) v[c] = p[c];
  }
}

}  // namespace rsd
