// Asynchronous global-to-shared copies (cp.async, sm_80 and later): a lane's copy lands in shared memory without
// passing through registers, and commit groups let a warp keep several input rows in flight while it computes.
#pragma once

#include <cstdint>

namespace ptb {

// 8 bytes from global to shared memory; both addresses 8-byte aligned.
__device__ __forceinline__ void CpAsync8(void* smemDst, const void* gmemSrc)
{
	const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smemDst));
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmemSrc) : "memory");
}

// Closes the lane's current group of copies (an empty group is allowed).
__device__ __forceinline__ void CpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// Waits until at most N of the lane's groups are still in flight.
template <int N> __device__ __forceinline__ void CpAsyncWait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

}  // namespace ptb
