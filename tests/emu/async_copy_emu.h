// CPU stand-in for palmtracer-cpp_b200/csrc/async_copy.cuh: the copy happens at once (so every wait is already
// satisfied); a misaligned address aborts, as it would fault on the GPU.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace ptb {

inline void CpAsync8(void* smemDst, const void* gmemSrc)
{
	if ((reinterpret_cast<uintptr_t>(smemDst) | reinterpret_cast<uintptr_t>(gmemSrc)) & 7u) {
		fprintf(stderr, "CpAsync8: misaligned %p <- %p\n", smemDst, gmemSrc);
		abort();
	}
	std::memcpy(smemDst, gmemSrc, 8);
}
inline void CpAsyncCommit() {}
template <int N> inline void CpAsyncWait() {}

}  // namespace ptb
