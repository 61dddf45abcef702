// CPU emulation shim for CUDA kernels: blocks run one after another, each thread of a block is a std::thread.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <barrier>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <thread>
#include <type_traits>
#include <vector>

#undef __shared__
#define __shared__ static
#undef __launch_bounds__
#define __launch_bounds__(...)

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern dim3 blockDim;
extern dim3 gridDim;

namespace emu {
extern std::barrier<>* blockBar;
extern std::vector<std::unique_ptr<std::barrier<>>> warpBar;
extern uint64_t xbuf[1024];
inline int lane() { return threadIdx.x & 31; }
inline int wid() { return threadIdx.x >> 5; }
inline void wsync() { warpBar[wid()]->arrive_and_wait(); }
template <class T> inline uint64_t bits(T v) { uint64_t b = 0; std::memcpy(&b, &v, sizeof(T)); return b; }
template <class T> inline T unbits(uint64_t b) { T v; std::memcpy(&v, &b, sizeof(T)); return v; }
template <class T> inline T shfl(T v, int src, bool valid)
{
	xbuf[threadIdx.x] = bits(v);
	wsync();
	const T r = valid ? unbits<T>(xbuf[wid() * 32 + src]) : v;
	wsync();
	return r;
}
}  // namespace emu

inline void __syncthreads() { emu::blockBar->arrive_and_wait(); }
inline void __syncwarp(unsigned = 0xffffffffu) { emu::wsync(); }
inline void __threadfence_block() {}
template <class T> inline T __shfl_sync(unsigned, T v, int src) { return emu::shfl(v, src & 31, true); }
template <class T> inline T __shfl_up_sync(unsigned, T v, unsigned d)
{
	const int s = emu::lane() - static_cast<int>(d);
	return emu::shfl(v, s < 0 ? 0 : s, s >= 0);
}
template <class T> inline T __shfl_down_sync(unsigned, T v, unsigned d)
{
	const int s = emu::lane() + static_cast<int>(d);
	return emu::shfl(v, s > 31 ? 31 : s, s <= 31);
}
template <class T> inline T __shfl_xor_sync(unsigned, T v, int m) { return emu::shfl(v, emu::lane() ^ m, true); }
inline unsigned __ballot_sync(unsigned, int pred)
{
	emu::xbuf[threadIdx.x] = pred ? 1u : 0u;
	emu::wsync();
	unsigned b = 0;
	for (int l = 0; l < 32; ++l) { if (emu::xbuf[emu::wid() * 32 + l]) { b |= 1u << l; } }
	emu::wsync();
	return b;
}
template <class T> inline unsigned __match_any_sync(unsigned, T v)
{
	emu::xbuf[threadIdx.x] = emu::bits(v);
	emu::wsync();
	unsigned b = 0;
	for (int l = 0; l < 32; ++l) { if (emu::xbuf[emu::wid() * 32 + l] == emu::bits(v)) { b |= 1u << l; } }
	emu::wsync();
	return b;
}
inline int __any_sync(unsigned m, int pred) { return __ballot_sync(m, pred) != 0; }
inline int __all_sync(unsigned m, int pred) { return __ballot_sync(m, !pred) == 0; }
inline int __popc(unsigned v) { return __builtin_popcount(v); }
inline size_t __cvta_generic_to_shared(const void* p) { return reinterpret_cast<uintptr_t>(p); }
inline unsigned __vimax3_u32(unsigned a, unsigned b, unsigned c) { return std::max(a, std::max(b, c)); }
inline int __ffs(int v) { return __builtin_ffs(v); }
inline int __clz(int v) { return v == 0 ? 32 : __builtin_clz(static_cast<unsigned>(v)); }
template <class T> inline T __ldg(const T* p) { return *p; }
template <class T> inline T __ldcg(const T* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
template <class T> inline T __ldca(const T* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline double __dadd_rn(double a, double b) { volatile double r = a + b; return r; }
inline double __dmul_rn(double a, double b) { volatile double r = a * b; return r; }
template <class T> inline T atomicAdd(T* p, T v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
inline unsigned atomicAdd(unsigned* p, unsigned v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
inline unsigned atomicExch(unsigned* p, unsigned v) { return __atomic_exchange_n(p, v, __ATOMIC_RELAXED); }
inline unsigned atomicCAS(unsigned* p, unsigned cmp, unsigned v)
{
	__atomic_compare_exchange_n(p, &cmp, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
	return cmp;
}
inline unsigned atomicOr(unsigned* p, unsigned v) { return __atomic_fetch_or(p, v, __ATOMIC_RELAXED); }
inline unsigned atomicMin(unsigned* p, unsigned v)
{
	unsigned old = __atomic_load_n(p, __ATOMIC_RELAXED);
	while (v < old && !__atomic_compare_exchange_n(p, &old, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
	return old;
}
inline unsigned atomicMax(unsigned* p, unsigned v)
{
	unsigned old = __atomic_load_n(p, __ATOMIC_RELAXED);
	while (v > old && !__atomic_compare_exchange_n(p, &old, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
	return old;
}
template <class A, class B> inline auto min(A a, B b) { using C = std::common_type_t<A, B>; return static_cast<C>(a) < static_cast<C>(b) ? static_cast<C>(a) : static_cast<C>(b); }
template <class A, class B> inline auto max(A a, B b) { using C = std::common_type_t<A, B>; return static_cast<C>(a) > static_cast<C>(b) ? static_cast<C>(a) : static_cast<C>(b); }

namespace emu {
template <class F, class... Args>
void Launch(dim3 grid, dim3 block, F kernel, Args... args)
{
	gridDim = grid;
	blockDim = block;
	const int n = block.x;
	for (unsigned b = 0; b < grid.x * grid.y * grid.z; ++b) {
		std::barrier<> bb(n);
		blockBar = &bb;
		warpBar.clear();
		for (int w = 0; w < (n + 31) / 32; ++w) { warpBar.emplace_back(new std::barrier<>(std::min(32, n - 32 * w))); }
		std::vector<std::thread> th;
		for (int t = 0; t < n; ++t) {
			th.emplace_back([=]() {
				threadIdx = make_uint3(t, 0, 0);
				blockIdx = make_uint3(b % grid.x, (b / grid.x) % grid.y, b / (grid.x * grid.y));
				kernel(args...);
				// an exited thread no longer takes part in the barriers (as on the GPU)
				warpBar[t >> 5]->arrive_and_drop();
				blockBar->arrive_and_drop();
			});
		}
		for (auto& x : th) { x.join(); }
	}
}
}  // namespace emu
