// Runs the detection kernel (DetectKernel of detect.cu) on a stack of frames on the CPU (each CUDA thread a host
// thread, shim.h). Every device array is a separate allocation, so AddressSanitizer reports any out-of-bounds access.
// Test harness only.
// Usage: emu_detect <in> <out>; in: int32 H, W, B, int64 threshold (2^-16 units), B * H * W uint16 pixels;
// out: uint32 ndom, nseed, overflow, B per-frame domain counts, B per-frame seed counts, P code bytes, P uint32 W1
// (as written: only domain pixels are defined), then the domain list and the seed list, each sorted.
#include "shim.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
dim3 blockDim;
dim3 gridDim;
namespace emu {
std::barrier<>* blockBar;
std::vector<std::unique_ptr<std::barrier<>>> warpBar;
uint64_t xbuf[1024];
}  // namespace emu

#include "detect_emu.inc"

#include <algorithm>
#include <cstdio>
#include <cstdlib>

namespace ptb {
void SetError(const std::string& m) { fprintf(stderr, "SetError %s\n", m.c_str()); }
bool CheckCuda(cudaError_t, const char*, const char*, int) { return true; }
void CountLaunch(uint64_t) {}

template <class T> static T* Alloc(size_t n, int fill)
{
	T* p = static_cast<T*>(malloc(std::max<size_t>(n, 1) * sizeof(T)));
	memset(p, fill, std::max<size_t>(n, 1) * sizeof(T));
	return p;
}
}  // namespace ptb

using namespace ptb;

int main(int argc, char** argv)
{
	if (argc < 3) { return 2; }
	FILE* fp = fopen(argv[1], "rb");
	int dims[3] = {0, 0, 0};
	long long thr = 0;
	if (!fp || fread(dims, 4, 3, fp) != 3 || fread(&thr, 8, 1, fp) != 1) { return 1; }
	const int H = dims[0], W = dims[1], B = dims[2];
	const size_t N = static_cast<size_t>(H) * W, P = N * B;
	uint16_t* img = Alloc<uint16_t>(P, 0);
	if (fread(img, 2, P, fp) != P) { return 1; }
	fclose(fp);

	Workspace ws{};
	ws.g.H = H;
	ws.g.W = W;
	ws.g.B = B;
	ws.g.N = static_cast<long long>(N);
	ws.g.P = static_cast<long long>(P);
	ws.img = img;
	ws.code = Alloc<uint8_t>(P, 0xAB);  // garbage, like uninitialised device memory
	ws.w1 = Alloc<uint32_t>(P, 0xAB);
	ws.capDom = static_cast<uint32_t>(P);
	ws.capSeed = static_cast<uint32_t>(P);
	ws.dom = Alloc<uint32_t>(P, 0xAB);
	ws.seeds = Alloc<uint32_t>(P, 0xAB);
	ws.cnt = Alloc<Counters>(1, 0);
	ws.frameDom = Alloc<uint32_t>(B + 1, 0);
	ws.frameSeeds = Alloc<uint32_t>(B + 1, 0);
	// widths the TMA can describe take the TMA staging path (emulated: the same box copy with zero fill, then the
	// kernel's own border replication), the others the per-thread loads, as on the GPU
	CUtensorMap map;
	std::memset(&map, 0, sizeof(map));
	const int useTma = (W % 8) == 0 ? 1 : 0;
	emu::Launch(dim3((W + TX - 1) / TX, (H + TY - 1) / TY, B), dim3(kThreads), DetectKernel,
	            static_cast<const uint16_t*>(img), ws, thr, map, useTma);
	const uint32_t nd = std::min(ws.cnt->ndom, ws.capDom), ns = std::min(ws.cnt->nseed, ws.capSeed);
	std::sort(ws.dom, ws.dom + nd);
	std::sort(ws.seeds, ws.seeds + ns);
	FILE* fo = fopen(argv[2], "wb");
	if (!fo) { return 1; }
	const uint32_t head[3] = {ws.cnt->ndom, ws.cnt->nseed, ws.cnt->overflow};
	fwrite(head, 4, 3, fo);
	fwrite(ws.frameDom, 4, B, fo);
	fwrite(ws.frameSeeds, 4, B, fo);
	fwrite(ws.code, 1, P, fo);
	fwrite(ws.w1, 4, P, fo);
	fwrite(ws.dom, 4, nd, fo);
	fwrite(ws.seeds, 4, ns, fo);
	fclose(fo);
	return 0;
}
