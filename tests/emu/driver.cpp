// Runs the segmentation kernels of one frame on the CPU (each CUDA thread a host thread, shim.h), every device array a
// separate allocation so that AddressSanitizer reports any out-of-bounds access. Test harness only.
// Usage: emu <in> <out> [mode]; in: int32 H, W, int64 threshold (2^-16 units), H * W int64 W1 values (2^-16 units);
// out: H * W uint32 labels, H * W code bytes, then 6 uint32 (routed, rank-tested, re-flooded, suspect pairs, fits, groups
// of the re-flooded frame re-flooded in global memory).
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

#include "segment_emu.inc"

#include <cstdio>
#include <cstdlib>

namespace ptb {
void SetError(const std::string& m) { fprintf(stderr, "SetError %s\n", m.c_str()); }
bool CheckCuda(cudaError_t, const char*, const char*, int) { return true; }
void CountLaunch(uint64_t) {}

bool ExclusiveScan(uint32_t* data, const uint32_t* nptr, uint32_t nconst, uint32_t cap, uint32_t*, uint32_t* totalOut,
                   cudaStream_t)
{
	const uint32_t n = nptr ? *nptr : nconst;
	if (n > cap) { fprintf(stderr, "scan n %u > cap %u\n", n, cap); abort(); }
	uint32_t s = 0;
	for (uint32_t i = 0; i < n; ++i) {
		const uint32_t v = data[i];
		data[i] = s;
		s += v;
	}
	data[n] = s;
	if (totalOut) { *totalOut = s; }
	return true;
}

template <class T> static T* Alloc(size_t n)
{
	T* p = static_cast<T*>(malloc(std::max<size_t>(n, 1) * sizeof(T)));
	memset(p, 0xAB, std::max<size_t>(n, 1) * sizeof(T));  // garbage, like uninitialised device memory
	return p;
}
}  // namespace ptb

using namespace ptb;

int main(int argc, char** argv)
{
	if (argc < 3) { return 2; }
	const int strictMode = argc > 3 ? atoi(argv[3]) : 0;
	FILE* fp = fopen(argv[1], "rb");
	int hw[2] = {0, 0};
	long long thr = 0;
	if (!fp || fread(hw, 4, 2, fp) != 2 || fread(&thr, 8, 1, fp) != 1) { return 1; }
	const int H = hw[0], W = hw[1], B = 1;
	std::vector<long long> w1u(static_cast<size_t>(H) * W);
	if (fread(w1u.data(), 8, w1u.size(), fp) != w1u.size()) { return 1; }
	fclose(fp);

	Workspace ws{};
	Geometry g{};
	g.H = H; g.W = W; g.B = B; g.words = (W + 31) / 32; g.N = static_cast<long long>(H) * W; g.P = g.N * B;
	g.divN = MakeFastDiv(static_cast<uint32_t>(g.N));
	g.divW = MakeFastDiv(static_cast<uint32_t>(W));
	ws.g = g;
	const size_t P = g.P;
	const uint32_t capComp = static_cast<uint32_t>(((H + 1) / 2) * ((W + 1) / 2) * B + 1);
	ws.capDom = P; ws.capSeed = P; ws.capComp = capComp; ws.capRegion = capComp;
	ws.capRows = std::min<uint32_t>(100000, capComp);
	const size_t rows = static_cast<size_t>(B) * H;
	ws.img = nullptr;
	ws.code = Alloc<uint8_t>(P); ws.w1 = Alloc<uint32_t>(P); ws.par = Alloc<uint32_t>(P); ws.lab = Alloc<uint32_t>(P);
	ws.rootmask = Alloc<uint32_t>(rows * g.words); ws.rowcnt = Alloc<uint32_t>(rows + 1);
	ws.dom = Alloc<uint32_t>(P); ws.seeds = Alloc<uint32_t>(P);
	ws.compRoot = Alloc<uint32_t>(capComp); ws.compSize = Alloc<uint32_t>(capComp); ws.compNRoot = Alloc<uint32_t>(capComp);
	ws.compNSeed = Alloc<uint32_t>(capComp); ws.compRegion = Alloc<uint32_t>(capComp); ws.multi = Alloc<uint32_t>(capComp);
	ws.gOff = Alloc<uint32_t>(capComp + 1); ws.gSeedOff = Alloc<uint32_t>(capComp + 1); ws.gRegOff = Alloc<uint32_t>(capComp + 1);
	ws.gCurPix = Alloc<uint32_t>(capComp + 1); ws.gCurSeed = Alloc<uint32_t>(capComp + 1); ws.gCurReg = Alloc<uint32_t>(capComp + 1);
	ws.gPix = Alloc<uint32_t>(P); ws.gSeed = Alloc<uint32_t>(P); ws.gReg = Alloc<uint32_t>(capComp);
	ws.heapKey = Alloc<double>(P); ws.heapPix = Alloc<uint32_t>(P);
	ws.regCount = Alloc<uint32_t>(capComp); ws.regSumVJ = Alloc<unsigned long long>(capComp);
	ws.regSumVI = Alloc<unsigned long long>(capComp); ws.regSumV = Alloc<unsigned long long>(capComp);
	ws.regFrame = Alloc<uint32_t>(capComp); ws.regCand = Alloc<uint32_t>(capComp + 1);
	ws.fuMaxWN = Alloc<double>(capComp); ws.fuMinP = Alloc<double>(capComp); ws.fuMaxP = Alloc<double>(capComp);
	ws.fuMaxPos = Alloc<uint32_t>(capComp); ws.fuWNPos = Alloc<uint32_t>(capComp); ws.fuNeighbour = Alloc<uint32_t>(capComp);
	ws.fuBecome = Alloc<uint32_t>(capComp); ws.fuLocked = Alloc<uint8_t>(capComp);
	ws.frameDom = Alloc<uint32_t>(B + 1); ws.frameSeeds = Alloc<uint32_t>(B + 1); ws.frameRoute = Alloc<uint32_t>(B + 1);
	ws.frameSuspect = Alloc<uint32_t>(B + 1);
	ws.frameReflood = Alloc<uint32_t>(B + 1);
	for (int f = 0; f <= B; ++f) { ws.frameDom[f] = ws.frameSeeds[f] = ws.frameRoute[f] = ws.frameSuspect[f] = ws.frameReflood[f] = 0; }
	ws.rfVals = Alloc<uint32_t>(static_cast<size_t>(kRefloodSlots) * 2 * kRefloodCap);
	ws.rfGrp = Alloc<uint32_t>(static_cast<size_t>(kRefloodSlots) * 2 * kRefloodCap);
	ws.rfOff = Alloc<uint32_t>(static_cast<size_t>(kRefloodSlots) * 2 * (kRefloodBuckets + 1));
	ws.rfInfo = Alloc<uint32_t>(kRefloodSlots * 8);
	ws.rfPix = Alloc<uint32_t>(static_cast<size_t>(kRefloodSlots) * g.N * kRfWords);
	ws.rfGroups = Alloc<uint32_t>(ws.capComp);
	ws.suspect = Alloc<uint4>(kSuspectCap); ws.capSuspect = kSuspectCap;
	ws.rankOrder = Alloc<uint32_t>(kSuspectCap); ws.rankSlotOff = Alloc<uint32_t>(kRankSlots + 1);
	ws.rankCount = Alloc<uint32_t>(2 * kSuspectCap);
	ws.frameRegBase = Alloc<uint32_t>(B + 1); ws.frameCandBase = Alloc<uint32_t>(B + 1); ws.frameKeep = Alloc<uint32_t>(B + 1);
	ws.frameOutBase = Alloc<uint32_t>(B + 1);
	ws.candRegion = Alloc<uint32_t>(ws.capRows); ws.candFrame = Alloc<uint32_t>(ws.capRows); ws.cand = Alloc<Cand>(ws.capRows);
	ws.rows = Alloc<double>(static_cast<size_t>(ws.capRows) * kCols); ws.sortedRows = Alloc<double>(static_cast<size_t>(ws.capRows) * kCols);
	ws.sortIdx = Alloc<uint32_t>(ws.capRows * 2); ws.sortKey = Alloc<double>(ws.capRows * 4); ws.fitFlag = Alloc<uint8_t>(ws.capRows);
	ws.scanBlock = Alloc<uint32_t>(P / 4096 + 64);
	ws.cnt = Alloc<Counters>(1);
	memset(ws.cnt, 0, sizeof(Counters));
	memset(ws.rootmask, 0, sizeof(uint32_t) * rows * g.words);

	// the detection kernel's outputs
	auto v0 = [&](int y, int x) -> long long { return (y < 0 || y >= H || x < 0 || x >= W) ? 0 : std::max(0ll, w1u[static_cast<size_t>(y) * W + x]); };
	uint32_t nd = 0, ns = 0;
	for (int y = 0; y < H; ++y) {
		for (int x = 0; x < W; ++x) {
			const size_t p = static_cast<size_t>(y) * W + x;
			const long long v = v0(y, x);
			const bool dom = v > thr && v > 0;
			long long m = 0;
			for (int dy = -1; dy <= 1; ++dy) for (int dx = -1; dx <= 1; ++dx) { m = std::max(m, v0(y + dy, x + dx)); }
			const bool seed = dom && v >= m;
			ws.code[p] = static_cast<uint8_t>((dom ? kDomain : 0) | (seed ? kSeed : 0));
			if (dom) { ws.w1[p] = static_cast<uint32_t>(v); ws.dom[nd++] = static_cast<uint32_t>(p); }
			if (seed) { ws.seeds[ns++] = static_cast<uint32_t>(p); }
		}
	}
	ws.cnt->ndom = nd; ws.cnt->nseed = ns; ws.frameDom[0] = nd; ws.frameSeeds[0] = ns;
	fprintf(stderr, "domain %u seeds %u\n", nd, ns);

	const dim3 one(1), t256(256), t1024(1024), t64(64);
	emu::Launch(one, t256, CclInit, ws);
	emu::Launch(one, t256, CclUnion, ws);
	emu::Launch(one, t256, CompEnumerate, ws);
	emu::Launch(one, t256, CompCount, ws);
	emu::Launch(one, t256, SeedParent, ws);
	emu::Launch(one, t256, RowCount, ws);
	ExclusiveScan(ws.rowcnt, nullptr, rows, rows, ws.scanBlock, &ws.cnt->nregion, nullptr);
	emu::Launch(one, t256, SeedLabel, ws);
	emu::Launch(one, t256, GroupEnumerate, ws);
	ExclusiveScan(ws.gOff, &ws.cnt->nmulti, 0, ws.capComp, ws.scanBlock, nullptr, nullptr);
	ExclusiveScan(ws.gSeedOff, &ws.cnt->nmulti, 0, ws.capComp, ws.scanBlock, nullptr, nullptr);
	ExclusiveScan(ws.gRegOff, &ws.cnt->nmulti, 0, ws.capComp, ws.scanBlock, nullptr, nullptr);
	fprintf(stderr, "components %u groups %u regions %u\n", ws.cnt->ncomp, ws.cnt->nmulti, ws.cnt->nregion);
	emu::Launch(one, t256, GroupScatter, ws, 0);
	uint32_t bigGroups = 0;
	const int rank = strictMode == 0 ? 1 : 0;  // mode 2: the first test only
	emu::Launch(one, t256, GroupFloodBox, ws, rank);
	fprintf(stderr, "flooded: suspect pairs %u routed %u\n", ws.cnt->nsuspect, ws.cnt->nroute);
	if (rank) {
		emu::Launch(one, t1024, SuspectPlan, ws);
		emu::Launch(one, t256, SuspectCount, ws);
		emu::Launch(one, t256, SuspectCheck, ws, 1);
		fprintf(stderr, "rank test: slots %u reflood %u routed %u\n", ws.cnt->nslots, ws.cnt->nreflood, ws.cnt->nroute);
		emu::Launch(one, t1024, RefloodPlan, ws);
		emu::Launch(one, t256, RefloodGather, ws);
		emu::Launch(dim3(kRefloodSlots * 2), t1024, RefloodBucket, ws);
		emu::Launch(one, t256, RefloodCounts, ws);
		emu::Launch(one, dim3(kRfWarps * 32), RefloodBox, ws);
		// groups of the re-flooded frame too large for the shared-memory box (re-flooded in global memory)
		for (uint32_t g = 0; g < ws.cnt->nrfgroup; ++g) {
			const uint32_t m = ws.rfGroups[g];
			int x0 = W, y0 = H, x1 = -1, y1 = -1;
			for (uint32_t i = ws.gOff[m]; i < ws.gOff[m + 1]; ++i) {
				const int y = static_cast<int>((ws.gPix[i] % (uint32_t)(H * W)) / W), x = static_cast<int>(ws.gPix[i] % W);
				x0 = std::min(x0, x); x1 = std::max(x1, x); y0 = std::min(y0, y); y1 = std::max(y1, y);
			}
			const int bw = std::min(x1 + 1, W - 1) - std::max(x0 - 1, 0) + 1, bh = std::min(y1 + 1, H - 1) - std::max(y0 - 1, 0) + 1;
			if (bw * bh > kBoxCap) { ++bigGroups; }
		}
		fprintf(stderr, "reflood: routed %u, groups re-flooded in global memory %u\n", ws.cnt->nroute, bigGroups);
		for (uint32_t i = 0; i < std::min(ws.cnt->nsuspect, 8u); ++i) {
			const uint4 r = ws.suspect[i];
			fprintf(stderr, "  pair %u: f %u c %u w1z %u zmax %u counts %u %u\n", i, r.x, r.y, r.z, r.w, ws.rankCount[2 * i], ws.rankCount[2 * i + 1]);
		}
	}
	emu::Launch(one, t1024, RedoOffsets, ws);
	emu::Launch(one, t256, GroupScatter, ws, 2);
	emu::Launch(one, t64, GroupFlood, ws, static_cast<uint32_t>(B), 1);
	emu::Launch(one, t256, RegionStats, ws);
	emu::Launch(one, t256, CandidateFlags, ws);
	ExclusiveScan(ws.regCand, &ws.cnt->nregion, 0, ws.capRegion, ws.scanBlock, &ws.cnt->ncand, nullptr);
	const uint32_t maxPoints = 100000;
	emu::Launch(dim3((B + 256) / 256), t256, FrameCandidates, ws, maxPoints);
	emu::Launch(dim3((B + 255) / 256), t256, FrameKeep, ws, maxPoints);
	memcpy(ws.frameOutBase, ws.frameKeep, sizeof(uint32_t) * B);
	ExclusiveScan(ws.frameOutBase, nullptr, B, B, ws.scanBlock, &ws.cnt->nfit, nullptr);
	emu::Launch(one, t256, CandidateEmit, ws, maxPoints);
	fprintf(stderr, "done: candidates %u fit %u overflow %u\n", ws.cnt->ncand, ws.cnt->nfit, ws.cnt->overflow);
	FILE* lf = fopen(argv[2], "wb");
	fwrite(ws.lab, sizeof(uint32_t), P, lf);
	fwrite(ws.code, 1, P, lf);
	const uint32_t st[6] = {ws.cnt->nroute, ws.cnt->nslots, ws.cnt->nreflood, ws.cnt->nsuspect, ws.cnt->nfit, bigGroups};
	fwrite(st, sizeof(uint32_t), 6, lf);
	fclose(lf);
	return 0;
}
