// Multi-page 16-bit TIFF reader (see tiff.h). Every offset and count read from the file is checked against the file
// size before use, so a truncated or malformed file is reported as an error rather than read past its end.
#include "tiff.h"

#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <unordered_set>

#include "pt_common.cuh"

namespace ptb {

namespace {

constexpr uint64_t kMaxPages = 1ull << 24;
constexpr uint64_t kMaxValues = 1ull << 24;  // values of one tag (strips of one page)

bool ReadAt(int fd, uint64_t off, void* dst, size_t n)
{
	char* p = static_cast<char*>(dst);
	while (n > 0) {
		const ssize_t r = pread(fd, p, n, static_cast<off_t>(off));
		if (r <= 0) { return false; }
		p += r;
		off += static_cast<uint64_t>(r);
		n -= static_cast<size_t>(r);
	}
	return true;
}

// Field access in the file's byte order.
struct Order {
	bool big;
	uint16_t U16(const uint8_t* b) const { return big ? static_cast<uint16_t>((b[0] << 8) | b[1]) : static_cast<uint16_t>((b[1] << 8) | b[0]); }
	uint32_t U32(const uint8_t* b) const
	{
		return big ? (static_cast<uint32_t>(b[0]) << 24) | (static_cast<uint32_t>(b[1]) << 16) | (static_cast<uint32_t>(b[2]) << 8) | b[3]
		           : (static_cast<uint32_t>(b[3]) << 24) | (static_cast<uint32_t>(b[2]) << 16) | (static_cast<uint32_t>(b[1]) << 8) | b[0];
	}
	uint64_t U64(const uint8_t* b) const
	{
		const uint64_t hi = U32(big ? b : b + 4), lo = U32(big ? b + 4 : b);
		return (hi << 32) | lo;
	}
};

enum : uint16_t {
	kTagNewSubfileType = 254, kTagWidth = 256, kTagHeight = 257, kTagBitsPerSample = 258, kTagCompression = 259,
	kTagStripOffsets = 273, kTagSamplesPerPixel = 277, kTagRowsPerStrip = 278, kTagStripByteCounts = 279,
	kTagPlanarConfig = 284, kTagTileWidth = 322, kTagTileOffsets = 324
};

size_t TypeSize(uint16_t type)
{
	switch (type) {
		case 1: case 2: case 6: case 7: return 1;   // BYTE, ASCII, SBYTE, UNDEFINED
		case 3: case 8: return 2;                   // SHORT, SSHORT
		case 4: case 9: case 11: case 13: return 4; // LONG, SLONG, FLOAT, IFD
		case 5: case 10: case 12: case 16: case 17: case 18: return 8;  // RATIONAL, SRATIONAL, DOUBLE, LONG8, SLONG8, IFD8
		default: return 0;
	}
}

}  // namespace

TiffStack::~TiffStack()
{
	if (fd_ >= 0) { close(fd_); }
}

bool TiffStack::Open(const char* path)
{
	if (path == nullptr) { SetError("TIFF path is null"); return false; }
	fd_ = open(path, O_RDONLY | O_CLOEXEC);
	if (fd_ < 0) { SetError(std::string("cannot open TIFF file: ") + path); return false; }
	const off_t end = lseek(fd_, 0, SEEK_END);
	if (end <= 0) { SetError("empty TIFF file"); return false; }
	fileSize_ = static_cast<uint64_t>(end);
	uint8_t hdr[16] = {};
	if (fileSize_ < 8 || !ReadAt(fd_, 0, hdr, std::min<uint64_t>(16, fileSize_))) { SetError("TIFF header unreadable"); return false; }
	if (!((hdr[0] == 'I' && hdr[1] == 'I') || (hdr[0] == 'M' && hdr[1] == 'M'))) { SetError("not a TIFF file (byte-order mark)"); return false; }
	const Order o{hdr[0] == 'M'};
	swap_ = o.big;  // the host is little-endian
	const uint16_t magic = o.U16(hdr + 2);
	const bool big = magic == 43;
	if (magic != 42 && !big) { SetError("not a TIFF file (version)"); return false; }
	if (big && (fileSize_ < 16 || o.U16(hdr + 4) != 8)) { SetError("unsupported BigTIFF offset size"); return false; }
	uint64_t ifd = big ? o.U64(hdr + 8) : o.U32(hdr + 4);
	const size_t entryBytes = big ? 20 : 12, countBytes = big ? 8 : 2, nextBytes = big ? 8 : 4, inlineBytes = big ? 8 : 4;
	std::unordered_set<uint64_t> seen;
	std::vector<uint8_t> buf;
	while (ifd != 0) {
		if (pages_.size() >= kMaxPages || !seen.insert(ifd).second) { SetError("TIFF directory chain loops or is too long"); return false; }
		uint8_t cnt[8];
		if (ifd + countBytes > fileSize_ || !ReadAt(fd_, ifd, cnt, countBytes)) { SetError("TIFF directory outside the file"); return false; }
		const uint64_t entries = big ? o.U64(cnt) : o.U16(cnt);
		if (entries > 65535 || ifd + countBytes + entries * entryBytes + nextBytes > fileSize_) { SetError("TIFF directory outside the file"); return false; }
		buf.resize(entries * entryBytes + nextBytes);
		if (!ReadAt(fd_, ifd + countBytes, buf.data(), buf.size())) { SetError("TIFF directory unreadable"); return false; }
		// tag values as unsigned integers (SHORT, LONG, LONG8 and IFD types); false for other types or bad offsets
		auto values = [&](const uint8_t* e, std::vector<uint64_t>& out) {
			const uint16_t type = o.U16(e + 2);
			const uint64_t n = big ? o.U64(e + 4) : o.U32(e + 4);
			const size_t sz = TypeSize(type);
			if (!(type == 3 || type == 4 || type == 13 || type == 16 || type == 18) || n == 0 || n > kMaxValues) { return false; }
			std::vector<uint8_t> raw(n * sz);
			const uint8_t* field = e + (big ? 12 : 8);
			if (n * sz <= inlineBytes) { std::memcpy(raw.data(), field, n * sz); }
			else {
				const uint64_t off = big ? o.U64(field) : o.U32(field);
				if (off > fileSize_ || n * sz > fileSize_ - off || !ReadAt(fd_, off, raw.data(), raw.size())) { return false; }
			}
			out.resize(n);
			for (uint64_t i = 0; i < n; ++i) {
				const uint8_t* v = raw.data() + i * sz;
				out[i] = sz == 2 ? o.U16(v) : sz == 4 ? o.U32(v) : o.U64(v);
			}
			return true;
		};
		uint64_t w = 0, h = 0, bps = 1, compression = 1, spp = 1, rps = ~0ull, planar = 1;
		std::vector<uint64_t> offsets, counts, v;
		bool tiled = false;
		for (uint64_t k = 0; k < entries; ++k) {
			const uint8_t* e = buf.data() + k * entryBytes;
			const uint16_t tag = o.U16(e);
			switch (tag) {
				case kTagWidth: if (!values(e, v)) { SetError("bad ImageWidth"); return false; } w = v[0]; break;
				case kTagHeight: if (!values(e, v)) { SetError("bad ImageLength"); return false; } h = v[0]; break;
				case kTagBitsPerSample: if (!values(e, v)) { SetError("bad BitsPerSample"); return false; } bps = v[0]; break;
				case kTagCompression: if (!values(e, v)) { SetError("bad Compression"); return false; } compression = v[0]; break;
				case kTagSamplesPerPixel: if (!values(e, v)) { SetError("bad SamplesPerPixel"); return false; } spp = v[0]; break;
				case kTagRowsPerStrip: if (!values(e, v)) { SetError("bad RowsPerStrip"); return false; } rps = v[0]; break;
				case kTagPlanarConfig: if (!values(e, v)) { SetError("bad PlanarConfiguration"); return false; } planar = v[0]; break;
				case kTagStripOffsets: if (!values(e, offsets)) { SetError("bad StripOffsets"); return false; } break;
				case kTagStripByteCounts: if (!values(e, counts)) { SetError("bad StripByteCounts"); return false; } break;
				case kTagTileWidth: case kTagTileOffsets: tiled = true; break;
				default: break;
			}
		}
		const uint64_t page = pages_.size();
		if (bps != 16) { SetError("the TIFF must have 16 bits per sample (page " + std::to_string(page) + ")"); return false; }
		if (spp != 1 || planar != 1) { SetError("the TIFF must have one sample per pixel"); return false; }
		if (tiled) { SetError("tiled TIFF pages are not supported"); return false; }
		if (compression != 1) { SetError("compressed TIFF pages are not supported (compression " + std::to_string(compression) + ")"); return false; }
		if (w == 0 || h == 0 || w > (1u << 30) || h > (1u << 30)) { SetError("bad TIFF page dimensions"); return false; }
		if (page == 0) { width_ = w; height_ = h; }
		else if (w != width_ || h != height_) { SetError("all TIFF pages must have the same dimensions"); return false; }
		rps = std::max<uint64_t>(1, std::min(rps, h));
		const uint64_t nStrips = (h + rps - 1) / rps;
		if (offsets.size() != nStrips || (!counts.empty() && counts.size() != nStrips)) { SetError("TIFF strip tables do not match the page"); return false; }
		Page p;
		p.strips.resize(nStrips);
		for (uint64_t s = 0; s < nStrips; ++s) {
			const uint64_t rows = std::min(rps, h - s * rps), bytes = rows * w * 2;
			if ((!counts.empty() && counts[s] < bytes) || offsets[s] > fileSize_ || bytes > fileSize_ - offsets[s]) {
				SetError("TIFF strip outside the file or shorter than its rows");
				return false;
			}
			p.strips[s] = {offsets[s], bytes};
		}
		pages_.push_back(std::move(p));
		const uint8_t* next = buf.data() + entries * entryBytes;
		ifd = big ? o.U64(next) : o.U32(next);
	}
	if (pages_.empty()) { SetError("TIFF file has no page"); return false; }
	return true;
}

bool TiffStack::Read(uint64_t first, uint64_t count, uint16_t* dst) const
{
	if (fd_ < 0) { SetError("TIFF file not open"); return false; }
	if (first > pages_.size() || count > pages_.size() - first) { SetError("TIFF page range outside the stack"); return false; }
	if (count == 0) { return true; }
	if (dst == nullptr) { SetError("TIFF destination is null"); return false; }
	// file ranges -> destination ranges, adjacent ones merged (pages written back to back read as one range)
	struct Seg {
		uint64_t off, bytes;
		char* dst;
	};
	std::vector<Seg> segs;
	char* out = reinterpret_cast<char*>(dst);
	const uint64_t frameBytes = width_ * height_ * 2;
	for (uint64_t p = first; p < first + count; ++p) {
		char* d = out + (p - first) * frameBytes;
		for (const Strip& s : pages_[p].strips) {
			if (!segs.empty() && segs.back().off + segs.back().bytes == s.offset && segs.back().dst + segs.back().bytes == d) {
				segs.back().bytes += s.bytes;
			}
			else { segs.push_back({s.offset, s.bytes, d}); }
			d += s.bytes;
		}
	}
	// pieces of at most 32 MiB (even sizes, so byte swapping never splits a pixel), read by up to 8 threads
	constexpr uint64_t kPiece = 32ull << 20;
	std::vector<Seg> pieces;
	uint64_t total = 0;
	for (const Seg& s : segs) {
		for (uint64_t o = 0; o < s.bytes; o += kPiece) { pieces.push_back({s.off + o, std::min(kPiece, s.bytes - o), s.dst + o}); }
		total += s.bytes;
	}
	const bool swap = swap_;
	std::atomic<size_t> nextPiece{0};
	std::atomic<bool> failed{false};
	auto worker = [&]() {
		for (size_t i = nextPiece++; i < pieces.size() && !failed; i = nextPiece++) {
			const Seg& s = pieces[i];
			if (!ReadAt(fd_, s.off, s.dst, s.bytes)) {
				failed = true;
				return;
			}
			if (swap) {
				uint16_t* v = reinterpret_cast<uint16_t*>(s.dst);
				for (uint64_t k = 0; k < s.bytes / 2; ++k) { v[k] = static_cast<uint16_t>((v[k] >> 8) | (v[k] << 8)); }
			}
		}
	};
	const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
	const size_t threads = std::min<size_t>({pieces.size(), static_cast<size_t>(std::min(hw, 8u)), static_cast<size_t>(total / (8ull << 20) + 1)});
	std::vector<std::thread> pool;
	for (size_t t = 1; t < threads; ++t) { pool.emplace_back(worker); }
	worker();
	for (auto& t : pool) { t.join(); }
	if (failed) { SetError("TIFF read failed (file truncated or unreadable)"); return false; }
	return true;
}

}  // namespace ptb
