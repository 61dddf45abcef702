// Multi-page 16-bit grayscale TIFF stacks (the input format of the reference's test harness,
// Tests_CPU/TiffManagement.hpp:8-55, which reads them with libtiff scanline by scanline).
//
// Reads classic TIFF and BigTIFF in either byte order, uncompressed strips, one 16-bit sample per pixel, every page
// the size of the first (the reference's checks: 16 bits per sample, equal dimensions). Pages are the IFD chain in
// file order. Pixels are read with pread straight into the caller's buffer (contiguous strips merged into one read,
// large reads split over threads) and byte-swapped in place for big-endian files.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ptb {

class TiffStack {
public:
	TiffStack() = default;
	~TiffStack();
	TiffStack(const TiffStack&) = delete;
	TiffStack& operator=(const TiffStack&) = delete;

	// Parses the header and every IFD; false (error recorded) on an unreadable or unsupported file.
	bool Open(const char* path);
	uint64_t Width() const { return width_; }
	uint64_t Height() const { return height_; }
	uint64_t Planes() const { return pages_.size(); }
	// Pages [first, first + count) into dst ([count][height][width], native byte order); false (error recorded) on a
	// short read or a range outside the stack.
	bool Read(uint64_t first, uint64_t count, uint16_t* dst) const;

private:
	struct Strip {
		uint64_t offset;  // file offset of the strip
		uint64_t bytes;   // bytes of pixel data taken from it (rows in the strip x width x 2)
	};
	struct Page {
		std::vector<Strip> strips;
	};
	int fd_ = -1;
	uint64_t fileSize_ = 0;
	bool swap_ = false;  // file byte order differs from the host's
	uint64_t width_ = 0, height_ = 0;
	std::vector<Page> pages_;
};

}  // namespace ptb
