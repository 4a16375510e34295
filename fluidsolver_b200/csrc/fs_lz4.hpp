// LZ4 frames (the container the reference's Lz4CompressedStream writes
// through the lz4 library's LZ4F_* functions, Lz4CompressedStream.cpp:24-180),
// written from the published LZ4 frame and block format descriptions:
//
//   frame  = magic 0x184D2204 (LE) | FLG | BD | [content size u64] | [dict id u32] | HC
//            | blocks | end mark 0x00000000 | [content checksum u32]
//   FLG    = version (bits 7-6 = 01) | block independence (5) | block checksum (4)
//            | content size (3) | content checksum (2) | dict id (0)
//   BD     = block max size code (bits 6-4): 4 -> 64 KB, 5 -> 256 KB, 6 -> 1 MB, 7 -> 4 MB
//   HC     = (XXH32(FLG .. last descriptor byte, seed 0) >> 8) & 0xFF
//   block  = size u32 (bit 31 set: stored uncompressed) | data | [block checksum u32]
//   LZ4 block: sequences of token (literal length << 4 | match length - 4), literal length
//            extension bytes (255 ... last), literals, offset u16 LE, match length
//            extension bytes; the last sequence holds literals only
//
// Skippable frames (magic 0x184D2A50..5F) are skipped; concatenated frames are
// decoded one after another. The encoder writes independent 64 KB blocks, no
// checksums, which every LZ4 frame reader accepts; its matches are found with a
// single hash table of 4-byte sequences (greedy parsing).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace fsio {

// XXH32 (the xxHash 32-bit digest, as published), used for the header checksum
// and, when a frame carries them, the block and content checksums
uint32_t xxh32(const uint8_t* data, size_t len, uint32_t seed);

// Decodes every frame of `in`, appending the content to `out`. Returns an
// empty string on success, else the reason.
std::string lz4_frame_decode(const uint8_t* in, size_t len, std::vector<uint8_t>& out);

// One frame holding `len` bytes: independent 64 KB blocks, no checksums.
std::vector<uint8_t> lz4_frame_encode(const uint8_t* data, size_t len);

// The raw block format, exposed for the tests: compress into at most
// lz4_block_bound(len) bytes; decode returns the decoded size or -1.
size_t lz4_block_bound(size_t len);
size_t lz4_block_compress(const uint8_t* src, size_t len, uint8_t* dst);
long long lz4_block_decompress(const uint8_t* src, size_t len, uint8_t* dst, size_t cap, const uint8_t* history_begin);

}  // namespace fsio
