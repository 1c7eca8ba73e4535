// Compressed neighbour lists of out-of-core blocks (internal to libgowalker.so).
//
// A block's neighbour ids cross the host link once per load, so the engine
// keeps a compressed copy of every block in pinned host memory and decodes it
// on the device into the block's cache slot.  Layout of one block's buffer:
//
//   u32 voff[nv + 1]      byte offset of each vertex's chunks in the payload
//   (pad to 16 bytes)
//   u32 split[3 * nsplit] for every vertex with more than 32 chunks, one
//                         entry (vertex, first chunk, byte offset) per group
//                         of 32 chunks, so no decoder task walks more than
//                         32 chunks in sequence (hub vertices have 10^5+)
//   (pad to 16 bytes)
//   payload               per vertex, ceil(deg / 32) chunks of up to 32 ids:
//                           u8  code    bits 0-5: c, the deltas' width w = c
//                                       zigzag-coded (c <= 32) or w = c - 32
//                                       stored as they are (c > 32: a sorted
//                                       chunk, one bit less each); bits 6-7:
//                                       the first id's bytes - 1
//                           first id    1-4 bytes, little endian, unaligned
//                           (k-1) deltas, packed LSB first at w bits
//   8 bytes of padding    so a decoder may read up to 5 bytes past a field
//
// Deltas are id[i] - id[i-1] modulo 2^32, zigzag-coded unless every delta of
// the chunk is narrower as it is, so any neighbour order (sorted or not,
// duplicates included) round-trips exactly; sorted lists give small deltas
// and need no sign bit, and a sorted list's first id is its smallest.  The offsets of every vertex are resident on the device, so
// the decoder knows each vertex's degree and output position without them
// crossing the link again.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

namespace gw {

constexpr uint32_t kChunkIds = 32;
// A chunk's code byte (layout above): width, whether the deltas are plain,
// bytes of the first id, bytes of the whole chunk of k ids.
__host__ __device__ inline uint32_t chunk_width(uint32_t code)
{
    const uint32_t c = code & 63u;
    return c > 32u ? c - 32u : c;
}
__host__ __device__ inline bool chunk_plain(uint32_t code) { return (code & 63u) > 32u; }
__host__ __device__ inline uint32_t chunk_first_bytes(uint32_t code) { return (code >> 6) + 1u; }
__host__ __device__ inline uint64_t chunk_bytes(uint32_t code, uint32_t k)
{
    return 1u + chunk_first_bytes(code) + (((uint64_t)(k - 1) * chunk_width(code) + 7) >> 3);
}
// A prefetched block is copied and decoded in kPieces vertex ranges of about
// equal payload (each a multiple of 32 vertices), so all but the last piece's
// decode overlap the copy of the pieces after it.
constexpr uint32_t kPieces = 4;

struct CompressedBlock {
    uint8_t *host = nullptr;   // pinned (cudaHostAlloc), owned by the handle
    uint64_t bytes = 0;        // whole buffer: offsets, payload, padding
    uint64_t split_off = 0;    // start of the split entries in the buffer
    uint32_t nsplit = 0;
    uint64_t payload_off = 0;  // start of the payload in the buffer
    uint64_t payload_bytes = 0;
    uint32_t piece_v[kPieces + 1] = {};  // first vertex of each piece (piece_v[kPieces] = nv)
    uint32_t piece_g[kPieces + 1] = {};  // first split group of each piece
};

// Encode block [beg[0], beg[nv]) (global edge ids; csr indexed from beg[0]).
// Checks that the offsets are non-decreasing and start and end at e0 / e1.
// Returns false with `why` set when they are not or the payload would exceed
// 2^32 bytes.  Uses up to `threads` host threads.
bool compress_block(const uint64_t *beg, const uint32_t *csr, uint32_t nv, uint64_t e0, uint64_t e1,
                    unsigned threads, CompressedBlock &out, std::string &why);

// Decode a block copied to the device at `src` (the layout above, 16-byte
// aligned) into `out` (neighbour slot, indexed from e0).  beg: resident
// offsets of every vertex, v0: the block's first vertex.  Any offset or
// payload read outside the buffer sets kErrBlock in *err and skips the
// vertex; an id >= nverts sets kErrVertexRange (the block's validation).
// piece < 0: the whole block; else only piece `piece`'s vertices, which need
// only the offsets, the split table and their payload bytes (plus 8) in place.
cudaError_t launch_decode_block(const uint8_t *src, const CompressedBlock &cb, uint32_t nv, const uint64_t *beg,
                                uint32_t v0, uint64_t e0, uint64_t ne, uint32_t nverts, uint32_t *out, uint32_t *err,
                                int num_sms, cudaStream_t s, int piece = -1);

}  // namespace gw
