// Compressed neighbour lists of out-of-core blocks: host encoder, device decoder.
// The format is described in gw_compress.cuh.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>
#include "gw_compress.cuh"
#include "gw_kernels.cuh"

namespace gw {

static inline uint32_t zigzag(uint32_t d) { return (d << 1) ^ (uint32_t)((int32_t)d >> 31); }
static inline uint32_t bit_length(uint32_t x) { return x ? 32u - (uint32_t)__builtin_clz(x) : 0u; }

// Code byte of the chunk ids[0, k): the deltas as they are when that is
// narrower (a sorted list: one bit less; at most 31 bits then), else
// zigzag-coded -- an OR has the same bit length as the maximum -- and the
// first id in as few bytes as hold it.
static inline uint32_t chunk_code(const uint32_t *ids, uint32_t k)
{
    uint32_t mz = 0, mr = 0;
    for (uint32_t i = 1; i < k; ++i) {
        mz |= zigzag(ids[i] - ids[i - 1]);
        mr |= ids[i] - ids[i - 1];
    }
    const uint32_t c = bit_length(mr) < bit_length(mz) ? 32u + bit_length(mr) : bit_length(mz);
    const uint32_t fb = std::max(1u, (bit_length(ids[0]) + 7u) / 8u);
    return c | ((fb - 1u) << 6);
}

// Bytes of a vertex's chunks; with `group` non-null, also the byte offset
// (from the vertex's first chunk) of every 32nd chunk.
static uint64_t vertex_bytes(const uint32_t *ids, uint64_t d, uint64_t *group)
{
    uint64_t s = 0, c = 0;
    for (uint64_t j = 0; j < d; j += kChunkIds, ++c) {
        if (group && c % kChunkIds == 0) group[c / kChunkIds] = s;
        const uint32_t k = (uint32_t)std::min<uint64_t>(kChunkIds, d - j);
        s += chunk_bytes(chunk_code(ids + j, k), k);
    }
    return s;
}

static inline uint64_t nchunks(uint64_t d) { return (d + kChunkIds - 1) / kChunkIds; }
static inline uint64_t ngroups(uint64_t d) { return nchunks(d) > kChunkIds ? (nchunks(d) + kChunkIds - 1) / kChunkIds : 0; }

static void encode_vertex(const uint32_t *ids, uint64_t d, uint8_t *p)
{
    for (uint64_t j = 0; j < d; j += kChunkIds) {
        const uint32_t k = (uint32_t)std::min<uint64_t>(kChunkIds, d - j);
        const uint32_t *c = ids + j;
        const uint32_t code = chunk_code(c, k), w = chunk_width(code);
        const bool plain = chunk_plain(code);
        *p++ = (uint8_t)code;
        for (uint32_t b = 0; b < chunk_first_bytes(code); ++b) *p++ = (uint8_t)(c[0] >> (8 * b));
        uint64_t acc = 0;
        uint32_t nbits = 0;
        for (uint32_t i = 1; i < k; ++i) {
            const uint32_t dl = c[i] - c[i - 1];
            acc |= (uint64_t)(plain ? dl : zigzag(dl)) << nbits;
            nbits += w;
            while (nbits >= 8) {
                *p++ = (uint8_t)acc;
                acc >>= 8;
                nbits -= 8;
            }
        }
        if (nbits) *p++ = (uint8_t)acc;
    }
}

bool compress_block(const uint64_t *beg, const uint32_t *csr, uint32_t nv, uint64_t e0, uint64_t e1,
                    unsigned threads, CompressedBlock &out, std::string &why)
{
    if (beg[0] != e0 || beg[nv] != e1) {
        why = "block offsets do not start and end at the block's first and last edge";
        return false;
    }
    for (uint32_t v = 0; v < nv; ++v)
        if (beg[v + 1] < beg[v]) {
            why = "block offsets are not non-decreasing";
            return false;
        }
    threads = std::max(1u, std::min(threads, 64u));
    // vertex ranges of about equal edge count
    std::vector<uint32_t> cut(threads + 1, nv);
    cut[0] = 0;
    for (unsigned t = 1; t < threads; ++t) {
        const uint64_t target = e0 + (e1 - e0) * t / threads;
        cut[t] = (uint32_t)(std::lower_bound(beg, beg + nv, target) - beg);
        cut[t] = std::max(cut[t], cut[t - 1]);
    }
    std::vector<uint64_t> off(nv + 1, 0), gstart(nv + 1, 0);
    for (uint32_t v = 0; v < nv; ++v) gstart[v + 1] = gstart[v] + ngroups(beg[v + 1] - beg[v]);
    const uint64_t nsplit = gstart[nv];
    std::vector<uint64_t> gofs(nsplit);  // byte offset of each group, from its vertex's first chunk
    auto run = [&](auto &&fn) {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < threads; ++t) pool.emplace_back(fn, cut[t], cut[t + 1]);
        for (auto &th : pool) th.join();
    };
    run([&](uint32_t a, uint32_t b) {
        for (uint32_t v = a; v < b; ++v) {
            const uint64_t d = beg[v + 1] - beg[v];
            off[v + 1] = vertex_bytes(csr + (beg[v] - e0), d, ngroups(d) ? gofs.data() + gstart[v] : nullptr);
        }
    });
    for (uint32_t v = 0; v < nv; ++v) off[v + 1] += off[v];
    const uint64_t payload = off[nv];
    if (payload >= (1ull << 32) || nsplit >= (1ull << 30)) {
        why = "block too large to compress (payload of 4 GB or more)";
        return false;
    }
    out.split_off = ((uint64_t)(nv + 1) * 4 + 15) & ~15ull;
    out.nsplit = (uint32_t)nsplit;
    out.payload_off = (out.split_off + nsplit * 12 + 15) & ~15ull;
    out.payload_bytes = payload;
    out.bytes = (out.payload_off + payload + 8 + 15) & ~15ull;
    if (cudaHostAlloc((void **)&out.host, out.bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        out.host = nullptr;
        why = "pinned allocation for a compressed block failed";
        return false;
    }
    memset(out.host, 0, out.payload_off);
    memset(out.host + out.payload_off + payload, 0, out.bytes - out.payload_off - payload);
    uint32_t *voff = (uint32_t *)out.host;
    for (uint32_t v = 0; v <= nv; ++v) voff[v] = (uint32_t)off[v];
    uint32_t *split = (uint32_t *)(out.host + out.split_off);
    for (uint32_t v = 0; v < nv; ++v)
        for (uint64_t g = gstart[v]; g < gstart[v + 1]; ++g) {
            split[3 * g] = v;
            split[3 * g + 1] = (uint32_t)((g - gstart[v]) * kChunkIds);
            split[3 * g + 2] = (uint32_t)(off[v] + gofs[g]);
        }
    uint8_t *pay = out.host + out.payload_off;
    run([&](uint32_t a, uint32_t b) {
        for (uint32_t v = a; v < b; ++v) encode_vertex(csr + (beg[v] - e0), beg[v + 1] - beg[v], pay + off[v]);
    });
    // pieces of about equal payload, cut at multiples of 32 vertices
    out.piece_v[0] = 0;
    out.piece_v[kPieces] = nv;
    for (uint32_t k = 1; k < kPieces; ++k) {
        const uint64_t target = payload * k / kPieces;
        uint32_t v = (uint32_t)(std::lower_bound(off.begin(), off.begin() + nv, target) - off.begin());
        v &= ~31u;
        out.piece_v[k] = std::max(v, out.piece_v[k - 1]);
    }
    for (uint32_t k = 0; k <= kPieces; ++k) out.piece_g[k] = (uint32_t)gstart[out.piece_v[k]];
    return true;
}

// One chunk of k ids at byte `pos` of the payload, decoded by the warp from
// its shared-memory window of the payload words [base, base + kWindowWords):
// lane 0 takes the first id, lane i < k delta i (its bits read straight from
// the window), and a warp prefix sum (mod 2^32) rebuilds the ids.  `end` is
// the byte past the chunks this task may read; a chunk reaching past it is
// malformed.  A chunk spans at most 3 + 5 + 124 bytes (alignment, code and
// first id, deltas), so its words lie in
// [off, off + 35) with off = pos / 4 - base; the caller keeps off <= kSlideAt.
__device__ __forceinline__ uint64_t decode_chunk_sm(const uint32_t *sm, uint64_t base, uint64_t pos, uint64_t end,
                                                    uint32_t k, uint32_t lane, uint32_t *__restrict__ row,
                                                    uint32_t nverts, bool &bad_id, bool &bad)
{
    const uint32_t off = (uint32_t)((pos >> 2) - base);
    const uint32_t sh = (uint32_t)(pos & 3u) * 8u;
    const uint64_t head = (((uint64_t)sm[off + 1] << 32) | sm[off]) >> sh;
    const uint32_t code = (uint32_t)head & 0xFFu, w = chunk_width(code), fb = chunk_first_bytes(code);
    const uint32_t zz = chunk_plain(code) ? 0u : 1u;  // zigzag-coded deltas
    const uint64_t size = chunk_bytes(code, k);
    if (pos + size > end) {
        bad = true;
        return pos;
    }
    const uint32_t bp = lane ? (lane - 1) * w : 0u;
    const uint32_t bo = sh + 8u + 8u * fb + bp;
    const uint32_t q = off + (bo >> 5);
    uint32_t x = 0;
    if (lane == 0) {
        x = (uint32_t)((head >> 8) & (0xFFFFFFFFull >> (32u - 8u * fb)));
    } else if (lane < k && w != 0) {
        const uint64_t acc = ((uint64_t)sm[q + 1] << 32) | sm[q];
        const uint64_t mask = (w == 32) ? 0xFFFFFFFFull : ((1ull << w) - 1);
        const uint32_t z = (uint32_t)((acc >> (bo & 31u)) & mask);
        x = zz ? (z >> 1) ^ (0u - (z & 1u)) : z;
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane < k) {
        row[lane] = x;
        bad_id |= x >= nverts;
    }
    return pos + size;
}

constexpr uint32_t kWindowWords = 1024 + 36;  // a warp's shared-memory window of the payload (4.1 KB)
constexpr uint32_t kSlideAt = 1024;           // a chunk starting past this word of the window slides it
constexpr uint32_t kDecodeThreads = 256;

// Warp tasks: task t < ntv decodes vertices [32t, 32t + 32) that have at most
// 32 chunks (lane i loads vertex 32t + i's payload offset and neighbour
// range, coalesced, and the warp walks the 32 in turn); task ntv + g decodes
// split group g (32 chunks of a larger vertex).  A task's chunks are read
// from a window of the payload in shared memory, filled by the warp with
// coalesced, independent loads and slid forward when the next chunk would
// run past it, so the only dependent chain -- each chunk's position follows
// from the previous chunk's width byte -- runs through shared memory.  Every
// id written is checked against nverts (the validation of a plain block
// copy, done here in the same pass).
__global__ void __launch_bounds__(kDecodeThreads)
    k_decode_block(const uint8_t *__restrict__ src, uint64_t split_off, uint32_t nsplit, uint64_t payload_off,
                   uint64_t payload_bytes, uint32_t nv, const uint64_t *__restrict__ beg, uint32_t v0, uint64_t e0,
                   uint64_t ne, uint32_t nverts, uint32_t *__restrict__ out, uint32_t *err, uint64_t t_lo,
                   uint64_t t_hi, uint64_t g_lo, uint64_t g_hi)
{
    __shared__ uint32_t s_win[kDecodeThreads / 32][kWindowWords];
    uint32_t *sm = s_win[threadIdx.x >> 5];
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t *voff = reinterpret_cast<const uint32_t *>(src);
    const uint32_t *split = reinterpret_cast<const uint32_t *>(src + split_off);
    const uint32_t *pay_words = reinterpret_cast<const uint32_t *>(src + payload_off);
    const uint64_t limit = (payload_bytes + 8) >> 2;  // whole words of payload and padding
    const uint64_t ntv = ((uint64_t)nv + 31) >> 5;
    // this launch's tasks: vertex batches [t_lo, t_hi), then split groups [g_lo, g_hi)
    const uint64_t nbt = t_hi - t_lo;
    const uint64_t ntasks = nbt + (g_hi - g_lo);
    bool bad_id = false, bad = false;
    uint64_t base = ~0ull;  // first payload word in the window (~0: empty)
    // make the window hold the chunk at byte `pos` (warp-uniform)
    auto cover = [&](uint64_t pos) {
        const uint64_t w = pos >> 2;
        if (base != ~0ull && w >= base && w - base <= kSlideAt) return;
        __syncwarp();  // every lane is done with the old window
        base = w;
        for (uint32_t i = lane; i < kWindowWords; i += 32) sm[i] = (base + i < limit) ? __ldg(pay_words + base + i) : 0u;
        __syncwarp();
    };
    for (uint64_t task = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; task < ntasks; task += nwarps) {
        const uint64_t t = task < nbt ? t_lo + task : ntv + g_lo + (task - nbt);
        if (t < ntv) {
            const uint64_t vi = (t << 5) + lane;
            uint64_t mpos = 0, mb0 = 0, mb1 = 0;
            if (vi < nv) {
                mpos = __ldg(voff + vi);
                mb0 = __ldg(beg + v0 + vi);
                mb1 = __ldg(beg + v0 + vi + 1);
            }
            const uint32_t nvt = (uint32_t)min((uint64_t)32, (uint64_t)nv - (t << 5));
            // the batch's payload: [first vertex's offset, the next batch's)
            const uint64_t p0 = __shfl_sync(0xFFFFFFFFu, mpos, 0);
            const uint64_t p1 = __ldg(voff + (t << 5) + nvt);
            if (p1 < p0 || p1 > payload_bytes) {
                bad = true;
                continue;
            }
            // every chunk of the batch reads words [p0 / 4, p1 / 4 + 2)
            const uint64_t b_base = p0 >> 2, nwords = ((p1 + 3) >> 2) - b_base + 2;
            if (nwords <= kWindowWords) {
                // ---- the whole batch in the window: one fill, then each lane
                // decodes its own vertex when it has one chunk (most do), and
                // the warp decodes the chunks of the batch's larger vertices
                __syncwarp();
                base = b_base;
                for (uint32_t i = lane; i < nwords; i += 32)
                    sm[i] = (base + i < limit) ? __ldg(pay_words + base + i) : 0u;
                __syncwarp();
                const bool mine = (uint64_t)lane < nvt;
                const bool range_ok = !mine || (mb1 >= mb0 && mb0 >= e0 && mb1 - e0 <= ne);
                bad |= !range_ok;
                const uint64_t d = (mine && range_ok) ? mb1 - mb0 : 0;
                if (d >= 1 && d <= kChunkIds) {
                    if (mpos < p0 || mpos + 2 > p1) {
                        bad = true;
                    } else {
                        const uint32_t off = (uint32_t)((mpos >> 2) - base);
                        const uint32_t sh = (uint32_t)(mpos & 3u) * 8u;
                        const uint64_t head = (((uint64_t)sm[off + 1] << 32) | sm[off]) >> sh;
                        const uint32_t code = (uint32_t)head & 0xFFu, w = chunk_width(code);
                        const uint32_t fb = chunk_first_bytes(code);
                        const bool zz = !chunk_plain(code);
                        if (mpos + chunk_bytes(code, (uint32_t)d) > p1) {
                            bad = true;
                        } else {
                            uint32_t *row = out + (mb0 - e0);
                            uint32_t x = (uint32_t)((head >> 8) & (0xFFFFFFFFull >> (32u - 8u * fb)));
                            row[0] = x;
                            bool over = x >= nverts;
                            const uint64_t mask = (w == 32) ? 0xFFFFFFFFull : ((1ull << w) - 1);
                            uint32_t bit = sh + 8u + 8u * fb;  // from word `off`
                            for (uint32_t i = 1; i < (uint32_t)d; ++i, bit += w) {
                                const uint32_t q = off + (bit >> 5);
                                const uint64_t acc = ((uint64_t)sm[q + 1] << 32) | sm[q];
                                const uint32_t z = (uint32_t)((acc >> (bit & 31u)) & mask);
                                x += zz ? (z >> 1) ^ (0u - (z & 1u)) : z;
                                row[i] = x;
                                over |= x >= nverts;
                            }
                            bad_id |= over;
                        }
                    }
                }
                // vertices of 2..32 chunks, one after another, a chunk per warp step
                for (unsigned mm = __ballot_sync(0xFFFFFFFFu, d > kChunkIds && d <= (uint64_t)kChunkIds * kChunkIds);
                     mm; mm &= mm - 1) {
                    const int j = __ffs(mm) - 1;
                    uint64_t pos = __shfl_sync(0xFFFFFFFFu, mpos, j);
                    const uint64_t b0 = __shfl_sync(0xFFFFFFFFu, mb0, j);
                    const uint64_t dj = __shfl_sync(0xFFFFFFFFu, d, j);
                    const uint64_t nch = (dj + kChunkIds - 1) / kChunkIds;
                    bool vbad = false;
                    for (uint64_t c = 0; c < nch && !vbad; ++c) {
                        const uint32_t k = (uint32_t)min((uint64_t)kChunkIds, dj - c * kChunkIds);
                        if (pos < p0 || pos + 2 > p1) {
                            vbad = true;
                            break;
                        }
                        pos = decode_chunk_sm(sm, base, pos, p1, k, lane, out + (b0 - e0) + c * kChunkIds, nverts,
                                              bad_id, vbad);
                    }
                    bad |= vbad;
                }
                base = ~0ull;  // the window holds this batch's words only
                continue;
            }
            // ---- a batch larger than the window: vertex by vertex, sliding it
            for (uint32_t j = 0; j < nvt; ++j) {
                uint64_t pos = __shfl_sync(0xFFFFFFFFu, mpos, j);
                const uint64_t b0 = __shfl_sync(0xFFFFFFFFu, mb0, j), b1 = __shfl_sync(0xFFFFFFFFu, mb1, j);
                if (b1 < b0 || b0 < e0 || b1 - e0 > ne) {
                    bad = true;
                    continue;
                }
                const uint64_t d = b1 - b0;
                const uint64_t nch = (d + kChunkIds - 1) / kChunkIds;
                if (nch > kChunkIds) continue;  // decoded by its split groups
                bool vbad = false;
                for (uint64_t c = 0; c < nch && !vbad; ++c) {
                    const uint32_t k = (uint32_t)min((uint64_t)kChunkIds, d - c * kChunkIds);
                    if (pos < p0 || pos + 2 > p1) {
                        vbad = true;
                        break;
                    }
                    cover(pos);
                    pos = decode_chunk_sm(sm, base, pos, p1, k, lane, out + (b0 - e0) + c * kChunkIds, nverts, bad_id,
                                          vbad);
                }
                bad |= vbad;
            }
        } else {
            const uint64_t g = t - ntv;
            const uint32_t v = __ldg(split + 3 * g), c0 = __ldg(split + 3 * g + 1);
            uint64_t pos = __ldg(split + 3 * g + 2);
            if (v >= nv) {
                bad = true;
                continue;
            }
            const uint64_t b0 = __ldg(beg + v0 + v), b1 = __ldg(beg + v0 + v + 1);
            if (b1 < b0 || b0 < e0 || b1 - e0 > ne) {
                bad = true;
                continue;
            }
            const uint64_t d = b1 - b0;
            const uint64_t nch = (d + kChunkIds - 1) / kChunkIds;
            const uint64_t c1 = min(nch, (uint64_t)c0 + kChunkIds);
            bool vbad = false;
            for (uint64_t c = c0; c < c1 && !vbad; ++c) {
                const uint32_t k = (uint32_t)min((uint64_t)kChunkIds, d - c * kChunkIds);
                if (pos + 2 > payload_bytes) {
                    vbad = true;
                    break;
                }
                cover(pos);
                pos = decode_chunk_sm(sm, base, pos, payload_bytes, k, lane, out + (b0 - e0) + c * kChunkIds, nverts,
                                      bad_id, vbad);
            }
            bad |= vbad;
        }
    }
    if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) atomicOr(err, kErrBlock);
    if (__any_sync(0xFFFFFFFFu, bad_id) && lane == 0) atomicOr(err, kErrVertexRange);
}

cudaError_t launch_decode_block(const uint8_t *src, const CompressedBlock &cb, uint32_t nv, const uint64_t *beg,
                                uint32_t v0, uint64_t e0, uint64_t ne, uint32_t nverts, uint32_t *out, uint32_t *err,
                                int num_sms, cudaStream_t s, int piece)
{
    if (nv == 0) return cudaSuccess;
    uint64_t t_lo = 0, t_hi = ((uint64_t)nv + 31) >> 5, g_lo = 0, g_hi = cb.nsplit;
    if (piece >= 0) {
        t_lo = cb.piece_v[piece] >> 5;
        t_hi = ((uint64_t)cb.piece_v[piece + 1] + 31) >> 5;
        g_lo = cb.piece_g[piece];
        g_hi = cb.piece_g[piece + 1];
        if (t_hi <= t_lo && g_hi <= g_lo) return cudaSuccess;
    }
    k_decode_block<<<num_sms * 4, kDecodeThreads, 0, s>>>(src, cb.split_off, cb.nsplit, cb.payload_off,
                                                         cb.payload_bytes, nv, beg, v0, e0, ne, nverts, out, err, t_lo,
                                                         t_hi, g_lo, g_hi);
    return cudaGetLastError();
}

}  // namespace gw
