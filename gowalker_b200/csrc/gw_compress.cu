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

// Width of the chunk ids[0, k): bits of the largest zigzag delta (an OR has
// the same bit length as the maximum).
static inline uint32_t chunk_width(const uint32_t *ids, uint32_t k)
{
    uint32_t m = 0;
    for (uint32_t i = 1; i < k; ++i) m |= zigzag(ids[i] - ids[i - 1]);
    return bit_length(m);
}

// Bytes of a vertex's chunks; with `group` non-null, also the byte offset
// (from the vertex's first chunk) of every 32nd chunk.
static uint64_t vertex_bytes(const uint32_t *ids, uint64_t d, uint64_t *group)
{
    uint64_t s = 0, c = 0;
    for (uint64_t j = 0; j < d; j += kChunkIds, ++c) {
        if (group && c % kChunkIds == 0) group[c / kChunkIds] = s;
        const uint32_t k = (uint32_t)std::min<uint64_t>(kChunkIds, d - j);
        s += 5 + ((uint64_t)(k - 1) * chunk_width(ids + j, k) + 7) / 8;
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
        const uint32_t w = chunk_width(c, k);
        *p++ = (uint8_t)w;
        for (int b = 0; b < 4; ++b) *p++ = (uint8_t)(c[0] >> (8 * b));
        uint64_t acc = 0;
        uint32_t nbits = 0;
        for (uint32_t i = 1; i < k; ++i) {
            acc |= (uint64_t)zigzag(c[i] - c[i - 1]) << nbits;
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
    return true;
}

// Eight bytes of `base` from byte offset `off`, read as two aligned 32-bit
// words (base 16-byte aligned): the low 40 bits or more are the bytes at off
// onwards.  Neighbouring lanes read the same words, so a chunk's fields load
// in one or two transactions instead of five byte loads per lane.
__device__ __forceinline__ uint64_t load_bytes64(const uint8_t *__restrict__ base, uint64_t off)
{
    const uint32_t *w = reinterpret_cast<const uint32_t *>(base + (off & ~3ull));
    const uint64_t v = (uint64_t)__ldg(w) | ((uint64_t)__ldg(w + 1) << 32);
    return v >> ((off & 3u) * 8u);
}

// Warp tasks: task t < nv decodes vertex t if it has at most 32 chunks;
// task nv + g decodes split group g (32 chunks of a larger vertex).  Within a
// chunk, lane i extracts delta i (lane 0 the first id) and a warp prefix sum
// (mod 2^32) rebuilds the ids.  Every id written is checked against nverts
// (the validation of a plain block copy, done here in the same pass).
__global__ void k_decode_block(const uint8_t *__restrict__ src, uint64_t split_off, uint32_t nsplit,
                               uint64_t payload_off, uint64_t payload_bytes, uint32_t nv,
                               const uint64_t *__restrict__ beg, uint32_t v0, uint64_t e0, uint64_t ne,
                               uint32_t nverts, uint32_t *__restrict__ out, uint32_t *err)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t *voff = reinterpret_cast<const uint32_t *>(src);
    const uint32_t *split = reinterpret_cast<const uint32_t *>(src + split_off);
    const uint8_t *pay = src + payload_off;
    const uint64_t ntasks = (uint64_t)nv + nsplit;
    bool bad_id = false;
    for (uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntasks; t += nwarps) {
        uint32_t v, c0;
        uint64_t pos;
        if (t < nv) {
            v = (uint32_t)t;
            c0 = 0;
            pos = __ldg(voff + v);
        } else {
            const uint64_t g = t - nv;
            v = __ldg(split + 3 * g);
            c0 = __ldg(split + 3 * g + 1);
            pos = __ldg(split + 3 * g + 2);
            if (v >= nv) {
                if (lane == 0) atomicOr(err, kErrBlock);
                continue;
            }
        }
        const uint64_t b0 = __ldg(beg + v0 + v), b1 = __ldg(beg + v0 + v + 1);
        bool bad = b1 < b0 || b0 < e0 || b1 - e0 > ne;
        const uint64_t d = bad ? 0 : b1 - b0;
        const uint64_t nch = (d + kChunkIds - 1) / kChunkIds;
        if (t < nv && nch > kChunkIds) continue;  // decoded by its split groups
        const uint64_t c1 = min(nch, (uint64_t)c0 + kChunkIds);
        for (uint64_t c = c0; c < c1; ++c) {
            const uint64_t j = c * kChunkIds;
            const uint32_t k = (uint32_t)min((uint64_t)kChunkIds, d - j);
            if (pos + 5 > payload_bytes) {
                bad = true;
                break;
            }
            const uint64_t head = load_bytes64(pay, pos);  // width byte, then the first id
            const uint32_t w = (uint32_t)head & 0xFFu;
            const uint64_t packed = ((uint64_t)(k - 1) * w + 7) >> 3;
            if (w > 32 || pos + 5 + packed > payload_bytes) {
                bad = true;
                break;
            }
            uint32_t x = 0;
            if (lane == 0) {
                x = (uint32_t)(head >> 8);
            } else if (lane < k && w != 0) {
                // bits [bp, bp + w) of the packed deltas: at most 39 bits from
                // the byte holding bit bp, inside the 8-byte pad past the payload
                const uint32_t bp = (lane - 1) * w;
                const uint64_t acc = load_bytes64(pay, pos + 5 + (bp >> 3));
                const uint64_t mask = (w == 32) ? 0xFFFFFFFFull : ((1ull << w) - 1);
                const uint32_t z = (uint32_t)((acc >> (bp & 7u)) & mask);
                x = (z >> 1) ^ (0u - (z & 1u));
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                if (lane >= (uint32_t)o) x += y;
            }
            if (lane < k) {
                out[b0 - e0 + j + lane] = x;
                bad_id |= x >= nverts;
            }
            pos += 5 + packed;
        }
        if (bad && lane == 0) atomicOr(err, kErrBlock);
    }
    if (__any_sync(0xFFFFFFFFu, bad_id) && lane == 0) atomicOr(err, kErrVertexRange);
}

cudaError_t launch_decode_block(const uint8_t *src, const CompressedBlock &cb, uint32_t nv, const uint64_t *beg,
                                uint32_t v0, uint64_t e0, uint64_t ne, uint32_t nverts, uint32_t *out, uint32_t *err,
                                int num_sms, cudaStream_t s)
{
    if (nv == 0) return cudaSuccess;
    k_decode_block<<<num_sms * 8, 256, 0, s>>>(src, cb.split_off, cb.nsplit, cb.payload_off, cb.payload_bytes, nv, beg,
                                               v0, e0, ne, nverts, out, err);
    return cudaGetLastError();
}

}  // namespace gw
