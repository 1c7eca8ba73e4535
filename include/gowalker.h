/*
 * gowalker.h -- C ABI of the B200 walk engine (libgowalker.so).
 *
 * The engine is a drop-in for the walk path of GOWalker: the Node2vec / SOPR /
 * SOSR second-order random-walk step, walker bucketing by (prev block, cur
 * block), the device block cache fed from pinned host memory, and block
 * choice.  GOWalker itself has no binary interface (each app is one nvcc
 * translation unit); every entry point below names the reference call site it
 * stands in for, as file:line inside the GOWalker sources.
 *
 * Conventions
 *   - Every call returns int status: GW_OK (0) or a negative GW_ERR_*; no call
 *     exits the process (the reference's checkCudaError calls exit(),
 *     api/types.hpp:28-35).  gw_last_error() gives the message of the last
 *     failure on a handle.
 *   - Plain pointers and sizes only.  Host buffers passed to gw_host_block are
 *     borrowed for the life of the handle (the reference keeps every block in
 *     pinned host memory, engine/engine.hpp:74-77); pin them (gw_host_alloc,
 *     cudaHostAlloc or cudaHostRegister) for full copy bandwidth.  The
 *     zero-copy tail reads pinned, mapped blocks in place and stages pageable
 *     ones into pinned memory of its own (it never registers caller pages).
 *   - One host thread per handle.  The handle owns its device memory and its
 *     CUDA streams.
 *   - Walks are bit-identical to the reference CPU step rule
 *     (engine/engine.hpp:158-404) driven by a Philox4x32-10 stream keyed by
 *     (seed, walker id, hop, attempt), whatever the block schedule, cache size
 *     or launch shape.
 */
#ifndef GOWALKER_H
#define GOWALKER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GW_ABI_VERSION 1

/* status codes */
#define GW_OK 0
#define GW_ERR_ARG (-1)      /* bad argument or configuration */
#define GW_ERR_CUDA (-2)     /* a CUDA runtime call failed */
#define GW_ERR_NOMEM (-3)    /* device or pinned allocation refused */
#define GW_ERR_STATE (-4)    /* call out of order (e.g. run before graph) */
#define GW_ERR_TIMEOUT (-5)  /* a bounded device wait gave up */
#define GW_ERR_DEVICE (-6)   /* a kernel reported an error word */
#define GW_ERR_GRAPH (-7)    /* graph data failed validation */

/* algorithms, in AlgorithmType order (api/types.hpp:27) */
#define GW_NODE2VEC 0u
#define GW_SOPR 1u
#define GW_SOSR 2u

/* walker initialisation */
#define GW_INIT_PER_VERTEX 0u    /* walkpersource walkers per vertex, id = v*wps+i
                                    (engine/walk.hpp:32-49) */
#define GW_INIT_SINGLE_SOURCE 1u /* SOPR: all at vertex 1; SOSR: first half at 1,
                                    rest at 3 (engine/walk.hpp:275-293, 355-384) */
#define GW_INIT_RANDOM 2u        /* numwalks walkers at Philox-drawn vertices
                                    (stands in for engine/walk.hpp:64-80) */

/* block-choice policies */
#define GW_POLICY_PLAIN 0u   /* GOwalker_scheduler_t::max_choose_blocks
                                (engine/schedule.hpp:70-138) on the device */
#define GW_POLICY_LEARNED 1u /* GOWalker's choice with learned parts (gw_config.learned_mode): the
                                zero-copy switch priced by measured costs, and eviction by the MLP's
                                forecast of incident walkers; judged run by run against the last plain
                                run of the same workload (more than 2 % more time per step loses, and
                                later learned runs of that workload are plain) */
#define GW_POLICY_SA 2u      /* SOwalker_scheduler_t::choose_blocks (engine/schedule.hpp:455-593):
                                an annealed block set, loaded block by block */

/* path recording */
#define GW_PATHS_NONE 0u   /* per-walker hash and length only */
#define GW_PATHS_FULL 1u   /* every vertex, walker-major rows of maxhops+1 */

typedef struct gw_handle gw_handle;

/* Run parameters.  The fields that have a graph_config counterpart
 * (engine/config.hpp:7-34) keep its meaning and default (apps/Node2vec.cu:35-59). */
typedef struct gw_config {
    uint64_t cache_size;      /* device block-cache bytes ("memory", GB on the CLI) */
    uint64_t blocksize;       /* bytes per block ("blocksize", MB on the CLI) */
    uint32_t algorithm;       /* GW_NODE2VEC / GW_SOPR / GW_SOSR */
    float p, q;               /* Node2vec return / in-out parameters */
    float alpha;              /* SOPR/SOSR restart weight */
    uint32_t maxhops;         /* walk length ("length") */
    uint32_t walkpersource;   /* walkers per vertex */
    uint32_t numwalks;        /* total walkers for SINGLE_SOURCE / RANDOM init */
    uint32_t blockpergrid;    /* 0 = chosen by the autotuner */
    uint32_t threadperblock;  /* 0 = chosen by the autotuner */
    uint32_t zero_threshold;  /* walkers a block must attract to be loaded */
    uint32_t zero_copy;       /* 1: finish stragglers reading mapped host CSR */
    uint32_t init_mode;       /* GW_INIT_* */
    float term_prob;          /* geometric termination per step at hop >= 1 (0 = off) */
    uint64_t seed;            /* Philox key of the walk stream */
    uint32_t record_paths;    /* GW_PATHS_* */
    int32_t device;           /* CUDA device ordinal */
    uint32_t strict_blocks;   /* out-of-core: 1 = a walker runs only when both its blocks are
                                 resident (the reference's rule); 0 = Node2vec walkers also run
                                 with only the current block until a trial needs N(prev) */
    uint32_t prefetch;        /* out-of-core: 1 = take each block choice one iteration ahead and
                                 copy the block on the copy stream while the step kernel runs
                                 (one cache slot stages the copy) */
    uint32_t compress_blocks; /* out-of-core: 1 = keep a compressed copy of every block's neighbour
                                 lists in pinned host memory (chunks of 32 ids, bit-packed deltas),
                                 copy that and decode it on the device: fewer host-link bytes */
    uint32_t learned_sync;    /* learned policy: 1 = evaluation mode: a decision waits for the
                                 predictor's training in flight and uses its weights at once, and
                                 the forecasts go on (and are scored) after the judge hands the run
                                 back to the plain rule; 0 = training never delays a decision
                                 (weights adopted when a training has finished) and the predictor
                                 stops once reverted */
    uint32_t launch_mode;     /* in-core: GW_LAUNCH_PERSISTENT (default) or GW_LAUNCH_PER_HOP, the
                                 plain form kept for comparison (unweighted walks only) */
    uint32_t learned_mode;    /* learned policy parts: GW_LEARNED_EVICT | GW_LEARNED_ZERO_SWITCH, or
                                 GW_LEARNED_AUTO (0, default): both parts on the first learned run of
                                 a workload, the switch alone on the next, then the faster */
    uint32_t reserved[2];
} gw_config;

/* learned policy parts (gw_config.learned_mode) */
#define GW_LEARNED_EVICT 1u        /* with a full cache, evict the cached block with the lowest forecast of
                                      incident walkers (GOWalker's choice of the block to load is kept) */
#define GW_LEARNED_ZERO_SWITCH 2u  /* zero-copy tail: switch when the next load's walkers, times the steps a
                                      runnable walker takes per iteration, times the mapped sectors a step
                                      reads, times the measured time per mapped sector, is below the
                                      measured time of an iteration (in place of the fixed zero_threshold,
                                      which is used until this handle has timed a zero-copy tail) */
#define GW_LEARNED_AUTO 0u

/* in-core launch modes */
#define GW_LAUNCH_PERSISTENT 0u /* one persistent work-stealing kernel runs every walker to the end */
#define GW_LAUNCH_PER_HOP 1u    /* one launch per hop, a thread per walker (the reference's grid-stride
                                   loop, gpu/gpuwalk.hpp:193-205, cut at each hop); same walks */

/* Per-run counters. */
typedef struct gw_stats {
    uint64_t steps;           /* real moves taken by all walkers */
    uint64_t trials;          /* rejection-sampling attempts */
    uint64_t walkers;         /* walkers finished */
    uint64_t h2d_bytes;       /* host->device bytes (blocks + walker records) */
    uint64_t d2h_bytes;       /* device->host bytes */
    uint64_t block_loads;     /* block copies into cache slots */
    uint64_t zero_copy_steps; /* steps taken in the mapped-host tail mode */
    uint32_t iterations;      /* scheduler iterations */
    uint32_t launches;        /* kernels launched by this run */
    float kernel_ms;          /* time inside the step kernels (CUDA events; out-of-core untraced
                                 runs include each iteration's runnable-bucket pass) */
    float total_ms;           /* whole run (CUDA events) */
    uint32_t learned_iterations; /* decisions the learned parts changed or took: forecast evictions,
                                    and the switch to the zero-copy tail */
    uint32_t policy_reverted;    /* 1 when the judge sent the run back to the plain policy */
    float train_loss;            /* predictor training loss (mean squared, log1p scale) */
    float pred_error;            /* learned: mean |prediction - realised target| per block, the target
                                    log1p(mean demand over the next 3 iterations) */
    uint32_t kernel_variant;     /* register-cap variant the autotuner picked (in-core) */
    float persist_error;         /* learned: the same error of the forecast without the network
                                    (this iteration's demand carried forward) */
    float bucket_ms;             /* out-of-core: time re-bucketing walkers (CUDA events) */
    uint32_t walker_chunk;       /* in-core: walkers a warp claims per atomic (the autotuner's pick) */
    uint64_t coop_small_steps;   /* hard steps decided from candidate positions (in-core) */
    uint64_t coop_small_attempts;
    uint64_t coop_large_steps;   /* hard steps evaluated with candidate loads (in-core) */
    uint64_t coop_large_attempts;
    uint32_t learned_parts;      /* learned out-of-core runs: the GW_LEARNED_* parts this run used */
    float copy_ms;               /* out-of-core with prefetch: time the copy stream spent on block copies
                                    (CUDA events around each upload) */
    uint64_t zero_copy_sectors;  /* 32-byte sectors the zero-copy tail read from mapped host memory (in
                                    h2d_bytes at 32 bytes each) */
} gw_stats;

/* ------------------------------------------------------------------ basics */

int gw_version(void);
const char *gw_status_string(int status);

/* Defaults of apps/Node2vec.cu:35-59 (p 0.5, q 2.0, alpha 0.2, length 30,
 * blocksize 1024 MB, memory 4 GB, walkpersource 1). */
int gw_config_default(gw_config *cfg);

/* Replaces the graph_engine constructor's device set-up
 * (engine/engine.hpp:54-102: initgpugraph, initgpucache, cudarand, initwalk). */
int gw_create(const gw_config *cfg, gw_handle **out);

/* Frees everything the handle owns (the reference never frees its device
 * state: gpu/memory.hpp:179-207 are never called). */
int gw_destroy(gw_handle *h);

int gw_last_error(gw_handle *h, char *buf, size_t n);

/* Update p, q, alpha, length, seed, termination or path mode between runs. */
int gw_set_config(gw_handle *h, const gw_config *cfg);

/* The handle's compute stream (a cudaStream_t), on which every step kernel
 * is launched; callers may record their own CUDA events on it.  The three
 * streams of the reference (gpu_stream, api/types.hpp:174-187) become one
 * compute stream and one copy stream. */
int gw_stream(gw_handle *h, void **stream);

/* ------------------------------------------------------------------ graph */

/* Block table: graph_block (engine/cache.hpp:150-175) from the .vert.blocks /
 * .edge.blocks files (vblocks: nblocks+1 u32, eblocks: nblocks+1 u64). */
int gw_set_graph_meta(gw_handle *h, uint32_t nverts, uint64_t nedges, uint32_t nblocks,
                      const uint32_t *vblocks, const uint64_t *eblocks);

/* Host copy of block blk: beg = its nverts+1 u64 offsets as stored in the
 * .beg file (absolute), csr = its nedges u32 neighbours.  Stands in for
 * graph_driver::load_block_info_all (engine/driver.hpp:71-90); the engine
 * copies from these buffers into device slots (gpu/memory.hpp:124-139). */
int gw_host_block(gw_handle *h, uint32_t blk, const uint64_t *beg, const uint32_t *csr);

/* Whole graph already resident on this device (d_beg: nverts+1, d_csr:
 * nedges), borrowed.  The engine then runs in-core without host copies. */
int gw_device_graph(gw_handle *h, const uint64_t *d_beg, const uint32_t *d_csr);

/* Edge weights (real_t, one per edge as in the reference's <base>.wht,
 * util/util.hpp:136-138), for weighted Node2vec: a step draws its candidate
 * in proportion to the weight of cur -> x (Walker's alias table per vertex,
 * built on the device) and accepts it by the unweighted rule.  The reference
 * loads weights (engine/cache.hpp:71, gpu/memory.hpp:134-137) but never
 * samples with them.  gw_host_weights borrows block blk's weights like
 * gw_host_block (every block with edges needs them before walks are
 * weighted); gw_device_weights gives the weights of a gw_device_graph graph
 * (NULL: unweighted again).  Weighted walks are Node2vec walks.
 * Out-of-core, every block's alias tables are built on the device from its
 * weights at the first run (scratch of 28 bytes per edge of the largest
 * block, freed after) and copied behind its neighbour list with each load
 * (8 bytes per edge, counted in h2d_bytes; the reference copies weights with
 * every block, gpu/memory.hpp:134-137); the zero-copy tail is refused.  A
 * weight that is not positive and finite fails the run with GW_ERR_GRAPH. */
int gw_host_weights(gw_handle *h, uint32_t blk, const float *w);
int gw_device_weights(gw_handle *h, const float *d_w);

/* Drop every cached block so the next run copies the graph from the host
 * blocks again. */
int gw_cache_reset(gw_handle *h);

/* ------------------------------------------------------------------ walks */

/* Replaces graph_walk::gpu_createwalk (engine/walk.hpp:272-389): sets the
 * walker population; walkers are generated on the device. */
int gw_init_walkers(gw_handle *h, uint32_t algo, uint32_t walkpersource, uint64_t seed);

/* One shard of that population: the walkers with ids [first, first+count)
 * of the population gw_init_walkers would set (ids as the reference assigns
 * them, engine/walk.hpp:32-49: v*walkpersource + i per vertex).  A walk
 * depends only on its id and the seed, so shards of one population walked on
 * different devices (or one after another) together give exactly the walks
 * of the whole population.  Per-walker results (gw_get_paths,
 * gw_path_hashes) are then indexed from the shard's first walker: row 0 is
 * walker `first`.  gw_init_walkers is the shard [0, all). */
int gw_init_walker_range(gw_handle *h, uint32_t algo, uint32_t walkpersource, uint64_t seed, uint64_t first,
                         uint64_t count);

/* Runs every walker to the end.  Replaces graph_engine::pipe_run
 * (engine/engine.hpp:517-638) with its pipeline / zero_gpujob launches
 * (406-515): the plain or learned block policy, device bucketing, and the
 * step kernels of gpu/gpuwalk.hpp. */
int gw_run(gw_handle *h, uint32_t policy, gw_stats *stats);

/* Walker count of the current population. */
int gw_num_walkers(gw_handle *h, uint64_t *n);

/* Paths of walkers [first, first+n) of the population (row 0 = its first
 * walker; see gw_init_walker_range): out = n rows of maxhops+1 u32 (zero
 * padded), lens = vertices per row.  Needs record_paths = GW_PATHS_FULL. */
int gw_get_paths(gw_handle *h, uint64_t first, uint64_t n, uint32_t *out, uint32_t *lens);

/* Vertices in each of walkers [first, first+n)'s paths (its steps + 1),
 * whether or not paths were recorded. */
int gw_path_lengths(gw_handle *h, uint64_t first, uint64_t n, uint32_t *lens);

/* 64-bit FNV-1a hash of each walker's path over its 32-bit vertex ids. */
int gw_path_hashes(gw_handle *h, uint64_t first, uint64_t n, uint64_t *out);

/* Hash of all path hashes (order-independent sum) and total steps, read back
 * as 16 bytes: the per-run checksum. */
int gw_checksum(gw_handle *h, uint64_t *hash_sum, uint64_t *steps);

/* Walker counts of the nblocks*nblocks (prev block, cur block) buckets after
 * the last scheduler iteration (walk_block::num, engine/walk.hpp:104-209). */
int gw_bucket_counts(gw_handle *h, uint32_t *out);

/* ------------------------------------------------------------------ graphs on the device */

/* Counter-based R-MAT graph built on the device: samples e in [0, nsamples)
 * take `scale` quadrant choices from Philox(e, level/4) against the u32
 * thresholds thr = {a, a+b, a+b+c} * 2^32.  Samples with an endpoint >=
 * nverts are rejected, self loops dropped, the edge set symmetrised when
 * `symmetric`, duplicates removed, adjacency sorted.  When target_edges is
 * non-zero the sorted unique edge list is thinned evenly to exactly that
 * many edges.  Allocates *d_beg (nverts+1 u64) and *d_csr (nedges u32) with
 * cudaMalloc on the current device; free them with gw_device_free. */
int gw_rmat_csr(uint32_t scale, uint32_t nverts, uint64_t nsamples, const uint32_t thr[3], uint64_t seed,
                int symmetric, uint64_t target_edges, uint64_t **d_beg, uint32_t **d_csr, uint64_t *nedges);

/* Edge list -> CSR on the device, in place of the reference's text-to-CSR
 * pass (graph_converter::convert, preprocess/graph_converter.hpp:286-449) and
 * its optional neighbour sort (sort_vertex_neighbors,
 * preprocess/precompute.hpp:42-133).  Edge i is (src[i], dst[i]); both
 * arrays may be host or device memory.  Self loops are dropped
 * (graph_converter.hpp:362-363).  Flags:
 *   GW_EDGES_SYMMETRIC  edge i also yields (dst[i], src[i]), right after it;
 *   GW_EDGES_SORT       each vertex's neighbours ascending (the `sorted` flag);
 *                       without it a vertex keeps its edges in input order,
 *                       which for a source-sorted list is the converter's CSR;
 *   GW_EDGES_DEDUP      repeated (src, dst) pairs kept once (implies SORT).
 * nverts 0 takes the largest id of a kept edge + 1 (the converter's
 * max_vert + 1); otherwise an id >= nverts fails with GW_ERR_ARG, as does an
 * id of 2^32-1 (no u32 vertex count covers it).  Allocates *d_beg (nverts+1
 * u64) and *d_csr (max(nedges,1) u32) on the current device; free them with
 * gw_device_free. */
#define GW_EDGES_SYMMETRIC 1u
#define GW_EDGES_SORT 2u
#define GW_EDGES_DEDUP 4u
int gw_edges_csr(const uint32_t *src, const uint32_t *dst, uint64_t n, uint32_t nverts, uint32_t flags,
                 uint64_t **d_beg, uint32_t **d_csr, uint64_t *nedges, uint32_t *nverts_out);

/* SOWalker's annealing block choice (SOwalker_scheduler_t::choose_blocks,
 * engine/schedule.hpp:455-593) on the device, exactly as GW_POLICY_SA runs
 * it: counts = nblocks*nblocks walkers per (prev, cur) block pair, cached =
 * the ncached resident blocks, k = cache slots; the annealing draws are
 * Philox4x32-10 (round, call, 0, 'SANN') under `seed` (the reference uses
 * std::rand).  Host memory in and out; writes the min(k, nblocks) chosen
 * blocks to out.  nblocks <= 1024. */
int gw_sa_choose_blocks(const uint32_t *counts, uint32_t nblocks, const uint32_t *cached, uint32_t ncached,
                        uint32_t k, uint64_t seed, uint32_t call, uint32_t *out);

/* GOWalker's block choice, GOwalker_scheduler_t::max_choose_blocks
 * (engine/schedule.hpp:70-138), on the device, exactly as GW_POLICY_PLAIN
 * takes it each iteration: counts = nblocks*nblocks walkers per (prev block,
 * cur block) pair; cached = the scheduler's list of the ncached resident
 * blocks in order (its `buckets`, distinct); nslots = cache slots
 * (graph_cache::ncblock).  out[0] = action: 0 when no block scores above 0
 * and zero_threshold (the reference returns false), 1 when block out[1] is
 * appended to the list (out[2] = ncached), 2 when out[1] replaces the block
 * at list position out[2].  Among equal best scores the lowest block id
 * wins (the reference's std::sort leaves that order open; its insertion sort
 * for at most 16 uncached blocks gives the same).  Host memory in and out;
 * nblocks <= 1024. */
int gw_plain_choose_block(const uint32_t *counts, uint32_t nblocks, const uint32_t *cached, uint32_t ncached,
                          uint32_t nslots, uint32_t zero_threshold, int32_t *out);

/* Block split points over CSR offsets beg[0..nverts] (host or device
 * memory), computed on the device.
 *   GW_SPLIT_REFERENCE   param = block size in bytes: the reference splitter
 *                        (split_blocks, preprocess/split.hpp:15-87), which cuts
 *                        when a block's edges pass param/4 (one vertex back) or
 *                        its vertices reach param/8;
 *   GW_SPLIT_EQUAL_EDGES param = block count: block k ends at the first vertex
 *                        whose offset reaches floor(k*E/param), at least one
 *                        vertex per block.
 * Writes nblocks+1 entries to vblocks (u32) and eblocks (u64), host memory
 * with room for cap+1 each; *nblocks gets the block count.  When it exceeds
 * cap nothing is written and the call fails with GW_ERR_ARG. */
#define GW_SPLIT_REFERENCE 0u
#define GW_SPLIT_EQUAL_EDGES 1u
int gw_split_blocks(const uint64_t *beg, uint32_t nverts, uint32_t mode, uint64_t param, uint32_t *vblocks,
                    uint64_t *eblocks, uint32_t cap, uint32_t *nblocks);

/* Web-shaped synthetic graph on the device (locality-ordered ids, the
 * full-pipeline workload's stand-in), directed.  Vertex v's out-degree is
 * floor(dmin / u^(1/tail)) capped at max_degree, u from Philox(v, 0, 0,
 * 'WDEG') -- a power law P(D >= d) = (d/dmin)^-tail (density exponent
 * 1 + tail), at least floor(dmin) per vertex.  Edge j of v: with probability
 * local_permille/1000 (Philox(j, v, 0, 'WEB0') lane 0 % 1000) it goes to
 * v + o, o uniform over [-window, -1] u [1, window], clipped to [0, nverts);
 * otherwise to a destination drawn from R-MAT's destination marginal over
 * `scale` levels (thr as gw_rmat_csr), rejected when >= nverts.  Self loops
 * and repeats dropped, adjacency sorted, then thinned evenly to target_edges
 * when non-zero (GW_ERR_ARG if fewer edges).  The power and log use fixed
 * IEEE-double steps so a CPU restatement reproduces the graph.  Outputs as
 * gw_rmat_csr. */
int gw_web_csr(uint32_t scale, uint32_t nverts, const uint32_t thr[3], double dmin, double tail, uint32_t max_degree,
               uint32_t local_permille, uint32_t window, uint64_t seed, uint64_t target_edges, uint64_t **d_beg,
               uint32_t **d_csr, uint64_t *nedges);

int gw_device_free(void *p);

/* Pinned host memory for graph blocks and walker batches, in place of the
 * reference's cudaHostAlloc calls (engine/cache.hpp:106-120,
 * api/graph_buffer.hpp:26-32), so a host program needs no CUDA runtime of its
 * own. */
int gw_host_alloc(uint64_t bytes, void **out);
int gw_host_free(void *p);

/* ------------------------------------------------------------------ block-demand predictor */

/* No counterpart in the reference (its block choice is the fixed rule of
 * engine/schedule.hpp:70-138): the learned policy's network, a 16 -> 64 ->
 * 64 -> 1 ReLU MLP in fp32 (GW_MLP_PARAMS weights, layout W1[64][16], b1[64],
 * W2[64][64], b2[64], W3[64], b3).  These calls run its hand-written kernels on
 * caller-owned device buffers (synchronous, default stream); the engine uses
 * the same kernels internally for GW_POLICY_LEARNED. */
#define GW_MLP_INPUTS 16
#define GW_MLP_PARAMS 5313
#define GW_MLP_GRAD_WS_FLOATS (32 * (GW_MLP_PARAMS + 1))

/* y[i] = mlp(x[i]) for n rows of GW_MLP_INPUTS floats. */
int gw_mlp_forward(const float *d_params, const float *d_x, uint32_t n, float *d_y);

/* Gradient of the mean squared error over n rows: d_grad (GW_MLP_PARAMS
 * floats), d_loss (1 float), workspace d_ws (GW_MLP_GRAD_WS_FLOATS floats). */
int gw_mlp_grad(const float *d_params, const float *d_x, const float *d_t, uint32_t n, float *d_grad, float *d_loss,
                float *d_ws);

/* Full-batch Adam for `epochs` steps at learning rate lr; seed != 0 first
 * re-initialises d_params.  d_ws holds GW_MLP_GRAD_WS_FLOATS + 3 *
 * GW_MLP_PARAMS + 1 floats.  *loss_out receives the final loss. */
int gw_mlp_train(float *d_params, const float *d_x, const float *d_t, uint32_t n, uint32_t epochs, float lr,
                 uint64_t seed, float *d_ws, float *loss_out);

/* ------------------------------------------------------------------ no-allocation walk */

/* No counterpart in the reference: an entry point for callers that cannot
 * let a library allocate device memory -- a plugin whose host owns all device
 * memory through its own pool, a runtime that forbids allocation after
 * start-up, a host language that manages the buffers itself.
 *
 * Walks every walker of `cfg` (algorithm, p, q, alpha, maxhops, term_prob,
 * seed, init_mode, walkpersource, numwalks, record_paths, blockpergrid,
 * device) over a CSR already on the device (d_beg: nverts+1 u64 offsets,
 * d_csr: nedges u32 ids, sorted per vertex), writing the caller's buffers:
 * d_hashes (nwalkers u64), d_lens (nwalkers u32) and, when record_paths is
 * GW_PATHS_FULL, d_paths (nwalkers rows of maxhops+1 u32, zero past each
 * walk's length, as gw_get_paths returns them).  The walks are the ones
 * gw_run produces for the same configuration, bit for bit.
 *
 * Allocates nothing: no cudaMalloc, no cudaFree, no allocating library call.
 * Its only other memory is a 256-byte array in the library (the run's work
 * cursor and counters, and the error word), which every device that loads
 * the library holds until the process exits and which this call clears
 * before use.  That array never grows: the size limits are the walk's own --
 * nwalkers must equal the population cfg implies and stay below 2^32 (walker
 * ids are 32-bit), otherwise the call returns GW_ERR_ARG without touching the
 * device.
 *
 * The first call on a device looks up the array's device address with that
 * device current (again after the device's context changes, e.g. after a
 * cudaDeviceReset); make that first call before any stream capture.  The
 * calling thread's current device is the same on return as before.  The call
 * runs on `stream` (a cudaStream_t, 0 for the default stream) and returns
 * after the walk has finished; it first checks the CSR (GW_ERR_GRAPH if
 * offsets are not monotone or an id is out of range).  Every call shares the
 * one array, so calls that overlap on the same device -- from two host
 * threads -- race: serialise them.  `stats` may be NULL. */
int gw_walk_noalloc(const gw_config *cfg, const uint64_t *d_beg, const uint32_t *d_csr, uint32_t nverts,
                    uint64_t nedges, uint64_t nwalkers, uint64_t *d_hashes, uint32_t *d_lens, uint32_t *d_paths,
                    void *stream, gw_stats *stats);

/* Issue rate of the walk's random draws on `device`: every thread evaluates
 * the step kernels' keyed Philox4x32-10 (per_thread evaluations, nothing
 * else), timed with CUDA events, best of three launches after a warm-up one.
 * *evals_per_s is the bound on rejection trials per second of any kernel
 * that draws once per trial; *ms (may be NULL) the best launch time.  No
 * counterpart in the reference (a measurement for the roofline of
 * trial-bound walks). */
int gw_philox_rate(int device, uint32_t per_thread, double *evals_per_s, float *ms);

/* Plain copy between any two host / device pointers (cudaMemcpyDefault),
 * synchronous: lets callers without their own CUDA runtime move the buffers
 * gw_rmat_csr returns. */
int gw_memcpy(void *dst, const void *src, uint64_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* GOWALKER_H */
