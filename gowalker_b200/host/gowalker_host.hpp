// C++ host side of the walk engine with GOWalker's interfaces.
//
// The classes keep the reference's names, members and call sequence so code
// written against GOWalker's engine reads the same (apps/Node2vec.cu:109-185):
//
//   graph_config conf{...};                 engine/config.hpp:7-34
//   metrics m(name);                        metrics/metrics.hpp:160-332
//   graph_block blocks(&conf);              engine/cache.hpp:144-193
//   graph_driver driver(&conf, m);          engine/driver.hpp:15-133
//   scheduler *s = new GOwalker_scheduler_t(m);   engine/schedule.hpp:58-366
//   graph_walk walk(conf, driver, blocks);  engine/walk.hpp:211-563
//   graph_cache cache(blocks.nblocks, bs), g_cache(nmblocks, bs);
//   graph_engine engine(cache, walk, driver, conf, m, g_cache, s);
//   engine.prologue(); engine.pipe_run(); engine.epilogue();
//   metrics_report(m);
//
// Underneath, every device action goes through the C ABI of libgowalker.so
// (include/gowalker.h): the host never launches a kernel itself.
#pragma once
#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <vector>
#include "gowalker.h"

typedef uint32_t vid_t;
typedef uint64_t eid_t;
typedef uint32_t bid_t;
typedef uint32_t hid_t;
typedef uint16_t tid_t;
typedef uint32_t wid_t;
typedef float real_t;
typedef enum { node2vec, SOPR, SOSR } AlgorithmType;  // api/types.hpp:27

// ---------------------------------------------------------------- cmdopts
// `name value` pairs and presence-only flags, scanned from the end of argv
// (api/cmdopts.hpp:108-246); `--key=value` pairs land in a map.
void set_argc(int argc, const char **argv);
int get_option_int(const char *name, int default_value);
uint64_t get_option_long(const char *name, uint64_t default_value);
float get_option_float(const char *name, float default_value);
std::string get_option_string(const char *name, const std::string &default_value);
bool get_option_bool(const char *name);
bool option_given(const char *name);

// ---------------------------------------------------------------- config
struct graph_config {  // field order of engine/config.hpp:7-34
    std::string base_name;
    size_t cache_size;
    size_t blocksize;
    tid_t nthreads;
    tid_t max_nthreads;
    vid_t nvertices;
    eid_t nedges;
    vid_t min_vert;
    bool is_weighted;
    wid_t numwalks;
    size_t walkpersource;
    size_t blockpergrid;
    size_t threadperblock;
    size_t cpu_threads;
    AlgorithmType algorithm;
    real_t p;
    real_t q;
    real_t alpha;
    hid_t maxhops;
    wid_t cpu_batch;
    wid_t gpu_batch;
    wid_t zero_threshold;
    bool gpu_schedule;
    bool cpu_schedule;
    bool walkaware;
};

// Settings the reference does not have (termination, seed, policy, device,
// path output), filled from the new flags.
struct walk_extras {
    float term_prob = 0.0f;
    uint64_t seed = 42;
    bool learned = false;
    bool zero_copy = false;
    int device = 0;
    uint32_t init_mode = GW_INIT_PER_VERTEX;
    std::string paths_file;      // text rows "v0 v1 ...", one walker per line
    std::string paths_bin_file;  // u32 rows of maxhops+1 then u32 lengths
    uint32_t launch_grid = 0;    // blockpergrid when given explicitly
};

// ---------------------------------------------------------------- metrics
// Name/value and timer entries written in the reference's file-reporter
// format (metrics/reps/file_reporter.hpp:56-90) so its scripts still parse.
class metrics {
public:
    explicit metrics(std::string name = "");
    void set(const std::string &key, double value);
    void set(const std::string &key, const std::string &value);
    void start_time(const std::string &key);
    void stop_time(const std::string &key);
    void add_time(const std::string &key, double seconds);
    double get(const std::string &key) const;
    void report(FILE *console, const std::string &file) const;
    std::string name;

private:
    struct entry {
        double value = 0, minv = 0, maxv = 0, sum = 0;
        size_t count = 0;
        bool is_time = false, is_string = false;
        std::string s;
        double started = 0;
    };
    std::map<std::string, entry> entries_;
};
void metrics_report(metrics &m);

// ---------------------------------------------------------------- graph
struct block_t {  // engine/cache.hpp:32-61
    bid_t blk = 0, cache_index = 0;
    vid_t start_vert = 0, nverts = 0;
    eid_t start_edge = 0, nedges = 0;
};

class graph_block {  // engine/cache.hpp:144-193
public:
    explicit graph_block(graph_config *conf);
    bid_t get_block(vid_t v) const;
    bid_t nblocks = 0;
    std::vector<block_t> blocks;
    std::vector<uint32_t> vblocks;
    std::vector<uint64_t> eblocks;
};

struct cache_block {  // engine/cache.hpp:63-121: pinned host copy of one block
    block_t *block = nullptr;
    eid_t *beg_pos = nullptr;
    vid_t *csr = nullptr;
    real_t *weights = nullptr;  // with `weighted`: <base>.wht, one real_t per edge
};

class graph_cache {  // engine/cache.hpp:195-223
public:
    graph_cache() = default;
    graph_cache(bid_t nblocks, size_t blocksize);
    ~graph_cache();
    graph_cache(const graph_cache &) = delete;
    graph_cache &operator=(const graph_cache &) = delete;
    bid_t ncblock = 0;
    std::vector<cache_block> cache_blocks;
};

class graph_driver {  // engine/driver.hpp:15-133: pread of block ranges
public:
    graph_driver(graph_config *conf, metrics &m);
    ~graph_driver();
    void load_block_info_all(graph_cache &cache, graph_block *global_blocks, bid_t cache_index, bid_t block_index,
                             size_t blocksize);
    int vertdesc = -1, edgedesc = -1, whtdesc = -1;
    bool _weighted = false;
    metrics &_m;
};

// ---------------------------------------------------------------- walks
class graph_walk {  // engine/walk.hpp:211-563: the walker population
public:
    graph_walk(graph_config &conf, graph_driver &driver, graph_block &blocks);
    wid_t nwalks() const { return remaining; }
    size_t numwalks;
    wid_t cpu_batch, gpu_batch;
    bid_t nblocks, totblocks;
    graph_block *global_blocks;
    wid_t remaining = 0;
};

class scheduler {  // engine/schedule.hpp:38-55
public:
    explicit scheduler(metrics &m) : _m(m) {}
    virtual ~scheduler() = default;
    virtual uint32_t policy() const { return GW_POLICY_PLAIN; }
    std::vector<bid_t> buckets;
    std::vector<bid_t> cpu_blk;

protected:
    metrics &_m;
};

class GOwalker_scheduler_t : public scheduler {  // engine/schedule.hpp:58-366 (plain rule on the device)
public:
    explicit GOwalker_scheduler_t(metrics &m, bool learned = false) : scheduler(m), learned_(learned) {}
    uint32_t policy() const override { return learned_ ? GW_POLICY_LEARNED : GW_POLICY_PLAIN; }

private:
    bool learned_;
};

class SOwalker_scheduler_t : public scheduler {  // engine/schedule.hpp:369-621 (annealing on the device)
public:
    explicit SOwalker_scheduler_t(metrics &m) : scheduler(m) {}
    uint32_t policy() const override { return GW_POLICY_SA; }
};

// ---------------------------------------------------------------- engine
class graph_engine {  // engine/engine.hpp:34-639
public:
    graph_engine(graph_cache &cache, graph_walk &manager, graph_driver &driver, graph_config &conf, metrics &m,
                 graph_cache &g_cache, scheduler *sched, const walk_extras &extras = walk_extras());
    ~graph_engine();
    void prologue();
    void pipe_run();
    void epilogue();
    int status() const { return status_; }
    const gw_stats &stats() const { return stats_; }
    std::string last_error() const;

    graph_cache *cache;
    graph_walk *walk_manager;
    graph_driver *driver;
    graph_config *conf;
    scheduler *block_scheduler;
    graph_cache *h_cache;

private:
    int check(int st, const char *what);
    void write_paths();
    metrics &_m;
    walk_extras extras_;
    gw_handle *h_ = nullptr;
    gw_stats stats_{};
    int status_ = GW_OK;
};

// The shared main of the Node2vec / SOPR / SOSR apps (apps/Node2vec.cu:22-187).
int walk_app_main(int argc, const char **argv, AlgorithmType algo);

// The reference's block splitter (preprocess/split.hpp:15-87), used when the
// dataset has no block files for the chosen block size.
size_t split_blocks(const std::string &base_name, size_t block_size);
std::string get_vert_blocks_name(const std::string &base_name, size_t blocksize);
std::string get_edge_blocks_name(const std::string &base_name, size_t blocksize);
std::string remove_extension(const std::string &filename);
