// C++ host side with GOWalker's interfaces (see gowalker_host.hpp).
#include "gowalker_host.hpp"

#include <fcntl.h>
#include <sys/stat.h>
#include <sys/time.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

// ---------------------------------------------------------------- cmdopts

static int g_argc = 0;
static const char **g_argv = nullptr;
static std::map<std::string, std::string> g_kv;  // --key=value pairs

void set_argc(int argc, const char **argv)
{
    g_argc = argc;
    g_argv = argv;
    g_kv.clear();
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a.compare(0, 2, "--") == 0) {
            const size_t eq = a.find('=');
            if (eq != std::string::npos) g_kv[a.substr(2, eq - 2)] = a.substr(eq + 1);
        }
    }
}

static const char *find_value(const char *name)
{
    for (int i = g_argc - 2; i >= 0; --i)
        if (std::strcmp(g_argv[i], name) == 0) return g_argv[i + 1];
    auto it = g_kv.find(name);
    return it == g_kv.end() ? nullptr : it->second.c_str();
}

int get_option_int(const char *name, int d)
{
    const char *v = find_value(name);
    return v ? std::atoi(v) : d;
}
uint64_t get_option_long(const char *name, uint64_t d)
{
    const char *v = find_value(name);
    return v ? (uint64_t)std::atol(v) : d;
}
float get_option_float(const char *name, float d)
{
    const char *v = find_value(name);
    return v ? (float)std::atof(v) : d;
}
std::string get_option_string(const char *name, const std::string &d)
{
    const char *v = find_value(name);
    return v ? std::string(v) : d;
}
bool get_option_bool(const char *name)
{
    for (int i = g_argc - 1; i >= 0; --i)
        if (std::strcmp(g_argv[i], name) == 0) return true;
    return false;
}
bool option_given(const char *name) { return find_value(name) != nullptr; }

// ---------------------------------------------------------------- metrics

static double now_seconds()
{
    timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + tv.tv_usec * 1e-6;
}

metrics::metrics(std::string n) : name(std::move(n)) { set("app", name); }

void metrics::set(const std::string &key, double v)
{
    entry &e = entries_[key];
    e.value = v;
    if (e.count == 0 || v < e.minv) e.minv = v;
    if (e.count == 0 || v > e.maxv) e.maxv = v;
    e.sum += v;
    e.count++;
}

void metrics::set(const std::string &key, const std::string &v)
{
    entry &e = entries_[key];
    e.is_string = true;
    e.s = v;
}

void metrics::start_time(const std::string &key)
{
    entry &e = entries_[key];
    e.is_time = true;
    e.started = now_seconds();
}

void metrics::stop_time(const std::string &key)
{
    entry &e = entries_[key];
    add_time(key, now_seconds() - e.started);
}

void metrics::add_time(const std::string &key, double secs)
{
    entry &e = entries_[key];
    e.is_time = true;
    e.value += secs;  // a timer accumulates, like metrics_entry::add for TIME entries
    if (e.count == 0 || secs < e.minv) e.minv = secs;
    if (e.count == 0 || secs > e.maxv) e.maxv = secs;
    e.sum += secs;
    e.count++;
}

double metrics::get(const std::string &key) const
{
    auto it = entries_.find(key);
    return it == entries_.end() ? 0.0 : it->second.value;
}

void metrics::report(FILE *console, const std::string &file) const
{
    if (console) {
        fprintf(console, "=== REPORT FOR %s ===\n", name.c_str());
        for (const auto &kv : entries_) {
            if (kv.second.is_string) fprintf(console, "%s: %s\n", kv.first.c_str(), kv.second.s.c_str());
            else fprintf(console, "%s: %lf\n", kv.first.c_str(), kv.second.value);
        }
    }
    if (file.empty()) return;
    FILE *f = fopen(file.c_str(), "a");
    if (!f) return;
    fprintf(f, "[%s:]\n", name.c_str());
    for (const auto &kv : entries_) {
        const entry &e = kv.second;
        const char *k = kv.first.c_str();
        if (e.is_string) {
            fprintf(f, ".%s=%s\n", k, e.s.c_str());
            continue;
        }
        const size_t n = e.count ? e.count : 1;
        fprintf(f, ".%s=%lf\n.%s.count=%lu\n.%s.min=%lf\n.%s.max=%lf\n.%s.avg=%lf\n", k, e.value, k,
                (unsigned long)e.count, k, e.minv, k, e.maxv, k, e.sum / (double)n);
    }
    fclose(f);
}

void metrics_report(metrics &m)
{
    m.report(stdout, get_option_string("metrics.reporter.filename", "randgraph_metrics.txt"));
}

// ---------------------------------------------------------------- names and files

std::string remove_extension(const std::string &filename)
{
    const size_t p = filename.find_last_of('.');
    return (p > 0 && p != std::string::npos) ? filename.substr(0, p) : filename;
}

static std::string block_folder(const std::string &base, size_t blocksize)
{
    const size_t p = base.rfind('/');
    const std::string dir = (p == std::string::npos) ? "./" : base.substr(0, p + 1);
    return dir + "sowalker_" + std::to_string(blocksize / (1024 * 1024));
}

static std::string file_part(const std::string &base)
{
    const size_t p = base.rfind('/');
    return p == std::string::npos ? base : base.substr(p + 1);
}

std::string get_vert_blocks_name(const std::string &base, size_t blocksize)
{
    return block_folder(base, blocksize) + "/" + file_part(base) + "_" + std::to_string(blocksize / (1024 * 1024)) +
           "MB.vert.blocks";
}

std::string get_edge_blocks_name(const std::string &base, size_t blocksize)
{
    return block_folder(base, blocksize) + "/" + file_part(base) + "_" + std::to_string(blocksize / (1024 * 1024)) +
           "MB.edge.blocks";
}

template <typename T>
static std::vector<T> read_all(const std::string &path)
{
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    fseek(f, 0, SEEK_END);
    const long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<T> v((size_t)n / sizeof(T));
    if (!v.empty() && fread(v.data(), sizeof(T), v.size(), f) != v.size()) {
        fclose(f);
        throw std::runtime_error("short read of " + path);
    }
    fclose(f);
    return v;
}

static void read_range(int fd, void *buf, size_t bytes, off_t off)
{
    char *p = (char *)buf;
    size_t done = 0;
    while (done < bytes) {
        const ssize_t r = pread(fd, p + done, bytes - done, off + (off_t)done);
        if (r <= 0) throw std::runtime_error("pread failed or short file");
        done += (size_t)r;
    }
}

static void load_meta(const std::string &base, vid_t *nv, eid_t *ne, vid_t *minv)
{
    FILE *f = fopen((base + ".meta").c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + base + ".meta");
    const bool ok = fread(nv, 4, 1, f) == 1 && fread(ne, 8, 1, f) == 1 && fread(minv, 4, 1, f) == 1;
    fclose(f);
    if (!ok) throw std::runtime_error(base + ".meta: expected 16 bytes");
}

size_t split_blocks(const std::string &base, size_t block_size)
{
    const std::vector<eid_t> beg = read_all<eid_t>(base + ".beg");
    if (beg.empty()) throw std::runtime_error(base + ".beg is empty");
    const size_t max_nedges = block_size / sizeof(vid_t), max_nverts = block_size / sizeof(eid_t);
    std::vector<vid_t> vb{0};
    std::vector<eid_t> eb{0};
    vid_t cur_pos = 0;
    eid_t rd_edges = 0;
    const size_t nv = beg.size();  // V+1 offsets: the reference's "nvertices"
    for (size_t v = 0; v < nv; ++v) {
        if (beg[v] - rd_edges > max_nedges && v > 0) {
            cur_pos = (vid_t)(v - 1);
            vb.push_back(cur_pos);
            rd_edges = beg[v - 1];
            eb.push_back(rd_edges);
        } else if (v - cur_pos >= max_nverts) {
            cur_pos = (vid_t)v;
            vb.push_back(cur_pos);
            rd_edges = beg[v];
            eb.push_back(rd_edges);
        }
    }
    vb.push_back((vid_t)(nv - 1));
    eb.push_back(beg[nv - 1]);
    mkdir(block_folder(base, block_size).c_str(), 0777);
    FILE *f = fopen(get_vert_blocks_name(base, block_size).c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write the vertex block file");
    fwrite(vb.data(), sizeof(vid_t), vb.size(), f);
    fclose(f);
    f = fopen(get_edge_blocks_name(base, block_size).c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write the edge block file");
    fwrite(eb.data(), sizeof(eid_t), eb.size(), f);
    fclose(f);
    return vb.size() - 1;
}

// ---------------------------------------------------------------- graph

graph_block::graph_block(graph_config *conf)
{
    vblocks = read_all<uint32_t>(get_vert_blocks_name(conf->base_name, conf->blocksize));
    eblocks = read_all<uint64_t>(get_edge_blocks_name(conf->base_name, conf->blocksize));
    if (vblocks.size() < 2 || vblocks.size() != eblocks.size())
        throw std::runtime_error("block files are missing or disagree");
    nblocks = (bid_t)vblocks.size() - 1;
    blocks.resize(nblocks);
    for (bid_t b = 0; b < nblocks; ++b) {
        blocks[b].blk = b;
        blocks[b].cache_index = nblocks;
        blocks[b].start_vert = vblocks[b];
        blocks[b].nverts = vblocks[b + 1] - vblocks[b];
        blocks[b].start_edge = eblocks[b];
        blocks[b].nedges = eblocks[b + 1] - eblocks[b];
    }
}

bid_t graph_block::get_block(vid_t v) const
{
    // binary search instead of the reference's linear scan (engine/cache.hpp:183-192)
    const auto it = std::upper_bound(vblocks.begin(), vblocks.end(), v);
    const bid_t b = (bid_t)(it - vblocks.begin());
    return b == 0 ? nblocks : std::min<bid_t>(b - 1, nblocks);
}

graph_cache::graph_cache(bid_t n, size_t) : ncblock(n), cache_blocks(n) {}

graph_cache::~graph_cache()
{
    for (auto &c : cache_blocks) {
        gw_host_free(c.beg_pos);
        gw_host_free(c.csr);
        gw_host_free(c.weights);
    }
}

graph_driver::graph_driver(graph_config *conf, metrics &m) : _m(m)
{
    vertdesc = open((conf->base_name + ".beg").c_str(), O_RDONLY);
    edgedesc = open((conf->base_name + ".csr").c_str(), O_RDONLY);
    _weighted = conf->is_weighted;
    if (vertdesc < 0 || edgedesc < 0) throw std::runtime_error("cannot open " + conf->base_name + ".beg/.csr");
    if (_weighted) {  // util/util.hpp:136-138
        whtdesc = open((conf->base_name + ".wht").c_str(), O_RDONLY);
        if (whtdesc < 0) throw std::runtime_error("weighted: cannot open " + conf->base_name + ".wht");
    }
}

graph_driver::~graph_driver()
{
    if (vertdesc >= 0) close(vertdesc);
    if (edgedesc >= 0) close(edgedesc);
    if (whtdesc >= 0) close(whtdesc);
}

void graph_driver::load_block_info_all(graph_cache &cache, graph_block *gb, bid_t ci, bid_t bi, size_t)
{
    cache_block &c = cache.cache_blocks[ci];
    block_t &b = gb->blocks[bi];
    c.block = &b;
    void *p = nullptr;
    if (gw_host_alloc((b.nverts + 1) * sizeof(eid_t), &p) != GW_OK) throw std::runtime_error("pinned allocation");
    c.beg_pos = (eid_t *)p;
    read_range(vertdesc, c.beg_pos, (b.nverts + 1) * sizeof(eid_t), (off_t)b.start_vert * sizeof(eid_t));
    if (b.nedges) {
        if (gw_host_alloc(b.nedges * sizeof(vid_t), &p) != GW_OK) throw std::runtime_error("pinned allocation");
        c.csr = (vid_t *)p;
        read_range(edgedesc, c.csr, b.nedges * sizeof(vid_t), (off_t)b.start_edge * sizeof(vid_t));
        if (_weighted) {
            if (gw_host_alloc(b.nedges * sizeof(real_t), &p) != GW_OK) throw std::runtime_error("pinned allocation");
            c.weights = (real_t *)p;
            read_range(whtdesc, c.weights, b.nedges * sizeof(real_t), (off_t)b.start_edge * sizeof(real_t));
        }
    }
}

graph_walk::graph_walk(graph_config &conf, graph_driver &, graph_block &blocks)
    : numwalks(conf.numwalks), cpu_batch(conf.cpu_batch), gpu_batch(conf.gpu_batch), nblocks(blocks.nblocks),
      totblocks(blocks.nblocks * blocks.nblocks), global_blocks(&blocks)
{
}

// ---------------------------------------------------------------- engine

graph_engine::graph_engine(graph_cache &_cache, graph_walk &manager, graph_driver &_driver, graph_config &_conf,
                           metrics &m, graph_cache &_g_cache, scheduler *sched, const walk_extras &extras)
    : cache(&_cache), walk_manager(&manager), driver(&_driver), conf(&_conf), block_scheduler(sched),
      h_cache(&_g_cache), _m(m), extras_(extras)
{
    gw_config c;
    gw_config_default(&c);
    c.cache_size = conf->cache_size;
    c.blocksize = conf->blocksize;
    c.algorithm = (uint32_t)conf->algorithm;
    c.p = conf->p;
    c.q = conf->q;
    c.alpha = conf->alpha;
    c.maxhops = conf->maxhops;
    c.walkpersource = (uint32_t)conf->walkpersource;
    c.numwalks = conf->numwalks;
    c.blockpergrid = extras.launch_grid;
    c.zero_threshold = conf->zero_threshold;
    c.zero_copy = extras.zero_copy ? 1u : 0u;
    c.init_mode = extras.init_mode;
    c.term_prob = extras.term_prob;
    c.seed = extras.seed;
    c.record_paths = (extras.paths_file.empty() && extras.paths_bin_file.empty()) ? GW_PATHS_NONE : GW_PATHS_FULL;
    c.device = extras.device;
    if (check(gw_create(&c, &h_), "gw_create")) return;
    graph_block *gb = walk_manager->global_blocks;
    _m.set("Graph blocks", (double)gb->nblocks);
    _m.set("Gpu memory blocks", (double)h_cache->ncblock);
    if (check(gw_set_graph_meta(h_, conf->nvertices, conf->nedges, gb->nblocks, gb->vblocks.data(),
                                gb->eblocks.data()),
              "gw_set_graph_meta"))
        return;
    // every block in pinned host memory, as the reference does (engine/engine.hpp:74-77)
    for (bid_t b = 0; b < cache->ncblock; ++b) {
        driver->load_block_info_all(*cache, gb, b, b, conf->blocksize);
        if (check(gw_host_block(h_, b, cache->cache_blocks[b].beg_pos, cache->cache_blocks[b].csr), "gw_host_block"))
            return;
        if (driver->_weighted && gb->eblocks[b + 1] > gb->eblocks[b] &&
            check(gw_host_weights(h_, b, cache->cache_blocks[b].weights), "gw_host_weights"))
            return;
    }
}

graph_engine::~graph_engine()
{
    if (h_) gw_destroy(h_);
}

int graph_engine::check(int st, const char *what)
{
    if (st != GW_OK && status_ == GW_OK) {
        status_ = st;
        char msg[512] = "";
        if (h_) gw_last_error(h_, msg, sizeof msg);
        fprintf(stderr, "%s failed: %s (%s)\n", what, gw_status_string(st), msg);
    }
    return st;
}

std::string graph_engine::last_error() const
{
    char msg[512] = "";
    if (h_) gw_last_error(h_, msg, sizeof msg);
    return msg;
}

void graph_engine::prologue()
{
    if (status_ != GW_OK) return;
    if (check(gw_init_walkers(h_, (uint32_t)conf->algorithm, (uint32_t)conf->walkpersource, extras_.seed),
              "gw_init_walkers"))
        return;
    uint64_t n = 0;
    gw_num_walkers(h_, &n);
    walk_manager->remaining = (wid_t)n;
}

void graph_engine::pipe_run()
{
    if (status_ != GW_OK) return;
    _m.start_time("0_Total_time");
    const int st = gw_run(h_, block_scheduler->policy(), &stats_);
    _m.stop_time("0_Total_time");
    if (check(st, "gw_run")) return;
    walk_manager->remaining = 0;
    // the reference's phase keys (engine/engine.hpp:408-447, 536-636)
    _m.add_time("1_GPUTime", stats_.total_ms / 1e3);
    _m.add_time("1.3_GPU_update", stats_.kernel_ms / 1e3);
    _m.add_time("1.1_transfer", std::max(0.0, (stats_.total_ms - stats_.kernel_ms) / 1e3));
    _m.add_time("2_CPUTime", 0.0);
    _m.add_time("3_Zero_Time", 0.0);
    _m.set("steps", (double)stats_.steps);
    _m.set("steps_per_sec", stats_.total_ms > 0 ? stats_.steps / (stats_.total_ms / 1e3) : 0.0);
    _m.set("h2d_bytes", (double)stats_.h2d_bytes);
    _m.set("h2d_bytes_per_step", stats_.steps ? (double)stats_.h2d_bytes / stats_.steps : 0.0);
    _m.set("block_loads", (double)stats_.block_loads);
    _m.set("iterations", (double)stats_.iterations);
    _m.set("trials", (double)stats_.trials);
    uint64_t hs = 0, steps = 0;
    gw_checksum(h_, &hs, &steps);
    char buf[32];
    snprintf(buf, sizeof buf, "%016llx", (unsigned long long)hs);
    _m.set("path_hash_sum", std::string(buf));
}

void graph_engine::write_paths()
{
    uint64_t n = 0;
    gw_num_walkers(h_, &n);
    const uint32_t stride = conf->maxhops + 1;
    const uint64_t chunk = 1 << 16;
    std::vector<uint32_t> rows(chunk * stride), lens(chunk);
    FILE *ft = extras_.paths_file.empty() ? nullptr : fopen(extras_.paths_file.c_str(), "w");
    FILE *fb = extras_.paths_bin_file.empty() ? nullptr : fopen(extras_.paths_bin_file.c_str(), "wb");
    std::vector<uint32_t> all_lens;
    for (uint64_t first = 0; first < n; first += chunk) {
        const uint64_t k = std::min(chunk, n - first);
        if (check(gw_get_paths(h_, first, k, rows.data(), lens.data()), "gw_get_paths")) break;
        for (uint64_t w = 0; w < k; ++w) {
            if (ft) {
                for (uint32_t j = 0; j < lens[w]; ++j) fprintf(ft, j ? " %u" : "%u", rows[w * stride + j]);
                fputc('\n', ft);
            }
        }
        if (fb) fwrite(rows.data(), sizeof(uint32_t), k * stride, fb);
        all_lens.insert(all_lens.end(), lens.begin(), lens.begin() + k);
    }
    if (fb) {
        fwrite(all_lens.data(), sizeof(uint32_t), all_lens.size(), fb);
        fclose(fb);
    }
    if (ft) fclose(ft);
}

void graph_engine::epilogue()
{
    if (status_ != GW_OK) return;
    if (!extras_.paths_file.empty() || !extras_.paths_bin_file.empty()) write_paths();
    fprintf(stdout, "walks: %llu walkers, %llu steps, %.3f ms (%.3e steps/s), h2d %.3e bytes/step\n",
            (unsigned long long)stats_.walkers, (unsigned long long)stats_.steps, stats_.total_ms,
            stats_.total_ms > 0 ? stats_.steps / (stats_.total_ms / 1e3) : 0.0,
            stats_.steps ? (double)stats_.h2d_bytes / stats_.steps : 0.0);
}

// ---------------------------------------------------------------- the apps

static void print_help()
{
    printf("- dataset:       the dataset path (<base>.beg/.csr/.meta in GOWalker's format)\n"
           "- weighted:      read <base>.wht (one float per edge): Node2vec draws each step in proportion to the\n"
           "                 edge weights (in-core); the reference loads weights but never samples with them\n"
           "- sorted:        whether the vertex neighbors are sorted (required)\n"
           "- skip:          use the preprocessed files as they are\n"
           "- blocksize:     the size (MB) of each block\n"
           "- memory:        the size (GB) of the device block cache\n"
           "- walkpersource: the number of walks for each vertex\n"
           "- numwalks:      total walks (overrides walkpersource)\n"
           "- length:        the number of steps of each walk\n"
           "- p, q:          node2vec parameters; alpha: SOPR/SOSR parameter\n"
           "- zero:          finish stragglers through mapped host memory (zero_threshold per block size)\n"
           "- GOWalker / SOWalker: block choice by the GOWalker rule or by SOWalker's annealed block set\n"
           "  (both on the device); gpu cpu walkaware: accepted, no effect\n"
           "- learned:       GOWalker's block choice with learned parts: the zero-copy switch priced by\n"
           "                 measured costs and eviction by a trained forecast (chosen run by run; the\n"
           "                 plain rule judges)\n"
           "- termination F: stop each walk with probability F per step (SOPR/SOSR workloads)\n"
           "- seed N, device N, keepblocks, persource, paths FILE, pathsbin FILE\n"
           "- h:             print this message\n");
}

int walk_app_main(int argc, const char **argv, AlgorithmType algo)
{
    if (argc < 2) {
        print_help();
        return 1;
    }
    set_argc(argc, argv);
    if (get_option_bool("h")) {
        print_help();
        return 0;
    }
    try {
        const std::string input = argv[1];
        const bool weighted = get_option_bool("weighted");
        const size_t blocksize_MB = get_option_long("blocksize", 1024);
        const size_t memory_size = get_option_int("memory", 4);
        wid_t walkpersource = (wid_t)get_option_int("walkpersource", 1);
        wid_t numwalks = (wid_t)get_option_int("numwalks", 0);
        const hid_t steps = (hid_t)get_option_int("length", 30);
        const real_t p = get_option_float("p", 0.5f);
        const real_t q = get_option_float("q", 2.0f);
        const real_t alpha = get_option_float("alpha", 0.2f);
        const size_t threadperblock = get_option_int("threadperblock", 512);
        const size_t blockpergrid = get_option_int("blockpergrid", 512);
        const size_t nthreads = get_option_int("nthreads", 70);
        const size_t cpu_threads = get_option_int("cpu_threads", 32);
        const wid_t walk_batch = get_option_int("walk_batch", 4096);
        wid_t zero_threshold = (wid_t)get_option_float("zero_threshold", algo == node2vec ? 2097152.f : 0.f);
        const bool zero = get_option_bool("zero");
        const bool gpu_schedule = get_option_bool("gpu");
        const bool cpu_schedule = get_option_bool("cpu");
        const bool walkaware = get_option_bool("walkaware");
        const bool GOWalker = get_option_bool("GOWalker");
        const bool SOWalker = get_option_bool("SOWalker");
        walk_extras ex;
        ex.term_prob = get_option_float("termination", 0.f);
        ex.seed = get_option_long("seed", 42);
        ex.learned = get_option_bool("learned");
        ex.device = get_option_int("device", 0);
        ex.paths_file = get_option_string("paths", "");
        ex.paths_bin_file = get_option_string("pathsbin", "");
        ex.launch_grid = option_given("blockpergrid") ? (uint32_t)blockpergrid : 0u;

        const std::string base_name = remove_extension(input);
        const size_t blocksize = blocksize_MB * 1024 * 1024;
        // the reference always re-splits blocks after conversion (preprocess/graph_converter.hpp:437-440)
        struct stat sb;
        if (!(get_option_bool("keepblocks") && stat(get_vert_blocks_name(base_name, blocksize).c_str(), &sb) == 0))
            split_blocks(base_name, blocksize);
        vid_t nvertices;
        eid_t nedges;
        vid_t minimum_id;
        load_meta(base_name, &nvertices, &nedges, &minimum_id);
        if (numwalks == 0) numwalks = walkpersource * nvertices;
        else walkpersource = 0;
        zero_threshold = zero ? (wid_t)(blocksize_MB * (1024 * 1024) / 128 / 24) : 0;
        ex.zero_copy = zero;
        if (algo == node2vec) ex.init_mode = walkpersource ? GW_INIT_PER_VERTEX : GW_INIT_RANDOM;
        else ex.init_mode = get_option_bool("persource") ? GW_INIT_PER_VERTEX : GW_INIT_SINGLE_SOURCE;
        if (ex.init_mode == GW_INIT_PER_VERTEX && walkpersource == 0) walkpersource = 1;

        graph_config conf = {base_name, memory_size * 1024ull * 1024 * 1024, blocksize, (tid_t)nthreads, (tid_t)1,
                             nvertices, nedges, minimum_id, weighted, numwalks, walkpersource, blockpergrid,
                             threadperblock, cpu_threads, algo, p, q, alpha, steps, walk_batch,
                             (wid_t)(blockpergrid * threadperblock * 16), zero_threshold, gpu_schedule, cpu_schedule,
                             walkaware};
        const std::string tag = (algo == node2vec) ? "node2vec" : "SOPR";
        metrics m(tag + "_numwalks_" + std::to_string(conf.numwalks) + "_steps_" + std::to_string(steps) +
                  "_dataset_" + input + (algo == node2vec ? std::string("_schedule_") + (GOWalker ? "GOWalker" : "") +
                                                                (SOWalker ? "SOWalker" : "")
                                                          : std::string()));
        m.set("gpu_schedule", gpu_schedule ? 1.0 : 0.0);
        m.set("cpu_schedule", cpu_schedule ? 1.0 : 0.0);
        if (get_option_bool("print-config")) {
            printf("{\"base_name\": \"%s\", \"cache_size\": %zu, \"blocksize\": %zu, \"nvertices\": %u, "
                   "\"nedges\": %llu, \"numwalks\": %u, \"walkpersource\": %zu, \"algorithm\": %d, \"p\": %.9g, "
                   "\"q\": %.9g, \"alpha\": %.9g, \"maxhops\": %u, \"zero_threshold\": %u, \"init_mode\": %u, "
                   "\"learned\": %d, \"term_prob\": %.9g, \"seed\": %llu}\n",
                   conf.base_name.c_str(), conf.cache_size, conf.blocksize, conf.nvertices,
                   (unsigned long long)conf.nedges, conf.numwalks, conf.walkpersource, (int)conf.algorithm, conf.p,
                   conf.q, conf.alpha, conf.maxhops, conf.zero_threshold, ex.init_mode, ex.learned ? 1 : 0,
                   ex.term_prob, (unsigned long long)ex.seed);
            return 0;
        }
        if (algo == node2vec && GOWalker == SOWalker) {
            printf("Please select one walker from GOWalker and SOWalker!\n");
            return 0;
        }
        graph_block blocks(&conf);
        graph_driver driver(&conf, m);
        GOwalker_scheduler_t go_sched(m, ex.learned);
        SOwalker_scheduler_t so_sched(m);
        scheduler &sched = (SOWalker && !GOWalker) ? static_cast<scheduler &>(so_sched) : go_sched;
        graph_walk walk(conf, driver, blocks);
        const bid_t nmblocks = (bid_t)std::max<size_t>(1, conf.cache_size / conf.blocksize);
        graph_cache cache(blocks.nblocks, blocksize);
        graph_cache g_cache(nmblocks, blocksize);
        graph_engine engine(cache, walk, driver, conf, m, g_cache, &sched, ex);
        engine.prologue();
        engine.pipe_run();
        engine.epilogue();
        if (engine.status() != GW_OK) {
            fprintf(stderr, "walk failed: %s\n", engine.last_error().c_str());
            return 2;
        }
        metrics_report(m);
    } catch (const std::exception &e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 3;
    }
    return 0;
}
