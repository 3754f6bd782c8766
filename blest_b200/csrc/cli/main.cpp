// blest -- command-line driver over libblest_b200 (the reference's
// `blest -d <dir> -g <graph> -j <0|1> -w <window>`, main.cu:19-131 and
// Benchmark::run, Benchmark.cuh:149-331), offline:
//  - the graph is <dir>/<graph>.mtx (Matrix Market, banner decides
//    symmetric/pattern), or synthesised with --gen;
//  - caches <dir>/<graph>_csc.bin (CSC.cuh:225-266 layout) and
//    <dir>/<graph>_ordering_j<J>_w<W>.bin (keyed on -j/-w, so changing them
//    never reuses a stale ordering);
//  - sources are original vertex ids, one per line, in <dir>/<graph>.txt
//    (written from a seeded sample when missing), mapped through the
//    ordering as Benchmark.cuh:67-85 does;
//  - one line per source in the reference's format, the average time, and
//    a TSV <dir>/<graph>.csv of Source / TotalLevels / TotalVisited / Time.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "blest.h"
#include "blest_kernels.hpp"

using blest_b200::check;

namespace {

struct Config {
    std::string directory, matrixName;
    bool jaccard = false;
    unsigned window = 0;
    std::string kernel = "bfs";
    std::string gen;
    unsigned sources = 64;
    unsigned long long seed = 1;
    int device = 0;
};

void usage(const char* prog) {
    std::cerr << "Usage: " << prog << " -d <directory> -g <graph_name> -j <0|1> -w <window_size>\n"
              << "          [-k bfs|cc|mbfs] [--gen rmat:S:EF|grid:W:H|er:LOGN:DEG] [--sources K] [--seed S]"
                 " [--device D]\n"
              << "  -d  directory holding <graph>.mtx and <graph>.txt (sources); caches and results go here\n"
              << "  -g  graph name\n"
              << "  -j  Jaccard reordering for social graphs (0 or 1)\n"
              << "  -w  Jaccard window (multiple of 8, e.g. 65536)\n"
              << "  -k  kernel: bfs (default), cc, mbfs (all sources in one multi-source run)\n"
              << "  --gen  synthesise the graph instead of reading <graph>.mtx\n"
              << "  --sources  number of seeded sources when <graph>.txt is missing (default 64)\n";
}

unsigned parse_unsigned(const std::string& v, const char* opt) {
    try {
        size_t pos = 0;
        const unsigned long x = std::stoul(v, &pos);
        if (pos != v.size() || x > std::numeric_limits<unsigned>::max()) throw std::out_of_range(opt);
        return (unsigned)x;
    } catch (const std::exception&) {
        throw std::runtime_error(std::string("Invalid value for ") + opt + " (expected unsigned integer), got: " + v);
    }
}

Config parse_args(int argc, char** argv) {
    Config c;
    bool jSet = false, wSet = false;
    auto value = [&](int& i, const char* opt) -> std::string {
        if (i + 1 >= argc) throw std::runtime_error(std::string("Missing value for ") + opt);
        return argv[++i];
    };
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "-h" || a == "--help") {
            usage(argv[0]);
            std::exit(0);
        } else if (a == "-d") {
            c.directory = value(i, "-d");
        } else if (a == "-g") {
            c.matrixName = value(i, "-g");
        } else if (a == "-j") {
            const std::string v = value(i, "-j");
            if (v != "0" && v != "1") throw std::runtime_error("Invalid value for -j (expected 0 or 1), got: " + v);
            c.jaccard = v == "1";
            jSet = true;
        } else if (a == "-w") {
            c.window = parse_unsigned(value(i, "-w"), "-w");
            wSet = true;
        } else if (a == "-k") {
            c.kernel = value(i, "-k");
            if (c.kernel != "bfs" && c.kernel != "cc" && c.kernel != "mbfs")
                throw std::runtime_error("Invalid value for -k (bfs, cc or mbfs), got: " + c.kernel);
        } else if (a == "--gen") {
            c.gen = value(i, "--gen");
        } else if (a == "--sources") {
            c.sources = parse_unsigned(value(i, "--sources"), "--sources");
        } else if (a == "--seed") {
            c.seed = parse_unsigned(value(i, "--seed"), "--seed");
        } else if (a == "--device") {
            c.device = (int)parse_unsigned(value(i, "--device"), "--device");
        } else {
            throw std::runtime_error("Unknown argument: " + a);
        }
    }
    if (c.directory.empty()) throw std::runtime_error("Missing required option: -d <directory>");
    if (c.matrixName.empty()) throw std::runtime_error("Missing required option: -g <graph_name>");
    if (!jSet) throw std::runtime_error("Missing required option: -j <0|1>");
    if (!wSet) throw std::runtime_error("Missing required option: -w <window_size>");
    if (c.directory.back() != '/') c.directory += '/';
    return c;
}

bool exists(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0;
}

struct CscPtr {
    blest_csc* p = nullptr;
    ~CscPtr() { blest_csc_destroy(p); }
};
struct BvssPtr {
    blest_bvss* p = nullptr;
    ~BvssPtr() { blest_bvss_destroy(p); }
};

blest_csc* make_graph(const Config& c) {
    blest_csc* g = nullptr;
    const std::string cache = c.directory + c.matrixName + "_csc.bin";
    if (exists(cache)) {
        check(blest_csc_load_bin(cache.c_str(), &g), "CSC cache");
        std::cout << "CSC read from binary." << std::endl;
        return g;
    }
    if (!c.gen.empty()) {
        std::vector<std::string> f;
        std::stringstream ss(c.gen);
        for (std::string x; std::getline(ss, x, ':');) f.push_back(x);
        if (f.size() == 3 && f[0] == "rmat")
            check(blest_csc_generate_rmat(parse_unsigned(f[1], "--gen"), parse_unsigned(f[2], "--gen"), 0.57, 0.19,
                                          0.19, c.seed, c.seed, &g),
                  "RMAT");
        else if (f.size() == 3 && f[0] == "grid")
            check(blest_csc_generate_grid(parse_unsigned(f[1], "--gen"), parse_unsigned(f[2], "--gen"), 0.05, 0.001,
                                          c.seed, 0, &g),
                  "grid");
        else if (f.size() == 3 && f[0] == "er") {
            const uint32_t n = 1u << parse_unsigned(f[1], "--gen");
            check(blest_csc_generate_er(n, (uint64_t)n * parse_unsigned(f[2], "--gen") / 2, c.seed, 0, &g), "ER");
        } else {
            throw std::runtime_error("Invalid value for --gen: " + c.gen);
        }
    } else {
        const std::string mtx = c.directory + c.matrixName + ".mtx";
        std::cout << "CSC construction started." << std::endl;
        check(blest_csc_read_mtx_auto(mtx.c_str(), &g), "Matrix Market");
    }
    check(blest_csc_save_bin(g, cache.c_str()), "CSC cache");
    std::cout << "CSC constructed." << std::endl;
    return g;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        const Config c = parse_args(argc, argv);
        CscPtr csc;
        csc.p = make_graph(c);
        blest_csc_view v;
        check(blest_csc_view_get(csc.p, &v), "CSC view");
        std::cout << "Number of vertices: " << v.n << "\nNumber of edges: " << v.nnz << "\nThe graph is "
                  << (v.is_social ? "" : "not ") << "a social network." << std::endl;

        // sources in original ids (before the ordering is applied)
        const std::string srcFile = c.directory + c.matrixName + ".txt";
        std::vector<uint32_t> sources;
        if (!exists(srcFile)) {
            sources.resize(std::max(1u, c.sources));
            uint32_t k = 0;
            check(blest_csc_sample_sources(csc.p, c.sources, c.seed, sources.data(), &k), "sources");
            sources.resize(k);
            std::ofstream out(srcFile);
            for (uint32_t s : sources) out << s << "\n";
        } else {
            std::ifstream in(srcFile);
            for (unsigned long s; in >> s;) {
                if (s >= v.n) throw std::runtime_error("source id out of range in " + srcFile);
                sources.push_back((uint32_t)s);
            }
        }

        // ordering (cached per -j/-w)
        std::vector<uint32_t> inv(v.n);
        const std::string ordFile = c.directory + c.matrixName + "_ordering_j" + (c.jaccard ? "1" : "0") + "_w" +
                                    std::to_string(c.window) + ".bin";
        if (exists(ordFile)) {
            check(blest_ordering_load_bin(ordFile.c_str(), v.n, inv.data()), "ordering cache");
            check(blest_csc_apply_permutation(csc.p, inv.data()), "ordering");
            std::cout << "Ordering read from binary." << std::endl;
        } else {
            blest_order_params op{};
            op.mode = BLEST_ORDER_AUTO;
            op.jaccard_enabled = c.jaccard ? 1 : 0;
            op.window = c.window ? c.window : 65536;
            op.rcm_rand_seed = 1;
            const auto t0 = std::chrono::steady_clock::now();
            check(blest_csc_reorder(csc.p, &op, inv.data()), "reorder");
            std::cout << "Time took to reorder: "
                      << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() << std::endl;
            check(blest_ordering_save_bin(ordFile.c_str(), inv.data(), v.n), "ordering cache");
        }
        for (uint32_t& s : sources) s = inv[s];

        BvssPtr bvss;
        check(blest_bvss_build(csc.p, -1, &bvss.p), "BVSS");
        uint64_t edges = 0;
        check(blest_bvss_edge_check(bvss.p, &edges), "BVSS check");
        std::cout << "BVSS constructed. Check: " << edges << std::endl;

        int sym = 0;
        check(blest_csc_check_symmetry(csc.p, &sym), "symmetry");
        CscPtr transposed;
        if (!sym) check(blest_csc_transpose(csc.p, &transposed.p), "transpose");
        check(blest_init(c.device), "device");
        blest_b200::DeviceGraph graph(bvss.p, sym ? csc.p : transposed.p);

        std::vector<uint32_t> perm(v.n);
        for (uint32_t old = 0; old < v.n; ++old) perm[inv[old]] = old;
        std::ofstream tsv(c.directory + c.matrixName + ".csv");
        tsv << "Source\tTotalLevels\tTotalVisited\tTime(ms)\n";
        double total = 0;
        if (c.kernel == "bfs") {
            std::cout << "BFS kernels launching..." << std::endl;
            blest_b200::B200BFSKernel kernel(&graph);
            for (uint32_t s : sources) {
                blest_b200::BFSResult r = kernel.run(s);
                r.sourceVertex = perm[r.sourceVertex];
                std::cout << "Source: " << r.sourceVertex << " - Number of levels processed: " << r.totalLevels
                          << " - Total visited: " << r.noVisited << " - Time took: " << r.time * 1000 << " ms."
                          << std::endl;
                tsv << r.sourceVertex << "\t" << r.totalLevels << "\t" << r.noVisited << "\t" << r.time * 1000 << "\n";
                total += r.time;
                delete[] r.levels;
            }
            total /= std::max<size_t>(1, sources.size());
        } else if (c.kernel == "cc") {
            std::cout << "CC kernels launching..." << std::endl;
            blest_b200::B200CCKernel kernel(&graph);
            blest_b200::CCResult r = kernel.run();
            std::cout << "Number of components identified: " << r.noComponents << std::endl;
            total = r.time;
            delete[] r.components;
        } else {
            std::cout << "MBFS kernel launching..." << std::endl;
            blest_b200::B200MBFSKernel kernel(&graph, sources);
            blest_b200::MBFSResult r = kernel.run();
            std::cout << "Sources: " << sources.size() << " - Time took: " << r.time * 1000 << " ms." << std::endl;
            total = r.time;
            for (unsigned* lv : r.levelArrays) delete[] lv;
        }
        std::cout << "Time: " << total * 1000 << " ms." << std::endl;
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << std::endl;
        usage(argv[0]);
        return 1;
    }
}
