// Command line of the self-join, a drop-in for the reference's
// `./main <dataset file> <epsilon> <dimensionality> 3` (main.cu:66-331).
//
//  * The dataset is read with the reference's grammar (import_dataset.cpp:49-95):
//    tokens split on ',' and then on whitespace, the flat list cut into tuples
//    of <dimensionality> values.
//  * The params.h switches are the library's build-time defaults; the
//    environment variables NUMINDEXEDDIM, REORDER, SHORTCIRCUIT, ILP, STAMP,
//    QUERYREORDER and DTYPE (float|double) override them without a rebuild.
//  * One line is appended to gpu_stats.txt in the reference's format
//    (main.cu:257-262).  The time covers everything after the import:
//    REORDER, index, join, and the copy of the neighbour table to the host.
//  * PRINTNEIGHBORTABLE=1 writes DSSJ_out.txt, one sorted list per line
//    (main.cu:544-565).
// Only algorithm 3 is provided; modes 0, 1 and 9 of the reference are CPU
// brute force, GPU brute force and a sequential R-tree.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "gpuselfjoin.h"

namespace {

template <typename T>
bool import_dataset(const char* fname, unsigned ndim, std::vector<T>& out, size_t& npts) {
    std::ifstream in(fname);
    if (!in) return false;
    std::vector<T> all;
    for (std::string f; std::getline(in, f, ',');) {
        T v;
        std::stringstream ss(f);
        while (ss >> v) {
            all.push_back(v);
            if (ss.peek() == ',') ss.ignore();
        }
    }
    npts = ndim ? all.size() / ndim : 0;
    all.resize(npts * ndim);
    out.swap(all);
    return true;
}

void env_override(const char* name, uint32_t& field) {
    const char* v = std::getenv(name);
    if (v && *v) field = (uint32_t)std::strtoul(v, nullptr, 10);
}

template <typename T>
int run(const char* fname, double eps_arg, unsigned ndim, gsj_config cfg) {
    std::vector<T> data;
    size_t N = 0;
    if (!import_dataset<T>(fname, ndim, data, N)) {
        std::fprintf(stderr, "\nERROR: cannot read dataset %s\n", fname);
        return 1;
    }
    const T epsilon = (T)eps_arg;  // DTYPE epsilon = atof(...) (main.cu:98)
    std::printf("\nDataset file: %s", fname);
    std::printf("\nEpsilon: %f", (double)epsilon);
    std::printf("\nNumber of dimensions (NDIM): %u\n", ndim);
    std::printf("\nData import: Total data points: %zu", N);
    gsj_context* ctx = nullptr;
    if (gsj_create(&ctx, cfg.device) != GSJ_OK) {
        std::fprintf(stderr, "\nERROR: %s\n", gsj_last_error(nullptr));
        return 1;
    }
    const auto t0 = std::chrono::steady_clock::now();
    gsj_stats st{};
    int rc = gsj_join(ctx, data.data(), N, (double)epsilon, &cfg, 0, &st);
    std::vector<uint32_t> counts(N), table;
    if (rc == GSJ_OK) rc = gsj_result_counts(ctx, counts.data(), 0);
    if (rc == GSJ_OK) {
        table.resize(st.total_pairs);
        rc = gsj_result_table(ctx, table.data(), table.size(), 0);
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (rc != GSJ_OK) {
        std::fprintf(stderr, "\nERROR: %s\n", gsj_last_error(ctx));
        gsj_destroy(ctx);
        return 1;
    }
    const double secs = std::chrono::duration<double>(t1 - t0).count();
    std::printf("\nTotal neighbors: %llu", (unsigned long long)st.total_pairs);
    std::printf("\nTime: %f\n", secs);
    {
        std::ofstream gpu_stats("gpu_stats.txt", std::ios::app);
        gpu_stats << secs << ", " << fname << ", " << epsilon << ", " << st.total_pairs
                  << ", GPUNUMDIM/NUMINDEXEDDIM/ILP/STAMP/SORT/REORDER/SHORTCIRCUIT/QUERYREORDER/DTYPE(float/double): "
                  << ndim << ", " << cfg.indexed_dims << ", " << cfg.ilp << ", " << cfg.stamp << ", " << 0 << ", "
                  << cfg.reorder << ", " << cfg.shortcircuit << ", " << cfg.query_reorder << ", "
                  << (sizeof(T) == 8 ? "double" : "float") << std::endl;
    }
    const char* pr = std::getenv("PRINTNEIGHBORTABLE");
    if (pr && std::atoi(pr) == 1) {
        std::ofstream out("DSSJ_out.txt");
        out << "#data point (line is the point id), neighbor point ids\n";
        size_t off = 0;
        for (size_t i = 0; i < N; i++) {
            std::sort(table.begin() + off, table.begin() + off + counts[i]);
            for (uint32_t j = 0; j < counts[i]; j++) out << table[off + j] << ", ";
            out << "\n";
            off += counts[i];
        }
        std::printf("\nOutputting neighbors to: DSSJ_out.txt\n");
    }
    gsj_destroy(ctx);
    return 0;
}

}  // namespace

int main(int argc, char* argv[]) {
    if (argc != 5) {
        std::cout << "\n\nIncorrect number of input parameters.  \nShould be dataset file, epsilon, number of "
                     "dimensions, searchmode\n";
        return 0;
    }
    const char* fname = argv[1];
    const double eps = std::atof(argv[2]);
    const unsigned ndim = (unsigned)std::atoi(argv[3]);
    const int mode = std::atoi(argv[4]);
    if (mode != 3) {
        std::printf("\nOnly search mode 3 (the GPU grid self-join) is provided.\n");
        return 0;
    }
    gsj_config cfg;
    gsj_default_config(&cfg);
    if (cfg.dim != 0 && cfg.dim != ndim) {
        std::printf("\nERROR: The number of dimensions defined for the GPU is not the same as the number of "
                    "dimensions\n passed into the computer program on the command line. GPUNUMDIM=%u, NDIM=%u "
                    "Exiting!!!",
                    cfg.dim, ndim);
        return 0;
    }
    cfg.dim = ndim;
    env_override("NUMINDEXEDDIM", cfg.indexed_dims);
    env_override("REORDER", cfg.reorder);
    env_override("SHORTCIRCUIT", cfg.shortcircuit);
    env_override("ILP", cfg.ilp);
    env_override("STAMP", cfg.stamp);
    env_override("QUERYREORDER", cfg.query_reorder);
    const char* dt = std::getenv("DTYPE");
    if (dt && !std::strcmp(dt, "double")) cfg.dtype = GSJ_FLOAT64;
    if (dt && !std::strcmp(dt, "float")) cfg.dtype = GSJ_FLOAT32;
    if (cfg.indexed_dims > ndim) {
        std::printf("\nNUMINDEXEDDIM=%u exceeds the dimensionality; using %u indexed dimensions\n",
                    cfg.indexed_dims, ndim);
        cfg.indexed_dims = ndim;
    }
    return cfg.dtype == GSJ_FLOAT64 ? run<double>(fname, eps, ndim, cfg) : run<float>(fname, eps, ndim, cfg);
}
