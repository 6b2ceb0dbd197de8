// Timing harness around the reference's own CPU self-join code (sequential
// R-tree, search mode 9): the R-tree of RTree.h, generateQueryMBB and
// filterCandidatesAddToTable (tree_index.cpp:191-233), built from the
// reference's sources by oracle/build_ref.sh.  TEST/BENCH INFRASTRUCTURE: the
// reference arm and cpu_baseline of bench.py.
//
// The reference's RtreeSearch (tree_index.cpp:37-185) inserts every point,
// then for each query searches the eps box and filters the candidates.  Its
// own timer sits inside the query loop (tree_index.cpp:105-157), so this
// harness times the same two phases externally: the full tree build over all
// N points, then a seeded sample of queries spread over T threads (each thread
// collects candidates through its own list; the reference's callback appends
// to a global vector).  The build runs once; then `steps` rounds of `sample`
// seeded queries each.  It prints one JSON line with the build time and, per
// round, the sample's pairs and wall time; the caller extrapolates the
// pairs/s of the full join, (pairs * N / sample) / (build + time * N / sample).
//
// usage: rtree_harness <points.bin float32 N x n> <N> <n> <eps> <threads> <steps> <sample> <seed>
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <random>
#include <vector>

#include "RTree.h"
#include "tree_index.h"

namespace {
bool collect(int id, void* ctx) {
    static_cast<std::vector<unsigned int>*>(ctx)->push_back((unsigned int)id);
    return true;
}
}  // namespace

int main(int argc, char** argv) {
    if (argc != 9) {
        std::fprintf(stderr, "usage: %s points.bin N n eps threads steps sample seed\n", argv[0]);
        return 2;
    }
    const size_t N = std::strtoull(argv[2], nullptr, 10);
    const unsigned n = (unsigned)std::atoi(argv[3]);
    const DTYPE eps = (DTYPE)std::atof(argv[4]);
    const int threads = std::atoi(argv[5]);
    const int steps = std::atoi(argv[6]);
    const size_t sample = std::strtoull(argv[7], nullptr, 10);
    const unsigned seed = (unsigned)std::atoi(argv[8]);
    if (n != GPUNUMDIM) {
        std::fprintf(stderr, "harness built for GPUNUMDIM=%d\n", GPUNUMDIM);
        return 2;
    }
    std::vector<float> raw(N * n);
    {
        std::ifstream in(argv[1], std::ios::binary);
        in.read(reinterpret_cast<char*>(raw.data()), raw.size() * sizeof(float));
        if (!in) return 3;
    }
    std::vector<std::vector<DTYPE>> pts(N, std::vector<DTYPE>(n));
    for (size_t i = 0; i < N; i++)
        for (unsigned j = 0; j < n; j++) pts[i][j] = (DTYPE)raw[i * n + j];
    raw.clear();
    raw.shrink_to_fit();

    using clk = std::chrono::steady_clock;
    // ---- build (RtreeSearch's insert loop, tree_index.cpp:61-82)
    const auto tb0 = clk::now();
    RTree<int, DTYPE, GPUNUMDIM, float> tree;
    std::vector<Rect> rects(N);
    createEntryMBBs(&pts, rects.data());
    for (size_t i = 0; i < N; i++) tree.Insert(rects[i].MBB_min, rects[i].MBB_max, rects[i].pid);
    const double t_build = std::chrono::duration<double>(clk::now() - tb0).count();

    // ---- rounds of seeded query samples
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<unsigned> pick(0u, (unsigned)(N - 1));
    std::vector<neighborTableLookupCPU> table(N);
    std::vector<unsigned> qs(sample);
    std::printf("{\"build_s\": %.4f, \"threads\": %d, \"N\": %zu, \"sample\": %zu, \"steps\": [", t_build,
                threads, N, sample);
    for (int step = 0; step < steps; step++) {
        for (auto& q : qs) q = pick(rng);
        unsigned long long rp = 0;
        const auto tq0 = clk::now();
#pragma omp parallel num_threads(threads) reduction(+ : rp)
        {
            std::vector<unsigned int> cand;
            std::vector<unsigned int> vect;
#pragma omp for schedule(dynamic, 64)
            for (long long t = 0; t < (long long)sample; t++) {
                const unsigned q = qs[t];
                DTYPE mn[GPUNUMDIM], mx[GPUNUMDIM];
                generateQueryMBB(&pts, q, eps, mn, mx);
                cand.clear();
                tree.Search(mn, mx, collect, &cand);
                rp += filterCandidatesAddToTable(&pts, q, eps, &cand, table.data(), &vect);
                vect.clear();
            }
        }
        const double tq = std::chrono::duration<double>(clk::now() - tq0).count();
        std::printf("%s{\"pairs\": %llu, \"query_s\": %.6f}", step ? ", " : "", rp, tq);
    }
    std::printf("]}\n");
    return 0;
}
