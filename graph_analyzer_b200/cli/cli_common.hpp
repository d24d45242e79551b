// cli_common.hpp - shared pieces of the command-line drivers (ga_tc, ga_densest, ga_dsg): argument scanning, the
// optional page-locked staging of the host CSR (--pinned), host wall-clock timing of the synchronous C-ABI calls and
// the clock-ramp burn-in. The drivers replace the reference's gpu_tc.cu, gpu_densest.cu and gpu_dsg.cu and print
// the same CSV columns; they call nothing but the C ABI / the C++ surface over it. The graph argument is a text edge
// list (load_graph's rules) or, when its name ends in ".gacsr", a binary CSR file written by ga_save_csr.
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ga/graph_analyzer.hpp"

namespace cli {

inline double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// A device graph created from the host CSR, timing the upload (+ validation); with `pinned` the CSR is first copied
// (untimed) into page-locked memory, as the reference's --pinned does.
struct Upload {
    ga_graph* g = nullptr;
    double h2d_ms = 0;
    double prepare_ms = 0;

    Upload(const ga::Graph& host, bool pinned) {
        {   // untimed: CUDA context, module load and memory pool set-up happen on the first graph of the process
            const uint32_t zero[2] = {0, 0};
            ga_graph* w = nullptr;
            ga::check(ga_graph_create(zero, nullptr, 1, 0, 0, nullptr, &w));
            ga_graph_destroy(w);
        }
        const uint32_t* rp = host.rowptr.data();
        const uint32_t* cl = host.m ? host.col.data() : nullptr;
        void* prp = nullptr;
        void* pcl = nullptr;
        if (pinned) {
            ga::check(ga_host_pinned_alloc(4ull * (host.n + 1), &prp));
            ga::check(ga_host_pinned_alloc(4ull * (host.m ? host.m : 1), &pcl));
            std::memcpy(prp, rp, 4ull * (host.n + 1));
            if (host.m) std::memcpy(pcl, cl, 4ull * host.m);
            rp = (const uint32_t*)prp;
            cl = host.m ? (const uint32_t*)pcl : nullptr;
        }
        const double t0 = now_ms();
        const ga_status s = ga_graph_create(rp, cl, host.n, host.m, 0, nullptr, &g);
        h2d_ms = now_ms() - t0;
        ga_host_pinned_free(prp);
        ga_host_pinned_free(pcl);
        ga::check(s);
        const double t1 = now_ms();
        ga::check(ga_graph_prepare(g));
        prepare_ms = now_ms() - t1;
    }
    ~Upload() { ga_graph_destroy(g); }
    Upload(const Upload&) = delete;
    Upload& operator=(const Upload&) = delete;
};

// Keeps the GPU busy ~1.5 s with counts so the SM clock has ramped before any timed run (the reference's burn-in).
inline void burn_in(ga_graph* g) {
    const double t0 = now_ms();
    uint64_t t = 0;
    do {
        ga::check(ga_tc_count(g, &t));
    } while (now_ms() - t0 < 1500.0);
}

inline void print_device() {
    int n = 0;
    ga_device_count(&n);
    std::fprintf(stderr, "devices visible: %d (library built for sm_100a)\n", n);
}

}  // namespace cli
