// ga_tc - triangle counting driver over the C ABI; replaces the reference's gpu_tc.cu (its kernels v1-v9).
// usage: ga_tc <edge_list.txt | graph.gacsr> [repeats] [--pinned] [--no-burnin]   (flags may appear anywhere)
// Rows (stdout, CSV, the reference's columns):  impl,graph,n,m,triangles,kernel_ms,h2d_ms,gpu_total_ms
//   gpu_hash_binned      the degree-binned shared-memory hash kernel (k_tc_hash)
//   gpu_edge_per_thread  one thread per oriented edge, two-list merge (k_tc_plain)
//   gpu_autotuned        the kernel the autotuner picks for this degree distribution
// (suffix "_pinned" with --pinned). kernel_ms = best of `repeats` (default 5) warm calls of ga_tc_count, host wall
// clock around the synchronous call (launch and the 8-byte result read included), after one untimed warm-up call.
// h2d_ms = ga_graph_create: upload of rowptr + col and the device-side validation; gpu_total_ms = kernel_ms + h2d_ms
// + the device-side index build (ga_graph_prepare, printed on stderr). Loading and orientation are not included.
// Every call's count must equal the first one's, across all rows; otherwise MISMATCH on stderr and exit code 1.
#include "cli_common.hpp"

int main(int argc, char** argv) {
    bool pinned = false, burnin = true;
    std::vector<const char*> pos;
    for (int i = 1; i < argc; i++) {
        if (std::strcmp(argv[i], "--pinned") == 0) pinned = true;
        else if (std::strcmp(argv[i], "--no-burnin") == 0) burnin = false;
        else pos.push_back(argv[i]);
    }
    if (pos.empty()) {
        std::fprintf(stderr, "usage: %s graph.txt [repeats] [--pinned] [--no-burnin]\n", argv[0]);
        return 2;
    }
    const char* path = pos[0];
    const int repeats = pos.size() > 1 ? std::max(1, std::atoi(pos[1])) : 5;
    try {
        cli::print_device();
        ga::Graph g;
        const double tl = cli::now_ms();
        if (!ga::load_any(path, g)) return 1;
        std::fprintf(stderr, "loaded n=%u m=%u max_out_deg=%u (%.1f ms)\n", g.n, g.m, g.max_out_degree,
                     cli::now_ms() - tl);
        cli::Upload up(g, pinned);
        std::fprintf(stderr, "upload %.3f ms, device index build %.3f ms\n", up.h2d_ms, up.prepare_ms);
        if (burnin) cli::burn_in(up.g);
        struct Variant { const char* name; int64_t kernel; };
        const Variant variants[] = {{"gpu_hash_binned", 2}, {"gpu_edge_per_thread", 1}, {"gpu_autotuned", 0}};
        bool ok = true, have = false;
        uint64_t expected = 0;
        for (const Variant& v : variants) {
            ga::check(ga_graph_set_option(up.g, GA_OPT_TC_KERNEL, v.kernel));
            double best = 1e300;
            uint64_t t = 0;
            for (int r = -1; r < repeats; r++) {   // r == -1: untimed warm-up
                const double t0 = cli::now_ms();
                ga::check(ga_tc_count(up.g, &t));
                const double ms = cli::now_ms() - t0;
                if (r >= 0) best = std::min(best, ms);
                if (!have) { expected = t; have = true; }
                if (t != expected) {
                    std::fprintf(stderr, "MISMATCH in %s (call %d): %llu vs %llu\n", v.name, r,
                                 (unsigned long long)t, (unsigned long long)expected);
                    ok = false;
                }
            }
            const std::string name = std::string(v.name) + (pinned ? "_pinned" : "");
            std::printf("%s,%s,%u,%u,%llu,%.3f,%.3f,%.3f\n", name.c_str(), path, g.n, g.m, (unsigned long long)t, best,
                        up.h2d_ms, best + up.h2d_ms + up.prepare_ms);
            std::fflush(stdout);
        }
        if (!ok) return 1;
        std::fprintf(stderr, "all kernels agree: %llu triangles\n", (unsigned long long)expected);
    } catch (const ga::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
