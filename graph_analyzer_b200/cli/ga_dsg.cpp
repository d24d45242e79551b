// ga_dsg - densest subgraph by triangle density over the C ABI; replaces the reference's gpu_dsg.cu: the
// (k, triangle)-core decomposition (dsg.h:724-751) and the pipeline after it (gpu_dsg.cu:318-369): lower bound
// max(kmax-core density, greedy density), prune to the ceil(lb)-core, Greedy++ and CoreExact seeded with it.
// usage: ga_dsg graph.txt [--T 10] [--repeats N] [--pinned] [--no-burnin] [--no-exact] [--no-greedy]
//                         [--no-greedypp] [--verify-full]
//   --T N          Greedy++ passes on the pruned graph (default 10)
//   --no-exact     stop after the cores, the greedy and the pruning
//   --no-greedy    lower bound = the kmax-core density only
//   --no-greedypp  no Greedy++ row (Greedy++ still runs as CoreExact's seed when CoreExact runs, as in the reference)
//   --verify-full  also CoreExact on the whole graph; its optimum must equal the pruned pipeline's
// Rows (stdout, CSV, the reference's dsg_row columns, printed only if everything verified):
//   impl,graph,n,m,triangles,vertices,density,time_ms,h2d_ms,total_ms,rounds,kmax
//   gpu_core_decomp       device-resident rounds in a CUDA graph with a conditional node (default); row = kmax-core
//   gpu_core_decomp_host  the same rounds driven from the host, one small read per round
//   greedy                Charikar's greedy (the reference's cpu_greedy): device core numbers and triangle lists, one
//                         removal sequence per core level on the host threads; rounds = n removals
//   prune_kcore           n,m = the pruned graph; triangles,vertices = the pruned graph; rounds = ceil(lb)
//   greedy_pp_pruned      Greedy++ on the pruned graph; rounds = T passes
//   core_exact_pruned_seeded  CoreExact on the pruned graph seeded with the Greedy++ result; rounds = max-flow calls
//   pipeline_gpu_core     time_ms = core decomposition (best) + greedy + prune + Greedy++ + CoreExact; h2d_ms = the
//                         upload of the graph (the pruned graph's upload is inside its stages' times)
//   core_exact_full       (--verify-full) CoreExact on the whole graph with the device core numbers
// (suffix "_pinned" on the gpu_ rows with --pinned). Core rows: time_ms = best of N (default 5) calls of
// ga_core_decomposition after one untimed verified call, host wall clock; EXCLUDES the upload (h2d_ms) and core[]'s
// download. Verification: every core call of both modes gives the same core numbers, kmax and rounds; CoreExact's
// optimum is not below the lower bound and not below Greedy++'s; --verify-full's optimum equals the pipeline's.
// Any failure: MISMATCH on stderr, exit 1, no rows.
#include "cli_common.hpp"

namespace {

struct Run {
    ga_core_result r{};
    std::vector<uint32_t> core;
};

Run cores_once(ga_graph* g, uint32_t n, double* ms) {
    Run run;
    run.core.assign(n, 0);
    const double t0 = cli::now_ms();
    ga::check(ga_core_decomposition(g, run.core.data(), &run.r));
    if (ms) *ms = cli::now_ms() - t0;
    return run;
}

std::string dsg_row(const std::string& impl, const char* graph, uint32_t n, uint32_t m, uint64_t tri, uint64_t verts,
                    double ms, double h2d, uint64_t rounds, uint64_t kmax) {
    char buf[1024];
    std::snprintf(buf, sizeof buf, "%s,%s,%u,%u,%llu,%llu,%.6f,%.3f,%.3f,%.3f,%llu,%llu", impl.c_str(), graph, n, m,
                  (unsigned long long)tri, (unsigned long long)verts, ga::density_value(tri, verts), ms, h2d, ms + h2d,
                  (unsigned long long)rounds, (unsigned long long)kmax);
    return buf;
}

ga::DsgResult must(ga::DsgResult r, const char* what) {
    if (!r.ok) throw ga::Error(GA_ERR_DEVICE_CHECK, std::string(what) + ": " + r.error);
    return r;
}

}  // namespace

int main(int argc, char** argv) {
    bool pinned = false, burnin = true, exact = true, greedy_on = true, gpp_row = true, verify_full = false;
    int repeats = 5;
    uint32_t T_pass = 10;
    std::vector<const char*> pos;
    for (int i = 1; i < argc; i++) {
        if (std::strcmp(argv[i], "--pinned") == 0) pinned = true;
        else if (std::strcmp(argv[i], "--no-burnin") == 0) burnin = false;
        else if (std::strcmp(argv[i], "--no-exact") == 0) exact = false;
        else if (std::strcmp(argv[i], "--no-greedy") == 0) greedy_on = false;
        else if (std::strcmp(argv[i], "--no-greedypp") == 0) gpp_row = false;
        else if (std::strcmp(argv[i], "--verify-full") == 0) verify_full = true;
        else if (std::strcmp(argv[i], "--T") == 0 && i + 1 < argc) T_pass = (uint32_t)std::max(1, std::atoi(argv[++i]));
        else if (std::strcmp(argv[i], "--repeats") == 0 && i + 1 < argc) repeats = std::max(1, std::atoi(argv[++i]));
        else pos.push_back(argv[i]);
    }
    if (pos.size() != 1) {
        std::fprintf(stderr, "usage: %s graph.txt [--T 10] [--repeats N] [--pinned] [--no-burnin] [--no-exact] "
                             "[--no-greedy] [--no-greedypp] [--verify-full]\n", argv[0]);
        return 2;
    }
    const char* path = pos[0];
    const std::string suffix = pinned ? "_pinned" : "";
    try {
        cli::print_device();
        ga::Graph g;
        if (!ga::load_any(path, g)) return 1;
        std::fprintf(stderr, "loaded n=%u m=%u max_out_deg=%u\n", g.n, g.m, g.max_out_degree);
        cli::Upload up(g, pinned);
        if (burnin) cli::burn_in(up.g);
        struct Mode { const char* name; int64_t loop; };
        const Mode modes[] = {{"gpu_core_decomp", 2}, {"gpu_core_decomp_host", 1}};
        std::vector<std::string> rows;
        bool ok = true, have = false;
        Run first;
        uint64_t kcore_tri = 0, kcore_verts = 0;
        double core_best = 0;
        for (const Mode& md : modes) {
            ga::check(ga_graph_set_option(up.g, GA_OPT_LOOP_MODE, md.loop));
            Run last = cores_once(up.g, g.n, nullptr);
            if (!have) {
                first = last;
                have = true;
                // the kmax-core: triangles of the subgraph induced by {v : core[v] >= kmax} (dsg.h:169-174)
                std::vector<uint8_t> in(g.n);
                for (uint32_t v = 0; v < g.n; v++) {
                    in[v] = first.core[v] >= first.r.kmax;
                    kcore_verts += in[v];
                }
                std::vector<uint32_t> tri(g.n);
                ga::check(ga_tc_participation(up.g, in.data(), tri.data(), &kcore_tri));
            }
            double best = 1e300;
            for (int i = -1; i < repeats && ok; i++) {
                double ms = 0;
                if (i >= 0) {
                    last = cores_once(up.g, g.n, &ms);
                    best = std::min(best, ms);
                }
                if (last.r.kmax != first.r.kmax || last.r.rounds != first.r.rounds || last.core != first.core) {
                    size_t v = 0;
                    while (v < g.n && last.core[v] == first.core[v]) v++;
                    std::fprintf(stderr, "MISMATCH in %s: kmax %u vs %u, rounds %u vs %u, first differing vertex %zu\n",
                                 md.name, last.r.kmax, first.r.kmax, last.r.rounds, first.r.rounds, v);
                    ok = false;
                }
            }
            if (md.loop == 2) core_best = best;
            rows.push_back(dsg_row(std::string(md.name) + suffix, path, g.n, g.m, kcore_tri, kcore_verts, best,
                                   up.h2d_ms, last.r.rounds, last.r.kmax));
        }
        if (!ok) {
            std::fprintf(stderr, "VERIFICATION FAILED - no timing rows printed\n");
            return 1;
        }
        ga::check(ga_graph_set_option(up.g, GA_OPT_LOOP_MODE, 2));
        const uint32_t kmax = first.r.kmax;
        const std::vector<uint32_t>& core = first.core;

        // ---- lower bound and pruning (gpu_dsg.cu:318-339) ----
        ga::Dens lb{kcore_tri, kcore_verts};
        double t_greedy = 0;
        if (greedy_on) {
            ga_dsg_result res{};
            std::vector<uint32_t> set(g.n);
            const double t0 = cli::now_ms();
            ga::check(ga_greedy_pp(up.g, 1, &res, set.data(), nullptr));
            t_greedy = cli::now_ms() - t0;
            rows.push_back(dsg_row("greedy", path, g.n, g.m, res.tri, res.verts, t_greedy, 0, g.n, 0));
            if (ga::dens_gt(ga::Dens{res.tri, res.verts}, lb)) lb = ga::Dens{res.tri, res.verts};
        }
        const uint64_t kprune = ga::dens_ceil(lb);
        ga::Graph gp;
        std::vector<uint32_t> old_id, core_p;
        double t0 = cli::now_ms();
        ga::prune_to_core(g, core, kprune, gp, old_id, core_p);
        const double t_prune = cli::now_ms() - t0;
        ga::DeviceGraph dp(gp);
        const uint64_t T_pruned = dp.triangles();
        rows.push_back(dsg_row("prune_kcore", path, gp.n, gp.m, T_pruned, gp.n, t_prune, 0, kprune, kmax));
        std::fprintf(stderr, "lower bound %llu/%llu = %.6f -> keep core >= %llu: pruned graph n=%u m=%u (of n=%u m=%u)\n",
                     (unsigned long long)lb.num, (unsigned long long)lb.den, ga::dens_value(lb),
                     (unsigned long long)kprune, gp.n, gp.m, g.n, g.m);

        // ---- Greedy++ and CoreExact on the pruned graph (gpu_dsg.cu:341-369) ----
        if (exact || gpp_row) {
            t0 = cli::now_ms();
            ga::DsgResult gpr = must(ga::greedy_pp(dp, T_pass), "greedy_pp");
            const double t_gpp = cli::now_ms() - t0;
            if (gpp_row)
                rows.push_back(dsg_row("greedy_pp_pruned", path, gp.n, gp.m, gpr.tri, gpr.verts, t_gpp, 0, T_pass, 0));
            if (exact) {
                t0 = cli::now_ms();
                ga::DsgResult ex = must(ga::core_exact(dp, core_p, true, &gpr), "core_exact");
                const double t_exact = cli::now_ms() - t0;
                rows.push_back(dsg_row("core_exact_pruned_seeded", path, gp.n, gp.m, ex.tri, ex.verts, t_exact, 0,
                                       ex.flow_calls, 0));
                if (ga::dens_cmp(ex.dens(), lb) < 0) {
                    std::fprintf(stderr, "MISMATCH: exact optimum below the lower bound\n");
                    return 1;
                }
                if (ga::dens_gt(gpr.dens(), ex.dens())) {
                    std::fprintf(stderr, "MISMATCH: greedy++ exceeds the exact optimum\n");
                    return 1;
                }
                rows.push_back(dsg_row("pipeline_gpu_core" + suffix, path, g.n, g.m, ex.tri, ex.verts,
                                       core_best + t_greedy + t_prune + t_gpp + t_exact, up.h2d_ms, first.r.rounds,
                                       kmax));
                if (verify_full) {
                    ga::DeviceGraph dfull(g);
                    t0 = cli::now_ms();
                    ga::DsgResult full = must(ga::core_exact(dfull, core), "core_exact (full)");
                    const double t_full = cli::now_ms() - t0;
                    if (ga::dens_cmp(full.dens(), ex.dens()) != 0) {
                        std::fprintf(stderr, "MISMATCH: full-graph CoreExact %llu/%llu vs pruned pipeline %llu/%llu\n",
                                     (unsigned long long)full.tri, (unsigned long long)full.verts,
                                     (unsigned long long)ex.tri, (unsigned long long)ex.verts);
                        return 1;
                    }
                    rows.push_back(dsg_row("core_exact_full", path, g.n, g.m, full.tri, full.verts, t_full, 0,
                                           full.flow_calls, 0));
                }
                std::fprintf(stderr, "optimum %llu/%llu = %.6f\n", (unsigned long long)ex.tri,
                             (unsigned long long)ex.verts, ga::dens_value(ex.dens()));
            }
        }
        for (auto& r : rows) std::puts(r.c_str());
        std::fflush(stdout);
        std::fprintf(stderr, "both loop modes agree element-wise (kmax %u, %u rounds)\n", first.r.kmax,
                     first.r.rounds);
    } catch (const ga::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
