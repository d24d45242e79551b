// api_check.cpp - the reference-names C++ surface (include/ga/graph_analyzer.hpp) used the way the reference's own
// drivers use graph.h / densest.h / dsg.h: load_graph, a device graph, batch_peel_loop with the CPU count as T_full,
// core_decomp_loop_inc, the support helpers and the densest-subgraph pipeline of gpu_dsg. Prints one line per result for the test to compare with the golden
// outputs. usage: api_check graph.txt eps_num eps_den T_full
#define GA_B200_GLOBAL_NAMES
#include "ga/graph_analyzer.hpp"

#include <cstdlib>

int main(int argc, char** argv) {
    if (argc != 5) return 2;
    Graph g;
    if (!load_graph(argv[1], g)) return 1;
    const uint64_t num = std::strtoull(argv[2], nullptr, 10), den = std::strtoull(argv[3], nullptr, 10);
    const uint64_t T_full = std::strtoull(argv[4], nullptr, 10);
    try {
        ga::DeviceGraph d(g);
        std::printf("triangles %llu\n", (unsigned long long)d.triangles());
        PeelResult r = batch_peel_loop(g.n, T_full, num, den, d);
        if (!r.ok) { std::fprintf(stderr, "peel: %s\n", r.error.c_str()); return 1; }
        unsigned long long rr = 0;
        for (uint32_t v = 0; v < g.n; v++) rr = rr * 1000003ull + r.removed_round[v];
        std::printf("peel %llu %llu %u %u %llx\n", (unsigned long long)r.best_num, (unsigned long long)r.best_den,
                    r.best_round, r.rounds, rr);
        std::vector<uint32_t> core;
        CoreLoopResult c = core_decomp_loop_inc(g.n, T_full, d, core);
        if (!c.ok) { std::fprintf(stderr, "cores: %s\n", c.error.c_str()); return 1; }
        unsigned long long ch = 0;
        for (uint32_t v = 0; v < g.n; v++) ch = ch * 1000003ull + core[v];
        std::printf("cores %u %u %llx\n", c.kmax, c.rounds, ch);
        const Dens kd = core_level_density(d, core, c.kmax);
        std::printf("kcore %llu %llu\n", (unsigned long long)kd.num, (unsigned long long)kd.den);
        std::vector<uint32_t> sup;
        std::vector<uint64_t> deg;
        std::printf("supports %llu %llu\n", (unsigned long long)d.edge_support(sup),
                    (unsigned long long)d.triangle_degrees(deg));
        // the gpu_dsg pipeline (gpu_dsg.cu:318-369) with the dsg.h names: lower bound, prune, Greedy++, CoreExact
        std::vector<uint8_t> in(g.n);
        uint64_t kverts = 0;
        for (uint32_t v = 0; v < g.n; v++) kverts += in[v] = core[v] >= c.kmax;
        std::vector<uint32_t> tri;
        Dens lb{d.triangle_participation(in, tri), kverts};
        DsgResult gr = greedy(g);
        if (!gr.ok) { std::fprintf(stderr, "greedy: %s\n", gr.error.c_str()); return 1; }
        if (dens_gt(gr.dens(), lb)) lb = gr.dens();
        Graph gp;
        std::vector<uint32_t> old_id, core_p;
        prune_to_core(g, core, dens_ceil(lb), gp, old_id, core_p);
        DsgResult gpp = greedy_pp(gp, 10);
        DsgResult ex = core_exact(gp, core_p, true, &gpp);
        if (!gpp.ok || !ex.ok) { std::fprintf(stderr, "dsg: %s%s\n", gpp.error.c_str(), ex.error.c_str()); return 1; }
        std::printf("dsg %llu %llu %u %u %llu %llu %llu %llu %u\n", (unsigned long long)gr.tri,
                    (unsigned long long)gr.verts, gp.n, gp.m, (unsigned long long)gpp.tri, (unsigned long long)gpp.verts,
                    (unsigned long long)ex.tri, (unsigned long long)ex.verts, ex.flow_calls);
        // the same graph twice in one batch, and through the request loop: each result equals the single-graph one
        {
            ga::DeviceBatch b({&g, &g});
            std::vector<uint64_t> bt;
            std::vector<PeelResult> bp = b.tc_peel(num, den, &bt);
            const bool same = bp.size() == 2 && bp[0] == r && bp[1] == r && bt[0] == T_full && bt[1] == T_full &&
                              b.triangles() == bt;
            ga::Server srv;
            const uint64_t id = srv.add_graph(g);
            std::vector<uint32_t> served_rr, served_core;   // the served vertex arrays
            const uint64_t t_tc = srv.submit(id, GA_REQ_TC),
                           t_peel = srv.submit(id, GA_REQ_PEEL, num, den, g.n, served_rr),
                           t_core = srv.submit(id, GA_REQ_CORE, 1, 1, g.n, served_core);
            const ga_request_result a = srv.wait(t_tc), p = srv.wait(t_peel), q = srv.wait(t_core);
            const bool served = a.status == GA_OK && a.triangles == T_full && p.status == GA_OK &&
                                p.peel.best_num == r.best_num && p.peel.best_den == r.best_den &&
                                p.peel.best_round == r.best_round && p.peel.rounds == r.rounds &&
                                q.status == GA_OK && q.core.kmax == c.kmax && q.core.rounds == c.rounds &&
                                served_rr == r.removed_round && served_core == core;
            std::printf("batch_serve %d %d\n", same ? 1 : 0, served ? 1 : 0);
        }
        // the refusals of batch_peel_loop (densest.h:65-78, 283-287): wrong T_full, eps out of range
        PeelResult bad = batch_peel_loop(g.n, T_full + 1, num, den, d);
        PeelResult bad_eps = batch_peel_loop(g.n, T_full, 1, 0, d);
        std::printf("refusals %d %d\n", bad.ok ? 1 : 0, bad_eps.ok ? 1 : 0);
    } catch (const ga::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
