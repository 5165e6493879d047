// ref_harness.cpp -- runs the REFERENCE decoder (its gpu/plp_common.hpp,
// compiled from the reference tree) over many restarts, for golden outputs
// and for the CPU baseline timing. Test infrastructure; built into
// oracle/_ref/ by `make -C oracle ref`.
//
//   ref_harness <instance> [<instance> ...] [--seed S] [--restarts R] [--passes P]
//               [--eps F] [--theta F | --no-theta] [--order volume|input]
//               [--first-fit] [--mu F] [--threads T] [--json] [--repeat N]
//
// Every instance gets restarts seed .. seed + R - 1; the threads share one
// work list of (instance, restart) pairs, so a sample drawn across a
// workload's instances is timed with its own mix of sizes. With --json the
// rows come out instance by instance, restart by restart.
//
// Restart k runs plp::run(inst, seed + k, ...) exactly as the reference CLI
// does for `--single-pass --seed (seed + k)` (gpu/plp_gpu.cpp:131-133). For
// P > 1 passes the reference only has a wall-clock loop, so a fixed count is
// composed from the same reference functions (PyRng carried across passes,
// decode_pass, stability_score and the strict-> selection of
// gpu/plp_common.hpp:493-511).
//
// Without --json it prints one timing line:
//   {"decodes": N, "seconds": T, "threads": K}
#include "plp_common.hpp"

#include <atomic>
#include <thread>

namespace {

// Serial feasibility backend over plp::check_feasible_one: the same loop as
// the reference HostBackend (gpu/plp_gpu.cpp:18-32).
struct SerialBackend : plp::FeasibilityBackend {
    std::vector<uint8_t> check_all(const std::vector<plp::Pt>& cand,
                                   const std::vector<plp::Pt>& ors,
                                   const std::vector<plp::FastBox>& fast,
                                   int L, int W, int H) override {
        std::vector<uint8_t> bits(cand.size() * ors.size(), 0);
        for (size_t ci = 0; ci < cand.size(); ci++)
            for (size_t oi = 0; oi < ors.size(); oi++)
                bits[ci * ors.size() + oi] = plp::check_feasible_one(
                    cand[ci][0], cand[ci][1], cand[ci][2], ors[oi], fast, L, W, H);
        return bits;
    }
};

plp::RunResult run_fixed(const plp::Instance& inst, int seed, int passes, double eps,
                         double* theta, const std::string& order, bool first_fit,
                         plp::FeasibilityBackend& be) {
    if (passes == 1)
        return plp::run(inst, seed, 0.0, eps, theta, order, first_fit, true, be);
    auto t0 = std::chrono::steady_clock::now();
    plp::PyRng rng((uint64_t)seed);
    struct Pack { long long vol; int n; double score; std::vector<plp::PlacedBox> placed; };
    std::vector<Pack> packs;
    for (int k = 0; k < passes; k++) {
        auto placed = plp::decode_pass(inst, order, first_fit, eps, rng, be);
        long long vol = 0;
        for (const auto& b : placed) vol += 1LL * b.w * b.d * b.h;
        packs.push_back(Pack{vol, (int)placed.size(), plp::stability_score(placed), std::move(placed)});
    }
    std::vector<const Pack*> pool;
    for (const auto& p : packs)
        if (theta == nullptr || p.score >= *theta) pool.push_back(&p);
    const bool fallback = pool.empty();
    if (fallback)
        for (const auto& p : packs) pool.push_back(&p);
    const Pack* best = pool[0];
    for (size_t i = 1; i < pool.size(); i++)
        if (pool[i]->vol > best->vol || (pool[i]->vol == best->vol && pool[i]->n > best->n))
            best = pool[i];
    plp::RunResult r;
    for (const auto& b : best->placed)
        r.placements.push_back({b.item_type, b.x, b.y, b.z, b.w, b.d, b.h});
    r.n_boxes = best->n;
    r.volume = best->vol;
    r.score = best->score;
    r.fallback = fallback;
    r.n_passes = passes;
    r.seed = seed;
    r.time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return r;
}

}  // namespace

int main(int argc, char** argv) {
    std::vector<std::string> paths;
    std::string order = "volume";
    int seed = 0, restarts = 1, passes = 1, threads = 1, repeat = 1;
    double eps = plp::EPS_QUALITY, theta = plp::THETA;
    bool no_theta = false, first_fit = false, as_json = false;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", a.c_str()); std::exit(2); }
            return argv[++i];
        };
        if (a == "--seed") seed = std::atoi(next().c_str());
        else if (a == "--restarts") restarts = std::atoi(next().c_str());
        else if (a == "--passes") passes = std::atoi(next().c_str());
        else if (a == "--eps") eps = std::strtod(next().c_str(), nullptr);
        else if (a == "--theta") theta = std::strtod(next().c_str(), nullptr);
        else if (a == "--no-theta") no_theta = true;
        else if (a == "--order") order = next();
        else if (a == "--first-fit") first_fit = true;
        else if (a == "--mu") plp::MU = std::strtod(next().c_str(), nullptr);
        else if (a == "--threads") threads = std::atoi(next().c_str());
        else if (a == "--repeat") repeat = std::atoi(next().c_str());
        else if (a == "--json") as_json = true;
        else if (!a.empty() && a[0] != '-') paths.push_back(a);
        else { std::fprintf(stderr, "unknown flag: %s\n", a.c_str()); return 2; }
    }
    if (paths.empty() || restarts < 1 || passes < 1 || threads < 1) {
        std::fprintf(stderr, "usage: ref_harness <instance> [<instance> ...] [flags]\n");
        return 2;
    }
    std::vector<plp::Instance> insts(paths.size());
    for (size_t i = 0; i < paths.size(); i++) {
        try {
            insts[i] = plp::load_instance(paths[i]);
        } catch (const plp::InstanceFormatError& e) {
            std::fprintf(stderr, "instance error: %s\n", e.what());
            return 1;
        }
    }
    const long long n_work = (long long)insts.size() * restarts;
    std::vector<plp::RunResult> res(n_work);
    double total_s = 0;
    for (int rep = 0; rep < repeat; rep++) {
        std::atomic<long long> next_w{0};
        auto t0 = std::chrono::steady_clock::now();
        auto work = [&]() {
            SerialBackend be;
            for (;;) {
                long long w = next_w.fetch_add(1);
                if (w >= n_work) break;
                const int k = (int)(w % restarts);
                res[w] = run_fixed(insts[w / restarts], seed + k, passes, eps,
                                   no_theta ? nullptr : &theta, order, first_fit, be);
            }
        };
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; t++) pool.emplace_back(work);
        for (auto& t : pool) t.join();
        total_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    if (as_json) {
        for (const auto& r : res) std::cout << plp::to_json(r) << "\n";
    } else {
        std::printf("{\"decodes\": %lld, \"seconds\": %.9f, \"threads\": %d}\n",
                    n_work * repeat, total_s, threads);
    }
    return 0;
}
