// cli_block.cpp -- plp_block: drop-in for the reference's block-building
// engine binaries plp_block (blockproof/plp_block.cpp:306-386) and
// plp_block_cuda (blockproof/plp_block_cuda.cu:1142-1254), on the C ABI.
//
//   plp_block <instance> [--seed N] [--time S] [--eps F] [--theta F | --no-theta]
//             [--amax A] [--bmax B] [--kmax K] [--topk N]
//             [--pick first|support|contact] [--single-pass] [--passes N]
//             [--device K] [--json]
//
// Every restart runs on the device (block engine, one warp per restart).
// Without --device the output is the CPU build's: one JSON line (plus
// fill_pct on stderr) or one text line. With --device K the rows are
// seed .. seed + K - 1 in one launch and the output is the CUDA build's: for
// K = 1 the plain JSON line, else the {"K", "n_passes", "time_s", "rows"}
// wrapper; text mode prints one "seed=..." line per row. Without
// --single-pass / --passes, --time S is the per-restart wall-clock budget.
// Exit codes: 0 ok; 1 instance, CUDA or device error; 2 usage.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/plp_capi.h"

namespace {

void usage(const char* prog) {
    std::fprintf(stderr,
                 "usage: %s <instance> [--seed N] [--time S] [--eps F] [--theta F | --no-theta]\n"
                 "                 [--amax A] [--bmax B] [--kmax K] [--topk N]\n"
                 "                 [--pick first|support|contact] [--single-pass] [--passes N]\n"
                 "                 [--device K] [--json]\n",
                 prog);
}

std::string json_of(const plp_result* r, int k) {
    size_t need = 0;
    plp_result_json(r, k, nullptr, 0, &need);
    std::string s(need + 1, '\0');
    plp_result_json(r, k, &s[0], s.size(), &need);
    s.resize(need);
    return s;
}

std::string repr(double v) {
    char b[64];
    plp_py_repr(v, b, sizeof b);
    return b;
}

}  // namespace

int main(int argc, char** argv) {
    std::string path;
    long long seed = 0;
    int amax = 3, bmax = 3, kmax = 4, topk = 8, pick = 0, device = 0, passes = 0;
    double time_s = 300.0, eps = 0.3, theta = 0.9;
    bool no_theta = false, single = false, as_json = false;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto next = [&](const char* what) -> std::string {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", what);
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--seed") seed = std::atoll(next("--seed").c_str());
        else if (a == "--time") time_s = std::strtod(next("--time").c_str(), nullptr);
        else if (a == "--eps") eps = std::strtod(next("--eps").c_str(), nullptr);
        else if (a == "--theta") theta = std::strtod(next("--theta").c_str(), nullptr);
        else if (a == "--no-theta") no_theta = true;
        else if (a == "--amax") amax = std::atoi(next("--amax").c_str());
        else if (a == "--bmax") bmax = std::atoi(next("--bmax").c_str());
        else if (a == "--kmax") kmax = std::atoi(next("--kmax").c_str());
        else if (a == "--topk") topk = std::max(1, std::atoi(next("--topk").c_str()));
        else if (a == "--pick") {
            const std::string v = next("--pick");
            if (v == "first") pick = 0;
            else if (v == "support") pick = 1;
            else if (v == "contact") pick = 2;
            else {
                std::fprintf(stderr, "bad --pick: %s (first|support|contact)\n", v.c_str());
                return 2;
            }
        }
        else if (a == "--single-pass") single = true;
        else if (a == "--passes") passes = std::atoi(next("--passes").c_str());
        else if (a == "--device") device = std::atoi(next("--device").c_str());
        else if (a == "--json") as_json = true;
        else if (a == "-h" || a == "--help") { usage(argv[0]); return 0; }
        else if (!a.empty() && a[0] != '-') {
            if (!path.empty()) { usage(argv[0]); return 2; }
            path = a;
        } else {
            std::fprintf(stderr, "unknown flag: %s\n", a.c_str());
            usage(argv[0]);
            return 2;
        }
    }
    if (path.empty()) { usage(argv[0]); return 2; }
    amax = std::max(1, amax);
    bmax = std::max(1, bmax);
    kmax = std::max(1, kmax);
    const bool dev_mode = device != 0;
    if (dev_mode && device < 1) {
        std::fprintf(stderr, "--device K must be >= 1\n");
        return 2;
    }
    if (passes < 0) {
        std::fprintf(stderr, "--passes N must be >= 1\n");
        return 2;
    }
    plp_instance* inst = nullptr;
    if (plp_instance_load(path.c_str(), &inst) != PLP_OK) {
        std::fprintf(stderr, "instance error: %s\n", plp_last_error(nullptr));
        return 1;
    }
    int32_t lwh[3] = {0, 0, 0}, n_types = 0, n_items = 0;
    plp_instance_info(inst, lwh, &n_types, &n_items);
    const double cvol = (double)(1LL * lwh[0] * lwh[1] * lwh[2]);
    plp_run_opts o;
    plp_default_opts(&o);
    o.seed = seed;
    o.restarts = dev_mode ? device : 1;
    o.eps = eps;
    o.theta = no_theta ? NAN : theta;
    o.mu = 0.2;   // the block engine scores with the default friction coefficient
    const bool fixed = single || passes > 0;
    o.passes = single ? 1 : (passes > 0 ? passes : 0);
    o.time_limit_s = fixed ? -1.0 : time_s;
    o.engine = 1;
    o.blk_amax = amax;
    o.blk_bmax = bmax;
    o.blk_kmax = kmax;
    o.blk_topk = topk;
    o.blk_pick = pick;
    plp_handle* h = nullptr;
    plp_result* res = nullptr;
    int st = plp_create(0, 0, &h);
    if (st == PLP_OK) {
        const plp_instance* one = inst;
        st = plp_solve(h, &one, 1, &o, 1, &res);
        if (st != PLP_OK) std::fprintf(stderr, "solve: %s\n", plp_last_error(h));
        plp_destroy(h);
    }
    plp_instance_free(inst);
    if (st != PLP_OK) {
        std::fprintf(stderr, "error: %s\n", plp_last_error(nullptr));
        return 1;
    }
    const int K = plp_result_restarts(res);
    for (int k = 0; k < K; k++) {
        plp_summary s;
        plp_result_summary(res, k, &s);
        if (s.err) {
            std::fprintf(stderr, "device decode error flag %d\n", s.err);
            plp_result_free(res);
            return 1;
        }
    }
    if (as_json) {
        if (K == 1) {
            plp_summary s;
            plp_result_summary(res, 0, &s);
            std::printf("%s\n", json_of(res, 0).c_str());
            std::fprintf(stderr, "fill_pct=%.4f\n", 100.0 * (double)s.volume / cvol);
        } else {
            plp_summary s0;
            plp_result_summary(res, 0, &s0);
            std::printf("{\"K\": %d, \"n_passes\": %d, \"time_s\": %s, \"rows\": [", K, s0.n_passes,
                        repr(s0.time_s).c_str());
            for (int k = 0; k < K; k++) std::printf("%s%s", k ? ", " : "", json_of(res, k).c_str());
            std::printf("]}\n");
        }
    } else {
        for (int k = 0; k < K; k++) {
            plp_summary s;
            plp_result_summary(res, k, &s);
            const double fill = 100.0 * (double)s.volume / cvol;
            if (dev_mode)
                std::printf("seed=%lld n_boxes=%d volume_cm3=%lld fill_pct=%.4f stability_score=%.4f fallback=%s "
                            "n_passes=%d time_s=%.3f\n",
                            (long long)s.seed, s.n_boxes, (long long)s.volume, fill, s.score,
                            s.fallback ? "true" : "false", s.n_passes, s.time_s);
            else
                std::printf("n_boxes=%d volume_cm3=%lld fill_pct=%.4f stability_score=%.4f fallback=%s n_passes=%d "
                            "time_s=%.3f\n",
                            s.n_boxes, (long long)s.volume, fill, s.score, s.fallback ? "true" : "false",
                            s.n_passes, s.time_s);
        }
    }
    plp_result_free(res);
    return 0;
}
