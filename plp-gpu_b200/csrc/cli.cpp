// cli.cpp -- plp_gpu: drop-in for the reference plp_gpu / plp_gpu_cuda CLI
// (gpu/plp_gpu.cpp:80-143, gpu/plp_gpu.cu:1563-1696), built on the C ABI.
//
//   plp_gpu <instance> [--seed N] [--time S] [--eps F] [--theta F | --no-theta]
//           [--order volume|input] [--first-fit] [--mu F] [--single-pass] [--json]
//           [--batch K | --device K] [--passes N] [--plain] [--multi]
//   plp_gpu --selftest | --rngdump N
//
// Modes:
//   --single-pass or --passes N   persistent device decoder, fixed pass count
//   neither (wall-clock budget)   persistent device decoder, passes until
//                                 --time has elapsed for the restart (the
//                                 decoder reads the GPU's global timer)
//   --batch K / --device K        K restarts (row k = seed + k) in one launch;
//                                 JSON wrapper {"K", "n_passes", "time_s", "rows"}
//   --plain                       the per-step path instead: host pass loop
//                                 with one device feasibility launch per step
//   --multi                       accept a file with P >= 1 instances (the
//                                 reference rejects P > 1) and solve all of
//                                 them in one batched launch; one output line
//                                 per instance, in file order
// Exit codes: 0 ok; 1 instance error, CUDA error or device error; 2 usage.
#include <cmath>
#include <fstream>
#include <sstream>
#include <vector>
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
                 "                 [--order volume|input] [--first-fit] [--mu F] [--single-pass]\n"
                 "                 [--batch K | --device K] [--passes N] [--plain] [--multi] [--json]\n"
                 "       %s --selftest | --rngdump N\n",
                 prog, prog);
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

int rngdump(int n) {
    if (n < 1) {
        std::fprintf(stderr, "--rngdump N must be >= 1\n");
        return 2;
    }
    std::vector<int64_t> seeds(n);
    for (int k = 0; k < n; k++) seeds[k] = k;
    std::vector<double> dr((size_t)n * 16);
    std::vector<uint32_t> db((size_t)n * 16);
    if (plp_rng_dump(seeds.data(), n, 16, 16, 13, dr.data(), db.data()) != PLP_OK) {
        std::fprintf(stderr, "rngdump: %s\n", plp_last_error(nullptr));
        return 1;
    }
    std::vector<double> hr((size_t)n * 16);
    std::vector<uint32_t> hb((size_t)n * 16);
    plp_rng_dump_host(seeds.data(), n, 16, 16, 13, hr.data(), hb.data());
    bool ok = true;
    for (int k = 0; k < n; k++) {
        bool row = true;
        for (int i = 0; i < 16; i++) {
            const size_t q = (size_t)k * 16 + i;
            if (hr[q] != dr[q]) {
                row = false;
                std::fprintf(stderr, "row %d random[%d]: host %s dev %s\n", k, i, repr(hr[q]).c_str(),
                             repr(dr[q]).c_str());
            }
            if (hb[q] != db[q]) {
                row = false;
                std::fprintf(stderr, "row %d getrandbits[%d]: host %u dev %u\n", k, i, hb[q], db[q]);
            }
        }
        std::printf("SEED %d: %s\n", k, row ? "PASS" : "FAIL");
        ok = ok && row;
    }
    std::printf("RNGDUMP: %s\n", ok ? "PASS" : "FAIL");
    return ok ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
    std::string path, order = "volume";
    long long seed = 0;
    double time_s = 300.0, eps = 0.3, theta = 0.9, mu = 0.2;
    bool no_theta = false, first_fit = false, single = false, as_json = false, plain = false, multi = false;
    int batch = 0, device = 0, passes = 0;
    if (const char* e = std::getenv("PLP_MU")) mu = std::strtod(e, nullptr);
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto next = [&](const char* what) -> std::string {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", what);
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--selftest") {
            size_t need = 0;
            plp_selftest(nullptr, 0, &need);
            std::string s(need + 1, '\0');
            plp_selftest(&s[0], s.size(), &need);
            std::fwrite(s.data(), 1, need, stdout);
            return 0;
        } else if (a == "--rngdump") return rngdump(std::atoi(next("--rngdump").c_str()));
        else if (a == "--seed") seed = std::atoll(next("--seed").c_str());
        else if (a == "--time") time_s = std::strtod(next("--time").c_str(), nullptr);
        else if (a == "--eps") eps = std::strtod(next("--eps").c_str(), nullptr);
        else if (a == "--mu") mu = std::strtod(next("--mu").c_str(), nullptr);
        else if (a == "--theta") theta = std::strtod(next("--theta").c_str(), nullptr);
        else if (a == "--no-theta") no_theta = true;
        else if (a == "--order") order = next("--order");
        else if (a == "--first-fit") first_fit = true;
        else if (a == "--single-pass") single = true;
        else if (a == "--json") as_json = true;
        else if (a == "--batch") batch = std::atoi(next("--batch").c_str());
        else if (a == "--device") device = std::atoi(next("--device").c_str());
        else if (a == "--passes") passes = std::atoi(next("--passes").c_str());
        else if (a == "--plain") plain = true;
        else if (a == "--multi") multi = true;
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
    std::vector<plp_instance*> insts;
    if (multi) {
        std::ifstream f(path, std::ios::binary);
        if (!f) {
            std::fprintf(stderr, "instance error: cannot open %s\n", path.c_str());
            return 1;
        }
        std::ostringstream ss;
        ss << f.rdbuf();
        const std::string text = ss.str();
        plp_instance** arr = nullptr;
        int32_t n = 0;
        if (plp_instance_parse_multi(text.data(), text.size(), &arr, &n) != PLP_OK) {
            std::fprintf(stderr, "instance error: %s\n", plp_last_error(nullptr));
            return 1;
        }
        insts.assign(arr, arr + n);
        plp_free(arr);
    } else {
        plp_instance* one = nullptr;
        if (plp_instance_load(path.c_str(), &one) != PLP_OK) {
            std::fprintf(stderr, "instance error: %s\n", plp_last_error(nullptr));
            return 1;
        }
        insts.push_back(one);
    }
    auto free_insts = [&]() {
        for (plp_instance* i : insts) plp_instance_free(i);
        insts.clear();
    };
    if (order != "volume" && order != "input") {
        std::fprintf(stderr, "unknown order %s\n", order.c_str());
        free_insts();
        return 2;
    }
    if (batch && device) {
        std::fprintf(stderr, "--device and --batch are mutually exclusive\n");
        return 2;
    }
    const int K = batch ? batch : device;
    if ((batch || device) && !as_json) {
        std::fprintf(stderr, "%s requires --json\n", batch ? "--batch" : "--device");
        return 2;
    }
    if ((batch || device) && K < 1) {
        std::fprintf(stderr, "%s K must be >= 1\n", batch ? "--batch" : "--device");
        return 2;
    }
    if (passes < 0) { std::fprintf(stderr, "--passes N must be >= 1\n"); return 2; }
    plp_run_opts o;
    plp_default_opts(&o);
    o.seed = seed;
    o.restarts = K ? K : 1;
    o.eps = eps;
    o.theta = no_theta ? NAN : theta;
    o.order = order == "volume" ? 0 : 1;
    o.first_fit = first_fit ? 1 : 0;
    o.mu = mu;
    const bool fixed = single || passes > 0;
    o.passes = single ? 1 : (passes > 0 ? passes : 0);   // 0: no cap under --time
    o.time_limit_s = fixed ? -1.0 : time_s;
    const int n_inst = (int)insts.size();
    std::vector<plp_result*> res(n_inst, nullptr);
    int st = PLP_OK;
    if (plain) {
        for (int i = 0; i < n_inst && st == PLP_OK; i++) st = plp_run_plain(insts[i], &o, &res[i]);
    } else {
        plp_handle* h = nullptr;
        st = plp_create(0, 0, &h);
        if (st == PLP_OK) {
            st = plp_solve(h, insts.data(), n_inst, &o, 1, res.data());
            if (st != PLP_OK) std::fprintf(stderr, "solve: %s\n", plp_last_error(h));
            plp_destroy(h);
        }
    }
    free_insts();
    auto free_res = [&]() {
        for (plp_result* r : res)
            if (r) plp_result_free(r);
    };
    if (st != PLP_OK) {
        std::fprintf(stderr, "error: %s\n", plp_last_error(nullptr));
        free_res();
        return 1;
    }
    for (plp_result* r : res) {
        for (int k = 0; k < plp_result_restarts(r); k++) {
            plp_summary s;
            plp_result_summary(r, k, &s);
            if (s.err) {
                std::fprintf(stderr, "device decode error flag %d\n", s.err);
                free_res();
                return 1;
            }
        }
    }
    for (plp_result* r : res) {
        if (K) {
            plp_summary s0;
            plp_result_summary(r, 0, &s0);
            std::printf("{\"K\": %d, \"n_passes\": %d, \"time_s\": %s, \"rows\": [", K, s0.n_passes,
                        repr(s0.time_s).c_str());
            for (int k = 0; k < K; k++) std::printf("%s%s", k ? ", " : "", json_of(r, k).c_str());
            std::printf("]}\n");
        } else if (as_json) {
            std::printf("%s\n", json_of(r, 0).c_str());
        } else {
            plp_summary s;
            plp_result_summary(r, 0, &s);
            std::printf("n_boxes=%d volume_cm3=%lld stability_score=%.4f fallback=%s n_passes=%d "
                        "time_s=%.3f\n",
                        s.n_boxes, (long long)s.volume, s.score, s.fallback ? "true" : "false",
                        s.n_passes, s.time_s);
        }
    }
    free_res();
    return 0;
}
