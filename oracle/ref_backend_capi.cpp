// ref_backend_capi.cpp -- the reference decoder (its gpu/plp_common.hpp,
// compiled from the reference tree) running on this library's one-step
// feasibility kernel through the C ABI: the binding a maintainer of the
// reference would add to drop the B200 backend in behind
// FeasibilityBackend::check_all (gpu/plp_common.hpp:326-332). Built into
// oracle/_ref/plp_gpu_capi by `make -C oracle ref`; the GPU tests compare its
// JSON with the reference's own host build (oracle/_ref/plp_gpu).
//
//   plp_gpu_capi <instance> [--seed N] [--eps F] [--theta F | --no-theta]
//                [--order volume|input] [--first-fit] [--single-pass] --json
#include "plp_common.hpp"
#include "plp_capi.h"

namespace {

struct CapiBackend : plp::FeasibilityBackend {
    std::vector<int32_t> c, o, f;
    std::vector<uint8_t> check_all(const std::vector<plp::Pt>& cand, const std::vector<plp::Pt>& ors,
                                   const std::vector<plp::FastBox>& fast, int L, int W,
                                   int H) override {
        c.clear();
        o.clear();
        f.clear();
        for (const auto& p : cand) c.insert(c.end(), {p[0], p[1], p[2]});
        for (const auto& p : ors) o.insert(o.end(), {p[0], p[1], p[2]});
        for (const auto& b : fast) f.insert(f.end(), {b.x, b.y, b.z, b.x2, b.y2, b.z2});
        std::vector<uint8_t> bits(cand.size() * ors.size(), 0);
        const int s = plp_feas_check_all(c.data(), (int32_t)cand.size(), o.data(), (int32_t)ors.size(),
                                         f.data(), (int32_t)fast.size(), L, W, H, bits.data());
        if (s != PLP_OK) {
            std::fprintf(stderr, "plp_feas_check_all: %s\n", plp_last_error(nullptr));
            std::exit(1);
        }
        return bits;
    }
};

}  // namespace

int main(int argc, char** argv) {
    std::string path, order = "volume";
    int seed = 0;
    double eps = plp::EPS_QUALITY, theta = plp::THETA;
    bool no_theta = false, first_fit = false;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        if (a == "--seed" && i + 1 < argc) seed = std::atoi(argv[++i]);
        else if (a == "--eps" && i + 1 < argc) eps = std::strtod(argv[++i], nullptr);
        else if (a == "--theta" && i + 1 < argc) theta = std::strtod(argv[++i], nullptr);
        else if (a == "--no-theta") no_theta = true;
        else if (a == "--order" && i + 1 < argc) order = argv[++i];
        else if (a == "--first-fit") first_fit = true;
        else if (a == "--single-pass" || a == "--json") continue;
        else if (!a.empty() && a[0] != '-') path = a;
        else { std::fprintf(stderr, "unknown flag: %s\n", a.c_str()); return 2; }
    }
    plp::Instance inst;
    try {
        inst = plp::load_instance(path);
    } catch (const plp::InstanceFormatError& e) {
        std::fprintf(stderr, "instance error: %s\n", e.what());
        return 1;
    }
    CapiBackend be;
    plp::RunResult r = plp::run(inst, seed, 0.0, eps, no_theta ? nullptr : &theta, order, first_fit, true, be);
    std::cout << plp::to_json(r) << "\n";
    return 0;
}
