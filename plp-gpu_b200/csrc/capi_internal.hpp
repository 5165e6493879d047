// capi_internal.hpp -- internal declarations shared by the C-ABI sources.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "../../include/plp_capi.h"
#include "device_common.cuh"
#include "host_core.hpp"

struct plp_instance {
    plpb::Instance inst;
};

// Results of one instance's restarts. Placements are kept in the device's
// packed form (8 bytes each) and expanded on request.
struct plp_result {
    int restarts = 0;
    // plain path: summaries and expanded rows
    std::vector<plp_summary> summ;
    std::vector<plpb::Placement> rows;
    std::vector<long long> row_off;           // restarts + 1 (plain path)
    // device path: the decoders' slot heads and packed placement words,
    // read in place from a host block shared by the results of one batch
    std::shared_ptr<const char> block;
    const plpb::SlotHead* heads = nullptr;    // one per restart
    const unsigned long long* packed = nullptr;   // `stride` words per kept restart
    bool kept_all = true;                     // false: only the best restart's placements
    long long seed0 = 0;                      // seed of restart 0
    double time_s = 0;
    int stride = 0;
    std::vector<plpb::TypeOrs> ors;
    int L = 0, W = 0, H = 0;
    std::vector<int> steps;                   // type of each decode step
    int best = -1;
    int best_fallback = 1;

    plp_summary summary(int k) const {
        if (!heads) return summ[k];
        const plpb::SlotHead& h = heads[k];
        plp_summary s;
        s.n_boxes = h.n_boxes;
        s.fallback = h.fallback;
        s.volume = h.volume;
        s.score = h.score;
        s.n_passes = h.n_passes;
        s.err = h.err;
        s.seed = seed0 + k;
        s.time_s = time_s;
        return s;
    }
    // index of restart k's placements in `packed` (-1: not kept)
    int packed_slot(int k) const { return kept_all ? k : (k == best ? 0 : -1); }
};

namespace plpb {

int set_error(int code, const std::string& msg);
int set_cuda_error(const char* what, cudaError_t e);
std::string plpb_last();
double now_seconds();

int run_plain(const Instance& inst, const plp_run_opts& o, std::vector<RunSummary>& summ,
              std::vector<std::vector<Placement>>& placements);
// device FSR of one packing (the plain path's scorer)
int device_fsr_score(const std::vector<Placement>& p, double mu, double* score);
// init_genrand(19650218) table on the current device (uploaded once)
const uint32_t* device_mt_init(int* status);
void mt_init_table(uint32_t out[624]);

}  // namespace plpb
