// feas.cu -- one-step feasibility kernel (kernel a) and the C-ABI entry
// points that replace the reference's per-step backend:
//   FeasibilityBackend::check_all   gpu/plp_common.hpp:326-332
//   CudaBackend::check_all          gpu/plp_gpu.cu:443-495 (one launch per step)
//
// One CTA stages the placed boxes in shared memory with 128-bit loads, orders
// them by top z (rank sort), and each thread evaluates one candidate point
// against every orientation (feas_eval.cuh). bits[ci * n_ors + oi] follow the
// reference's candidate-major order. The optional first-feasible output is a
// warp-ballot argmin folded across warps with atomicMin.
#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "capi_internal.hpp"
#include "device_common.cuh"
#include "engine.hpp"
#include "feas_eval.cuh"

namespace plpb {

constexpr int FEAS_BLOCK = 256;

__global__ void __launch_bounds__(FEAS_BLOCK) feas_kernel(
    const int* __restrict__ cand, int n_cand, const int* __restrict__ ors, int n_ors,
    const int* __restrict__ fast6, int n_fast, int L, int W, int H,
    unsigned char* __restrict__ bits, int* __restrict__ first_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // raw copy of fast6 (6 ints per box, padded to a 16-byte multiple), then
    // the top-sorted tables
    int* raw = reinterpret_cast<int*>(smem_raw);
    const int raw_ints = (6 * n_fast + 3) & ~3;
    int4* bx = reinterpret_cast<int4*>(smem_raw + 4 * raw_ints);
    int* bz = reinterpret_cast<int*>(bx + n_fast);
    int* z2 = bz + n_fast;
    const bool aligned = (reinterpret_cast<uintptr_t>(fast6) & 15) == 0;
    const int n4 = (6 * n_fast) / 4;
    if (aligned) {
        const int4* src = reinterpret_cast<const int4*>(fast6);
        for (int i = threadIdx.x; i < n4; i += blockDim.x) reinterpret_cast<int4*>(raw)[i] = src[i];
        for (int i = 4 * n4 + threadIdx.x; i < 6 * n_fast; i += blockDim.x) raw[i] = fast6[i];
    } else {
        for (int i = threadIdx.x; i < 6 * n_fast; i += blockDim.x) raw[i] = fast6[i];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_fast; i += blockDim.x) {
        const int* b = raw + 6 * i;
        int rank = 0;
        for (int j = 0; j < n_fast; j++) {
            const int t = raw[6 * j + 5];
            rank += t < b[5] || (t == b[5] && j < i);
        }
        bx[rank] = make_int4(b[0], b[1], b[3], b[4]);
        bz[rank] = b[2];
        z2[rank] = b[5];
    }
    __syncthreads();
    const Boxes B{bx, bz, z2, n_fast};
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    int first = INT_MAX;
    if (ci < n_cand) {
        const int x = cand[3 * ci], y = cand[3 * ci + 1], z = cand[3 * ci + 2];
        for (int o0 = 0; o0 < n_ors; o0 += 6) {
            const int no = min(6, n_ors - o0);
            int ow[6], od[6], oh[6];
#pragma unroll
            for (int o = 0; o < 6; o++) {
                ow[o] = o < no ? ors[3 * (o0 + o)] : 0;
                od[o] = o < no ? ors[3 * (o0 + o) + 1] : 0;
                oh[o] = o < no ? ors[3 * (o0 + o) + 2] : 0;
            }
            const unsigned m = eval_point<long long>(x, y, z, ow, od, oh, no, L, W, H, B);
            for (int o = 0; o < no; o++) bits[(long long)ci * n_ors + o0 + o] = (m >> o) & 1u;
            if (m && first == INT_MAX) first = ci * n_ors + o0 + __ffs(m) - 1;
        }
    }
    if (first_out) {
        // candidates are contiguous per warp, so the lowest lane holding a
        // feasible pair holds the warp's smallest pair index
        const unsigned bal = __ballot_sync(FULL, first != INT_MAX);
        if (bal && (threadIdx.x & 31) == __ffs(bal) - 1) atomicMin(first_out, first);
    }
}

static int feas_smem_bytes(int n_fast) {
    const int raw_ints = (6 * n_fast + 3) & ~3;
    return 4 * raw_ints + 24 * n_fast;
}

cudaError_t launch_feas(const int* cand, int n_cand, const int* ors, int n_ors, const int* fast6,
                        int n_fast, int L, int W, int H, unsigned char* bits, int* first_out,
                        cudaStream_t st) {
    if (n_cand <= 0 || n_ors <= 0) return cudaSuccess;
    const int smem = feas_smem_bytes(n_fast);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(feas_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
    }
    const int grid = (n_cand + FEAS_BLOCK - 1) / FEAS_BLOCK;
    feas_kernel<<<grid, FEAS_BLOCK, smem, st>>>(cand, n_cand, ors, n_ors, fast6, n_fast, L, W, H,
                                                bits, first_out);
    return cudaGetLastError();
}

// largest placed-box list one launch stages in shared memory (227 KB opt-in)
constexpr int FEAS_MAX_FAST = (227 * 1024) / 48;

// ---------------------------------------------------------------------------
// per-thread context of the host-buffer entry point and the plain path
// ---------------------------------------------------------------------------
struct StepCtx {
    cudaStream_t stream = nullptr;
    int device = -1;
    char* h_stage = nullptr;   // pinned: [cand | ors | fast | first] in, bits out
    char* d_stage = nullptr;
    size_t cap = 0;
    ~StepCtx() {
        if (h_stage) cudaFreeHost(h_stage);
        if (d_stage) cudaFree(d_stage);
        if (stream) cudaStreamDestroy(stream);
    }
    cudaError_t ensure(size_t need) {
        cudaError_t e = cudaSuccess;
        if (!stream) {
            e = cudaGetDevice(&device);
            if (e != cudaSuccess) return e;
            e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
            if (e != cudaSuccess) return e;
        }
        if (need <= cap) return cudaSuccess;
        size_t nc = cap ? cap : 1 << 16;
        while (nc < need) nc *= 2;
        if (h_stage) cudaFreeHost(h_stage);
        if (d_stage) cudaFree(d_stage);
        h_stage = nullptr;
        d_stage = nullptr;
        cap = 0;
        e = cudaMallocHost(&h_stage, nc);
        if (e != cudaSuccess) return e;
        e = cudaMalloc(&d_stage, nc);
        if (e != cudaSuccess) return e;
        cap = nc;
        return cudaSuccess;
    }
};

static StepCtx& step_ctx() {
    thread_local StepCtx ctx;
    return ctx;
}

static size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

// One step on the thread's stream: copy inputs in one transfer, launch, copy
// the bits back, synchronise. Returns the smallest feasible pair index (or
// INT_MAX) through first (when non-null).
static int step_check(const int32_t* cand, int n_cand, const int32_t* ors, int n_ors,
                      const int32_t* fast6, int n_fast, int L, int W, int H, uint8_t* bits_out,
                      int* first) {
    StepCtx& c = step_ctx();
    const size_t o_cand = 0;
    const size_t o_ors = align16(o_cand + 12 * (size_t)n_cand);
    const size_t o_fast = align16(o_ors + 12 * (size_t)n_ors);
    const size_t o_first = align16(o_fast + 24 * (size_t)n_fast);
    const size_t o_bits = align16(o_first + 16);
    const size_t nbits = (size_t)n_cand * n_ors;
    const size_t total = o_bits + nbits;
    cudaError_t e = c.ensure(total);
    if (e != cudaSuccess) return set_cuda_error("plp_feas_check_all: allocation", e);
    std::memcpy(c.h_stage + o_cand, cand, 12 * (size_t)n_cand);
    std::memcpy(c.h_stage + o_ors, ors, 12 * (size_t)n_ors);
    if (n_fast) std::memcpy(c.h_stage + o_fast, fast6, 24 * (size_t)n_fast);
    *reinterpret_cast<int*>(c.h_stage + o_first) = INT_MAX;
    e = cudaMemcpyAsync(c.d_stage, c.h_stage, o_bits, cudaMemcpyHostToDevice, c.stream);
    if (e != cudaSuccess) return set_cuda_error("plp_feas_check_all: copy in", e);
    int* d_first = reinterpret_cast<int*>(c.d_stage + o_first);
    e = launch_feas(reinterpret_cast<const int*>(c.d_stage + o_cand), n_cand,
                    reinterpret_cast<const int*>(c.d_stage + o_ors), n_ors,
                    reinterpret_cast<const int*>(c.d_stage + o_fast), n_fast, L, W, H,
                    reinterpret_cast<unsigned char*>(c.d_stage + o_bits), d_first, c.stream);
    if (e != cudaSuccess) return set_cuda_error("plp_feas_check_all: launch", e);
    e = cudaMemcpyAsync(c.h_stage + o_first, c.d_stage + o_first, o_bits - o_first + nbits,
                        cudaMemcpyDeviceToHost, c.stream);
    if (e != cudaSuccess) return set_cuda_error("plp_feas_check_all: copy out", e);
    e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) return set_cuda_error("plp_feas_check_all: sync", e);
    if (bits_out) std::memcpy(bits_out, c.h_stage + o_bits, nbits);
    if (first) *first = *reinterpret_cast<int*>(c.h_stage + o_first);
    return PLP_OK;
}

static int check_feas_args(int n_cand, int n_ors, int n_fast, int L, int W, int H,
                           const void* cand, const void* ors, const void* fast, const void* out) {
    if (n_cand < 0 || n_ors < 0 || n_fast < 0)
        return set_error(PLP_E_INVALID, "plp_feas_check_all: negative size");
    if ((n_cand && !cand) || (n_ors && !ors) || (n_fast && !fast) || (n_cand && n_ors && !out))
        return set_error(PLP_E_INVALID, "plp_feas_check_all: null buffer");
    if (n_fast > FEAS_MAX_FAST)
        return set_error(PLP_E_CAPACITY, "plp_feas_check_all: more than " +
                                             std::to_string(FEAS_MAX_FAST) + " placed boxes");
    (void)L; (void)W; (void)H;
    return PLP_OK;
}

}  // namespace plpb

using namespace plpb;

extern "C" int plp_feas_check_all(const int32_t* cand_xyz, int32_t n_cand, const int32_t* ors_wdh,
                                  int32_t n_ors, const int32_t* fast6, int32_t n_fast, int32_t L,
                                  int32_t W, int32_t H, uint8_t* bits_out) {
    int s = check_feas_args(n_cand, n_ors, n_fast, L, W, H, cand_xyz, ors_wdh, fast6, bits_out);
    if (s != PLP_OK) return s;
    if ((long long)n_cand * n_ors == 0) return PLP_OK;
    return step_check(cand_xyz, n_cand, ors_wdh, n_ors, fast6, n_fast, L, W, H, bits_out, nullptr);
}

extern "C" int plp_feas_check_all_dev(const int32_t* d_cand_xyz, int32_t n_cand,
                                      const int32_t* d_ors_wdh, int32_t n_ors,
                                      const int32_t* d_fast6, int32_t n_fast, int32_t L, int32_t W,
                                      int32_t H, uint8_t* d_bits_out, void* stream) {
    int s = check_feas_args(n_cand, n_ors, n_fast, L, W, H, d_cand_xyz, d_ors_wdh, d_fast6,
                            d_bits_out);
    if (s != PLP_OK) return s;
    cudaError_t e = launch_feas(d_cand_xyz, n_cand, d_ors_wdh, n_ors, d_fast6, n_fast, L, W, H,
                                d_bits_out, nullptr, reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return set_cuda_error("plp_feas_check_all_dev: launch", e);
    return PLP_OK;
}

namespace plpb {

// ---------------------------------------------------------------------------
// plain path: the reference's host decode loop (gpu/plp_common.hpp:404-456)
// with one feasibility launch per item step, and the device FSR per pass.
// ---------------------------------------------------------------------------
int run_plain(const Instance& inst, const plp_run_opts& o, std::vector<RunSummary>& summ,
              std::vector<std::vector<Placement>>& placements) {
    const std::vector<int> seq = item_sequence(inst, o.order);
    std::vector<std::vector<Dims>> ors;
    for (const auto& t : inst.types) ors.push_back(orientations(t));
    const bool has_theta = !std::isnan(o.theta);
    const bool randomized = !(o.first_fit || o.eps == 0.0);
    summ.assign(o.restarts, RunSummary{});
    placements.assign(o.restarts, {});
    std::vector<int32_t> cand, fast, orsf;
    std::vector<uint8_t> bits;
    for (int r = 0; r < o.restarts; r++) {
        const long long seed = o.seed + r;
        PyRng rng((uint64_t)(seed < 0 ? -seed : seed));
        const double t0 = now_seconds();
        bool have_acc = false, have_any = false;
        long long best_vol = 0;
        int best_n = 0;
        double best_score = 0;
        std::vector<Placement> best, cur;
        int k = 0;
        for (;;) {
            cur.clear();
            cand.assign({0, 0, 0});
            fast.clear();
            long long vol = 0;
            for (int t : seq) {
                const auto& ot = ors[t];
                if (ot.empty()) continue;
                orsf.clear();
                for (const auto& d : ot) orsf.insert(orsf.end(), d.begin(), d.end());
                const int nc = (int)cand.size() / 3, no = (int)ot.size();
                bits.resize((size_t)nc * no);
                int first = INT_MAX;
                int s = step_check(cand.data(), nc, orsf.data(), no, fast.data(),
                                   (int)fast.size() / 6, inst.L, inst.W, inst.H, bits.data(), &first);
                if (s != PLP_OK) return s;
                if (first == INT_MAX) continue;
                int pick = first;
                if (randomized && rng.random() >= 1.0 - o.eps) {
                    int cnt = 0;
                    for (size_t p = (size_t)first; p < bits.size(); p++) cnt += bits[p];
                    int idx = rng.randrange(cnt);
                    for (size_t p = (size_t)first; p < bits.size(); p++)
                        if (bits[p] && idx-- == 0) { pick = (int)p; break; }
                }
                const int ci = pick / no, oi = pick % no;
                const int x = cand[3 * ci], y = cand[3 * ci + 1], z = cand[3 * ci + 2];
                const int w = ot[oi][0], d = ot[oi][1], h = ot[oi][2];
                cur.push_back({t, x, y, z, w, d, h});
                vol += 1LL * w * d * h;
                fast.insert(fast.end(), {x, y, z, x + w, y + d, z + h});
                // extreme points: drop those strictly inside, add 8 corners,
                // keep sorted by (z, y, x) and unique
                std::vector<std::array<int, 3>> pts;
                pts.reserve(nc + 8);
                for (int i = 0; i < nc; i++) {
                    const int px = cand[3 * i], py = cand[3 * i + 1], pz = cand[3 * i + 2];
                    if (x < px && px < x + w && y < py && py < y + d && z < pz && pz < z + h) continue;
                    pts.push_back({pz, py, px});
                }
                for (int c = 0; c < 8; c++)
                    pts.push_back({z + ((c & 4) ? h : 0), y + ((c & 2) ? d : 0), x + ((c & 1) ? w : 0)});
                std::sort(pts.begin(), pts.end());
                pts.erase(std::unique(pts.begin(), pts.end()), pts.end());
                cand.clear();
                for (const auto& p : pts) cand.insert(cand.end(), {p[2], p[1], p[0]});
            }
            k++;
            double score = 0;
            int s = device_fsr_score(cur, o.mu, &score);
            if (s != PLP_OK) return s;
            const int n = (int)cur.size();
            const bool acc = !has_theta || score >= o.theta;
            bool take;
            if (acc) take = !have_acc || vol > best_vol || (vol == best_vol && n > best_n);
            else take = !have_acc && (!have_any || vol > best_vol || (vol == best_vol && n > best_n));
            if (take) {
                best_vol = vol;
                best_n = n;
                best_score = score;
                best = cur;
            }
            have_any = true;
            have_acc = have_acc || acc;
            const bool done = o.time_limit_s < 0
                                  ? k >= o.passes
                                  : now_seconds() - t0 >= o.time_limit_s || (o.passes > 0 && k >= o.passes);
            if (done) break;
        }
        RunSummary& S = summ[r];
        S.n_boxes = best_n;
        S.volume = best_vol;
        S.score = best_score;
        S.fallback = !have_acc;
        S.n_passes = k;
        S.seed = seed;
        S.time_s = now_seconds() - t0;
        placements[r] = std::move(best);
    }
    return PLP_OK;
}

}  // namespace plpb
