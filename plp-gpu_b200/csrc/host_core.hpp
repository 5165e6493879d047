// host_core.hpp -- host-side instance model, thpack parser, orientation and
// item-order tables, a CPython-compatible MT19937, and the reference JSON
// writer. Built with -ffp-contract=off like the reference host build.
//
// Reference semantics (pqant/plp-gpu):
//   parser + errors   gpu/plp_common.hpp:68-151 (messages kept verbatim so the
//                     CLI's "instance error: ..." lines match)
//   orientations      gpu/plp_common.hpp:269-280, plp/parser.py:142-156
//   item order        gpu/plp_common.hpp:335-351, plp/solver.py:169-177
//   PyRng             gpu/plp_common.hpp:164-250
//   py_repr / JSON    gpu/plp_common.hpp:535-610, plp/solver.py:297-307
#pragma once

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace plpb {

struct BoxType {
    int l = 0, w = 0, h = 0;
    bool lf = false, wf = false, hf = false;
    int qty = 0;
    long long volume() const { return 1LL * l * w * h; }
};

struct Instance {
    int L = 0, W = 0, H = 0;
    std::vector<BoxType> types;
    int n_items() const {
        long long n = 0;
        for (const auto& t : types) n += t.qty;
        return (int)n;
    }
};

class FormatError : public std::runtime_error {
public:
    explicit FormatError(const std::string& m) : std::runtime_error(m) {}
};

// thpack "original" format; throws FormatError.
std::vector<Instance> parse_thpack(const std::string& text);
Instance load_single(const std::string& path);   // exactly one instance

using Dims = std::array<int, 3>;                 // (w, d, h) along x, y, z
// Allowed (w, d, h) placements of one type, parser order, duplicates removed.
std::vector<Dims> orientations(const BoxType& t);
// Type index of each decode step; order 0 = volume-descending with ties by
// (type, copy), 1 = input order.
std::vector<int> item_sequence(const Instance& inst, int order);

// CPython random.Random(int) stream (init_by_array seeding, genrand_res53
// random(), getrandbits, randrange via rejection of getrandbits(k)).
class PyRng {
public:
    explicit PyRng(uint64_t seed_abs);
    uint32_t next32();
    double random();
    uint32_t getrandbits(int k);
    int randrange(int n);
private:
    uint32_t mt_[624];
    int pos_;
};

// init_by_array state for |seed| right after seeding (before the first twist).
void mt_seed_state(uint64_t seed_abs, uint32_t out[624]);

std::string py_repr(double x);

struct Placement { int type, x, y, z, w, d, h; };

struct RunSummary {
    int n_boxes = 0;
    long long volume = 0;
    double score = 0.0;
    bool fallback = false;
    int n_passes = 0;
    double time_s = 0.0;
    long long seed = 0;
};

std::string to_json(const RunSummary& s, const std::vector<Placement>& p);

}  // namespace plpb
