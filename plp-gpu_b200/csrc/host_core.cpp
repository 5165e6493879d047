// host_core.cpp -- see host_core.hpp.
#include "host_core.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace plpb {

// ---------------------------------------------------------------------------
// parser (gpu/plp_common.hpp:68-141): non-blank lines, whitespace tokens,
// strtoll for every integer, the same checks in the same order.
// ---------------------------------------------------------------------------
namespace {

long long to_int(const std::string& s, const char* what) {
    char* end = nullptr;
    long long v = std::strtoll(s.c_str(), &end, 10);
    if (end == s.c_str() || *end != '\0')
        throw FormatError(std::string("not an integer: ") + s + " (" + what + ")");
    return v;
}

}  // namespace

std::vector<Instance> parse_thpack(const std::string& text) {
    std::vector<std::vector<std::string>> lines;
    {
        std::istringstream in(text);
        std::string line;
        while (std::getline(in, line)) {
            if (!line.empty() && line.back() == '\r') line.pop_back();
            std::istringstream ls(line);
            std::vector<std::string> t;
            for (std::string w; ls >> w;) t.push_back(w);
            if (!t.empty()) lines.push_back(std::move(t));
        }
    }
    if (lines.empty()) throw FormatError("empty file");
    const long long P = to_int(lines[0][0], "instance count");
    if (P <= 0 || lines.size() < 2) throw FormatError("instance count must be >= 1");
    std::vector<Instance> out;
    size_t ln = 1;
    for (long long p = 0; p < P; p++) {
        if (ln >= lines.size() || lines[ln].size() > 2) throw FormatError("malformed problem line");
        ln++;
        if (ln >= lines.size() || lines[ln].size() != 3)
            throw FormatError("container line must have 3 dimensions");
        long long dim[3];
        for (int i = 0; i < 3; i++) dim[i] = to_int(lines[ln][i], "container dimension");
        if (dim[0] <= 0 || dim[1] <= 0 || dim[2] <= 0)
            throw FormatError("container dimensions must be positive");
        ln++;
        if (ln >= lines.size() || lines[ln].size() != 1)
            throw FormatError("type-count line must be a single integer");
        const long long n = to_int(lines[ln][0], "type count");
        ln++;
        Instance inst;
        inst.L = (int)dim[0];
        inst.W = (int)dim[1];
        inst.H = (int)dim[2];
        for (long long k = 1; k <= n; k++) {
            if (ln >= lines.size()) throw FormatError("instance truncated");
            const auto& t = lines[ln++];
            if (t.size() != 8) throw FormatError("item line must have 8 tokens");
            if (to_int(t[0], "item index") != k) throw FormatError("item index must be sequential");
            const long long l = to_int(t[1], "item dimension");
            const long long w = to_int(t[3], "item dimension");
            const long long h = to_int(t[5], "item dimension");
            if (l <= 0 || w <= 0 || h <= 0) throw FormatError("item dimensions must be positive");
            for (int f : {2, 4, 6})
                if (t[f] != "0" && t[f] != "1") throw FormatError("orientation flags must be 0/1");
            const long long q = to_int(t[7], "item qty");
            if (q < 0) throw FormatError("item qty must be >= 0");
            BoxType bt;
            bt.l = (int)l; bt.w = (int)w; bt.h = (int)h;
            bt.lf = t[2] == "1"; bt.wf = t[4] == "1"; bt.hf = t[6] == "1";
            bt.qty = (int)q;
            inst.types.push_back(bt);
        }
        out.push_back(std::move(inst));
    }
    if (ln != lines.size()) throw FormatError("trailing data after last instance");
    return out;
}

Instance load_single(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw FormatError("cannot open " + path);
    std::ostringstream ss;
    ss << f.rdbuf();
    auto v = parse_thpack(ss.str());
    if (v.size() != 1)
        throw FormatError("expected exactly 1 instance, got " + std::to_string(v.size()));
    return v[0];
}

// ---------------------------------------------------------------------------
// orientation table and item order
// ---------------------------------------------------------------------------
std::vector<Dims> orientations(const BoxType& t) {
    std::vector<Dims> out;
    auto push = [&](int w, int d, int h) {
        const Dims v{w, d, h};
        if (std::find(out.begin(), out.end(), v) == out.end()) out.push_back(v);
    };
    // vertical edge l, then w, then h; two rotations each (plp/parser.py:142-156)
    if (t.lf) { push(t.w, t.h, t.l); push(t.h, t.w, t.l); }
    if (t.wf) { push(t.l, t.h, t.w); push(t.h, t.l, t.w); }
    if (t.hf) { push(t.l, t.w, t.h); push(t.w, t.l, t.h); }
    return out;
}

std::vector<int> item_sequence(const Instance& inst, int order) {
    struct Key { long long vol; int type, copy; };
    std::vector<Key> k;
    for (int t = 0; t < (int)inst.types.size(); t++)
        for (int c = 0; c < inst.types[t].qty; c++) k.push_back({inst.types[t].volume(), t, c});
    if (order == 0)
        std::sort(k.begin(), k.end(), [](const Key& a, const Key& b) {
            if (a.vol != b.vol) return a.vol > b.vol;
            if (a.type != b.type) return a.type < b.type;
            return a.copy < b.copy;
        });
    std::vector<int> out(k.size());
    for (size_t i = 0; i < k.size(); i++) out[i] = k[i].type;
    return out;
}

// ---------------------------------------------------------------------------
// MT19937, CPython seeding (Matsumoto-Nishimura init_by_array with the
// little-endian 32-bit words of |seed|)
// ---------------------------------------------------------------------------
void mt_seed_state(uint64_t seed_abs, uint32_t mt[624]) {
    uint32_t key[2];
    int nkey = 0;
    uint64_t v = seed_abs;
    do {
        key[nkey++] = (uint32_t)v;
        v >>= 32;
    } while (v);
    mt[0] = 19650218u;
    for (uint32_t i = 1; i < 624; i++) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i;
    int i = 1, j = 0;
    for (int k = 624; k > 0; k--) {
        mt[i] = (mt[i] ^ ((mt[i - 1] ^ (mt[i - 1] >> 30)) * 1664525u)) + key[j] + (uint32_t)j;
        if (++i >= 624) { mt[0] = mt[623]; i = 1; }
        if (++j >= nkey) j = 0;
    }
    for (int k = 623; k > 0; k--) {
        mt[i] = (mt[i] ^ ((mt[i - 1] ^ (mt[i - 1] >> 30)) * 1566083941u)) - (uint32_t)i;
        if (++i >= 624) { mt[0] = mt[623]; i = 1; }
    }
    mt[0] = 0x80000000u;
}

PyRng::PyRng(uint64_t seed_abs) {
    mt_seed_state(seed_abs, mt_);
    pos_ = 624;
}

uint32_t PyRng::next32() {
    if (pos_ >= 624) {
        for (int i = 0; i < 624; i++) {
            const uint32_t y = (mt_[i] & 0x80000000u) | (mt_[(i + 1) % 624] & 0x7fffffffu);
            const uint32_t v = mt_[(i + 397) % 624] ^ (y >> 1);
            mt_[i] = (y & 1u) ? (v ^ 0x9908b0dfu) : v;
        }
        pos_ = 0;
    }
    uint32_t y = mt_[pos_++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

double PyRng::random() {
    const uint32_t a = next32() >> 5;
    const uint32_t b = next32() >> 6;
    return ((double)a * 67108864.0 + (double)b) * (1.0 / 9007199254740992.0);
}

uint32_t PyRng::getrandbits(int k) { return next32() >> (32 - k); }

int PyRng::randrange(int n) {
    int k = 0;
    for (unsigned v = (unsigned)n; v; v >>= 1) k++;
    uint32_t r;
    do {
        r = getrandbits(k);
    } while (r >= (uint32_t)n);
    return (int)r;
}

// ---------------------------------------------------------------------------
// CPython float repr: shortest digit string that round-trips, fixed notation
// when the decimal exponent d (value = 0.DIGITS x 10^d) has -4 < d <= 16.
// ---------------------------------------------------------------------------
std::string py_repr(double x) {
    if (std::isnan(x)) return "nan";
    if (std::isinf(x)) return x < 0 ? "-inf" : "inf";
    if (x == 0.0) return std::signbit(x) ? "-0.0" : "0.0";
    const double a = std::fabs(x);
    char tmp[40];
    for (int prec = 1; prec <= 17; prec++) {
        std::snprintf(tmp, sizeof tmp, "%.*e", prec - 1, a);
        if (std::strtod(tmp, nullptr) == a) break;
    }
    const char* e = std::strchr(tmp, 'e');
    std::string digits;
    for (const char* c = tmp; c < e; c++)
        if (*c != '.') digits.push_back(*c);
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    const int decpt = std::atoi(e + 1) + 1;
    const int nd = (int)digits.size();
    std::string out = x < 0 ? "-" : "";
    if (decpt > -4 && decpt <= 16) {
        if (decpt <= 0) out += "0." + std::string((size_t)-decpt, '0') + digits;
        else if (decpt >= nd) out += digits + std::string((size_t)(decpt - nd), '0') + ".0";
        else out += digits.substr(0, (size_t)decpt) + "." + digits.substr((size_t)decpt);
    } else {
        out += digits[0];
        if (nd > 1) out += "." + digits.substr(1);
        const int ex = decpt - 1;
        char eb[16];
        std::snprintf(eb, sizeof eb, "e%c%02d", ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
        out += eb;
    }
    return out;
}

std::string to_json(const RunSummary& s, const std::vector<Placement>& p) {
    std::string o;
    o.reserve(160 + p.size() * 40);
    o += "{\"n_boxes\": " + std::to_string(s.n_boxes);
    o += ", \"volume_cm3\": " + std::to_string(s.volume);
    o += ", \"stability_score\": " + py_repr(s.score);
    o += std::string(", \"fallback\": ") + (s.fallback ? "true" : "false");
    o += ", \"n_passes\": " + std::to_string(s.n_passes);
    o += ", \"time_s\": " + py_repr(s.time_s);
    o += ", \"seed\": " + std::to_string(s.seed);
    o += ", \"placements\": [";
    char b[96];
    for (size_t i = 0; i < p.size(); i++) {
        const auto& q = p[i];
        std::snprintf(b, sizeof b, "%s[%d, %d, %d, %d, %d, %d, %d]", i ? ", " : "", q.type, q.x,
                      q.y, q.z, q.w, q.d, q.h);
        o += b;
    }
    o += "]}";
    return o;
}

}  // namespace plpb
