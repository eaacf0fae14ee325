// Spatial and temporal envelopes of the command line (--pump, --potential,
// --pulse, --fftMask, --initState, --initReservoir): the parser of
// Envelope::fromCommandlineArguments (source/system/envelope.cpp:143-312),
// the point-wise evaluation of Envelope::calculate (envelope.cpp:332-410) and
// the temporal shapes of Envelope::updateTemporal (envelope.cpp:466-500,
// include/system/envelope.hpp:165-175).
//
// Evaluation keeps the reference's arithmetic types: positions are formed in
// double (-L/2 + dx*col), the Gaussian argument is rounded to the build
// precision T before pow/exp, the charge and momentum phases are std::exp of
// a complex<T>, and complex products are std::complex<T> products, so the
// matrices equal the reference's on the same host math library.
#pragma once

#include <algorithm>
#include <bit>
#include <cmath>
#include <complex>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "phx_io.hpp"

namespace phxio {

// include/system/envelope.hpp:38-85
enum EnvType : uint32_t { kGauss = 1, kOuterExponent = 2, kRing = 4, kNoDivide = 8, kLocal = 16 };
enum Pol : uint32_t { kPlus = 1, kMinus = 2, kBoth = 3 };
enum Behavior : uint32_t { kAdd = 1, kMultiply = 2, kReplace = 4, kAdaptive = 8, kComplex = 16 };
enum TemporalKind : uint32_t { kTIExp = 1, kTCos = 2, kTGauss = 4, kTConstant = 8, kTLoaded = 16 };

// the reference's operator& on these flags: true when the common bits form a
// single bit (envelope.hpp:152-157)
inline bool has(uint32_t a, uint32_t b) {
    const uint32_t x = a & b;
    return x != 0 && (x & (x - 1)) == 0;
}

inline uint32_t flags_of(const std::string& s, const std::map<std::string, uint32_t>& m, const std::string& what) {
    uint32_t r = 0;
    size_t prev = 0, pos;
    auto one = [&](const std::string& sub) {
        auto it = m.find(sub);
        if (it == m.end()) throw std::runtime_error("unknown " + what + " '" + sub + "'");
        r |= it->second;
    };
    while ((pos = s.find('+', prev)) != std::string::npos) {
        one(s.substr(prev, pos - prev));
        prev = pos + 1;
    }
    one(s.substr(prev));
    return r;
}

inline const std::map<std::string, uint32_t>& type_names() {
    static const std::map<std::string, uint32_t> m = {
        {"gauss", kGauss}, {"outerExponent", kOuterExponent}, {"ring", kRing}, {"noDivide", kNoDivide}, {"local", kLocal}};
    return m;
}
inline const std::map<std::string, uint32_t>& pol_names() {
    static const std::map<std::string, uint32_t> m = {{"plus", kPlus}, {"minus", kMinus}, {"both", kBoth}};
    return m;
}
inline const std::map<std::string, uint32_t>& behavior_names() {
    static const std::map<std::string, uint32_t> m = {
        {"add", kAdd}, {"multiply", kMultiply}, {"replace", kReplace}, {"adaptive", kAdaptive}, {"complex", kComplex}};
    return m;
}
inline const std::map<std::string, uint32_t>& temporal_names() {
    static const std::map<std::string, uint32_t> m = {
        {"gauss", kTGauss}, {"iexp", kTIExp}, {"osc", kTIExp}, {"cos", kTCos}, {"constant", kTConstant}};
    return m;
}

// ---- argv scanning as PHOENIX::CLIO (source/misc/commandline_io.cpp:110-158)
struct Args {
    std::vector<std::string> v;
    int find(const std::vector<std::string>& keys, int start = 0, const std::string& prefix = "") const {
        for (int i = start; i < (int)v.size(); ++i)
            for (const auto& k : keys)
                if (v[i] == prefix + k) return i;
        return -1;
    }
    int find(const std::string& key, int start = 0) const { return find(std::vector<std::string>{key}, start); }
    // getNextInput: std::stod of the token, 0 past the end (index not advanced)
    double num(int& i, const std::string& name) const {
        if (i >= (int)v.size()) return 0.0;
        try {
            return std::stod(v[i++]);
        } catch (const std::exception&) {
            throw std::runtime_error("parsing variable '" + name + "' as '" + v[i - 1] + "' cannot be converted to a numerical value");
        }
    }
    std::string str(int& i) const {
        if (i >= (int)v.size()) return "";
        return v[i++];
    }
};

template <typename T>
struct Envelope {
    using C = std::complex<T>;
    // spatial components
    std::vector<T> amp, width_x, width_y, x, y, exponent, k0_x, k0_y;
    std::vector<uint32_t> type, pol, behavior;
    std::vector<int> m;
    std::vector<std::string> load_path;
    std::vector<int> group_identifier;
    // temporal groups
    std::vector<T> t0, sigma, freq;
    std::vector<uint32_t> temporal;
    std::vector<std::string> load_path_temporal;
    std::map<std::string, int> group_of;
    std::vector<std::vector<std::vector<T>>> temporal_points;  // loaded groups: columns t, re, im

    int size() const { return (int)amp.size(); }
    int group_size() const { return (int)group_of.size(); }

    void add_spatial(T a, T wx, T wy, T px, T py, T e, const std::string& st, const std::string& sp, const std::string& sb,
                     const std::string& sm, T kx, T ky) {
        amp.push_back(a), width_x.push_back(wx), width_y.push_back(wy), x.push_back(px), y.push_back(py);
        exponent.push_back(e), k0_x.push_back(kx), k0_y.push_back(ky);
        type.push_back(flags_of(st, type_names(), "envelope type"));
        pol.push_back(flags_of(sp, pol_names(), "polarization"));
        behavior.push_back(flags_of(sb, behavior_names(), "behaviour"));
        m.push_back((sm == "None" || sm == "none") ? 0 : std::stoi(sm));
        load_path.push_back("");
    }
    void add_loaded(const std::string& path, T a, const std::string& sb, const std::string& sp) {
        amp.push_back(a), width_x.push_back(0), width_y.push_back(0), x.push_back(0), y.push_back(0);
        exponent.push_back(0), k0_x.push_back(0), k0_y.push_back(0);
        type.push_back(kGauss);
        pol.push_back(flags_of(sp, pol_names(), "polarization"));
        behavior.push_back(flags_of(sb, behavior_names(), "behaviour"));
        m.push_back(0);
        load_path.push_back(path);
    }
    // Envelope::addTemporal: envelopes with equal (t0, sigma, freq, kind) share a group
    void add_temporal(T a_t0, T a_sigma, T a_freq, const std::string& kind) {
        const std::string key = std::to_string(a_t0) + std::to_string(a_sigma) + std::to_string(a_freq) + kind;
        if (!group_of.count(key)) {
            const int g = (int)group_of.size();
            group_of[key] = g;
            t0.push_back(a_t0), sigma.push_back(a_sigma), freq.push_back(a_freq);
            temporal.push_back(flags_of(kind, temporal_names(), "temporal kind"));
            load_path_temporal.push_back("");
        }
        group_identifier.push_back(group_of[key]);
    }
    void add_temporal_file(const std::string& path) {
        if (!group_of.count(path)) {
            const int g = (int)group_of.size();
            group_of[path] = g;
            t0.push_back(0), sigma.push_back(0), freq.push_back(0);
            temporal.push_back(kTLoaded);
            load_path_temporal.push_back(path);
        }
        group_identifier.push_back(group_of[path]);
    }

    // Envelope::fromCommandlineArguments: the legacy positional form
    //   --key amp behaviour wx wy x y pol exponent charge type [momenta kx ky] [time kind t0 sigma freq | time load path]
    // the named form
    //   --key amp behaviour [width wx wy] [pos x y] [pol p] [exponent e] [charge m] [type t] [momenta kx ky]
    //                       [time kind t0 sigma freq | time load path]
    // and the loaded form  --key load path amp behaviour pol [time ...]
    static Envelope parse(const Args& a, const std::vector<std::string>& keys, bool time) {
        Envelope e;
        int index = 0;
        while ((index = a.find(keys, index, "--")) != -1) {
            ++index;
            int peek = index;
            if (a.str(peek) == "load") {
                index = peek;
                const std::string path = a.str(index);
                const T amp_ = (T)a.num(index, "amp");
                const std::string sb = a.str(index);
                const std::string sp = a.str(index);
                e.add_loaded(path, amp_, sb, sp);
            } else {
                const T amp_ = (T)a.num(index, "amp");
                const std::string sb = a.str(index);
                int p2 = index;
                const std::string syntax = a.str(p2);
                const bool named = syntax == "width" || syntax == "pos" || syntax == "pol" || syntax == "exponent" ||
                                   syntax == "charge" || syntax == "type" || syntax == "momenta" || syntax == "time";
                T wx = 0, wy = 0, px = 0, py = 0, ex = 1, kx = 0, ky = 0;
                std::string sp, sm, st;
                if (named) {
                    sp = "both", sm = "none", st = "gauss+noDivide";
                    bool temporal_handled = false;
                    std::string t_type = "constant", t_path;
                    T tt0 = 0, tsig = 0, tfreq = 0;
                    auto keyword = [&](const std::string& kw) -> bool {
                        if (kw == "width") {
                            wx = (T)a.num(index, "width_x"), wy = (T)a.num(index, "width_y");
                        } else if (kw == "pos") {
                            px = (T)a.num(index, "X"), py = (T)a.num(index, "Y");
                        } else if (kw == "pol") {
                            sp = a.str(index);
                        } else if (kw == "exponent") {
                            ex = (T)a.num(index, "exponent");
                        } else if (kw == "charge") {
                            sm = a.str(index);
                        } else if (kw == "type") {
                            st = a.str(index);
                        } else if (kw == "momenta") {
                            kx = (T)a.num(index, "k0_x"), ky = (T)a.num(index, "k0_y");
                        } else if (kw == "time") {
                            temporal_handled = true;
                            const std::string tp = a.str(index);
                            if (tp == "load") {
                                t_path = a.str(index);
                            } else {
                                t_type = tp;
                                tt0 = (T)a.num(index, "t0"), tsig = (T)a.num(index, "sigma"), tfreq = (T)a.num(index, "freq");
                            }
                        } else {
                            return false;
                        }
                        return true;
                    };
                    index = p2;
                    keyword(syntax);
                    while (true) {
                        const int before = index;
                        const std::string kw = a.str(index);
                        if (!keyword(kw)) {
                            index = before < (int)a.v.size() ? index - 1 : index;
                            break;
                        }
                    }
                    e.add_spatial(amp_, wx, wy, px, py, ex, st, sp, sb, sm, kx, ky);
                    if (temporal_handled) {
                        if (!t_path.empty())
                            e.add_temporal_file(t_path);
                        else
                            e.add_temporal(tt0, tsig, tfreq, t_type);
                    } else {
                        e.add_temporal(0, 0, 0, "constant");
                    }
                    continue;
                }
                wx = (T)a.num(index, "width_x"), wy = (T)a.num(index, "width_y");
                px = (T)a.num(index, "X"), py = (T)a.num(index, "Y");
                sp = a.str(index);
                ex = (T)a.num(index, "exponent");
                sm = a.str(index);
                st = a.str(index);
                int p3 = index;
                if (a.str(p3) == "momenta") {
                    index = p3;
                    kx = (T)a.num(index, "k0_x"), ky = (T)a.num(index, "k0_y");
                }
                e.add_spatial(amp_, wx, wy, px, py, ex, st, sp, sb, sm, kx, ky);
            }
            int p4 = index;
            const std::string next = a.str(p4);
            if (!time || next != "time") {
                e.add_temporal(0, 0, 0, "constant");
                continue;
            }
            index = p4;
            int p5 = index;
            if (a.str(p5) == "load") {
                index = p5;
                e.add_temporal_file(a.str(index));
            } else {
                const std::string kind = a.str(index);
                const T tt0 = (T)a.num(index, "t0");
                const T tsig = (T)a.num(index, "sigma");
                const T tfreq = (T)a.num(index, "freq");
                e.add_temporal(tt0, tsig, tfreq, kind);
            }
        }
        return e;
    }

    // loaded spatial components (read again on every evaluation, like the
    // reference's cache) and loaded temporal tables
    bool load_tables(std::string& err) {
        temporal_points.assign(load_path_temporal.size(), {});
        for (size_t g = 0; g < load_path_temporal.size(); ++g) {
            if (load_path_temporal[g].empty()) continue;
            temporal_points[g] = load_list<T>(load_path_temporal[g]);
            if (temporal_points[g].size() != 3 || temporal_points[g][0].empty()) {
                err = "temporal envelope file '" + load_path_temporal[g] + "' must have 3 columns: time, real, imag";
                return false;
            }
        }
        return true;
    }

    struct Dims {
        uint32_t N_c, N_r;
        T L_x, L_y, dx, dy;
    };

    // Envelope::calculate: group < 0 evaluates every group
    bool calculate(C* buffer, int group, uint32_t polarization, const Dims& dim, T default_value, std::string& err) const {
        std::vector<std::vector<C>> cache(load_path.size());
        for (size_t c = 0; c < load_path.size(); ++c) {
            if (load_path[c].empty()) continue;
            uint32_t fc = 0, fr = 0;
            if (load_complex_txt<T>(load_path[c], cache[c], fc, fr) < 0) {
                err = "unable to load '" + load_path[c] + "'";
                return false;
            }
            if (fc != dim.N_c || fr != dim.N_r) {
                err = "'" + load_path[c] + "' holds a " + std::to_string(fc) + " x " + std::to_string(fr) +
                      " matrix, the grid is " + std::to_string(dim.N_c) + " x " + std::to_string(dim.N_r);
                return false;
            }
        }
        for (uint32_t row = 0; row < dim.N_r; ++row)
            for (uint32_t col = 0; col < dim.N_c; ++col) {
                const size_t i = (size_t)row * dim.N_c + col;
                buffer[i] = C(0.0, 0.0);
                bool set = false;
                for (int c = 0; c < size(); ++c) {
                    if (group >= 0 && group_identifier[c] != group) continue;
                    if (pol[c] != kBoth && pol[c] != polarization && polarization != kBoth) continue;
                    double cx = -dim.L_x / 2.0 + dim.dx * (T)col;
                    double cy = -dim.L_y / 2.0 + dim.dy * (T)row;
                    if (has(type[c], kLocal)) {
                        cx = -1.0 + 2.0 * col / (dim.N_c - 1);
                        cy = -1.0 + 2.0 * row / (dim.N_r - 1);
                    }
                    set = true;
                    C amplitude(amp[c], 0.0);
                    T exp_factor = 1, pre = 1, exp_function = 1;
                    C charge(1.0, 0);
                    if (!load_path[c].empty()) {
                        amplitude = cache[c][i] * amp[c];
                    } else {
                        const T ax = (T)((cx - x[c]) / width_x[c]);
                        const T ay = (T)((cy - y[c]) / width_y[c]);
                        exp_factor = (T)(0.5 * (ax * ax + ay * ay));
                        exp_function = std::exp(-std::pow(exp_factor, exponent[c]));
                        if (has(type[c], kOuterExponent)) exp_function = std::pow(std::exp(-exp_factor), exponent[c]);
                        pre = 1.0;
                        if (has(type[c], kRing)) pre = exp_factor;
                        charge = std::exp(C(0.0, m[c] * std::atan2(cx - x[c], cy - y[c])));
                        if (!has(type[c], kNoDivide)) amplitude = amplitude / (T)std::sqrt((T)(2 * 3.1415 * width_x[c] * width_y[c]));
                    }
                    const C momentum = std::exp(C(0.0, k0_x[c] * (cx - x[c]) + k0_y[c] * (cy - y[c])));
                    if (has(behavior[c], kAdaptive)) amplitude = amp[c] * buffer[i];
                    if (has(behavior[c], kComplex)) amplitude = C(0.0, amplitude.real());
                    const C contribution = amplitude * pre * exp_function * charge * momentum;
                    if (has(behavior[c], kAdd))
                        buffer[i] = buffer[i] + contribution;
                    else if (behavior[c] == kMultiply)
                        buffer[i] = buffer[i] * contribution;
                    else if (behavior[c] == kReplace)
                        buffer[i] = contribution;
                }
                if (!set) buffer[i] = C(default_value, 0);
            }
        return true;
    }

    // Envelope::updateTemporal for one group
    C temporal_value(int g, T t) const {
        if (has(temporal[g], kTConstant)) return C(1.0, 0.0);
        C v(1.0, 0.0);
        if (has(temporal[g], kTLoaded)) {
            const auto& P = temporal_points[g];
            if (t > P[0].back()) return C(P[1].back(), P[2].back());
            const auto it = std::lower_bound(P[0].begin(), P[0].end(), t);
            const size_t idx = std::min<size_t>(std::max<size_t>(1, (size_t)std::distance(P[0].begin(), it)), P[0].size() - 1);
            const T t1 = P[0][idx - 1], t2 = P[0][idx];
            const C v1(P[1][idx - 1], P[2][idx - 1]), v2(P[1][idx], P[2][idx]);
            v = v1 + (v2 - v1) * (t - t1) / (t2 - t1);
        }
        if (has(temporal[g], kTIExp)) {
            v = std::exp(-C((t - t0[g]) * (t - t0[g]) / (T(2.0) * sigma[g] * sigma[g]), freq[g] * (t - t0[g])));
        } else if (has(temporal[g], kTCos)) {
            const auto p = (t - t0[g]) / sigma[g];
            v = C((T)(std::exp(-0.5 * p * p) * (1.0 + std::cos(freq[g] * (t - t0[g]))) / 2.0), 0);
        } else if (has(temporal[g], kTGauss)) {
            const auto p = (t - t0[g]) / sigma[g];
            v = C((T)std::exp(-0.5 * std::pow(p * p, freq[g])), 0);
        }
        return v;
    }
};

}  // namespace phxio
