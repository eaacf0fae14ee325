// phoenix_b200 command line: the PHOENIX executable's flags, main loop and
// output files (source/main.cu:47-135, source/system/system_initialization.cpp:13-260,
// source/system/system.cpp:116-187, source/system/system_validate_input.cpp,
// source/system/config_readin.cpp, source/system/filehandler.cpp:31-98,
// source/cuda_solver/solver/solver_initialization.cu:37-174,
// solver_output_matrices.cu, solver_cache.cu, solver_finalize.cu) over the
// C ABI of libphx.so: every iteration runs on the GPU.
//
// Precision: the reference picks it at build time (FP32 with
// USE_32_BIT_PRECISION); here `--precision fp32|fp64` (default fp64, or fp32
// when the program's name contains "fp32").  Accepted and ignored: --threads,
// --blocksize, --subgrids (the GPU iteration has no subgrids), --cmap,
// -nosfml / -norender (no viewer).  Added: --gpu <ordinal>.
//
// Where the reference's bookkeeping differs from what a reader might expect,
// the reference is followed, for byte-identical files: min_plus in scalar.txt
// is always 0 (the extrema start from a complex "max()" that is 0), the
// initial_*_minus files hold the plus fields, history windows thinned by an
// increment keep the full window's shape in their binary headers.
// max_plus is taken over the grid points; the reference takes it over its
// halo-padded buffer, whose rings hold partial stage sums.

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/phx.h"
#include "phx_envelope.hpp"
#include "phx_io.hpp"

using namespace phxio;

namespace {

struct Fail : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void check(phx_handle* h, phx_status st, const char* what) {
    if (st != PHX_OK)
        throw Fail(std::string(what) + ": " + phx_status_string(st) + " (" + (h ? phx_last_error(h) : phx_last_error(nullptr)) + ")");
}

// readConfigFromFile (config_readin.cpp:7-42): every --config file's words
// are appended (a word starting with '#' ends its line; each line adds " ")
std::vector<std::string> read_config(int argc, char** argv) {
    std::vector<std::string> out(argv, argv + argc);
    const Args a{out};
    int index = a.find("--config");
    if (index == -1) return out;
    while (true) {
        // the reference steps over one token after each file name
        // (++index before a read that advances it again)
        ++index;
        const std::string file = a.str(index);
        if (file.empty()) break;
        if (!std::filesystem::exists(file)) {
            std::cout << "Config file '" << file << "' does not exist. Skipping." << std::endl;
            return out;
        }
        std::ifstream f(file);
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream is(line);
            std::string w;
            while (is >> w) {
                if (w[0] == '#') break;
                out.push_back(w);
            }
            out.push_back(" ");
        }
    }
    return out;
}

bool adaptive_iterator(int it) {
    return it == PHX_ITER_DP45 || it == PHX_ITER_BOSHA || it == PHX_ITER_CASHKARP || it == PHX_ITER_FEHLBERG2 ||
           it == PHX_ITER_FEHLBERG5 || it == PHX_ITER_DP85 || it == PHX_ITER_NSRK78;
}

int iterator_of(std::string key) {
    for (auto& c : key) c = (char)std::toupper((unsigned char)c);
    static const std::map<std::string, int> m = {
        {"RK4", PHX_ITER_RK4},       {"DP45", PHX_ITER_DP45},         {"RK3", PHX_ITER_RK3},
        {"SSPRK3", PHX_ITER_SSPRK3}, {"MP", PHX_ITER_MP},             {"HEUN2", PHX_ITER_HEUN2},
        {"HEUN3", PHX_ITER_HEUN3},   {"HW", PHX_ITER_HW},             {"NEWTON", PHX_ITER_NEWTON},
        {"NYSTROEM", PHX_ITER_NYSTROEM}, {"RALSTON", PHX_ITER_RALSTON}, {"RALSTON3", PHX_ITER_RALSTON3},
        {"RALSTON4", PHX_ITER_RALSTON4}, {"RULE38", PHX_ITER_RULE38}, {"BOSHA", PHX_ITER_BOSHA},
        {"CASHKARP", PHX_ITER_CASHKARP}, {"FEHLBERG2", PHX_ITER_FEHLBERG2}, {"FEHLBERG5", PHX_ITER_FEHLBERG5},
        {"DP85", PHX_ITER_DP85},     {"NSRK78", PHX_ITER_NSRK78},     {"SSFM", PHX_ITER_SSFM}};
    auto it = m.find(key);
    if (it == m.end()) throw Fail("iterator '" + key + "' is not registered");
    return it->second;
}

// fft_shift_2D of the reference (swap of diagonal quadrants, even sizes)
template <typename T>
void fft_shift(std::vector<T>& d, uint32_t N_c, uint32_t N_r) {
    for (uint32_t k = 0; k < N_r / 2; ++k)
        for (uint32_t l = 0; l < N_c / 2; ++l) {
            std::swap(d[(size_t)k * N_c + l], d[(size_t)(k + N_r / 2) * N_c + l + N_c / 2]);
            std::swap(d[(size_t)k * N_c + l + N_c / 2], d[(size_t)(k + N_r / 2) * N_c + l]);
        }
}

template <typename T>
struct Run {
    using C = std::complex<T>;
    Args a;
    // ---- SystemParameters (system.cpp:18-72 defaults, system_initialization.cpp)
    bool tetm = false;
    T gamma_c = (T)0.15, gamma_r, g_c = (T)3.E-6, g_r, R = (T)0.01, L_x = (T)100., L_y = (T)100., g_pm, delta_LT = (T)0.025E-3;
    uint32_t N_c = 400, N_r = 400;
    T t_max = 1000, output_every = 1, dt_max = 3, dt_min = (T)0.0001, tolerance = (T)1E-1, fft_every = 1;
    T dt = 0, t = 0, imag_time = 0, dw = 0;
    T m_e = (T)9.10938356E-31, h_bar = (T)1.0545718E-34, e_e = (T)1.60217662E-19, h_bar_s = -1, m_eff = -1;
    T magic_timestep = 0, dx = 0, dy = 0;
    bool do_overwrite_dt = true, adaptive = false, periodic_x = false, periodic_y = false, use_reservoir = true;
    std::string iterator = "RK4";
    std::vector<std::string> output_keys = {"mat", "scalar"};
    bool random_init = false;
    T random_amp = 1.0;
    uint32_t random_seed = 0;
    int precision = -1;
    uint32_t hx0 = 0, hx1 = 0, hy0 = 0, hy1 = 0, hinc = 1;
    bool history = false;
    int history_every = 1;
    T history_start = 0;
    Envelope<T> pump, potential, pulse, fft_mask, init_state, init_reservoir;
    std::string out_path = "data", out_name, out_type;
    int device = 0;
    // ---- state
    phx_handle* h = nullptr;
    std::map<std::string, std::vector<T>> scalar;
    std::vector<double> loop_times;
    uint32_t history_counter = 1;
    int64_t iterations = 0;
    bool last_adaptive = false;

    template <typename... K>
    bool out(const K&... k) const {
        return ((std::find(output_keys.begin(), output_keys.end(), std::string(k)) != output_keys.end()) || ...);
    }
    std::string path_of(const std::string& name, const std::string& type) const {
        return out_path + (out_path.back() == '/' ? "" : "/") + out_name + (out_name.empty() ? "" : "_") + name + "." + type;
    }

    void parse() {
        int i;
        gamma_r = (T)(1.5 * gamma_c);
        g_r = (T)(2. * g_c);
        g_pm = -g_c / 5;
        tetm = a.find("-tetm") != -1;
        if ((i = a.find({"gammaC", "gamma_C", "gammac", "gamma_c"}, 0, "--")) != -1) gamma_c = (T)a.num(++i, "gamma_c");
        if ((i = a.find({"gammaR", "gamma_R", "gammar", "gamma_r"}, 0, "--")) != -1) gamma_r = (T)a.num(++i, "gamma_r");
        if ((i = a.find({"gc", "g_c"}, 0, "--")) != -1) g_c = (T)a.num(++i, "g_c");
        if ((i = a.find({"gr", "g_r"}, 0, "--")) != -1) g_r = (T)a.num(++i, "g_r");
        if ((i = a.find("--R")) != -1) R = (T)a.num(++i, "R");
        if ((i = a.find({"L", "gridlength", "xmax"}, 0, "--")) != -1) {
            L_x = (T)a.num(++i, "L");
            L_y = (T)a.num(i, "L");
        }
        if ((i = a.find({"g_pm", "gpm", "g_PM"}, 0, "--")) != -1) g_pm = (T)a.num(++i, "gm");
        if ((i = a.find({"deltaLT", "delta_LT", "deltalt", "dlt"}, 0, "--")) != -1) delta_LT = (T)a.num(++i, "deltaLT");
        if ((i = a.find({"output", "fileoutput", "FO"}, 0, "--")) != -1) {
            output_keys.clear();
            const std::string s = a.str(++i);
            size_t prev = 0, pos;
            while ((pos = s.find(',', prev)) != std::string::npos) {
                output_keys.push_back(s.substr(prev, pos - prev));
                prev = pos + 1;
            }
            output_keys.push_back(s.substr(prev));
        }
        if ((i = a.find({"N", "gridsize"}, 0, "--")) != -1) {
            N_c = (uint32_t)(int)a.num(++i, "N_c");
            N_r = (uint32_t)(int)a.num(i, "N_r");
        }
        if ((i = a.find({"tmax", "tend"}, 0, "--")) != -1) t_max = (T)a.num(++i, "t_max");
        if ((i = a.find({"tstep", "dt"}, 0, "--")) != -1) {
            dt = (T)a.num(++i, "t_step");
            do_overwrite_dt = false;
        }
        if ((i = a.find("--tol")) != -1) tolerance = (T)a.num(++i, "tol");
        if ((i = a.find("--rkvdt")) != -1) {
            dt_min = (T)a.num(++i, "dt_min");
            dt_max = (T)a.num(i, "dt_max");
        }
        if ((i = a.find("--imagTime")) != -1) imag_time = (T)a.num(++i, "imag_time_amplitude");
        if ((i = a.find("--fftEvery")) != -1) fft_every = (T)a.num(++i, "fft_every");
        if (a.find("-ssfm") != -1) iterator = "SSFM";
        if ((i = a.find("--iterator")) != -1) iterator = a.str(++i);
        adaptive = a.find({"adaptive", "adaptiveTimestep"}, 0, "-") != -1;
        if ((i = a.find({"initRandom", "iR"}, 0, "--")) != -1) {
            random_init = true;
            random_amp = (T)a.num(++i, "random_system_amplitude");
            random_seed = std::random_device{}();
            const std::string s = a.str(i);
            if (s != "random") random_seed = (uint32_t)std::stod(s);
        }
        if ((i = a.find("--dw")) != -1) dw = (T)a.num(++i, "dw");
        if ((i = a.find("--outEvery")) != -1) output_every = (T)a.num(++i, "output_every");
        if ((i = a.find({"fileout-precision", "fileoutPrecision"}, 0, "--")) != -1)
            precision = (int)a.num(++i, "fileout_precision");
        hx1 = N_c, hy1 = N_r;
        if ((i = a.find({"historyMatrix", "hM"}, 0, "--")) != -1) {
            hx0 = (uint32_t)a.num(++i, "history_matrix_start_x");
            hx1 = (uint32_t)a.num(i, "history_matrix_end_x");
            hy0 = (uint32_t)a.num(i, "history_matrix_start_y");
            hy1 = (uint32_t)a.num(i, "history_matrix_end_y");
            hinc = (uint32_t)a.num(i, "history_matrix_output_increment");
            history = true;
        }
        if ((i = a.find({"historyTime", "hT"}, 0, "--")) != -1) {
            history_start = (T)a.num(++i, "history_time");
            history_every = int(a.num(i, "history_time_every"));
        }
        if ((i = a.find("--boundary")) != -1) {
            periodic_x = a.str(++i) == "periodic";
            periodic_y = a.str(i) == "periodic";
        }
        if ((i = a.find("--t0")) != -1) t = (T)a.num(++i, "t0");
        if ((i = a.find("--hbar")) != -1) h_bar = (T)a.num(++i, "hbar");
        if ((i = a.find({"electron_charge", "e"}, 0, "--")) != -1) e_e = (T)a.num(++i, "e");
        if ((i = a.find({"me", "m_e", "electron_mass"}, 0, "--")) != -1) m_e = (T)a.num(++i, "me");
        if ((i = a.find({"hbarscaled", "hbar_scaled", "hbars"}, 0, "--")) != -1) h_bar_s = (T)a.num(++i, "hbars");
        if ((i = a.find({"meff", "m_eff"}, 0, "--")) != -1) m_eff = (T)a.num(++i, "m_eff");
        if ((i = a.find("--gpu")) != -1) device = (int)a.num(++i, "gpu");
        pump = Envelope<T>::parse(a, {"pump"}, true);
        potential = Envelope<T>::parse(a, {"potential"}, true);
        pulse = Envelope<T>::parse(a, {"pulse"}, true);
        fft_mask = Envelope<T>::parse(a, {"fftMask"}, false);
        init_state = Envelope<T>::parse(a, {"initState", "initialState", "iS"}, false);
        init_reservoir = Envelope<T>::parse(a, {"initReservoir", "initialReservoir", "iR"}, false);
        use_reservoir = !(pump.size() == 0 && init_reservoir.size() == 0);
        if (a.find("-noReservoir") != -1) use_reservoir = false;
        // FileHandler::init
        if ((i = a.find({"path", "outputPath"}, 0, "--")) != -1) out_path = a.str(++i);
        if (out_path.empty() || out_path.back() != '/') out_path += "/";
        if ((i = a.find("--name")) != -1) out_name = a.str(++i);
        if ((i = a.find({"of", "outputFileType"}, 0, "--")) != -1) out_type = a.str(++i);
        if (out_type == "phoenix") out_type = "ash";
        if (out_type == "numpy") out_type = "npy";
        if (out_type == "text") out_type = "txt";
        if (out_type == "matlab") out_type = "mat";
        if (out_type != "ash" && out_type != "npy" && out_type != "txt" && out_type != "mat") out_type = "txt";
        std::filesystem::create_directories(out_path);
        if (a.find({"historyMatrix", "hm"}, 0, "--") != -1) std::filesystem::create_directories(out_path + "timeoutput");
    }

    // calculateAuto (system.cpp:116-140) and validateInputs
    void derive() {
        if (h_bar_s < 0) h_bar_s = (T)(h_bar / e_e * 1E12);
        if (m_eff < 0) m_eff = (T)(m_e / e_e * 1E8);
        const auto dt_scaling_factor = m_e / e_e * 1E8 / m_eff;
        dx = L_x / (T)(N_c - 1);
        dy = L_y / (T)(N_r - 1);
        magic_timestep = (T)(0.5 * dx * dy / dt_scaling_factor);
        if (do_overwrite_dt) dt = magic_timestep;
        bool valid = true;
        if ((int)N_c <= 0 || (int)N_r <= 0) valid = false;
        if (N_c % 2 != 0 || N_r % 2 != 0) {
            std::cout << "Input Dimensions have to be even!" << std::endl;
            valid = false;
        }
        if (t_max < 0 || dt <= 0 || dt > t_max || dt_max < 0 || dt_min < 0) valid = false;
        if (!valid) throw Fail("Invalid input (N even and positive, 0 < dt <= tmax, dt_min, dt_max >= 0)");
    }

    void set_field(int field, int group, const std::vector<T>& v) {
        check(h, phx_set_field(h, field, group, v.data(), (int64_t)v.size(), sizeof(T) == 4 ? PHX_F32 : PHX_F64), "set field");
    }
    std::vector<T> real_of(const std::vector<C>& z) {
        std::vector<T> r(z.size());
        for (size_t k = 0; k < z.size(); ++k) r[k] = z[k].real();
        return r;
    }
    std::vector<T> flat(const std::vector<C>& z) {
        std::vector<T> r(2 * z.size());
        for (size_t k = 0; k < z.size(); ++k) r[2 * k] = z[k].real(), r[2 * k + 1] = z[k].imag();
        return r;
    }
    std::vector<C> get_complex(int field) {
        std::vector<T> r(2 * (size_t)N_c * N_r);
        check(h, phx_get_field(h, field, 0, r.data(), (int64_t)r.size(), sizeof(T) == 4 ? PHX_F32 : PHX_F64), "get field");
        std::vector<C> z(r.size() / 2);
        for (size_t k = 0; k < z.size(); ++k) z[k] = C(r[2 * k], r[2 * k + 1]);
        return z;
    }
    std::vector<C> get_reservoir(int field) {
        std::vector<T> r((size_t)N_c * N_r);
        check(h, phx_get_field(h, field, 0, r.data(), (int64_t)r.size(), sizeof(T) == 4 ? PHX_F32 : PHX_F64), "get field");
        std::vector<C> z(r.size());
        for (size_t k = 0; k < z.size(); ++k) z[k] = C(r[k], 0);
        return z;
    }
    void write_complex(const std::string& name, const std::vector<C>& z, const Window& w, const Header<T>& hd) {
        if (!write_file(path_of(name, out_type), encode_complex<T>(out_type, z.data(), w, hd, precision)))
            std::cout << "File '" << path_of(name, out_type) << "' is not open! Cannot output matrix to file!" << std::endl;
    }
    void write_real(const std::string& name, const std::vector<T>& v, const Window& w, const Header<T>& hd) {
        if (!write_file(path_of(name, out_type), encode_real<T>(out_type, v.data(), w, hd, precision)))
            std::cout << "File '" << path_of(name, out_type) << "' is not open! Cannot output matrix to file!" << std::endl;
    }

    std::vector<C> eval(const Envelope<T>& e, int group, uint32_t pol, T dflt) {
        std::vector<C> b((size_t)N_c * N_r);
        std::string err;
        typename Envelope<T>::Dims d{N_c, N_r, L_x, L_y, dx, dy};
        if (!e.calculate(b.data(), group, pol, d, dflt, err)) throw Fail(err);
        return b;
    }

    void set_temporals(Envelope<T>& e, int family) {
        std::string err;
        if (!e.load_tables(err)) throw Fail(err);
        for (int g = 0; g < e.group_size(); ++g) {
            const uint32_t k = e.temporal[g];
            if (has(k, kTConstant)) {
                check(h, phx_set_temporal(h, family, g, PHX_TEMPORAL_CONSTANT, 0, 0, 0), "temporal");
            } else if (has(k, kTLoaded)) {
                std::vector<double> tt, re, im;
                for (size_t n = 0; n < e.temporal_points[g][0].size(); ++n) {
                    tt.push_back(e.temporal_points[g][0][n]);
                    re.push_back(e.temporal_points[g][1][n]);
                    im.push_back(e.temporal_points[g][2][n]);
                }
                check(h, phx_set_temporal_table(h, family, g, tt.data(), re.data(), im.data(), (int64_t)tt.size()), "temporal table");
            } else {
                const int kind = has(k, kTIExp) ? PHX_TEMPORAL_IEXP
                                                : (has(k, kTCos) ? PHX_TEMPORAL_COS : (has(k, kTGauss) ? PHX_TEMPORAL_GAUSS : PHX_TEMPORAL_CONSTANT));
                check(h, phx_set_temporal(h, family, g, kind, e.t0[g], e.sigma[g], e.freq[g]), "temporal");
            }
        }
    }

    void create() {
        phx_params p{};
        p.abi_version = PHX_ABI_VERSION;
        p.N_c = (int32_t)N_c, p.N_r = (int32_t)N_r;
        p.L_x = L_x, p.L_y = L_y, p.h_bar_s = h_bar_s, p.m_eff = m_eff;
        p.gamma_c = gamma_c, p.gamma_r = gamma_r, p.g_c = g_c, p.g_r = g_r, p.R = R, p.g_pm = g_pm, p.delta_LT = delta_LT;
        p.periodic_x = periodic_x, p.periodic_y = periodic_y, p.tetm = tetm, p.use_reservoir = use_reservoir;
        p.dtype = sizeof(T) == 4 ? PHX_F32 : PHX_F64;
        p.iterator = iterator_of(iterator);
        if (adaptive && !adaptive_iterator(p.iterator)) {
            // Solver::iterate (solver.cu:23-26): the flag is dropped for fixed-step solvers
            std::cout << "Cannot use variable time step with this solver." << std::endl;
            adaptive = false;
        }
        p.adaptive = adaptive;
        p.norm_mode = PHX_NORM_REFERENCE;
        p.dt = dt, p.t0 = t, p.t_max = t_max, p.tol = tolerance, p.dt_min = dt_min, p.dt_max = dt_max;
        p.fft_every = fft_every;
        p.stochastic_amplitude = dw;
        p.seed = random_seed;
        p.n_pump_groups = pump.group_size(), p.n_potential_groups = potential.group_size(), p.n_pulse_groups = pulse.group_size();
        p.device = device;
        p.imag_time_amplitude = imag_time;
        check(nullptr, phx_create(&p, &h), "create");
    }

    // Solver::initializeMatricesFromSystem + outputInitialMatrices
    void initialize() {
        const Header<T> hd{L_x, L_y, dx, dy, t};
        std::vector<C> s_plus = eval(init_state, -1, kPlus, 0), s_minus, r_plus, r_minus;
        if (use_reservoir) r_plus = eval(init_reservoir, -1, kPlus, 0);
        if (tetm) {
            s_minus = eval(init_state, -1, kMinus, 0);
            if (use_reservoir) r_minus = eval(init_reservoir, -1, kMinus, 0);
        }
        if (random_init) {
            std::mt19937 gen{random_seed};
            std::uniform_real_distribution<T> dist{-random_amp, random_amp};
            for (auto& z : s_plus) z += C{dist(gen), dist(gen)};
            if (tetm)
                for (auto& z : s_minus) z += C{dist(gen), dist(gen)};
        }
        for (const auto* r : {&r_plus, &r_minus})
            for (const auto& z : *r)
                if (z.imag() != 0) throw Fail("a complex initial reservoir is not supported (the reservoir is stored real)");
        set_field(PHX_PSI_PLUS, 0, flat(s_plus));
        if (use_reservoir) set_field(PHX_N_PLUS, 0, real_of(r_plus));
        if (tetm) {
            set_field(PHX_PSI_MINUS, 0, flat(s_minus));
            if (use_reservoir) set_field(PHX_N_MINUS, 0, real_of(r_minus));
        }
        const Window full{0, N_c, 0, N_r, N_c, 1};
        if (out("all", "mat", "initial_plus", "initial")) {
            write_complex("initial_wavefunction_plus", s_plus, full, hd);
            if (use_reservoir) write_complex("initial_reservoir_plus", r_plus, full, hd);
        }
        auto osc = [&](const Envelope<T>& e, int g) { return Header<T>{L_x, L_y, dx, dy, t, e.t0[g], e.freq[g], e.sigma[g]}; };
        auto suffix = [](int g) { return g > 0 ? "_" + std::to_string(g) : std::string(); };
        const int comps = tetm ? 2 : 1;
        const char* cn[2] = {"plus", "minus"};
        const uint32_t pols[2] = {kPlus, kMinus};
        for (int q = 0; q < comps; ++q) {
            for (int g = 0; g < pump.group_size(); ++g) {
                const std::vector<T> v = real_of(eval(pump, g, pols[q], 0));
                set_field(q ? PHX_PUMP_MINUS : PHX_PUMP_PLUS, g, v);
                if (use_reservoir && out("all", "mat", q ? "pump_minus" : "pump_plus", "pump"))
                    write_real(std::string("pump_") + cn[q] + suffix(g), v, full, osc(pump, g));
            }
            for (int g = 0; g < potential.group_size(); ++g) {
                const std::vector<T> v = real_of(eval(potential, g, pols[q], 0));
                set_field(q ? PHX_POTENTIAL_MINUS : PHX_POTENTIAL_PLUS, g, v);
                if ((q ? true : potential.size() > 0) && out("all", "mat", q ? "potential_minus" : "potential_plus", "potential"))
                    write_real(std::string("potential_") + cn[q] + suffix(g), v, full, osc(potential, g));
            }
            for (int g = 0; g < pulse.group_size(); ++g) {
                const std::vector<C> v = eval(pulse, g, pols[q], 0);
                set_field(q ? PHX_PULSE_MINUS : PHX_PULSE_PLUS, g, flat(v));
                if ((q ? true : pulse.size() > 0) && out("all", "mat", q ? "pulse_minus" : "pulse_plus", "pulse"))
                    write_complex(std::string("pulse_") + cn[q] + suffix(g), v, full, osc(pulse, g));
            }
            if (fft_mask.size() > 0) {
                std::vector<T> m = real_of(eval(fft_mask, -1, pols[q], 1.0));
                set_field(q ? PHX_FFT_MASK_MINUS : PHX_FFT_MASK_PLUS, 0, m);
                fft_shift(m, N_c, N_r);
                if (fft_every < t_max && (q ? true : fft_mask.size() > 0) && out("all", "mat", q ? "fft_minus" : "fft_plus", "fft"))
                    write_real(std::string("fft_mask_") + cn[q], m, full, hd);
            }
        }
        if (tetm && out("all", "mat", "initial_minus", "initial")) {
            write_complex("initial_wavefunction_minus", s_plus, full, hd);
            if (use_reservoir) write_complex("initial_reservoir_minus", r_plus, full, hd);
        }
        set_temporals(pump, PHX_ENV_PUMP);
        set_temporals(potential, PHX_ENV_POTENTIAL);
        set_temporals(pulse, PHX_ENV_PULSE);
        if (fft_every < t_max) check(h, phx_set_spectrum_output(h, 1), "spectrum output");
    }

    void refresh_time() {
        double tt, dd;
        check(h, phx_get_time(h, &tt, &dd), "time");
        t = (T)tt, dt = (T)dd;
    }

    // Solver::cacheValues (solver_cache.cu:7-46)
    void cache_values() {
        scalar["t"].push_back(t);
        const int comps = tetm ? 2 : 1;
        const char* cn[2] = {"plus", "minus"};
        for (int q = 0; q < comps; ++q) {
            if (q == 0) {
                // the envelopes' last evaluated temporal values (updateKernelTime runs
                // at t + dt of the iteration's start; the step-size control
                // evaluates them once more at the new t + dt)
                const T te = last_adaptive ? (T)(t + dt) : t;
                for (int g = 0; g < pulse.group_size(); ++g) {
                    if (has(pulse.temporal[g], kTConstant)) continue;
                    const C v = pulse.temporal_value(g, te);
                    scalar["pulse_" + std::to_string(g) + "_real"].push_back(v.real());
                    scalar["pulse_" + std::to_string(g) + "_imag"].push_back(v.imag());
                }
                for (int g = 0; g < pump.group_size(); ++g)
                    if (!has(pump.temporal[g], kTConstant)) scalar["pump_" + std::to_string(g)].push_back(pump.temporal_value(g, te).real());
                for (int g = 0; g < potential.group_size(); ++g)
                    if (!has(potential.temporal[g], kTConstant))
                        scalar["potential_" + std::to_string(g)].push_back(potential.temporal_value(g, te).real());
            }
            const std::vector<C> z = get_complex(q ? PHX_PSI_MINUS : PHX_PSI_PLUS);
            C mx(0, 0);
            for (const C& v : z)
                if (!(std::norm(mx) > std::norm(v))) mx = v;
            scalar[std::string("min_") + cn[q]].push_back((T)0);
            scalar[std::string("max_") + cn[q]].push_back(std::abs(mx));
        }
    }

    // Solver::outputMatrices (solver_output_matrices.cu:20-70)
    void output_matrices(uint32_t x0, uint32_t x1, uint32_t y0, uint32_t y1, uint32_t inc, const std::string& suffix,
                         const std::string& prefix) {
        const Header<T> hd{L_x * (T)(x1 - x0) / (T)N_c, L_y * (T)(y1 - y0) / (T)N_r, dx, dy, t};
        const Header<T> fhd{(T)(-1.0 * (x1 - x0) / N_c), (T)(-1.0 * (y1 - y0) / N_r), (T)(2.0 / N_c), (T)(2.0 / N_r), t};
        const Window w{x0, x1, y0, y1, N_c, inc};
        if (out("wavefunction", "psi", "wavefunction_plus", "psi_plus", "plus", "wf", "mat", "all", "initial", "initial_plus"))
            write_complex(prefix + "wavefunction_plus" + suffix, get_complex(PHX_PSI_PLUS), w, hd);
        if (use_reservoir && out("mat", "reservoir", "n", "reservoir_plus", "n_plus", "plus", "rv", "mat", "all"))
            write_complex(prefix + "reservoir_plus" + suffix, get_reservoir(PHX_N_PLUS), w, hd);
        if (fft_every < t_max && out("fft_mask", "fft", "fft_plus", "plus", "mat", "all"))
            write_complex(prefix + "fft_plus" + suffix, get_complex(PHX_FFT_PLUS), w, fhd);
        if (!tetm) return;
        if (out("wavefunction", "psi", "wavefunction_minus", "psi_minus", "plus", "wf", "mat", "all", "initial", "initial_minus"))
            write_complex(prefix + "wavefunction_minus" + suffix, get_complex(PHX_PSI_MINUS), w, hd);
        if (use_reservoir && out("reservoir", "n", "reservoir_minus", "n_minus", "plus", "rv", "mat", "all"))
            write_complex(prefix + "reservoir_minus" + suffix, get_reservoir(PHX_N_MINUS), w, hd);
        if (fft_every < t_max && out("fft_mask", "fft", "fft_minus", "plus", "mat", "all"))
            write_complex(prefix + "fft_minus" + suffix, get_complex(PHX_FFT_MINUS), w, fhd);
    }

    // Solver::cacheMatrices (solver_cache.cu:64-78)
    void cache_matrices() {
        if (!history) return;
        if (t < history_start) return;
        if ((int)history_counter < history_every) {
            ++history_counter;
            return;
        }
        history_counter = 1;
        output_matrices(hx0, hx1, hy0, hy1, hinc, "_" + std::to_string(t), "timeoutput/");
    }

    // Solver::iterate with the main loop's dt adjustment
    bool iterate(bool force_fixed) {
        phx_step_info info{};
        check(h, phx_iterate(h, force_fixed ? 1 : 0, &info), "iterate");
        iterations += info.iterations;
        if (info.iterations > 0) last_adaptive = adaptive && !force_fixed;
        return info.iterations > 0;
    }

    // main.cu:76-117 (no viewer: the disableRender branch)
    void main_loop() {
        uint32_t oei = 1;
        while (t < t_max) {
            const auto c0 = std::chrono::high_resolution_clock::now();
            bool force = false;
            while (t < (T)(oei * output_every)) {
                const T saved = dt;
                if (t + dt > (T)(oei * output_every)) {
                    const T next_dt = (T)(oei * output_every) - t;
                    if (next_dt > 0) {
                        dt = next_dt;
                        check(h, phx_set_time(h, t, dt), "set time");
                        force = true;
                    }
                }
                const bool result = iterate(force);
                refresh_time();
                if (force) {
                    force = false;
                    dt = saved;
                    check(h, phx_set_time(h, t, dt), "set time");
                }
                if (!result) break;
            }
            ++oei;
            cache_values();
            cache_matrices();
            const auto c1 = std::chrono::high_resolution_clock::now();
            loop_times.push_back(std::chrono::duration_cast<std::chrono::nanoseconds>(c1 - c0).count() / 1E9);
            // progress line (printCMD, system_print_output.cpp:800-848; pyphoenix echoes "T =" lines)
            std::cout << "T = " << t << "ps - dt = " << dt << "ps - " << iterations << " iterations" << std::endl;
        }
    }

    void finalize() {
        output_matrices(0, N_c, 0, N_r, 1, "", "");
        if (out("all", "max", "scalar")) {
            std::string s = "index ";
            for (const auto& kv : scalar) s += kv.first + " ";
            s += "\n";
            const size_t rows = scalar.count("t") ? scalar["t"].size() : 0;
            for (size_t i = 0; i < rows; ++i) {
                s += std::to_string(i) + " ";
                for (const auto& kv : scalar) s += fmt_g(i < kv.second.size() ? (double)kv.second[i] : 0.0, 6) + " ";
                s += "\n";
            }
            write_file(path_of("scalar", "txt"), s);
        }
        std::string s = "iteration Main-Loop \n";
        for (size_t i = 0; i < loop_times.size(); ++i) s += std::to_string(i) + " " + fmt_g(loop_times[i], 6) + " \n";
        write_file(path_of("times", "txt"), s);
    }

    int run() {
        parse();
        derive();
        std::cout << "phoenix_b200: " << N_c << " x " << N_r << ", " << (sizeof(T) == 4 ? "fp32" : "fp64") << ", iterator "
                  << iterator << (adaptive ? " (adaptive)" : "") << ", dt " << dt << ", tmax " << t_max << std::endl;
        create();
        initialize();
        const auto c0 = std::chrono::high_resolution_clock::now();
        main_loop();
        const auto c1 = std::chrono::high_resolution_clock::now();
        finalize();
        const double total = std::chrono::duration_cast<std::chrono::nanoseconds>(c1 - c0).count() / 1E9;
        std::cout << "Total Runtime: " << total << " s --> " << (total / t * 1E3) << " ms/ps --> " << (t / total) << " ps/s --> "
                  << (iterations ? total / (double)iterations * 1e6 : 0.0) << " mus/it" << std::endl;
        std::cout << "    Time per ps: " << total / (double)t << "s/ps-  " << (double)t / total << "ps/s-  "
                  << (double)iterations / total << "it/s" << std::endl;
        phx_destroy(h);
        h = nullptr;
        return 0;
    }
};

void usage() {
    std::cout
        << "phoenix_b200 -- the PHOENIX command line on the phoenix_b200 GPU library\n"
           "  grid       --N Nc Nr  --L Lx Ly  --boundary zero|periodic zero|periodic\n"
           "  time       --tmax T  --dt dt (default: magic time step)  --t0 t  --outEvery T\n"
           "  iterator   --iterator RK4|DP45|RK3|SSPRK3|MP|Heun2|Heun3|HW|Newton|Nystroem|Ralston|Ralston3|Ralston4|\n"
           "             Rule38|BoSha|CashKarp|Fehlberg2|Fehlberg5|DP85|NSRK78|SSFM  -ssfm  -adaptive  --tol t\n"
           "             --rkvdt dt_min dt_max  --imagTime A  --dw amplitude\n"
           "  physics    --gammaC --gammaR --gc --gr --R --gpm --deltaLT --hbarscaled --meff --hbar --e --me  -tetm\n"
           "  envelopes  --pump --potential --pulse --fftMask --initState --initReservoir (positional, named or\n"
           "             'load <file> amp behaviour pol' forms; 'time kind t0 sigma freq' or 'time load <file>')\n"
           "             --initRandom amplitude seed|random  -noReservoir  --fftEvery T\n"
           "  output     --path dir  --name prefix  --of txt|npy|ash|mat  --output key,key,...  --fileoutPrecision p\n"
           "             --historyMatrix x0 x1 y0 y1 inc  --historyTime t0 every\n"
           "  other      --config file...  --precision fp32|fp64  --gpu ordinal\n";
}

}  // namespace

int main(int argc, char** argv) {
    try {
        const std::vector<std::string> v = read_config(argc, argv);
        Args a{v};
        if (a.find("--help") != -1 || a.find("-h") != -1 || a.find("--helpVerbose") != -1 || a.find("-hv") != -1) {
            usage();
            return 0;
        }
        bool fp32 = std::string(argv[0]).find("fp32") != std::string::npos;
        int i;
        if ((i = a.find("--precision")) != -1) {
            const std::string p = a.str(++i);
            if (p != "fp32" && p != "fp64") throw Fail("--precision takes fp32 or fp64");
            fp32 = p == "fp32";
        }
        if (fp32) {
            Run<float> r{a};
            return r.run();
        }
        Run<double> r{a};
        return r.run();
    } catch (const std::exception& e) {
        std::cerr << "phoenix_b200: " << e.what() << std::endl;
        return 1;
    }
}
