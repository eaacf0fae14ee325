// Host-side arithmetic that must round exactly like the reference build of
// the same precision: derived kernel constants (calculateAuto,
// source/system/system.cpp:116-160), temporal envelopes
// (Envelope::updateTemporal, source/system/envelope.cpp:466-500, with the
// helpers of include/system/envelope.hpp:165-175) and the per-stage
// interpolation amp*(1-w) + w*amp_next (kernel_gp_compute.cuh:79,93,102).
// Compiled with -ffp-contract=off so no multiply-add is fused.
#pragma once

#include <cmath>
#include <algorithm>
#include <complex>
#include <vector>
#include <initializer_list>
#include <cstdint>

#include "../../include/phx.h"

namespace phx {

template <typename T>
struct Derived {
    T dx, dy, dV, odx2, ody2, m2, meff, ohb;
};

template <typename T>
Derived<T> derive(const phx_params& p) {
    Derived<T> d;
    const T L_x = (T)p.L_x, L_y = (T)p.L_y, hbs = (T)p.h_bar_s, m_eff = (T)p.m_eff;
    d.dx = L_x / (T)(unsigned)(p.N_c - 1);
    d.dy = L_y / (T)(unsigned)(p.N_r - 1);
    d.dV = d.dx * d.dy;
    d.odx2 = (T)1.0 / (d.dx * d.dx);
    d.ody2 = (T)1.0 / (d.dy * d.dy);
    d.m2 = (T)-2.0 * (d.odx2 + d.ody2);
    d.meff = (T)(-0.5 * (double)hbs * (double)hbs / (double)m_eff);
    d.ohb = (T)(1.0 / (double)hbs);
    return d;
}

struct TemporalSpec {
    int kind = PHX_TEMPORAL_CONSTANT;
    double t0 = 0, sigma = 0, freq = 0;
    std::vector<double> tt, re, im;  // PHX_TEMPORAL_LOADED
};

template <typename T>
std::complex<T> temporal_value(const TemporalSpec& s, T t) {
    const T t0 = (T)s.t0, sigma = (T)s.sigma, freq = (T)s.freq;
    switch (s.kind) {
        case PHX_TEMPORAL_LOADED: {
            // the table in the build precision: the last point after its end, else
            // v1 + (v2 - v1) (t - t1) / (t2 - t1) between the neighbours of the
            // first point >= t (index clamped to 1..n-1)
            const size_t n = s.tt.size();
            if (t > (T)s.tt[n - 1]) return std::complex<T>((T)s.re[n - 1], (T)s.im[n - 1]);
            const auto it = std::lower_bound(s.tt.begin(), s.tt.end(), t, [](double a, T b) { return (T)a < b; });
            const size_t idx = std::min<size_t>(std::max<size_t>(1, (size_t)(it - s.tt.begin())), n - 1);
            const T t1 = (T)s.tt[idx - 1], t2 = (T)s.tt[idx];
            const std::complex<T> v1((T)s.re[idx - 1], (T)s.im[idx - 1]), v2((T)s.re[idx], (T)s.im[idx]);
            return v1 + (v2 - v1) * (t - t1) / (t2 - t1);
        }
        case PHX_TEMPORAL_IEXP: {
            const T a = (t - t0) * (t - t0) / ((T)2.0 * sigma * sigma);
            const T b = freq * (t - t0);
            return std::exp(std::complex<T>(-a, -b));
        }
        case PHX_TEMPORAL_COS: {
            const T q = (t - t0) / sigma;
            return std::complex<T>((T)(std::exp(-0.5 * q * q) * (1.0 + (double)std::cos(freq * (t - t0))) / 2.0), (T)0);
        }
        case PHX_TEMPORAL_GAUSS: {
            const T q = (t - t0) / sigma;
            return std::complex<T>((T)std::exp(-0.5 * (double)std::pow(q * q, freq)), (T)0);
        }
        default:
            return std::complex<T>((T)1, (T)0);
    }
}

template <typename T>
std::complex<T> interp(std::complex<T> amp, std::complex<T> next, T w) {
    const T omw = (T)1.0 - w;
    return std::complex<T>(amp.real() * omw + w * next.real(), amp.imag() * omw + w * next.imag());
}

// Fixed-step explicit tableaux of the reference's registered iterators, as
// their step() functions call CALCULATE_K(s, c_s), INTERMEDIATE_SUM_K(s, a_s..)
// and FINAL_SUM_K(S, b..): weight lists zeros included, in the build
// precision.  Two reference entries are not well defined and follow the
// method instead: RK3's final sum lists a fourth weight for three stages
// (runge_kutta.cu:46; the printed tableau, :28-30, has three) and Ralston4
// declares k_max 3 for four stages (ralston.cu:92-93).
struct Tableau {
    int S = 0;          // stages of the fixed-step sequence (index of the final sum)
    int H = 0;          // k_max_ = halo_size_ (S unless set)
    double c[16] = {};  // envelope time weight of stage s
    int nw[16] = {};    // weights of intermediate sum s
    double a[16][16] = {};
    int nb = 0;         // weights of the final / solution sum
    double b[16] = {};
    // adaptive iterators: the solution sum goes to the buffer, an extra stage
    // S + 1 when fsal, ERROR_K(e_1..e_E), adaptTimeStep(power)
    bool adaptive = false, fsal = false;
    bool inverted = false;  // DP85: the reference swaps its fixed and variable branches
    int E = 0;
    double e[16] = {};
    double power = 0.25;
};

inline bool tableau_for(int it, Tableau& t) {
    t = Tableau();
    auto row = [&](int s, std::initializer_list<double> w) {
        t.nw[s] = (int)w.size();
        int q = 0;
        for (double v : w) t.a[s][q++] = v;
    };
    auto fin = [&](std::initializer_list<double> w) {
        t.nb = (int)w.size();
        int q = 0;
        for (double v : w) t.b[q++] = v;
    };
    auto cs = [&](std::initializer_list<double> w) {
        t.S = (int)w.size();
        int q = 0;
        for (double v : w) t.c[q++] = v;
    };
    auto err = [&](std::initializer_list<double> w) {
        t.E = (int)w.size();
        int q = 0;
        for (double v : w) t.e[q++] = v;
    };
    auto adaptive = [&](int S, int H, bool fsal, double power) {
        t.S = S, t.H = H, t.adaptive = true, t.fsal = fsal, t.power = power;
    };
    switch (it) {
        case PHX_ITER_RK4:  // runge_kutta.cu:74-94 (the k-stack form; real-time RK4 runs the fused iteration)
            cs({0.0, 0.5, 0.5, 1.0});
            row(0, {0.5}), row(1, {0.5}), row(2, {1.0}), fin({1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0});
            return true;
        case PHX_ITER_RK3:  // runge_kutta.cu:33-47
            cs({0.0, 1.0 / 2.0, 1.0});
            row(0, {0.5}), row(1, {-1.0, 2.0}), fin({1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0});
            return true;
        case PHX_ITER_SSPRK3:  // SSPRK3.cu:27-41
            cs({0.0, 1.0, 1.0});
            row(0, {1.0}), row(1, {1.0 / 4.0, 1.0 / 4.0}), fin({1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0});
            return true;
        case PHX_ITER_MP:  // explicit_mp.cu:28-38
            cs({0.0, 0.5});
            row(0, {0.5}), fin({0.0, 1.0});
            return true;
        case PHX_ITER_HEUN2:  // heun.cu:31-41
            cs({0.0, 1.0});
            row(0, {1.0}), fin({0.5, 0.5});
            return true;
        case PHX_ITER_HEUN3:  // heun.cu:66-80
            cs({0.0, 1.0 / 3.0, 2.0 / 3.0});
            row(0, {1.0 / 3.0}), row(1, {0.0, 2.0 / 3.0}), fin({1.0 / 4.0, 0.0, 3.0 / 4.0});
            return true;
        case PHX_ITER_HW:  // houwen_wray.cu:27-41
            cs({0.0, 8.0 / 15.0, 2.0 / 3.0});
            row(0, {8.0 / 15.0}), row(1, {1.0 / 4.0, 5.0 / 12.0}), fin({1.0 / 4.0, 0.0, 3.0 / 4.0});
            return true;
        case PHX_ITER_NEWTON:  // newton.cu:24-30
            cs({0.0});
            fin({1.0});
            return true;
        case PHX_ITER_NYSTROEM:  // nystroem.cu:30-56
            cs({0.0, 1.0 / 3.0, 2.0 / 5.0, 1.0, 2.0 / 3.0, 4.0 / 5.0});
            row(0, {1.0 / 3.0}), row(1, {4.0 / 25.0, 6.0 / 25.0}), row(2, {1.0 / 4.0, -3.0, 15.0 / 4.0});
            row(3, {2.0 / 27.0, 10.0 / 9.0, -(50.0 / 81.0), 8.0 / 81.0});
            row(4, {2.0 / 25.0, 12.0 / 25.0, 2.0 / 15.0, 8.0 / 75.0});
            fin({23.0 / 192.0, 0.0, 125.0 / 192.0, 0.0, -(27.0 / 64.0), 125.0 / 192.0});
            return true;
        case PHX_ITER_RALSTON:  // ralston.cu:31-41
            cs({0.0, 2.0 / 3.0});
            row(0, {2.0 / 3.0}), fin({1.0 / 4.0, 3.0 / 4.0});
            return true;
        case PHX_ITER_RALSTON3:  // ralston.cu:66-80
            cs({0.0, 1.0 / 2.0, 3.0 / 4.0});
            row(0, {1.0 / 2.0}), row(1, {0.0, 3.0 / 4.0}), fin({2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0});
            return true;
        case PHX_ITER_RALSTON4:  // ralston.cu:106-124
            cs({0.0, 0.4, 0.51823725421, 0.51823725421});
            row(0, {0.4}), row(1, {0.29697760924, 0.15875964497}), row(2, {0.21810038822, -3.05096514869, 3.83286476047});
            fin({0.17476028226, -0.55148066287, 1.2055355994, 0.17118478122});
            return true;
        case PHX_ITER_RULE38:  // rule38.cu:28-47
            cs({0.0, 1.0 / 3.0, 2.0 / 3.0, 1.0});
            row(0, {1.0 / 3.0}), row(1, {-1.0 / 3.0, 1.0}), row(2, {1.0, -1.0, 1.0});
            fin({1.0 / 8.0, 3.0 / 8.0, 3.0 / 8.0, 1.0 / 8.0});
            return true;
        case PHX_ITER_DP45:  // dormand_prince.cu:37-95
            cs({0.0, 1.0 / 5.0, 3.0 / 10.0, 4.0 / 5.0, 8.0 / 9.0, 1.0, 1.0});
            adaptive(6, 7, true, 1.0 / 4.0);
            row(0, {1.0 / 5.0}), row(1, {3.0 / 40.0, 9.0 / 40.0}), row(2, {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0});
            row(3, {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0});
            row(4, {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0});
            fin({35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0});
            err({35.0 / 384.0 - 5179.0 / 57600.0, 0.0, 500.0 / 1113.0 - 7571.0 / 16695.0, 125.0 / 192.0 - 393.0 / 640.0,
                 -2187.0 / 6784.0 + 92097.0 / 339200.0, 11.0 / 84.0 - 187.0 / 2100.0, -1.0 / 40.0});
            return true;
        case PHX_ITER_BOSHA:  // bogacki.cu:27-76 (a_32 as the reference writes it at :42: 3/9)
            cs({0.0, 1.0 / 2.0, 3.0 / 4.0, 1.0});
            adaptive(3, 4, true, 1.0 / 3.0);
            row(0, {1.0 / 2.0}), row(1, {0.0, 3.0 / 9.0}), fin({2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0});
            err({2.0 / 9.0 - 7.0 / 24.0, 1.0 / 3.0 - 1.0 / 4.0, 4.0 / 9.0 - 1.0 / 3.0, 0.0 - 1.0 / 8.0});
            return true;
        case PHX_ITER_CASHKARP:  // cash_karp.cu:31-84
            cs({0.0, 1.0 / 5.0, 3.0 / 10.0, 3.0 / 5.0, 1.0, 7.0 / 8.0});
            adaptive(6, 6, false, 1.0 / 4.0);
            row(0, {1.0 / 5.0}), row(1, {3.0 / 40.0, 9.0 / 40.0}), row(2, {3.0 / 1.0, -9.0 / 10.0, 6.0 / 5.0});
            row(3, {-11.0 / 54.0, 5.0 / 2.0, -70.0 / 27.0, 35.0 / 27.0});
            row(4, {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0});
            fin({37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0});
            err({37.0 / 378.0 - 2825.0 / 27648.0, 0.0, 250.0 / 621.0 - 18575.0 / 48384.0, 125.0 / 594.0 - 13525.0 / 55296.0,
                 0.0 - 2187.0 / 6784.0, 512.0 / 1771.0 - 1.0 / 4.0});
            return true;
        case PHX_ITER_FEHLBERG2:  // fehlberg.cu:33-73
            cs({0.0, 1.0 / 2.0, 1.0});
            adaptive(3, 3, false, 1.0 / 4.0);
            row(0, {1.0 / 2.0}), row(1, {1.0 / 256.0, 255.0 / 256.0}), fin({1.0 / 512.0, 255.0 / 256.0, 1.0 / 512.0});
            err({1.0 / 512.0 - 1.0 / 256.0, 0.0, 1.0 / 512.0});
            return true;
        case PHX_ITER_FEHLBERG5:  // fehlberg.cu:100-153
            cs({0.0, 1.0 / 4.0, 3.0 / 8.0, 12.0 / 13.0, 1.0, 1.0 / 2.0});
            adaptive(6, 6, false, 1.0 / 4.0);
            row(0, {1.0 / 4.0}), row(1, {3.0 / 32.0, 9.0 / 32.0}), row(2, {1932.0 / 2197.0, -7200.0 / 2197.0, 7296.0 / 2197.0});
            row(3, {439.0 / 216.0, -8.0, 3680.0 / 513.0, -845.0 / 4104.0});
            row(4, {-8.0 / 27.0, 2.0, -3544.0 / 2565.0, 1859.0 / 4104.0, -11.0 / 40.0});
            fin({16.0 / 135.0, 0.0, 6656.0 / 12825.0, 28561.0 / 56430.0, -9.0 / 50.0, 2.0 / 55.0});
            err({16.0 / 135.0 - 25.0 / 216.0, 0.0, 6656.0 / 12825.0 - 1408.0 / 2565.0, 28561.0 / 56430.0 - 2197.0 / 4104.0,
                 -9.0 / 50.0 - 1.0 / 5.0, 2.0 / 55.0});
            return true;
        case PHX_ITER_DP85:  // dormand_prince.cu:128-204
            cs({0.0, 0.05260015196, 0.07890022794, 0.1183503419, 0.2816496581, 0.3333333333, 0.25, 0.3076923077, 0.6512820513, 0.6, 0.8571428571, 1.0});
            adaptive(12, 12, false, 1.0 / 4.0);
            t.inverted = true;  // dormand_prince.cu:182-190 tests `if (variable_time_step)`
            row(0, {5.260015195876773e-2});
            row(1, {1.9725056984537899e-2, 5.9175170953613698e-2});
            row(2, {2.9587585476806849e-2, 0.0, 8.8762756430420548e-2});
            row(3, {2.4136513415926669e-1, 0.0, -8.8454947932828610e-1, 9.2483400326179200e-1});
            row(4, {3.7037037037037037e-2, 0.0, 0.0, 1.7082860872947387e-1, 1.2546768756682243e-1});
            row(5, {3.7109375e-2, 0.0, 0.0, 1.7025221101954404e-1, 6.0216538980455961e-2, -1.7578125e-2});
            row(6, {3.7092000118504793e-2, 0.0, 0.0, 1.7038392571223999e-1, 1.0726203044637328e-1, -1.5319437748624402e-2, 8.2737891638140229e-3});
            row(7, {6.2411095871607572e-1, 0.0, 0.0, -3.3608926294469413e+0, -8.6821934684172601e-1, 2.7592099699446708e+1, 2.0154067550477893e+1, -4.3489884181069959e+1});
            row(8, {4.7766253643826437e-1, 0.0, 0.0, -2.4881146199716676e+0, -5.9029082683684300e-1, 2.1230051448181194e+1, 1.5279233632882424e+1, -3.3288210968984863e+1, -2.0331201708508626e-2});
            row(9, {-9.3714243008598733e-1, 0.0, 0.0, 5.1863724288440637e+0, 1.0914373489967296e+0, -8.1497870107469261e+0, -1.8520065659996960e+1, 2.2739487099350504e+1, 2.4936055526796524e+0, -3.0467644718982195e+0});
            row(10, {2.2733101475165382e+0, 0.0, 0.0, -1.0534495466737250e+1, -2.0008720582248625e+0, -1.7958931863118799e+1, 2.7948884529419960e+1, -2.8589982771350237e+0, -8.8728569335306295e+0, 1.2360567175794303e+1, 6.4339274601576353e-1});
            fin({5.4293734116568762e-2, 0.0, 0.0, 0.0, 0.0, 4.4503128927524089e+0, 1.8915178993145004e+0, -5.8012039600105848e+0, 3.1116436695781989e-1, -1.5216094966251608e-1, 2.0136540080403035e-1, 4.4710615727772591e-2});
            err({4.1173689122373888e-2, 0.0, 0.0, 0.0, 0.0, 5.6754693391286133e+0, 2.3872768489717506e+0, -7.4655811424655713e+0, 6.6149321570779360e-1, -4.8634006837553356e-1, 1.1944219431891464e-1, 6.7065923591658886e-2});
            return true;
        case PHX_ITER_NSRK78:  // NSRK78.cu:37-117
            cs({0.0, 0.001, 0.1111111111, 0.1666666667, 0.4166666667, 0.5, 0.8333333333, 0.1666666667, 0.6666666667, 0.76, 0.84, 1.0, 1.0});
            adaptive(13, 13, false, 1.0 / 8.0);
            row(0, {1.0 / 1000.0});
            row(1, {-491.0 / 81.0, 500.0 / 81.0});
            row(2, {1.0 / 24.0, 0.0, 1.0 / 8.0});
            row(3, {5.0 / 12.0, 0.0, -25.0 / 16.0, 25.0 / 16.0});
            row(4, {1.0 / 20.0, 0.0, 0.0, 1.0 / 4.0, 1.0 / 5.0});
            row(5, {-43.0 / 180.0, 0.0, 0.0, 127.0 / 108.0, -329.0 / 135.0, 7.0 / 3.0});
            row(6, {27931.0 / 240300.0, 0.0, 0.0, -631.0 / 16020.0, 2459.0 / 6675.0, -3572.0 / 12015.0, 5.0 / 267.0});
            row(7, {26114.0 / 12015.0, 0.0, 0.0, -7480.0 / 801.0, 67264.0 / 4005.0, -30640.0 / 2403.0, 1051.0 / 1335.0, 3.0});
            row(8, {33096587331.0 / 17382812500.0, 0.0, 0.0, -1828977848.0 / 173828125.0, 62801809904.0 / 4345703125.0, -9389764774.0 / 869140625.0, 6380757669.0 / 8691406250.0, 98417891.0 / 19531250.0, -1692691.0 / 39062500.0});
            row(9, {-1456295425347.0 / 2642187500000.0, 0.0, 0.0, 110740056.0 / 34765625.0, -21221682384.0 / 4345703125.0, 58859060169.0 / 13906250000.0, -177381525069.0 / 1529687500000.0, -28942485159.0 / 27812500000.0, -1272297.0 / 312500000.0, 5151.0 / 297616.0});
            row(10, {844300798.0 / 137013275.0, 0.0, 0.0, -9997568.0 / 206035.0, 49636624.0 / 1030175.0, -3358834871.0 / 91067470.0, -40456983.0 / 1813108.0, 495817135.0 / 16647628.0, -149375.0 / 84266.0, 7470703125.0 / 1567431866.0, 1562500000.0 / 72342361.0});
            row(11, {-26225423.0 / 37371100.0, 0.0, 0.0, 807744.0 / 98345.0, -205584.0 / 37825.0, 5882202.0 / 1278485.0, -84543.0 / 432718.0, -223415.0 / 39338.0, -3625.0 / 6188.0, 292968750.0 / 374084711.0, 0.0, 0.0});
            fin({4241.0 / 88200.0, 0.0, 0.0, 0.0, 0.0, 9946.0 / 23205.0, -10449.0 / 1925.0, 415449.0 / 1573075.0, -2025.0 / 5096.0, 48828125.0 / 44900856.0, 48828125.0 / 9843561.0, 463.0 / 12600.0, 0.0});
            err({4241.0 / 88200.0 - 3799.0 / 79800.0, 0.0, 0.0, 0.0, 0.0, 9946.0 / 23205.0 - 538.0 / 1365.0, -10449.0 / 1925.0 - 351.0 / 1925.0, 415449.0 / 1573075.0 - 4149.0 / 15575.0, -2025.0 / 5096.0 - ( -45.0 / 392.0 ), 48828125.0 / 44900856.0 - 48828125.0 / 284372088.0, 48828125.0 / 9843561.0 - 0.0, 463.0 / 12600.0 - 0.0, 0.0 - 221.0 / 4200.0});
            return true;
        default:
            return false;
    }
}

inline bool tableau_resolve(int it, Tableau& t) {
    if (!tableau_for(it, t)) return false;
    if (t.H == 0) t.H = t.S;  // fixed-step iterators: halo_size_ = k_max_ = stages
    return true;
}

}  // namespace phx
