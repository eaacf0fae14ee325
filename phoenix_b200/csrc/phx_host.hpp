// Host-side arithmetic that must round exactly like the reference build of
// the same precision: derived kernel constants (calculateAuto,
// source/system/system.cpp:116-160), temporal envelopes
// (Envelope::updateTemporal, source/system/envelope.cpp:466-500, with the
// helpers of include/system/envelope.hpp:165-175) and the per-stage
// interpolation amp*(1-w) + w*amp_next (kernel_gp_compute.cuh:79,93,102).
// Compiled with -ffp-contract=off so no multiply-add is fused.
#pragma once

#include <cmath>
#include <complex>
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
};

template <typename T>
std::complex<T> temporal_value(const TemporalSpec& s, T t) {
    const T t0 = (T)s.t0, sigma = (T)s.sigma, freq = (T)s.freq;
    switch (s.kind) {
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

}  // namespace phx
