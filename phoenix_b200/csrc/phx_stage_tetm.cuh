// Fused RK stage kernel for the TE/TM spinor: psi+, psi-, n+, n- in one pass.
//
// Right-hand side of gp_scalar's TE/TM branch
// (include/kernel/kernel_gp_compute.cuh:112-235): both polarisations with
// g_pm cross-interaction and the TE-TM splitting term delta_LT * H_cross,
// whose mixed derivative reads the diagonal neighbours of the other
// component.  A warp keeps three rows of both components in registers
// (with their left/right neighbours from shuffles and edge loads), so the
// nine-point stencil needs no shared-memory halo and no halo kernel.
#pragma once

#include "phx_stage.cuh"

namespace phx {

template <typename T>
struct TetmParams {
    StageParams<T> p;  // plus component and every shared constant
    // minus component planes
    const cx<T>* psi_in;
    const T* n_in;
    const cx<T>* psi0;
    const T* n0;
    cx<T>* psi_out;
    T* n_out;
    cx<T>* acc_psi;
    T* acc_n;
    cx<T>* k_psi;
    T* k_n;
    const T* pump;
    const T* pot;
    const cx<T>* pulse;
    // TE/TM constants
    T ohb_meff;  // one_over_h_bar_s * m_eff_scaled
    T ohb_gpm;   // one_over_h_bar_s * g_pm
    T ohb_dlt;   // one_over_h_bar_s * delta_LT
    cx<T> hidd;  // half_i / dx / dy
};

template <typename T>
struct Row {
    Pack<T> v;
    cx<T> el, er;  // left neighbour of lane 0, right neighbour of lane 31
};

template <typename T>
__device__ __forceinline__ Row<T> load_row(const cx<T>* base, long long rowo, int cl, int c_left, int c_right, int lane) {
    Row<T> r;
    r.v = ldp(base + rowo + cl);
    r.el = mk((T)0, (T)0);
    r.er = mk((T)0, (T)0);
    if (lane == 0) r.el = ld1(base + rowo + c_left);
    if (lane == 31) r.er = ld1(base + rowo + c_right);
    return r;
}

// left / right neighbours of point j of this lane
template <typename T>
__device__ __forceinline__ void neighbours(const Row<T>& r, int lane, cx<T>* L, cx<T>* R) {
    constexpr int CPT = Pack<T>::CPT;
    cx<T> l0 = shfl_up1(r.v.v[CPT - 1]);
    cx<T> rN = shfl_dn1(r.v.v[0]);
    if (lane == 0) l0 = r.el;
    if (lane == 31) rN = r.er;
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
        L[j] = j == 0 ? l0 : r.v.v[j - 1];
        R[j] = j == CPT - 1 ? rN : r.v.v[j + 1];
    }
}

// Both polarisations at one point: k of psi+, n+, psi-, n-; the pointwise
// inputs come from `src` (TetmGlobalSrc or a shared-memory copy).  The
// reference multiplies complex numbers whose imaginary part is exactly zero
// (the reservoir, stored real here) or whose real part is (half_i / dx / dy),
// and multiplies by -1 to negate; this keeps only the products that are not
// with that zero and negates directly, which changes no result except,
// possibly, the sign of an exact zero.
template <typename T, typename Src>
__device__ __forceinline__ void rhs_tetm_src(const TetmParams<T>& Q, const Src& src, cx<T> wp, cx<T> upp, cx<T> dnp, cx<T> lp,
                                             cx<T> rp, cx<T> ulp, cx<T> urp, cx<T> dlp, cx<T> drp, cx<T> wm, cx<T> upm,
                                             cx<T> dnm, cx<T> lm, cx<T> rm, cx<T> ulm, cx<T> urm, cx<T> dlm, cx<T> drm, T rvp,
                                             T rvm, cx<T>& kwp, T& krp, cx<T>& kwm, T& krm) {
    const StageParams<T>& P = Q.p;
    const cx<T> in_wf_plus_mi = mk(wp.im, -wp.re);
    const cx<T> in_wf_minus_mi = mk(wm.im, -wm.re);
    const cx<T> horizontal_plus = smul(P.odx2, cadd(rp, lp));
    const cx<T> vertical_plus = smul(P.ody2, cadd(dnp, upp));
    const cx<T> horizontal_minus = smul(P.odx2, cadd(rm, lm));
    const cx<T> vertical_minus = smul(P.ody2, cadd(dnm, upm));
    // psi[i+ro+1] + psi[i-ro-1] - psi[i+ro-1] - psi[i-ro+1]
    const cx<T> diag_m = csub(csub(cadd(drm, ulm), dlm), urm);
    const cx<T> diag_p = csub(csub(cadd(drp, ulp), dlp), urp);
    // hidd = (0, h): (0 a - h b, 0 b + h a) = (-h b, h a)
    cx<T> hcp = cadd(csub(horizontal_minus, vertical_minus), mk(-rmul(Q.hidd.im, diag_m.im), rmul(Q.hidd.im, diag_m.re)));
    cx<T> hcm = csub(csub(horizontal_plus, vertical_plus), mk(-rmul(Q.hidd.im, diag_p.im), rmul(Q.hidd.im, diag_p.re)));
    cx<T> hrp = cadd(cadd(smul(P.m2, wp), horizontal_plus), vertical_plus);
    cx<T> hrm = cadd(cadd(smul(P.m2, wm), horizontal_minus), vertical_minus);
    const T npl = abs2(wp), nmi = abs2(wm);
    hrp = mk(hrp.im, -hrp.re);
    hrm = mk(hrm.im, -hrm.re);
    hcp = mk(hcp.im, -hcp.re);
    hcm = mk(hcm.im, -hcm.re);

    // wavefunction plus
    cx<T> res = smul(Q.ohb_meff, hrp);
    for (int g = 0; g < P.n_pot; ++g) {
        const cx<T> pot = smul(src.pot(0, g), P.pot_c[g]);
        res = cadd(res, cmul(smul(P.ohb, pot), in_wf_plus_mi));
    }
    res = cadd(res, smul(rmul(P.ohb_gc, npl), in_wf_plus_mi));
    res = cadd(res, smul(rmul(P.ohb_gr, rvp), in_wf_plus_mi));
    res = cadd(res, smul(rmul(P.half_R, rvp), wp));
    res = csub(res, smul(P.half_gamma_c, wp));
    res = cadd(res, smul(rmul(Q.ohb_gpm, nmi), in_wf_plus_mi));
    res = cadd(res, smul(Q.ohb_dlt, hcp));
    for (int g = 0; g < P.n_pulse; ++g) res = cadd(res, cmul(smul(P.ohb, src.pulse(0, g)), P.pulse_c[g]));
    if (P.noise.on) res = csub(res, noise_drift(P, in_wf_plus_mi));
    kwp = res;
    // reservoir plus
    T r = rmul(-radd(P.gamma_r, rmul(P.R, npl)), rvp);
    for (int g = 0; g < P.n_pump; ++g) r = radd(r, rmul(src.pump(0, g), P.pump_c[g].re));
    if (P.noise.on) r = radd(r, rdiv(rmul(P.R, rvp), P.dV));
    krp = r;
    // wavefunction minus
    res = smul(Q.ohb_meff, hrm);
    for (int g = 0; g < P.n_pot; ++g) {
        const cx<T> pot = smul(src.pot(1, g), P.pot_c[g]);
        res = cadd(res, cmul(smul(P.ohb, pot), in_wf_minus_mi));
    }
    res = cadd(res, smul(rmul(P.ohb_gc, nmi), in_wf_minus_mi));
    res = cadd(res, smul(rmul(P.ohb_gr, rvm), in_wf_minus_mi));
    res = cadd(res, smul(rmul(P.half_R, rvm), wm));
    res = csub(res, smul(P.half_gamma_c, wm));
    res = cadd(res, smul(rmul(Q.ohb_gpm, npl), in_wf_minus_mi));
    res = cadd(res, smul(Q.ohb_dlt, hcm));
    for (int g = 0; g < P.n_pulse; ++g) res = cadd(res, cmul(smul(P.ohb, src.pulse(1, g)), P.pulse_c[g]));
    if (P.noise.on) res = csub(res, noise_drift(P, in_wf_minus_mi));
    kwm = res;
    // reservoir minus
    r = rmul(-radd(P.gamma_r, rmul(P.R, nmi)), rvm);
    for (int g = 0; g < P.n_pump; ++g) r = radd(r, rmul(src.pump(1, g), P.pump_c[g].re));
    if (P.noise.on) r = radd(r, rdiv(rmul(P.R, rvm), P.dV));
    krm = r;
}

// The pointwise inputs of one point (pump, potential, pulse of group g of
// component c) read from the global planes
template <typename T>
struct TetmGlobalSrc {
    const TetmParams<T>& Q;
    long long idx;
    __device__ __forceinline__ T pump(int c, int g) const { return __ldg((c ? Q.pump : Q.p.pump) + idx + g * Q.p.plane); }
    __device__ __forceinline__ T pot(int c, int g) const { return __ldg((c ? Q.pot : Q.p.pot) + idx + g * Q.p.plane); }
    __device__ __forceinline__ cx<T> pulse(int c, int g) const { return ld1((c ? Q.pulse : Q.p.pulse) + idx + g * Q.p.plane); }
};

// Both polarisations at one point, the pointwise inputs from the global planes
template <typename T>
__device__ __forceinline__ void rhs_tetm(const TetmParams<T>& Q, long long idx, cx<T> wp, cx<T> upp, cx<T> dnp, cx<T> lp, cx<T> rp,
                                         cx<T> ulp, cx<T> urp, cx<T> dlp, cx<T> drp, cx<T> wm, cx<T> upm, cx<T> dnm, cx<T> lm,
                                         cx<T> rm, cx<T> ulm, cx<T> urm, cx<T> dlm, cx<T> drm, T rvp, T rvm, cx<T>& kwp, T& krp,
                                         cx<T>& kwm, T& krm) {
    rhs_tetm_src<T>(Q, TetmGlobalSrc<T>{Q, idx}, wp, upp, dnp, lp, rp, ulp, urp, dlp, drp, wm, upm, dnm, lm, rm, ulm, urm, dlm,
                    drm, rvp, rvm, kwp, krp, kwm, krm);
}

template <typename T, int KIND, int RB, int WARPS>
__global__ void __launch_bounds__(32 * WARPS) stage_tetm_kernel(const __grid_constant__ TetmParams<T> Q) {
    constexpr int CPT = Pack<T>::CPT;
    const StageParams<T>& P = Q.p;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int c_base = P.c0 + blockIdx.x * (32 * CPT);
    const int c = c_base + lane * CPT;
    const int rs = P.r0 + (blockIdx.y * WARPS + warp) * RB;
    const int re = min(rs + RB, P.r1);
    const bool active = c < P.c1;
    const int cl = min(c, P.c1);
    const int c_left = c_base - 1;
    const int c_right = min(c_base + 32 * CPT, P.c1);
    const long long pitch = P.pitch;
    double err_acc = 0.0, norm_acc = 0.0;

    if (rs < P.r1) {
        Row<T> upP = load_row(P.psi_in, (long long)(rs - 1) * pitch, cl, c_left, c_right, lane);
        Row<T> ceP = load_row(P.psi_in, (long long)rs * pitch, cl, c_left, c_right, lane);
        Row<T> upM = load_row(Q.psi_in, (long long)(rs - 1) * pitch, cl, c_left, c_right, lane);
        Row<T> ceM = load_row(Q.psi_in, (long long)rs * pitch, cl, c_left, c_right, lane);
        for (int r = rs; r < re; ++r) {
            const long long rowo = (long long)r * pitch;
            const Row<T> dnP = load_row(P.psi_in, rowo + pitch, cl, c_left, c_right, lane);
            const Row<T> dnM = load_row(Q.psi_in, rowo + pitch, cl, c_left, c_right, lane);
            cx<T> uLp[CPT], uRp[CPT], cLp[CPT], cRp[CPT], dLp[CPT], dRp[CPT];
            cx<T> uLm[CPT], uRm[CPT], cLm[CPT], cRm[CPT], dLm[CPT], dRm[CPT];
            neighbours(upP, lane, uLp, uRp);
            neighbours(ceP, lane, cLp, cRp);
            neighbours(dnP, lane, dLp, dRp);
            neighbours(upM, lane, uLm, uRm);
            neighbours(ceM, lane, cLm, cRm);
            neighbours(dnM, lane, dLm, dRm);
            const long long idx = rowo + cl;
            const RPack<T> nip = ldr(P.n_in + idx);
            const RPack<T> nim = ldr(Q.n_in + idx);
            if (active) {
                Pack<T> owp, owm;
                RPack<T> orp, orm;
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    rhs_tetm<T>(Q, idx + j, ceP.v.v[j], upP.v.v[j], dnP.v.v[j], cLp[j], cRp[j], uLp[j], uRp[j], dLp[j], dRp[j],
                                ceM.v.v[j], upM.v.v[j], dnM.v.v[j], cLm[j], cRm[j], uLm[j], uRm[j], dLm[j], dRm[j], nip.v[j],
                                nim.v[j], owp.v[j], orp.v[j], owm.v[j], orm.v[j]);
                }
                if constexpr (KIND == kRk4First || KIND == kRk4Mid || KIND == kRk4Last) {
                    // per component: (psi_in, n_in) are y0 in stage 1
                    const Pack<T> y0p = KIND == kRk4First ? ceP.v : ldp(P.psi0 + idx);
                    const Pack<T> y0m = KIND == kRk4First ? ceM.v : ldp(Q.psi0 + idx);
                    const RPack<T> n0p = KIND == kRk4First ? nip : ldr(P.n0 + idx);
                    const RPack<T> n0m = KIND == kRk4First ? nim : ldr(Q.n0 + idx);
                    Pack<T> ap, am;
                    RPack<T> anp, anm;
                    if constexpr (KIND != kRk4First) {
                        ap = ldp_rw(P.acc_psi + idx);
                        am = ldp_rw(Q.acc_psi + idx);
                        anp = ldr_rw(P.acc_n + idx);
                        anm = ldr_rw(Q.acc_n + idx);
                    }
#pragma unroll
                    for (int j = 0; j < CPT; ++j) {
                        if constexpr (KIND == kRk4First) {
                            ap.v[j] = smul(P.b, owp.v[j]);
                            am.v[j] = smul(P.b, owm.v[j]);
                            anp.v[j] = rmul(P.b, orp.v[j]);
                            anm.v[j] = rmul(P.b, orm.v[j]);
                        } else if constexpr (KIND == kRk4Mid) {
                            ap.v[j] = cadd(ap.v[j], smul(P.b, owp.v[j]));
                            am.v[j] = cadd(am.v[j], smul(P.b, owm.v[j]));
                            anp.v[j] = radd(anp.v[j], rmul(P.b, orp.v[j]));
                            anm.v[j] = radd(anm.v[j], rmul(P.b, orm.v[j]));
                        }
                        if constexpr (KIND != kRk4Last) {
                            owp.v[j] = cadd(y0p.v[j], smul(P.dtw, owp.v[j]));
                            owm.v[j] = cadd(y0m.v[j], smul(P.dtw, owm.v[j]));
                            orp.v[j] = radd(n0p.v[j], rmul(P.dtw, orp.v[j]));
                            orm.v[j] = radd(n0m.v[j], rmul(P.dtw, orm.v[j]));
                        } else {
                            owp.v[j] = cadd(y0p.v[j], smul(P.dt, cadd(ap.v[j], smul(P.b, owp.v[j]))));
                            owm.v[j] = cadd(y0m.v[j], smul(P.dt, cadd(am.v[j], smul(P.b, owm.v[j]))));
                            orp.v[j] = radd(n0p.v[j], rmul(P.dt, radd(anp.v[j], rmul(P.b, orp.v[j]))));
                            orm.v[j] = radd(n0m.v[j], rmul(P.dt, radd(anm.v[j], rmul(P.b, orm.v[j]))));
                        }
                        if (P.noise.on) {
                            // one noise value for both polarisations, scaled by the plus
                            // reservoir; the final sum updates n+ in place before the minus
                            // wavefunction's sum runs (cuda_macro.cuh:200-229), so psi- sees
                            // the new n+ there
                            const cx<T> xi = stage_xi(P, r, c + j);
                            owp.v[j] = cadd(owp.v[j], stage_noise_of<T, true>(P, xi, n0p.v[j]));
                            owm.v[j] = cadd(owm.v[j], stage_noise_of<T, true>(P, xi, KIND == kRk4Last ? orp.v[j] : n0p.v[j]));
                        }
                    }
                    if constexpr (KIND != kRk4Last) {
                        stp(P.acc_psi + idx, ap);
                        stp(Q.acc_psi + idx, am);
                        str(P.acc_n + idx, anp);
                        str(Q.acc_n + idx, anm);
                    }
                } else {
                    const long long kofs = (long long)(P.stage - 1) * P.plane;
                    if constexpr (KIND == kStack) {
                        stp(P.k_psi + kofs + idx, owp);
                        stp(Q.k_psi + kofs + idx, owm);
                        str(P.k_n + kofs + idx, orp);
                        str(Q.k_n + kofs + idx, orm);
                    }
                    if constexpr (KIND == kStackError) {
                        // the reference's TE/TM error re-reads k of psi+ (cuda_macro.cuh:244)
#pragma unroll
                        for (int j = 0; j < CPT; ++j) {
                            cx<T> e = mk((T)0, (T)0);
                            for (int q = 0; q < P.nw; ++q) {
                                if (P.w[q] == (T)0) continue;
                                const cx<T> kq = (q == P.stage - 1) ? owp.v[j] : ld1(P.k_psi + (long long)q * P.plane + idx + j);
                                e = cadd(e, smul(P.w[q], kq));
                            }
                            err_acc += (double)abs2(smul(P.dt, e)) * (double)P.error_passes;
                            norm_acc += (double)abs2(ceP.v.v[j]);
                        }
                    } else {
                        const Pack<T> y0p = P.stage == 1 ? ceP.v : ldp(P.psi0 + idx);
                        const Pack<T> y0m = P.stage == 1 ? ceM.v : ldp(Q.psi0 + idx);
                        const RPack<T> n0p = P.stage == 1 ? nip : ldr(P.n0 + idx);
                        const RPack<T> n0m = P.stage == 1 ? nim : ldr(Q.n0 + idx);
#pragma unroll
                        for (int j = 0; j < CPT; ++j) {
                            if (P.nw == 1) {
                                owp.v[j] = cadd(y0p.v[j], smul(P.dtw, owp.v[j]));
                                owm.v[j] = cadd(y0m.v[j], smul(P.dtw, owm.v[j]));
                                orp.v[j] = radd(n0p.v[j], rmul(P.dtw, orp.v[j]));
                                orm.v[j] = radd(n0m.v[j], rmul(P.dtw, orm.v[j]));
                            } else {
                                // summation order as in the scalar kernel (7 weights or fewer:
                                // left to right; more: zeros dropped, nested from the right)
                                const bool wide = P.nw > 7;
                                cx<T> a1 = mk((T)0, (T)0), a2 = mk((T)0, (T)0);
                                T b1 = (T)0, b2 = (T)0;
                                bool have = false;
                                for (int u = 0; u < P.nw; ++u) {
                                    const int q = wide ? P.nw - 1 - u : u;
                                    if (wide && P.w[q] == (T)0) continue;
                                    cx<T> k1, k2;
                                    T kn1, kn2;
                                    if (q == P.stage - 1) {
                                        k1 = owp.v[j], k2 = owm.v[j], kn1 = orp.v[j], kn2 = orm.v[j];
                                    } else {
                                        const long long o = (long long)q * P.plane + idx + j;
                                        k1 = ld1(P.k_psi + o), k2 = ld1(Q.k_psi + o), kn1 = P.k_n[o], kn2 = Q.k_n[o];
                                    }
                                    const cx<T> t1 = smul(P.w[q], k1), t2 = smul(P.w[q], k2);
                                    const T u1 = rmul(P.w[q], kn1), u2 = rmul(P.w[q], kn2);
                                    if (!have) {
                                        a1 = t1, a2 = t2, b1 = u1, b2 = u2, have = true;
                                    } else if (wide) {
                                        a1 = cadd(t1, a1), a2 = cadd(t2, a2), b1 = radd(u1, b1), b2 = radd(u2, b2);
                                    } else {
                                        a1 = cadd(a1, t1), a2 = cadd(a2, t2), b1 = radd(b1, u1), b2 = radd(b2, u2);
                                    }
                                }
                                owp.v[j] = cadd(y0p.v[j], smul(P.dt, a1));
                                owm.v[j] = cadd(y0m.v[j], smul(P.dt, a2));
                                orp.v[j] = radd(n0p.v[j], rmul(P.dt, b1));
                                orm.v[j] = radd(n0m.v[j], rmul(P.dt, b2));
                            }
                            if (P.noise.on) {
                                const cx<T> xi = stage_xi(P, r, c + j);
                                owp.v[j] = cadd(owp.v[j], stage_noise_of<T, true>(P, xi, n0p.v[j]));
                                owm.v[j] = cadd(owm.v[j],
                                                stage_noise_of<T, true>(P, xi, KIND == kStackFinal ? orp.v[j] : n0p.v[j]));
                            }
                        }
                    }
                }
                if constexpr (KIND != kStackError) {
                    stp(P.psi_out + idx, owp);
                    stp(Q.psi_out + idx, owm);
                    str(P.n_out + idx, orp);
                    str(Q.n_out + idx, orm);
                    if (P.img_x | P.img_y) {
#pragma unroll
                        for (int j = 0; j < CPT; ++j) {
                            write_images(P, P.psi_out, r, c + j, owp.v[j]);
                            write_images(P, Q.psi_out, r, c + j, owm.v[j]);
                            write_images(P, P.n_out, r, c + j, orp.v[j]);
                            write_images(P, Q.n_out, r, c + j, orm.v[j]);
                        }
                    }
                }
            }
            upP = ceP;
            ceP = dnP;
            upM = ceM;
            ceM = dnM;
        }
    }
    if constexpr (KIND == kStackError) {
        __shared__ double red[2 * WARPS];
        block_reduce2<32 * WARPS>(err_acc, norm_acc, red);
        if (threadIdx.x == 0) {
            const long long b = (long long)blockIdx.y * gridDim.x + blockIdx.x;
            P.partials[2 * b] = err_acc;
            P.partials[2 * b + 1] = norm_acc;
        }
    }
}

}  // namespace phx
