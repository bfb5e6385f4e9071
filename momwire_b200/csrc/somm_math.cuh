// Sommerfeld-integral mathematics shared by the device kernels and host
// builds of the same code (sm_100a + host).
//
// The six lambda-integrals of the NEC-2 theory manual (eqs 148-153, kernels
// D1/D2 of eqs 154-155) on the deformed contours of figs 13-14, and the four
// interpolation surfaces (eqs 156-159, R1 -> 0 limits eqs 169-172), as the
// reference evaluates them (_sommerfeld.py:208-584, C++ six_integrals
// _accelerators.cpp:5723-5785): the same contour waypoints, 24-point
// Gauss-Legendre rule, bisection depth 14 with a segment-relative tolerance
// and the same two-quiet-panel tail rule, so that grid tables agree with the
// reference's to the quadrature's rounding.
//
// Complex Bessel and Hankel functions of order 0 and 1 are this file's own:
//   * ascending series (A&S 9.1.10, 9.1.11, 9.1.13) for |z| < 14 or, for
//     H^(2) below the real axis, |z| < 2;
//   * H^(2) for Im z <= 0, 2 <= |z| < 30 from K_0, K_1 of i z by Steed's
//     continued fraction as formulated by Temme (J. Comput. Phys. 19 (1975)
//     324-337), H^(2)_nu(z) = (2/pi) i^(nu+1) K_nu(i z) (A&S 9.6.4) -- the
//     series J - iY loses exp(2|Im z|) there;
//   * the Hankel expansion (DLMF 10.17.5-6) beyond.
// Accuracy against scipy.special is ~1e-13 relative or better.
#pragma once

#include <math.h>

#include "common.cuh"

#define MW_HD __host__ __device__

namespace mw {
namespace somm {

constexpr double kEulerGamma = 0.57721566490153286061;
constexpr double kTwoOverPi = 0.63661977236758134308;
constexpr int kGaussN = 24;
constexpr int kAdaptDepth = 14;
constexpr int kMaxTailPanels = 800;

// 24-point Gauss-Legendre rule on [-1, 1] (filled on the host).
struct GL24 {
    double x[kGaussN], w[kGaussN];
};

MW_HD inline cd cexp_(cd z) {
    const double e = exp(z.re);
    return cd{e * cos(z.im), e * sin(z.im)};
}
MW_HD inline cd clog_(cd z) { return cd{log(hypot(z.re, z.im)), atan2(z.im, z.re)}; }
MW_HD inline double cabs_(cd z) { return hypot(z.re, z.im); }
MW_HD inline cd cinv(cd z) { return cdiv(cd{1.0, 0.0}, z); }
MW_HD inline cd cscale(cd z, double s) { return cd{z.re * s, z.im * s}; }
MW_HD inline cd mul_i(cd z) { return cd{-z.im, z.re}; }    // i z
MW_HD inline cd mul_mi(cd z) { return cd{z.im, -z.re}; }   // -i z

// ------------------------------------------------------------ Bessel/Hankel
// Ascending series: J0, J1/z, and with_y: Y0, Y1/z (principal log).
MW_HD inline void bessel_series(cd z, bool with_y, cd* j0, cd* j1z, cd* y0, cd* y1z) {
    const cd q = cscale(z * z, -0.25);
    cd a{1.0, 0.0};
    cd s_j0 = a, s_j1 = cscale(a, 0.5);
    cd s_y0{0.0, 0.0};
    cd s_y1 = cscale(a, 1.0 - 2.0 * kEulerGamma);  // k = 0: H_0 + H_1 - 2 gamma
    double hk = 0.0;
    const double az = cabs_(z);
    for (int k = 1; k < 80; ++k) {
        a = cscale(a * q, 1.0 / ((double)k * (double)k));
        const double hk1 = hk + 1.0 / (double)(k + 1) + 1.0 / (double)k;  // H_{k+1}
        hk += 1.0 / (double)k;                                              // H_k
        const cd b = cscale(a, 1.0 / (double)(k + 1));
        s_j0 = s_j0 + a;
        s_j1 = s_j1 + cscale(b, 0.5);
        if (with_y) {
            s_y0 = s_y0 + cscale(a, hk);
            s_y1 = s_y1 + cscale(b, hk + hk1 - 2.0 * kEulerGamma);
        }
        if ((double)k > 0.5 * az + 1.0 && cabs_(a) * (1.0 + 2.0 * hk1) <= 1e-17 * fmax(cabs_(s_j0), 1e-300)) break;
    }
    *j0 = s_j0;
    *j1z = s_j1;
    if (with_y) {
        const cd L = clog_(cscale(z, 0.5));
        *y0 = cscale(cd{L.re + kEulerGamma, L.im} * s_j0 - s_y0, kTwoOverPi);
        const cd iz2 = cinv(z * z);
        *y1z = cscale(iz2, -kTwoOverPi) + cscale(L * s_j1, kTwoOverPi) - cscale(s_y1, 0.5 / kPi);
    }
}

// Hankel expansion of H^(kind)_0 and H^(kind)_1 (kind 1 or 2).
MW_HD inline void hankel_asym(cd z, int kind, cd* h0, cd* h1) {
    const double s = kind == 1 ? 1.0 : -1.0;
    const cd m = cscale(mul_i(cinv(z)), s);  // s i / z
    cd t0{1.0, 0.0}, t1{1.0, 0.0}, s0{1.0, 0.0}, s1{1.0, 0.0};
    double p0 = 1e300, p1 = 1e300;
    bool go0 = true, go1 = true;
    for (int k = 1; k < 64 && (go0 || go1); ++k) {
        const double o = (double)(2 * k - 1) * (double)(2 * k - 1);
        if (go0) {
            const cd t = cscale(t0 * m, (0.0 - o) / (8.0 * k));
            const double at = cabs_(t);
            if (at > p0) {
                go0 = false;
            } else {
                t0 = t;
                p0 = at;
                s0 = s0 + t;
                if (at < 1e-17 * cabs_(s0)) go0 = false;
            }
        }
        if (go1) {
            const cd t = cscale(t1 * m, (4.0 - o) / (8.0 * k));
            const double at = cabs_(t);
            if (at > p1) {
                go1 = false;
            } else {
                t1 = t;
                p1 = at;
                s1 = s1 + t;
                if (at < 1e-17 * cabs_(s1)) go1 = false;
            }
        }
    }
    const cd pref = csqrt_p(cscale(cinv(z), kTwoOverPi));
    const double qp = 0.25 * kPi;
    const cd w0 = cscale(mul_i(cd{z.re - qp, z.im}), s);        // s i (z - pi/4)
    const cd w1 = cscale(mul_i(cd{z.re - 3.0 * qp, z.im}), s);  // s i (z - 3 pi/4)
    *h0 = pref * cexp_(w0) * s0;
    *h1 = pref * cexp_(w1) * s1;
}

// K_0(x), K_1(x) for Re x > 0, |x| >= 2: Steed/Temme continued fraction.
MW_HD inline void bessel_k01_cf(cd x, cd* k0, cd* k1) {
    cd b = cscale(cd{1.0 + x.re, x.im}, 2.0);
    cd d = cinv(b);
    cd h = d, delh = d;
    cd q1{0.0, 0.0}, q2{1.0, 0.0};
    const double a1 = 0.25;
    cd q{a1, 0.0}, c{a1, 0.0};
    double a = -a1;
    cd s = cd{1.0, 0.0} + cscale(delh, a1);
    for (int i = 1; i < 400; ++i) {
        a -= 2.0 * i;
        c = cscale(c, -a / (double)(i + 1));
        const cd qn = cscale(q1 - b * q2, 1.0 / a);
        q1 = q2;
        q2 = qn;
        q = q + c * qn;
        b = cd{b.re + 2.0, b.im};
        d = cinv(b + cscale(d, a));
        delh = (b * d - cd{1.0, 0.0}) * delh;
        h = h + delh;
        const cd dels = q * delh;
        s = s + dels;
        if (cabs_(dels) < 1e-17 * cabs_(s)) break;
    }
    h = cscale(h, a1);
    const cd kk0 = cdiv(csqrt_p(cscale(cinv(x), 0.5 * kPi)) * cexp_(cd{-x.re, -x.im}), s);
    *k0 = kk0;
    *k1 = cdiv(kk0 * cd{x.re + 0.5 - h.re, x.im - h.im}, x);
}

// J0(z) and J1(z)/z for the Bessel-form contour (both even in z).
MW_HD inline void bessel_j0_j1z(cd z, cd* j0, cd* j1z) {
    if (z.re < 0.0) z = cd{-z.re, -z.im};
    if (cabs_(z) < 14.0) {
        cd y0, y1z;
        bessel_series(z, false, j0, j1z, &y0, &y1z);
        return;
    }
    cd a0, a1, b0, b1;
    hankel_asym(z, 1, &a0, &a1);
    hankel_asym(z, 2, &b0, &b1);
    *j0 = cscale(a0 + b0, 0.5);
    *j1z = cdiv(cscale(a1 + b1, 0.5), z);
}

// H^(2)_0(z) and H^(2)_1(z)/z for the Hankel-form contour, which stays
// out of the quadrant Re z < 0 < Im z (the expansion's edge at ph z = pi).
MW_HD inline void hankel2_h0_h1z(cd z, cd* h0, cd* h1z) {
    const double az = cabs_(z);
    if (az >= 30.0 || (az >= 14.0 && z.im > 0.0)) {
        cd h1;
        hankel_asym(z, 2, h0, &h1);
        *h1z = cdiv(h1, z);
        return;
    }
    if (z.im <= 0.0 && az >= 2.0) {
        cd k0, k1;
        bessel_k01_cf(mul_i(z), &k0, &k1);  // i z has Re >= 0
        *h0 = cscale(mul_i(k0), kTwoOverPi);  // (2/pi) i K0(iz)
        *h1z = cdiv(cscale(k1, -kTwoOverPi), z);  // -(2/pi) K1(iz) / z
        return;
    }
    cd j0, j1z, y0, y1z;
    bessel_series(z, true, &j0, &j1z, &y0, &y1z);
    *h0 = j0 - mul_i(y0);
    *h1z = j1z - mul_i(y1z);
}

// --------------------------------------------------------------- integrands
struct SixParams {
    cd k1;       // k2 sqrt(eps~), Im <= 0
    double k2;
    double rho, h;
    bool bessel;  // fig-13 (J0) form, else fig-14 (H0^(2)) form
};

// (lambda^2 - k^2)^(1/2) with NEC's vertical cuts:
// sqrt(-i (lambda - k)) sqrt(i (lambda + k)), principal roots.
MW_HD inline cd gamma_cut(cd lam, cd k) {
    return csqrt_p(mul_mi(lam - k)) * csqrt_p(mul_i(lam + k));
}

// The six integrands of eqs 148-153 at lambda.
MW_HD inline void integrand6(const SixParams& P, cd lam, cd out[6]) {
    const cd k1 = P.k1, k2{P.k2, 0.0};
    const cd g1 = gamma_cut(lam, k1), g2 = gamma_cut(lam, k2);
    const cd k1s = k1 * k1;
    const cd k2s{P.k2 * P.k2, 0.0};
    const cd ks = k1s + k2s;
    const cd two{2.0, 0.0};
    const cd d1 = cdiv(two, g1 + g2) - cdiv(cscale(k2s, 2.0), g2 * ks);
    const cd d2 = cdiv(two, k1s * g2 + k2s * g1) - cdiv(two, g2 * ks);
    const cd e = cexp_(cd{-(g2.re * P.h), -(g2.im * P.h)});
    const cd x = cscale(lam, P.rho);
    cd b0, b1x;
    if (P.bessel) {
        bessel_j0_j1z(x, &b0, &b1x);
    } else {
        hankel2_h0_h1z(x, &b0, &b1x);
        b0 = cscale(b0, 0.5);
        b1x = cscale(b1x, 0.5);
    }
    const cd l2 = lam * lam, l3 = l2 * lam;
    const cd c = d2 * e;
    out[0] = c * (b1x - b0) * l3;
    out[1] = c * g2 * g2 * b0 * lam;
    out[2] = c * g2 * (b1x * x) * l2;
    const cd m3 = c * b1x * l3;
    out[3] = cd{-m3.re, -m3.im};
    out[4] = c * b0 * lam;
    out[5] = d1 * e * b0 * lam;
}

// ---------------------------------------------------------------- quadrature
// A Rule integrates the six integrands over the straight segment z0 -> z1
// with the 24-point rule: rule(z0, z1, out).  The drivers below are written
// once; the host rule loops over the nodes, the device rule spreads them
// over a warp (every lane ends with the same sums, so control flow stays
// warp-uniform).
MW_HD inline double max_abs6(const cd v[6]) {
    double m = 0.0;
    for (int i = 0; i < 6; ++i) m = fmax(m, cabs_(v[i]));
    return m;
}

#pragma nv_exec_check_disable
template <class Rule>
MW_HD inline void adaptive6(const Rule& rule, cd z0, cd z1, double rtol, cd acc[6]) {
    struct Frame {
        cd z0, z1, whole[6];
        int depth;
    };
    Frame st[kAdaptDepth + 2];
    int top = 0;
    st[0].z0 = z0;
    st[0].z1 = z1;
    st[0].depth = kAdaptDepth;
    rule(z0, z1, st[0].whole);
    top = 1;
    while (top > 0) {
        Frame f = st[--top];
        const cd mid = cscale(f.z0 + f.z1, 0.5);
        cd left[6], right[6], better[6];
        rule(f.z0, mid, left);
        rule(mid, f.z1, right);
        double err = 0.0, scale = 0.0;
        for (int i = 0; i < 6; ++i) {
            better[i] = left[i] + right[i];
            err = fmax(err, cabs_(better[i] - f.whole[i]));
            scale = fmax(scale, cabs_(better[i]));
        }
        if (f.depth <= 0 || err <= rtol * fmax(scale, 1e-300)) {
            for (int i = 0; i < 6; ++i) acc[i] = acc[i] + better[i];
            continue;
        }
        // right pushed first so the left half is processed first
        Frame& r = st[top++];
        r.z0 = mid;
        r.z1 = f.z1;
        r.depth = f.depth - 1;
        for (int i = 0; i < 6; ++i) r.whole[i] = right[i];
        Frame& l = st[top++];
        l.z0 = f.z0;
        l.z1 = mid;
        l.depth = f.depth - 1;
        for (int i = 0; i < 6; ++i) l.whole[i] = left[i];
    }
}

#pragma nv_exec_check_disable
template <class Rule>
MW_HD inline void tail6(const Rule& rule, cd z0, cd dir, double panel, double rtol, double ref_scale, double panel0,
                        cd out[6]) {
    cd total[6];
    for (int i = 0; i < 6; ++i) total[i] = cd{0.0, 0.0};
    int quiet = 0;
    cd z = z0;
    double step = panel0 > 0.0 ? fmin(panel0, panel) : panel;
    for (int it = 0; it < kMaxTailPanels; ++it) {
        const cd zn = z + cscale(dir, step);
        cd c[6];
        rule(z, zn, c);
        for (int i = 0; i < 6; ++i) total[i] = total[i] + c[i];
        z = zn;
        step = fmin(2.0 * step, panel);
        const double scale = fmax(max_abs6(total), ref_scale);
        const double cmax = max_abs6(c);
        if (cmax == 0.0 || cmax < rtol * scale) {
            if (++quiet >= 2) break;
        } else {
            quiet = 0;
        }
    }
    for (int i = 0; i < 6; ++i) out[i] = total[i];
}

// The six integrals at one (rho, h), R1 > 0; out[] = (V_rr, V_zz, V_rz,
// V_r1, V, U).  eps~ == 1 gives zeros (D1 = D2 = 0 identically).
#pragma nv_exec_check_disable
template <class Rule>
MW_HD inline void six_integrals(Rule& rule, cd eps_t, double k2, double rho, double h, double rtol, cd out[6]) {
    for (int i = 0; i < 6; ++i) out[i] = cd{0.0, 0.0};
    if (eps_t.re == 1.0 && eps_t.im == 0.0) return;
    cd k1 = cscale(csqrt_p(eps_t), k2);
    if (k1.im > 0.0) k1.im = -k1.im;
    const double scale = fmax(rho, h);
    const double panel = 0.2 * kPi / scale;
    const double ak1 = cabs_(k1);
    const double kmax = fmax(ak1, k2);
    const double kcap = 1.2 * k2 + 50.0 / scale;
    const double kmax_eff = fmin(kmax, kcap);
    const double qtol = fmin(rtol, 1e-11);
    rule.P.k1 = k1;
    rule.P.k2 = k2;
    rule.P.rho = rho;
    rule.P.h = h;
    rule.P.bessel = rho < 2.0 * h;
    if (rule.P.bessel) {
        const double p = fmin(rho > 0.0 ? 1.0 / rho : INFINITY, 1.0 / h);
        const cd brk{p, p};
        const cd end_adapt{1.3 * kmax_eff + 3.0 * p, p};
        cd tot[6];
        for (int i = 0; i < 6; ++i) tot[i] = cd{0.0, 0.0};
        adaptive6(rule, cd{0.0, 0.0}, brk, qtol, tot);
        cd start = brk;
        if (end_adapt.re > brk.re) {
            cd part[6];
            for (int i = 0; i < 6; ++i) part[i] = cd{0.0, 0.0};
            adaptive6(rule, brk, end_adapt, qtol, part);
            for (int i = 0; i < 6; ++i) tot[i] = tot[i] + part[i];
            start = end_adapt;
        }
        cd tl[6];
        tail6(rule, start, cd{1.0, 0.0}, panel, rtol, max_abs6(tot), -1.0, tl);
        for (int i = 0; i < 6; ++i) out[i] = tot[i] + tl[i];
        return;
    }
    const double r1 = hypot(rho, h);
    const cd dir_r{h / r1, -rho / r1}, dir_l{-h / r1, -rho / r1};
    const cd a{0.0, -0.4 * k2}, b{0.6 * k2, 0.2 * k2}, c{1.02 * k2, 0.2 * k2};
    const bool k1_dead = k1.re * h - k1.im * rho >= 50.0;
    const double cap_d = (k1_dead || ak1 > 200.0 * k2) ? kcap : fmax(kcap, 1.01 * k1.re);
    cd d;
    if (1.01 * k1.re <= cap_d)
        d = cd{1.01 * k1.re, 0.99 * fmax(k1.im, -cap_d)};
    else
        d = cd{cap_d, 0.0};
    if (d.re < 1.1 * k2) d.re = 1.1 * k2;
    cd s1[6], s2[6], s3[6];
    for (int i = 0; i < 6; ++i) s1[i] = s2[i] = s3[i] = cd{0.0, 0.0};
    adaptive6(rule, a, b, qtol, s1);
    adaptive6(rule, b, c, qtol, s2);
    adaptive6(rule, c, d, qtol, s3);
    cd tot[6];
    for (int i = 0; i < 6; ++i) tot[i] = (s1[i] + s2[i]) + s3[i];
    const double ref = max_abs6(tot);
    const double p0 = 0.5 * kmax;
    cd tr[6], tl[6];
    tail6(rule, d, dir_r, panel, rtol, ref, p0, tr);
    tail6(rule, a, dir_l, panel, rtol, ref, p0, tl);
    for (int i = 0; i < 6; ++i) out[i] = (tot[i] + tr[i]) - tl[i];
}

// Eq 123 normalisation -j omega mu / (4 pi k2^2) of a unit current moment.
MW_HD inline cd c1_norm(double k2, double omega, double mu) { return cd{0.0, -omega * mu / (4.0 * kPi * k2 * k2)}; }

// The four surfaces (I_rho^V, I_z^V, I_rho^H, I_phi^H) at one node.
#pragma nv_exec_check_disable
template <class Rule>
MW_HD inline void surfaces(Rule& rule, cd eps_t, double k2, double omega, double mu, double r1, double rho, double h,
                           double theta, double rtol, cd out[4]) {
    const cd k1s = cscale(eps_t, k2 * k2);
    const double k2s = k2 * k2;
    const cd c1 = c1_norm(k2, omega, mu);
    if (r1 == 0.0) {
        // eqs 169-172
        const cd den = k1s + cd{k2s, 0.0};
        const cd c2 = cdiv(cd{k1s.re - k2s, k1s.im}, den);
        const cd c3 = cdiv(cscale(cd{k1s.re - k2s, k1s.im}, k2s), den * den);
        const double sn = sin(theta), co = cos(theta);
        const bool near = fabs(co) < 1e-8;
        const double q1 = near ? 0.0 : (1.0 - sn) / co;
        const double q2 = near ? 0.5 : (1.0 - sn) / (co * co);
        const cd c13k = c1 * c3 * k1s;
        out[0] = cscale(c13k, q1);
        out[1] = c13k;
        out[2] = cscale(c1, k2s) * (c2 - c3 + cscale(c3, q2));
        const cd t = cscale(c1, k2s) * (c2 - cscale(c3, q2));
        out[3] = cd{-t.re, -t.im};
        return;
    }
    cd six[6];
    six_integrals(rule, eps_t, k2, rho, h, rtol, six);
    const cd phase = cscale(cd{cos(k2 * r1), sin(k2 * r1)}, r1);
    const cd cp = c1 * phase;
    out[0] = cp * k1s * six[2];
    out[1] = cp * k1s * (six[1] + cscale(six[4], k2s));
    out[2] = cscale(cp, k2s) * (six[0] + six[5]);
    const cd t = cscale(cp, k2s) * (six[3] + six[5]);
    out[3] = cd{-t.re, -t.im};
}

// Host rule: the 24 nodes in a loop.
struct HostRule {
    SixParams P;
    const GL24* g;
    void operator()(cd z0, cd z1, cd out[6]) const {
        const cd mid = cscale(z0 + z1, 0.5), half = cscale(z1 - z0, 0.5);
        for (int i = 0; i < 6; ++i) out[i] = cd{0.0, 0.0};
        for (int n = 0; n < kGaussN; ++n) {
            cd v[6];
            integrand6(P, mid + cscale(half, g->x[n]), v);
            for (int i = 0; i < 6; ++i) out[i] = out[i] + cscale(v[i], g->w[n]);
        }
        for (int i = 0; i < 6; ++i) out[i] = out[i] * half;
    }
};

}  // namespace somm
}  // namespace mw
