// Sommerfeld remainder field: interpolation of the four surfaces on an
// (R1, theta) grid and the eqs 143-147 projection (sm_100a device code shared
// by the grid and surrogate remainder kernels).  Restates proj_one of the
// reference (_accelerators.cpp:5906-5963; _sommerfeld.py:831-875, 940-1035).
#pragma once

#include "common.cuh"

namespace mw {

struct GridDev {
    int n_region;
    int n_r[6], n_th[6];
    int64_t off[6];
    double r0[6], dr[6], th0[6], dth[6];
    double r1_max, r_break, th_split, r_near, tiny, vscale;
    const double2* vals;  // (nodes, 4) complex
};

__device__ __forceinline__ void lagrange4(double u, double w[4]) {
    const double u0 = u, u1 = u - 1.0, u2 = u - 2.0, u3 = u - 3.0;
    w[0] = -u1 * u2 * u3 / 6.0;
    w[1] = u0 * u2 * u3 / 2.0;
    w[2] = -u0 * u1 * u3 / 2.0;
    w[3] = u0 * u1 * u2 / 6.0;
}

// Source tangent split into horizontal unit (ux, uy), horizontal magnitude
// and vertical part (_sommerfeld.py:985-990).
struct SrcTangent {
    double ux, uy, th, tz;
};
__host__ __device__ __forceinline__ SrcTangent split_tangent(double tx, double ty, double tz) {
    SrcTangent s;
    s.th = hypot(tx, ty);
    const bool safe = s.th > 1e-12;
    s.ux = safe ? tx / s.th : 1.0;
    s.uy = safe ? ty / s.th : 0.0;
    s.tz = tz;
    return s;
}

// Image-geometry coordinates of an (observer, source) point pair.
struct PairGeom {
    double dx, dy, rho, hh, r1, theta;
};

__device__ __forceinline__ PairGeom pair_geom(double gz, double ox, double oy, double oz, double sx, double sy,
                                              double sz) {
    PairGeom p;
    p.dx = ox - sx;
    p.dy = oy - sy;
    p.rho = hypot(p.dx, p.dy);
    p.hh = (oz - gz) + (sz - gz);
    p.r1 = sqrt(p.rho * p.rho + p.hh * p.hh);
    const double th = atan2(p.hh, p.rho);
    p.theta = fmin(fmax(th, 0.0), 0.5 * kPi);
    return p;
}

// 4x4 Lagrange interpolation of the four surfaces at (r1, theta).
__device__ __forceinline__ void grid_surfaces(const GridDev& G, double r1, double theta, cd surf[4]) {
    const double r1c = fmin(r1, G.r1_max);
    const int reg = (r1c <= G.r_break) ? (theta <= G.th_split ? 0 : 1)
                                       : (r1c <= G.r_near ? (theta <= G.th_split ? 2 : 3)
                                                          : (theta <= G.th_split ? 4 : 5));
    const double fr = (r1c - G.r0[reg]) / G.dr[reg];
    const double ft = (theta - G.th0[reg]) / G.dth[reg];
    int i0 = (int)floor(fr) - 1, j0 = (int)floor(ft) - 1;
    i0 = min(max(i0, 0), G.n_r[reg] - 4);
    j0 = min(max(j0, 0), G.n_th[reg] - 4);
    double wr[4], wt[4];
    lagrange4(fr - i0, wr);
    lagrange4(ft - j0, wt);
    const double2* V = G.vals + (G.off[reg] + (int64_t)i0 * G.n_th[reg] + j0) * 4;
#pragma unroll
    for (int s = 0; s < 4; ++s) surf[s] = cd{0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double2* row = V + (int64_t)i * G.n_th[reg] * 4;
        cd rs[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) rs[s] = cd{0.0, 0.0};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const double2 v = __ldg(row + j * 4 + s);
                rs[s].re += v.x * wt[j];
                rs[s].im += v.y * wt[j];
            }
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            surf[s].re += rs[s].re * wr[i];
            surf[s].im += rs[s].im * wr[i];
        }
    }
}

// t_obs . F . t_src from the surfaces (eqs 143-147); vscale multiplies the
// surfaces, tiny is the rho below which the azimuth degenerates.
__device__ __forceinline__ cd project_surfaces(const PairGeom& p, const cd surf[4], double k, double vscale,
                                               double tiny, double tox, double toy, double toz,
                                               const SrcTangent& ts) {
    double sn, cs;
    sincos(k * p.r1, &sn, &cs);
    const double ir = vscale / p.r1;
    const cd g{cs * ir, -sn * ir};
    const bool safe_r = p.rho > tiny;
    const double inv_rho = safe_r ? 1.0 / p.rho : 0.0;
    const double dhx = safe_r ? p.dx * inv_rho : ts.ux;
    const double dhy = safe_r ? p.dy * inv_rho : ts.uy;
    const double cphi = ts.ux * dhx + ts.uy * dhy;
    const double sphi = ts.ux * dhy - ts.uy * dhx;
    const cd e_rho = g * cd{ts.tz * surf[0].re + ts.th * cphi * surf[2].re, ts.tz * surf[0].im + ts.th * cphi * surf[2].im};
    const cd e_phi = g * cd{ts.th * sphi * surf[3].re, ts.th * sphi * surf[3].im};
    const cd e_z = g * cd{ts.tz * surf[1].re - ts.th * cphi * surf[0].re, ts.tz * surf[1].im - ts.th * cphi * surf[0].im};
    const double ax = tox * dhx + toy * dhy, ay = toy * dhx - tox * dhy;
    return cd{ax * e_rho.re + ay * e_phi.re + toz * e_z.re, ax * e_rho.im + ay * e_phi.im + toz * e_z.im};
}

// t_obs . F(obs, src) . t_src: interpolation, then projection.
__device__ __forceinline__ cd proj_one(const GridDev& G, double gz, double k, double ox, double oy, double oz,
                                       double tox, double toy, double toz, double sx, double sy, double sz,
                                       const SrcTangent& ts) {
    const PairGeom p = pair_geom(gz, ox, oy, oz, sx, sy, sz);
    cd surf[4];
    grid_surfaces(G, p.r1, p.theta, surf);
    return project_surfaces(p, surf, k, G.vscale, G.tiny, tox, toy, toz, ts);
}

}  // namespace mw
