// Host-side fill tiling: the greedy split of the basis list into runs of
// consecutive bases whose wings touch at most max_seg distinct segments
// (the tiles the fill kernel stages in shared memory).  Plain C++ on the
// host; no device work.
#include <algorithm>
#include <thread>
#include <vector>

#include "common.cuh"

extern "C" mw_status mw_build_tiles(const int32_t* supp, int64_t n_b, int32_t wings, int32_t max_basis,
                                    int32_t max_seg, int32_t* first, int32_t* nb, int32_t* ns, int32_t* seg,
                                    int32_t* loc, int64_t* n_tile) {
    MW_REQUIRE(n_b >= 0 && wings >= 1 && wings <= 8, "bad basis sizes");
    MW_REQUIRE(max_basis >= 1 && max_seg >= 1 && max_seg <= 64, "bad tile limits");
    MW_REQUIRE(n_tile != nullptr, "NULL argument");
    *n_tile = 0;
    if (n_b == 0) return MW_OK;
    MW_REQUIRE(supp && first && nb && ns && seg && loc, "NULL argument");
    int32_t cur[64];
    int64_t t = 0, m = 0;
    while (m < n_b) {
        int nc = 0, cnt = 0;
        while (m + cnt < n_b && cnt < max_basis) {
            // distinct new segments of basis m + cnt
            int32_t add[8];
            int na = 0;
            const int32_t* row = supp + (m + cnt) * wings;
            for (int a = 0; a < wings; ++a) {
                const int32_t sg = row[a];
                if (sg < 0) continue;
                bool seen = false;
                for (int i = 0; i < nc && !seen; ++i) seen = cur[i] == sg;
                for (int i = 0; i < na && !seen; ++i) seen = add[i] == sg;
                if (!seen) add[na++] = sg;
            }
            if (nc + na > max_seg) break;
            for (int i = 0; i < na; ++i) cur[nc++] = add[i];
            ++cnt;
        }
        MW_REQUIRE(cnt > 0, "basis %lld touches more segments than a tile holds", (long long)m);
        // sorted segment list of the tile (insertion sort, <= 64 entries)
        for (int i = 1; i < nc; ++i) {
            const int32_t v = cur[i];
            int j = i - 1;
            while (j >= 0 && cur[j] > v) {
                cur[j + 1] = cur[j];
                --j;
            }
            cur[j + 1] = v;
        }
        first[t] = (int32_t)m;
        nb[t] = cnt;
        ns[t] = nc;
        int32_t* srow = seg + t * max_seg;
        for (int i = 0; i < max_seg; ++i) srow[i] = i < nc ? cur[i] : -1;
        for (int64_t b = m; b < m + cnt; ++b)
            for (int a = 0; a < wings; ++a) {
                const int32_t sg = supp[b * wings + a];
                int32_t l = -1;
                if (sg >= 0)
                    for (int i = 0; i < nc; ++i)
                        if (cur[i] == sg) {
                            l = i;
                            break;
                        }
                loc[b * wings + a] = l;
            }
        ++t;
        m += cnt;
    }
    *n_tile = t;
    return MW_OK;
}

// Host-side basis polynomials: for every kept basis b (local index js[b] on
// wire bw[b]) and wing a, the segment it covers and the monomial
// coefficients of the basis on that segment in the local arc length u:
// values of the d+1 B-splines active on the segment's knot span at d+1
// uniform points (Cox-de Boor on the clamped knot vector), then the inverse
// of the Vandermonde matrix of those points.  garc holds every wire's knot
// arc positions back to back (wire w at arc_off[w], wire_n[w] + 1 values).
extern "C" mw_status mw_basis_polys(const double* garc, const int64_t* arc_off, const int64_t* wire_n,
                                    const int64_t* wire_first, int64_t n_wires, int32_t degree, const int64_t* js,
                                    const int64_t* bw, int64_t m, int32_t* supp, double* poly) {
    MW_REQUIRE(degree == 1 || degree == 2, "degree must be 1 or 2 (got %d)", degree);
    MW_REQUIRE(n_wires >= 0 && m >= 0, "sizes must be >= 0");
    if (m == 0) return MW_OK;
    MW_REQUIRE(garc && arc_off && wire_n && wire_first && js && bw && supp && poly, "NULL argument");
    const int d = degree, NM = d + 1;
    // inverse of U[i][p] = (i/d)^p
    static const double kUinv1[2][2] = {{1.0, 0.0}, {-1.0, 1.0}};
    static const double kUinv2[3][3] = {{1.0, 0.0, 0.0}, {-3.0, 4.0, -1.0}, {2.0, -4.0, 2.0}};
    for (int64_t b = 0; b < m; ++b)
        MW_REQUIRE(bw[b] >= 0 && bw[b] < n_wires, "basis %lld: wire out of range", (long long)b);
    // every basis is independent: contiguous chunks on host threads for
    // large structures (the same arithmetic per basis, so the same bits)
    auto one = [&](int64_t b) {
        const int64_t w = bw[b], j = js[b];
        const int64_t nw = wire_n[w], off = arc_off[w];
        const double* arc = garc + off;
        const int64_t lo = j - d > 0 ? j - d : 0, hi = nw < j + 1 ? nw : j + 1;
        for (int a = 0; a < NM; ++a) {
            const int64_t s = lo + a;
            int32_t* sp = supp + b * NM + a;
            double* pc = poly + (b * NM + a) * NM;
            if (s >= hi) {
                *sp = -1;
                for (int p = 0; p < NM; ++p) pc[p] = 0.0;
                continue;
            }
            *sp = (int32_t)(wire_first[w] + s);
            const int c = (int)(j - s);  // active index of basis j on span s
            // knots of spans s+1-d .. s+d: arc positions clip(s+t, 0, n_w)
            double K[4];
            for (int t = 1 - d; t <= d; ++t) {
                int64_t q = s + t;
                q = q < 0 ? 0 : (q > nw ? nw : q);
                K[t - 1 + d] = arc[q];
            }
            const double a0 = arc[s], h = arc[s + 1] - a0;
            double vals[3];  // basis c at the d+1 sample points
            for (int i = 0; i < NM; ++i) {
                const double x = a0 + h * (d == 1 ? (double)i : 0.5 * i);
                double N[3] = {1.0, 0.0, 0.0}, left[3] = {0, 0, 0}, right[3] = {0, 0, 0};
                for (int jj = 1; jj <= d; ++jj) {
                    left[jj] = x - K[(1 - jj) - 1 + d];  // knot at span + 1 - jj
                    right[jj] = K[jj - 1 + d] - x;       // knot at span + jj
                    double saved = 0.0;
                    for (int r = 0; r < jj; ++r) {
                        const double tmp = N[r] / (right[r + 1] + left[jj - r]);
                        N[r] = saved + right[r + 1] * tmp;
                        saved = left[jj - r] * tmp;
                    }
                    N[jj] = saved;
                }
                vals[i] = N[c];
            }
            double hp = 1.0;
            for (int p = 0; p < NM; ++p) {
                double acc = 0.0;
                for (int i = 0; i < NM; ++i) acc += (d == 1 ? kUinv1[p][i] : kUinv2[p][i]) * vals[i];
                pc[p] = acc / hp;
                hp *= h;
            }
        }
    };
    const unsigned hw = std::thread::hardware_concurrency();
    const int64_t nt = std::min<int64_t>(std::min<int64_t>(hw ? hw : 1, 8), m / 1024);
    if (nt <= 1) {
        for (int64_t b = 0; b < m; ++b) one(b);
    } else {
        std::vector<std::thread> pool;
        const int64_t chunk = (m + nt - 1) / nt;
        for (int64_t t = 0; t < nt; ++t)
            pool.emplace_back([&, t] {
                const int64_t b1 = std::min(m, (t + 1) * chunk);
                for (int64_t b = t * chunk; b < b1; ++b) one(b);
            });
        for (auto& th : pool) th.join();
    }
    return MW_OK;
}
