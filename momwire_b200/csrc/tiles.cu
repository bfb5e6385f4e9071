// Host-side fill tiling: the greedy split of the basis list into runs of
// consecutive bases whose wings touch at most max_seg distinct segments
// (the tiles the fill kernel stages in shared memory).  Plain C++ on the
// host; no device work.
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
