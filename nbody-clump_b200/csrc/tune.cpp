// tune.cpp -- choice of hierarchical-grid levels from the radius distribution.
//
// The reference sizes its single-level cells at 3 x the largest radius
// (src/dem_subsphere_io.cu:195-230), so with a wide radius distribution
// every subsphere scans cells sized for the largest one.  Its hierarchical
// grid reads the levels from a grid.bt file the user writes
// (src/dem_io.cu:204-248).  Here the levels are chosen from the radii:
// radius bands, level 0 the coarsest, cell of a level = 3 x the largest
// radius in it (so a pair's cutoff 1.5 (ri + rj) never exceeds the cell of
// the coarser partner's level).  The search work of a band choice is
// estimated as sum_t n_t sum_{l<=t} cell_l^3 n_l (a subsphere of level t
// scans 27 cells of its own and of every coarser level); for each band count
// the band edges are placed by coordinate descent over radius quantiles, and
// an extra level is taken only when it cuts the estimate by 10 %.
#include <algorithm>
#include <cmath>
#include <functional>
#include <vector>

#include "../../include/nbc.h"

namespace {

// cuts: ascending indices into the descending radii where a finer band starts
double band_cost(const std::vector<double>& r, const std::vector<int>& cuts) {
    const int n = (int)r.size();
    double S = 0, tot = 0;
    int b0 = 0;
    for (size_t k = 0; k <= cuts.size(); k++) {
        const int b1 = k < cuts.size() ? cuts[k] : n;
        if (b1 <= b0) return INFINITY;
        const double cell = 3.0 * r[b0], nk = (double)(b1 - b0);
        S += cell * cell * cell * nk;
        tot += nk * S;
        b0 = b1;
    }
    return tot;
}

}  // namespace

extern "C" int nbc_choose_levels(const double* radius, int n, int max_levels, int* level, double* level_cell) {
    if (n <= 0 || !radius) return 0;
    max_levels = std::max(1, std::min(max_levels, NBC_MAX_LEVELS));
    std::vector<double> r(radius, radius + n);
    std::sort(r.begin(), r.end(), std::greater<double>());
    // candidate cuts: radius quantiles moved onto a change of radius, so that
    // equal radii always share a band
    const int Q = 48;
    std::vector<int> cand;
    for (int q = 1; q < Q; q++) {
        int c = (int)((long long)n * q / Q);
        while (c < n && c > 0 && !(r[c] < r[c - 1])) c++;
        if (c > 0 && c < n && (cand.empty() || cand.back() != c)) cand.push_back(c);
    }
    std::vector<int> best_cuts;
    double best_cost = band_cost(r, best_cuts);
    for (int L = 2; L <= max_levels && (int)cand.size() >= L - 1; L++) {
        double bc = INFINITY;
        std::vector<int> bcut;
        // starts: L-1 evenly spaced candidates, and every shift of that pattern
        for (int s0 = 0; s0 < (int)cand.size(); s0 += std::max(1, (int)cand.size() / 8)) {
            std::vector<int> cuts;
            for (int k = 1; k < L; k++) cuts.push_back(cand[std::min((int)cand.size() - 1, (s0 + k * (int)cand.size() / L) % (int)cand.size())]);
            std::sort(cuts.begin(), cuts.end());
            cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
            if ((int)cuts.size() != L - 1) continue;
            double c = band_cost(r, cuts);
            for (bool improved = true; improved;) {
                improved = false;
                for (int k = 0; k < L - 1; k++)
                    for (int q : cand) {
                        std::vector<int> t = cuts;
                        t[k] = q;
                        std::sort(t.begin(), t.end());
                        if (std::adjacent_find(t.begin(), t.end()) != t.end()) continue;
                        const double ct = band_cost(r, t);
                        if (ct < c) { c = ct; cuts = t; improved = true; }
                    }
            }
            if (c < bc) { bc = c; bcut = cuts; }
        }
        if (bc < 0.9 * best_cost) {  // an extra level must earn 10 %
            best_cost = bc;
            best_cuts = bcut;
        }
    }
    const int L = (int)best_cuts.size() + 1;
    if (level)
        for (int i = 0; i < n; i++) {
            int l = 0;
            for (int c : best_cuts) l += radius[i] <= r[c];
            level[i] = l;
        }
    if (level_cell) {
        level_cell[0] = 3.0 * r[0];
        for (int k = 0; k < L - 1; k++) level_cell[k + 1] = 3.0 * r[best_cuts[k]];
    }
    return L;
}
