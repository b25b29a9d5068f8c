// tune.cpp -- choice of hierarchical-grid levels from the radius distribution.
//
// The reference sizes its single-level cells at 3 x the largest radius
// (src/dem_subsphere_io.cu:195-230), so with a wide radius distribution
// every subsphere scans cells sized for the largest one.  Its hierarchical
// grid reads the levels from a grid.bt file the user writes
// (src/dem_io.cu:204-248).  Here the levels are chosen from the radii:
// geometric radius bands, level 0 the coarsest, cell of a level = 3 x the
// largest radius in it (so a pair's cutoff 1.5 (ri + rj) never exceeds the
// cell of the coarser partner's level), and the band count that minimises
// the estimated search work sum_t n_t sum_{l<=t} cell_l^3 n_l (a subsphere
// of level t scans 27 cells of its own and of every coarser level).
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/nbc.h"

extern "C" int nbc_choose_levels(const double* radius, int n, int max_levels, int* level, double* level_cell) {
    if (n <= 0 || !radius) return 0;
    if (max_levels < 1) max_levels = 1;
    if (max_levels > 4) max_levels = 4;
    double rmin = radius[0], rmax = radius[0];
    for (int i = 1; i < n; i++) {
        rmin = std::min(rmin, radius[i]);
        rmax = std::max(rmax, radius[i]);
    }
    int best_L = 1;
    double best_cost = 0;
    std::vector<int> best_lv(n, 0);
    std::vector<double> best_cell(1, 3.0 * rmax);
    for (int L = 1; L <= max_levels; L++) {
        std::vector<double> edge(L + 1);
        for (int k = 0; k <= L; k++) edge[k] = rmax * std::pow(rmin / rmax, (double)k / L);
        std::vector<int> lv(n);
        std::vector<long long> cnt(L, 0);
        std::vector<double> rmx(L, 0.0);
        for (int i = 0; i < n; i++) {
            int b = 0;
            while (b < L - 1 && radius[i] <= edge[b + 1]) b++;
            lv[i] = b;
            cnt[b]++;
            rmx[b] = std::max(rmx[b], radius[i]);
        }
        // drop empty bands, renumbering so level 0 stays the coarsest
        std::vector<int> remap(L, -1);
        std::vector<double> cell;
        std::vector<long long> c2;
        for (int b = 0; b < L; b++)
            if (cnt[b] > 0) {
                remap[b] = (int)cell.size();
                cell.push_back(3.0 * rmx[b]);
                c2.push_back(cnt[b]);
            }
        for (int i = 0; i < n; i++) lv[i] = remap[lv[i]];
        double cost = 0;
        for (size_t t = 0; t < cell.size(); t++) {
            double vol = 0;
            for (size_t l = 0; l <= t; l++) vol += cell[l] * cell[l] * cell[l] * (double)c2[l];
            cost += (double)c2[t] * vol;
        }
        if (L == 1 || cost < 0.9 * best_cost) {  // extra levels must earn 10 %
            best_cost = cost;
            best_L = (int)cell.size();
            best_lv = lv;
            best_cell = cell;
        }
    }
    if (level)
        for (int i = 0; i < n; i++) level[i] = best_lv[i];
    if (level_cell)
        for (int l = 0; l < best_L; l++) level_cell[l] = best_cell[l];
    return best_L;
}
