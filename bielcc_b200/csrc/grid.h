// grid.h — host-side choice of the cell-split count of a (tiles x splits)
// grid whose CTAs each sweep one split of the cells for one tile of points.
#pragma once
#include <algorithm>
#include <cstddef>
#include <functional>
#include <queue>
#include <vector>

namespace bielcc_gpu {

// Cells per split rounded up to a multiple of 32 (one near-mask word).
inline int round_cells_per_split(int n_cells, int splits) {
    int cps = (n_cells + splits - 1) / splits;
    return (cps + 31) / 32 * 32;
}

// Slot utilisation of a (tiles x splits) grid on `slots` resident CTAs.
// CTAs start in block order (tiles fastest) and run for a time proportional
// to their cell count, so the grid is full waves of full-split CTAs, then a
// tail: the remaining full-split CTAs and the CTAs of the last, shorter split,
// each taking the earliest free slot.
inline double split_grid_utilisation(int tiles, int splits, int cps, int n_cells, int slots) {
    const long long full = (long long)tiles * (splits - 1);
    const long long fw = full / slots, r = full % slots;
    const long long t0 = fw * cps, last = n_cells - (long long)(splits - 1) * cps;
    // slots free at t0 (slots - r of them) and at t0 + cps (r of them)
    std::priority_queue<long long, std::vector<long long>, std::greater<long long>> q;
    for (long long i = 0; i < slots; i++) q.push(i < r ? t0 + cps : t0);
    long long end = r ? t0 + cps : t0;
    for (int t = 0; t < tiles; t++) {
        const long long f = q.top() + last;
        q.pop();
        q.push(f);
        end = std::max(end, f);
    }
    return (double)tiles * n_cells / ((double)slots * (double)end);
}

// Split count: at least one full wave of CTAs, at most eight waves, at least
// 32 cells per split and at most max_splits; the count with the highest slot
// utilisation wins (the fewest splits within 0.5 %).
inline int choose_cell_splits(int tiles, int n_cells, int slots, int max_splits) {
    if (tiles <= 0 || n_cells <= 32) return 1;
    const int cap = std::max(1, std::min(n_cells / 32, max_splits));
    const int lo = std::min(cap, std::max(1, (slots + tiles - 1) / tiles));
    const int hi = std::min(cap, 8 * lo);
    int best = 0;
    double best_u = -1.0;
    for (int s = lo; s <= hi; s++) {
        const int cps = round_cells_per_split(n_cells, s);
        if ((n_cells + cps - 1) / cps != s) continue;  // the same grid as a smaller count
        const double u = split_grid_utilisation(tiles, s, cps, n_cells, slots);
        if (u > best_u + 0.005) {
            best_u = u;
            best = s;
        }
    }
    if (best > 0) return best;
    const int cps = round_cells_per_split(n_cells, lo);
    return (n_cells + cps - 1) / cps;
}

}  // namespace bielcc_gpu
