// Host side of the coordination step runs (coord_run.cuh): the tile-major step
// list of a set of coordination items and the balanced per-CTA ranges.
#include <algorithm>
#include <cmath>
#include <vector>

#include "kernels.hpp"

namespace glued {

int buildCoordSteps(std::vector<CoordItem>& items, int ra, int ch, std::vector<CoordStep>& steps, int itemsPerSys) {
    const int TA = COORD_NW * ra;
    steps.clear();
    int rows = 0;
    for (size_t i = 0; i < items.size(); i++) {
        CoordItem& it = items[i];
        it.row0 = rows;
        if (it.cells) {
            it.tilesA = 0;
            rows += it.nA + it.nB;
            continue;
        }
        it.tilesA = std::max(1, (it.nA + TA - 1) / TA);
        const int nCh = std::max(1, (it.nB + ch - 1) / ch);
        for (int ta = 0; ta < it.tilesA; ta++) {
            const int nAv = std::min(TA, it.nA - ta * TA);
            for (int c = 0; c < nCh; c++) {
                CoordStep s{};
                s.item = (int)i;
                s.aStart = it.a0 + ta * TA;
                s.bStart = it.b0 + c * ch;
                s.rowA = rows + ta * TA;
                s.rowB = rows + it.nA + c * ch;
                const int nBv = std::min(ch, it.nB - c * ch);
                int fl = (c == 0 ? COORD_F_FIRST : 0) | (c == nCh - 1 ? COORD_F_LAST : 0);
                s.packed = stepPack(nAv, nBv, fl);
                s.pieceSlot = -1;
                s.sys = (int)i / std::max(1, itemsPerSys);
                steps.push_back(s);
            }
        }
        rows += it.nA + it.nB;
    }
    return rows;
}

std::vector<int> balanceRanges(int numSteps, int grid) {
    // the split the kernels compute themselves (coordRange): equal counts +-1
    std::vector<int> begin(std::max(grid, 0) + 1, 0);
    for (int b = 0; b <= grid; b++) begin[b] = grid > 0 ? coordRange(numSteps, grid, b) : 0;
    return begin;
}

int buildCoordPieces(std::vector<CoordStep>& steps, const std::vector<int>& begin, std::vector<CoordItem>& items) {
    std::vector<std::vector<int>> per(items.size());
    for (size_t b = 0; b + 1 < begin.size(); b++)
        for (int s = begin[b]; s < begin[b + 1]; s++) {
            const int fl = stepFlags(steps[s].packed);
            steps[s].pieceSlot = -1;
            if (s == begin[b + 1] - 1 || (fl & COORD_F_LAST)) per[steps[s].item].push_back(s);
        }
    int slot = 0;
    for (size_t i = 0; i < items.size(); i++) {
        std::sort(per[i].begin(), per[i].end());
        items[i].pieceBegin = slot;
        for (int s : per[i]) steps[s].pieceSlot = slot++;
        items[i].pieceEnd = slot;
    }
    return slot;
}

bool coordNeedsHi(const std::vector<CoordItem>& items, const double box[9], bool periodic) {
    if (!periodic) return true;
    // longest minimum-image distance: half of |a| + |b| + |c| bounds it
    double la = std::sqrt(box[0] * box[0] + box[1] * box[1] + box[2] * box[2]);
    double lb = std::sqrt(box[3] * box[3] + box[4] * box[4] + box[5] * box[5]);
    double lc = std::sqrt(box[6] * box[6] + box[7] * box[7] + box[8] * box[8]);
    const double dmax = 0.5 * (la + lb + lc);
    for (const CoordItem& it : items) {
        if (it.rc2 > 0.0f && (double)it.rc2 < dmax * dmax) return true;
        const double x = dmax / (double)it.r0;
        if (x * x >= 0.9e6) return true;
    }
    return false;
}

}  // namespace glued
