// compact_host.h -- the lockstep engine's compact layout of a square CSR pattern, computed on the
// host once per pattern (setup_host.cpp); batch.cu uploads it.  Internal header (not installed).
#pragma once

#include <vector>

namespace femd {

constexpr int CL_TILE = 32;    // rows per slice (and per tile of the column-window bounds)
constexpr int CL_SORT = 256;   // rows per window of the sort by row length

// The reverse Cuthill-McKee order of a square pattern, order[new] = old.
void rcm_order(int n, const std::vector<int> &ip, const std::vector<int> &ix, std::vector<int> &order);

// The RCM order with the rows of every CL_SORT sorted by length, longest first (iperm: original
// row -> reordered row); the entries in slices of CL_TILE reordered rows, column-major and padded
// to the slice's longest row: entry j of reordered row k at rstart[k] + CL_TILE j (rstart[n] =
// nsell, the slots with padding); off[slot] = the entry's reordered column minus k (0 in the
// padding); dst[q] = the slot of original entry q; per slice the smallest and largest column
// (tlo, thi; the row indices themselves included).  ok = false when the layout does not apply:
// a column offset over 32767 (bw is then the bandwidth) or more slots than an int indexes.
struct CompactLayout {
    std::vector<int> iperm, rstart, dst, tlo, thi;
    std::vector<short> off;
    long long nsell = 0;
    int bw = 0;
    bool ok = false;
};

void compact_layout(int n, const std::vector<int> &ip, const std::vector<int> &ix, CompactLayout &L);

}  // namespace femd
