// layout.h -- host builders for the sweep's site lists and the FP64 quartet table.
#pragma once
#include <vector>
#include <cstdint>
#include "internal.h"

namespace pspin {

struct QuartetRec {
    int i, j, k, l;   // sorted
    int ch;           // 0, 1, 2
    double g;         // rescaled coupling (real)
};

struct SiteLists {
    std::vector<int2> entries;         // sample-relative
    std::vector<int64_t> chunk_start;  // sample-relative entry offset of each chunk (no sentinel)
    std::vector<int> site_chunks;      // N*(kSplit+1) sample-relative chunk indices
};

// Per-site lists in the group format, or (records) as 16-byte records
// {g, o2, p<<16|o1, last}: the same groups, one record per data entry, so a
// record's position never depends on an earlier header and the loads of
// consecutive records overlap; the sweep kernels read site lists this way.
void build_site_lists(int N, const double* g2re, int h2_active, const std::vector<QuartetRec>& qs,
                      SiteLists& out, bool records = false);
// Sub-lists of the terms that couple the two sites of a pair (same group
// format): for i < j and P = j(j-1)/2 + i, list 2P holds site i's terms that
// contain a_j, list 2P+1 site j's terms that contain a_i.  Each term of a
// site list is in 3 of them (one per other site of its quartet).
void build_pair_lists(int N, const double* g2re, int h2_active, const std::vector<QuartetRec>& qs,
                      SiteLists& out);
// fully connected tiles from the dense g4 (channel 0 everywhere) and g2
void build_site_tiles_fc(int N, const double* g2re, int h2_active, const double* g4re, SiteLists& out);
void build_q64(const std::vector<QuartetRec>& qs, std::vector<Q64>& out);
// site lists in the record format: does every record end its group?
bool records_single_groups(const SiteLists& L);

// FP32 operations the sweep kernels execute, per replica, to accumulate the
// lists of all N sites once (the expected work of one sweep's N/2 moves over
// their two sites each), walking the packed chunks exactly as
// accumulate_chunk / accumulate_records / accumulate_tiles do (padding
// words included).
double list_exec_flops(const SiteLists& L, int N, bool tiles, bool records = false);
// every active (q, ch) of a dense mask in q order
void dense_quartets(int N, const double* g4re, const uint8_t* mask, std::vector<QuartetRec>& out);

}  // namespace pspin
