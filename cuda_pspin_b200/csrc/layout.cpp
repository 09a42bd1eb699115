// layout.cpp -- host construction of the sweep's per-site lists and of the
// FP64 quartet table, from one sample's active (quartet, channel) list.
//
// Channel classes (disorder.h:9-16) for sorted i<j<k<l:
//   ch 0: unconjugated {i,j}, conjugated {k,l}
//   ch 1: unconjugated {i,l}, conjugated {j,k}
//   ch 2: unconjugated {i,k}, conjugated {j,l}
// Member m of a quartet has a partner p (the other site of m's class) and
// an opposite pair {o1<o2}.  Site m's list holds, for every quartet of m,
// the record (p, o1, o2, g).  Records are sorted by (p, o1, o2); each run of
// equal (p, o1) is stored as a header {len, p<<16 | o1} followed by len data
// entries {g as float bits, o2}, with runs cut at kGroupMax entries.  The
// list is cut in 32 balanced parts and each part packed in TMA chunks.
#include "layout.h"

#include <algorithm>
#include <cstring>

namespace pspin {

static inline void class_of(const int q[4], int ch, int m_pos, int& partner, int& o1, int& o2) {
    // positions of the unconjugated pair for each channel
    static const int U[3][2] = {{0, 1}, {0, 3}, {0, 2}};
    static const int C[3][2] = {{2, 3}, {1, 2}, {1, 3}};
    const int* mine;
    const int* opp;
    if (m_pos == U[ch][0] || m_pos == U[ch][1]) { mine = U[ch]; opp = C[ch]; }
    else { mine = C[ch]; opp = U[ch]; }
    partner = q[mine[0] == m_pos ? mine[1] : mine[0]];
    const int a = q[opp[0]], b = q[opp[1]];
    o1 = a < b ? a : b;
    o2 = a < b ? b : a;
}

struct Rec {
    int32_t key;   // p<<16 | o1
    int32_t o2;
    float g;
};

void build_site_lists(int N, const double* g2re, int h2_active, const std::vector<QuartetRec>& qs,
                      SiteLists& out) {
    std::vector<std::vector<Rec>> per(N);
    std::vector<int64_t> cnt(N, 0);
    for (const QuartetRec& r : qs) { cnt[r.i]++; cnt[r.j]++; cnt[r.k]++; cnt[r.l]++; }
    for (int m = 0; m < N; m++) per[m].reserve(cnt[m] + (h2_active ? N : 0));
    for (const QuartetRec& r : qs) {
        const int q[4] = {r.i, r.j, r.k, r.l};
        const float g = (float)r.g;
        for (int pos = 0; pos < 4; pos++) {
            int p, o1, o2;
            class_of(q, r.ch, pos, p, o1, o2);
            per[q[pos]].push_back(Rec{(p << 16) | o1, o2, g});
        }
    }
    if (h2_active) {
        // 2-body field h2_m = sum_{j != m} g_mj conj(a_j): partner and first
        // opposite site are the virtual unit site N
        for (int m = 0; m < N; m++)
            for (int j = 0; j < N; j++) {
                if (j == m) continue;
                const double g = g2re[(size_t)m * N + j];
                if (g != 0.0) per[m].push_back(Rec{(N << 16) | N, j, (float)g});
            }
    }
    out.entries.clear();
    out.chunk_start.clear();
    out.site_chunks.assign((size_t)N * (kSplit + 1), 0);
    std::vector<std::pair<int64_t, int64_t>> groups;   // [begin, end) in a site-local list
    std::vector<int2> site;
    for (int m = 0; m < N; m++) {
        std::vector<Rec>& v = per[m];
        std::sort(v.begin(), v.end(), [](const Rec& a, const Rec& b) {
            return a.key != b.key ? a.key < b.key : a.o2 < b.o2;
        });
        // groups of equal (p, o1), cut at kGroupMax data entries
        site.clear();
        groups.clear();
        size_t t = 0;
        while (t < v.size()) {
            size_t e = t;
            while (e < v.size() && v[e].key == v[t].key && (int)(e - t) < kGroupMax) e++;
            const int64_t gb = (int64_t)site.size();
            site.push_back(make_int2((int)(e - t), v[t].key));
            for (size_t u = t; u < e; u++) {
                int bits;
                std::memcpy(&bits, &v[u].g, sizeof(int));
                site.push_back(make_int2(bits, v[u].o2));
            }
            groups.push_back({gb, (int64_t)site.size()});
            t = e;
        }
        // 32 parts of nearly equal size, cut at group starts
        const int64_t total = (int64_t)site.size();
        std::vector<size_t> part_first(kSplit + 1, groups.size());
        part_first[0] = 0;
        size_t g = 0;
        for (int part = 1; part < kSplit; part++) {
            const int64_t target = (total * part) / kSplit;
            while (g < groups.size() && groups[g].first < target) g++;
            part_first[part] = g;
        }
        // every part packed in chunks of whole groups, <= kStage entries,
        // padded with an empty group to an even length (16-byte granules)
        int* sc = &out.site_chunks[(size_t)m * (kSplit + 1)];
        for (int part = 0; part < kSplit; part++) {
            sc[part] = (int)out.chunk_start.size();
            size_t gi = part_first[part];
            const size_t ge = std::max(part_first[part], part_first[part + 1]);
            while (gi < ge) {
                const int64_t cb = (int64_t)out.entries.size();
                out.chunk_start.push_back(cb);
                int64_t len = 0;
                while (gi < ge) {
                    const int64_t gl = groups[gi].second - groups[gi].first;
                    if (len > 0 && len + gl + 1 > kStage) break;
                    out.entries.insert(out.entries.end(), site.begin() + groups[gi].first,
                                       site.begin() + groups[gi].second);
                    len += gl;
                    gi++;
                }
                if (len & 1) out.entries.push_back(make_int2(0, 0));
            }
        }
        sc[kSplit] = (int)out.chunk_start.size();
    }
}

void build_q64(const std::vector<QuartetRec>& qs, std::vector<Q64>& out) {
    out.resize(qs.size());
    for (size_t t = 0; t < qs.size(); t++) {
        const QuartetRec& r = qs[t];
        out[t].i = (uint16_t)r.i;
        out[t].j = (uint16_t)r.j;
        out[t].k = (uint16_t)r.k;
        out[t].lch = (uint16_t)(r.l | (r.ch << 14));
        out[t].g = r.g;
    }
}

void dense_quartets(int N, const double* g4re, const uint8_t* mask, std::vector<QuartetRec>& out) {
    out.clear();
    int64_t q = 0;
    for (int l = 3; l < N; l++)
        for (int k = 2; k < l; k++)
            for (int j = 1; j < k; j++)
                for (int i = 0; i < j; i++, q++) {
                    const uint8_t m = mask[q];
                    const double g = g4re[q];
                    if (m == 0 || g == 0.0) continue;       // mc.cu:249
                    for (int ch = 0; ch < 3; ch++)
                        if (m & (1 << ch)) out.push_back(QuartetRec{i, j, k, l, ch, g});
                }
}

}  // namespace pspin
