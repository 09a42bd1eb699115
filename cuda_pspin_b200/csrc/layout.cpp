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

// Cuts one site's records (groups or tiles, [begin, end) in int2 units of
// `site`) into kSplit/stride pieces of nearly equal size, piece q in part
// q*stride (the other parts empty), and packs every part in TMA chunks of
// whole records, <= kStage entries, padded to an even length.  stride 1 for
// site lists; short lists use a larger stride so that a warp fetches one
// chunk rather than several tiny ones (a warp owns kSplit/W consecutive
// parts for any W dividing kSplit).
static void pack_site(const std::vector<int2>& site, const std::vector<std::pair<int64_t, int64_t>>& groups, int m,
                      SiteLists& out, int stride = 1) {
    const int64_t total = (int64_t)site.size();
    const int pieces = kSplit / stride;
    std::vector<size_t> bound(pieces + 1, groups.size());
    bound[0] = 0;
    size_t g = 0;
    for (int q = 1; q < pieces; q++) {
        const int64_t target = (total * q) / pieces;
        while (g < groups.size() && groups[g].first < target) g++;
        bound[q] = g;
    }
    std::vector<size_t> part_first(kSplit + 1, groups.size());
    for (int part = 0; part < kSplit; part++)
        part_first[part] = (part % stride == 0) ? bound[part / stride] : bound[part / stride + 1];
    int* sc = &out.site_chunks[(size_t)m * (kSplit + 1)];
    for (int part = 0; part < kSplit; part++) {
        sc[part] = (int)out.chunk_start.size();
        size_t gi = part_first[part];
        const size_t ge = std::max(part_first[part], part_first[part + 1]);
        while (gi < ge) {
            out.chunk_start.push_back((int64_t)out.entries.size());
            int64_t len = 0;
            while (gi < ge) {
                const int64_t gl = groups[gi].second - groups[gi].first;
                if (len > 0 && len + gl + 1 > kStage) break;
                out.entries.insert(out.entries.end(), site.begin() + groups[gi].first, site.begin() + groups[gi].second);
                len += gl;
                gi++;
            }
            if (len & 1) out.entries.push_back(make_int2(0, 0));
        }
    }
    sc[kSplit] = (int)out.chunk_start.size();
}

// Sorts one list's records by (p, o1, o2), cuts groups of equal (p, o1) at
// kGroupMax data entries and packs them as list `id`: as a header and data
// entries, or (records) as one 16-byte record {g, o2, p<<16|o1, last} per
// data entry, `last` marking the group's final record.
static void group_and_pack(std::vector<Rec>& v, int id, std::vector<int2>& site,
                           std::vector<std::pair<int64_t, int64_t>>& groups, SiteLists& out, int stride = 1,
                           bool records = false) {
    std::sort(v.begin(), v.end(), [](const Rec& a, const Rec& b) {
        return a.key != b.key ? a.key < b.key : a.o2 < b.o2;
    });
    site.clear();
    groups.clear();
    size_t t = 0;
    while (t < v.size()) {
        size_t e = t;
        while (e < v.size() && v[e].key == v[t].key && (int)(e - t) < kGroupMax) e++;
        const int64_t gb = (int64_t)site.size();
        if (!records) site.push_back(make_int2((int)(e - t), v[t].key));
        for (size_t u = t; u < e; u++) {
            int bits;
            std::memcpy(&bits, &v[u].g, sizeof(int));
            site.push_back(make_int2(bits, v[u].o2));
            if (records) site.push_back(make_int2(v[t].key, u + 1 == e ? 1 : 0));
        }
        groups.push_back({gb, (int64_t)site.size()});
        t = e;
    }
    pack_site(site, groups, id, out, stride);
}

void build_pair_lists(int N, const double* g2re, int h2_active, const std::vector<QuartetRec>& qs,
                      SiteLists& out) {
    const int npairs = N * (N - 1) / 2;
    auto list_id = [](int m, int x) {   // m's terms that contain x
        return m < x ? 2 * (x * (x - 1) / 2 + m) : 2 * (m * (m - 1) / 2 + x) + 1;
    };
    std::vector<std::vector<Rec>> per((size_t)2 * npairs);
    for (const QuartetRec& r : qs) {
        const int q[4] = {r.i, r.j, r.k, r.l};
        const float g = (float)r.g;
        for (int pos = 0; pos < 4; pos++) {
            int p, o1, o2;
            class_of(q, r.ch, pos, p, o1, o2);
            const Rec rec{(p << 16) | o1, o2, g};
            per[list_id(q[pos], p)].push_back(rec);
            per[list_id(q[pos], o1)].push_back(rec);
            per[list_id(q[pos], o2)].push_back(rec);
        }
    }
    if (h2_active)
        for (int m = 0; m < N; m++)
            for (int j = 0; j < N; j++) {
                if (j == m) continue;
                const double g = g2re[(size_t)m * N + j];
                if (g != 0.0) per[list_id(m, j)].push_back(Rec{(N << 16) | N, j, (float)g});
            }
    out.entries.clear();
    out.chunk_start.clear();
    out.site_chunks.assign((size_t)2 * npairs * (kSplit + 1), 0);
    std::vector<std::pair<int64_t, int64_t>> groups;
    std::vector<int2> site;
    for (int id = 0; id < 2 * npairs; id++) {
        group_and_pack(per[id], id, site, groups, out, 4);      // 8 pieces: one chunk per warp at 8 warps
        std::vector<Rec>().swap(per[id]);
    }
}

void build_site_lists(int N, const double* g2re, int h2_active, const std::vector<QuartetRec>& qs,
                      SiteLists& out, bool records) {
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
    for (int m = 0; m < N; m++) group_and_pack(per[m], m, site, groups, out, 1, records);
}

static inline int64_t encode_sorted(int a, int b, int c, int d) {
    int v[4] = {a, b, c, d};
    std::sort(v, v + 4);
    return (int64_t)v[3] * (v[3] - 1) * (v[3] - 2) * (v[3] - 3) / 24 + (int64_t)v[2] * (v[2] - 1) * (v[2] - 2) / 6 +
           (int64_t)v[1] * (v[1] - 1) / 2 + v[0];
}

static inline int fbits(float f) {
    int b;
    std::memcpy(&b, &f, sizeof(int));
    return b;
}

void build_site_tiles_fc(int N, const double* g2re, int h2_active, const double* g4re, SiteLists& out) {
    out.entries.clear();
    out.chunk_start.clear();
    out.site_chunks.assign((size_t)N * (kSplit + 1), 0);
    std::vector<int2> site;
    std::vector<std::pair<int64_t, int64_t>> tiles;
    std::vector<int> partners;
    for (int m = 0; m < N; m++) {
        site.clear();
        tiles.clear();
        // one tile: header + (hi-lo) rows of 4 couplings; coef(k, t) for partner k, inner t
        auto emit = [&](int outer, int lo, int hi, const int* p, auto coef) {
            const int64_t b = (int64_t)site.size();
            site.push_back(make_int2(outer | (lo << 16), hi));
            site.push_back(make_int2(p[0] | (p[1] << 16), p[2] | (p[3] << 16)));
            for (int t = lo; t < hi; t++) {
                site.push_back(make_int2(fbits(coef(0, t)), fbits(coef(1, t))));
                site.push_back(make_int2(fbits(coef(2, t)), fbits(coef(3, t))));
            }
            tiles.push_back({b, (int64_t)site.size()});
        };
        if (h2_active) {
            const int pv[4] = {N, N, N, N};
            for (int lo = 0; lo < N; lo += kGroupMax) {
                const int hi = std::min(N, lo + kGroupMax);
                emit(N, lo, hi, pv, [&](int k, int t) {
                    return (k == 0 && t != m) ? (float)g2re[(size_t)m * N + t] : 0.0f;
                });
            }
        }
        // m among the two smallest: outer o1 > m, partners p < o1, inner o2 in (o1, N)
        // m among the two largest: outer o2 < m, partners p > o2, inner o1 in [0, o2)
        for (int side = 0; side < 2; side++) {
            const int o_begin = side == 0 ? m + 1 : 0, o_end = side == 0 ? N : m;
            for (int outer = o_begin; outer < o_end; outer++) {
                const int ilo = side == 0 ? outer + 1 : 0, ihi = side == 0 ? N : outer;
                if (ilo >= ihi) continue;
                partners.clear();
                if (side == 0) { for (int p = 0; p < outer; p++) if (p != m) partners.push_back(p); }
                else { for (int p = outer + 1; p < N; p++) if (p != m) partners.push_back(p); }
                for (size_t pb = 0; pb < partners.size(); pb += 4) {
                    int pv[4];
                    bool real[4];
                    for (int k = 0; k < 4; k++) {
                        real[k] = pb + k < partners.size();
                        pv[k] = real[k] ? partners[pb + k] : N;
                    }
                    for (int lo = ilo; lo < ihi; lo += kGroupMax) {
                        const int hi = std::min(ihi, lo + kGroupMax);
                        emit(outer, lo, hi, pv, [&](int k, int t) {
                            return real[k] ? (float)g4re[encode_sorted(m, pv[k], outer, t)] : 0.0f;
                        });
                    }
                }
            }
        }
        pack_site(site, tiles, m, out);
    }
}

// Per record, per replica: the group format costs 14 operations per header
// (a_p conj(a_o1): 2 FMA + 2 MUL; the field update: 4 FMA) and 4 per data
// entry (2 FMA); a fully connected tile costs 56 per header (4 partners x 14)
// and 16 per row (8 FMA: 4 couplings times one gathered amplitude).
double list_exec_flops(const SiteLists& L, int N, bool tiles, bool records) {
    double total = 0.0;
    const int64_t nchunks = (int64_t)L.chunk_start.size();
    for (int m = 0; m < N; m++) {
        const int c0 = L.site_chunks[(size_t)m * (kSplit + 1)];
        const int c1 = L.site_chunks[(size_t)m * (kSplit + 1) + kSplit];
        for (int c = c0; c < c1; c++) {
            const int64_t b = L.chunk_start[c];
            const int64_t e = (c + 1 < nchunks) ? L.chunk_start[c + 1] : (int64_t)L.entries.size();
            const int2* R = L.entries.data() + b;
            const int64_t n = e - b;
            if (tiles) {
                for (int64_t u = 0; u < n / 2;) {
                    const int lo = R[2 * u].x >> 16, hi = R[2 * u].y;
                    total += 56.0 + 16.0 * (hi - lo);
                    u += 1 + (hi - lo);
                }
            } else if (records) {
                for (int64_t u = 0; u + 1 < n; u += 2) total += 4.0 + (R[u + 1].y ? 14.0 : 0.0);
            } else {
                for (int64_t u = 0; u < n;) {
                    const int len = R[u].x;
                    total += 14.0 + 4.0 * len;
                    u += len + 1;
                }
            }
        }
    }
    return total;
}

bool records_single_groups(const SiteLists& L) {
    for (size_t u = 0; u + 1 < L.entries.size(); u += 2)
        if (L.entries[u + 1].y != 1) return false;
    return true;
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
