// Host-side forest of one unit-square block with p4est semantics:
// leaves kept in Morton (z-) order, neighbour relations found by point
// location (binary search over Morton keys), refinement with ForestClaw's
// smooth-refine target levels, family coarsening and 2:1 balance across
// faces and corners (P4EST_CONNECT_FULL, the balance fclaw2d_domain_new_unitsquare
// asks of p4est_wrap).
//
// References: src/forestclaw2d.c (level iteration :224-294, face neighbours
// :443-541, corner neighbours :986-1112, mark refine/coarsen :1400-1450,
// iterate_families :267-294, iterate_adapted :1453-1507) and
// src/fclaw2d_convenience.c:498-680 (fclaw2d_domain_adapt).
#pragma once
#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <vector>

namespace fcb {

enum Rel : int { REL_BOUNDARY = 0, REL_HALFSIZE = 1, REL_SAMESIZE = 2, REL_DOUBLESIZE = 3 };

struct Leaf {
    uint64_t key;  // Morton key of the lower-left corner at the finest resolution
    int32_t x, y;  // lower-left corner, units of 2^-kMaxLevel
    int32_t level;
};

struct Neighbors {
    int face_rel[4];
    int face_nbr[4][2];
    int face_pos[4];
    int corner_rel[4];  // 0 = no corner neighbour (boundary or hanging node)
    int corner_nbr[4];
    // periodic domains: the neighbour adjacent to this leaf is the stored leaf
    // moved by img * (block width) in x and y (0 unless a periodic side is crossed)
    int face_img[4][2];
    int corner_img[4][2];
    int has_fine;       // fclaw2d_patch_has_finegrid_neighbors
    int on_cf;          // fclaw2d_patch_on_coarsefine_interface
};

class QuadForest {
  public:
    static constexpr int kMaxLevel = 28;
    static constexpr int32_t kRoot = (int32_t)1 << kMaxLevel;
    std::vector<Leaf> leaves;
    // a periodic brick (p4est brick connectivity with periodic_i / periodic_j):
    // points across a periodic side wrap to the opposite side
    bool periodic_x = false, periodic_y = false;

    static int32_t width(int level) { return (int32_t)1 << (kMaxLevel - level); }
    // bit b of v (b < 32) to bit 2b
    static uint64_t spread(uint32_t v) {
        uint64_t k = v;
        k = (k | (k << 16)) & 0x0000FFFF0000FFFFull;
        k = (k | (k << 8)) & 0x00FF00FF00FF00FFull;
        k = (k | (k << 4)) & 0x0F0F0F0F0F0F0F0Full;
        k = (k | (k << 2)) & 0x3333333333333333ull;
        k = (k | (k << 1)) & 0x5555555555555555ull;
        return k;
    }
    // z-order key of the low kMaxLevel bits: x in the even bits, y in the odd
    static uint64_t morton(int32_t x, int32_t y) {
        constexpr uint32_t mask = ((uint32_t)1 << kMaxLevel) - 1;
        return spread((uint32_t)x & mask) | (spread((uint32_t)y & mask) << 1);
    }
    static Leaf make(int level, int32_t x, int32_t y) { return Leaf{morton(x, y), x, y, level}; }

    void uniform(int level) {
        leaves.clear();
        const int n = 1 << level;
        const int32_t h = width(level);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) leaves.push_back(make(level, i * h, j * h));
        sort();
    }
    void sort() {
        std::sort(leaves.begin(), leaves.end(), [](const Leaf& a, const Leaf& b) { return a.key < b.key; });
    }
    // Wrap a point across the periodic sides (img: -1 / +1 per direction it
    // wrapped); false if it lies outside a non-periodic side.
    bool wrap(int32_t& x, int32_t& y, int* img = nullptr) const {
        int ix = 0, iy = 0;
        if (x < 0 || x >= kRoot) {
            if (!periodic_x) return false;
            ix = x < 0 ? -1 : 1;
            x -= ix * kRoot;
        }
        if (y < 0 || y >= kRoot) {
            if (!periodic_y) return false;
            iy = y < 0 ? -1 : 1;
            y -= iy * kRoot;
        }
        if (img) { img[0] = ix; img[1] = iy; }
        return true;
    }
    // Leaf containing finest-resolution point (x, y) (wrapped on periodic
    // sides), or -1 outside the block.
    int locate(int32_t x, int32_t y, int* img = nullptr) const {
        if (!wrap(x, y, img)) return -1;
        const uint64_t k = morton(x, y);
        auto it = std::upper_bound(leaves.begin(), leaves.end(), k,
                                   [](uint64_t v, const Leaf& l) { return v < l.key; });
        if (it == leaves.begin()) throw std::runtime_error("forest: point not covered");
        const int p = (int)(it - leaves.begin()) - 1;
        const Leaf& l = leaves[p];
        const int32_t h = width(l.level);
        if (x < l.x || y < l.y || x >= l.x + h || y >= l.y + h) throw std::runtime_error("forest: not a partition");
        return p;
    }
    int min_level() const {
        int m = kMaxLevel;
        for (auto& l : leaves) m = std::min(m, (int)l.level);
        return m;
    }
    int max_level() const {
        int m = 0;
        for (auto& l : leaves) m = std::max(m, (int)l.level);
        return m;
    }
    bool is_first_sibling(int p) const {
        if (p + 4 > (int)leaves.size()) return false;
        const Leaf& a = leaves[p];
        if (a.level == 0) return false;
        const int32_t h = width(a.level);
        if ((a.x % (2 * h)) != 0 || (a.y % (2 * h)) != 0) return false;
        for (int k = 1; k < 4; ++k) {
            const Leaf& b = leaves[p + k];
            if (b.level != a.level || b.x != a.x + (k & 1) * h || b.y != a.y + (k >> 1) * h) return false;
        }
        return true;
    }

    Neighbors neighbors(int p) const {
        Neighbors n{};
        const Leaf& l = leaves[p];
        const int32_t h = width(l.level);
        for (int f = 0; f < 4; ++f) {
            n.face_nbr[f][0] = n.face_nbr[f][1] = -1;
            n.face_pos[f] = -1;
            n.face_img[f][0] = n.face_img[f][1] = 0;
            // a point just across the face, at the face's low end
            int32_t px = l.x, py = l.y;
            if (f == 0) px = l.x - 1;
            else if (f == 1) px = l.x + h;
            else if (f == 2) py = l.y - 1;
            else py = l.y + h;
            const int a = locate(px, py, n.face_img[f]);
            if (a < 0) { n.face_rel[f] = REL_BOUNDARY; continue; }
            const int la = leaves[a].level;
            if (la == l.level) { n.face_rel[f] = REL_SAMESIZE; n.face_nbr[f][0] = a; }
            else if (la == l.level - 1) {
                n.face_rel[f] = REL_DOUBLESIZE;
                n.face_nbr[f][0] = a;
                n.face_pos[f] = (f < 2) ? (l.y - leaves[a].y) / h : (l.x - leaves[a].x) / h;
            } else if (la == l.level + 1) {
                n.face_rel[f] = REL_HALFSIZE;
                n.face_nbr[f][0] = a;
                const int b = (f < 2) ? locate(px, py + h / 2) : locate(px + h / 2, py);
                if (b < 0 || leaves[b].level != l.level + 1) throw std::runtime_error("forest: unbalanced face");
                n.face_nbr[f][1] = b;
            } else {
                throw std::runtime_error("forest: unbalanced face");
            }
        }
        for (int c = 0; c < 4; ++c) {
            n.corner_rel[c] = 0;
            n.corner_nbr[c] = -1;
            n.corner_img[c][0] = n.corner_img[c][1] = 0;
            const int sx = (c & 1) ? 1 : -1, sy = (c & 2) ? 1 : -1;
            const int32_t X = l.x + ((c & 1) ? h : 0), Y = l.y + ((c & 2) ? h : 0);
            const int a = locate(sx > 0 ? X : X - 1, sy > 0 ? Y : Y - 1, n.corner_img[c]);
            if (a < 0) continue;
            const Leaf& d = leaves[a];
            if (d.level == l.level) { n.corner_rel[c] = REL_SAMESIZE; n.corner_nbr[c] = a; }
            else if (d.level == l.level + 1) { n.corner_rel[c] = REL_HALFSIZE; n.corner_nbr[c] = a; }
            else if (d.level == l.level - 1) {
                const int32_t hd = width(d.level);
                // the neighbour's image adjacent to this leaf
                const int32_t dx0 = d.x + n.corner_img[c][0] * kRoot, dy0 = d.y + n.corner_img[c][1] * kRoot;
                const bool corner = (X == dx0 || X == dx0 + hd) && (Y == dy0 || Y == dy0 + hd);
                if (corner) { n.corner_rel[c] = REL_DOUBLESIZE; n.corner_nbr[c] = a; }
                // otherwise a hanging node: no corner neighbour
            } else {
                throw std::runtime_error("forest: unbalanced corner");
            }
        }
        n.has_fine = 0;
        n.on_cf = 0;
        for (int f = 0; f < 4; ++f)
            if (n.face_rel[f] == REL_HALFSIZE || n.face_rel[f] == REL_DOUBLESIZE) {
                n.on_cf = 1;
                if (n.face_rel[f] == REL_HALFSIZE) n.has_fine = 1;
            }
        for (int c = 0; c < 4; ++c)
            if (n.corner_rel[c] == REL_HALFSIZE || n.corner_rel[c] == REL_DOUBLESIZE) {
                n.on_cf = 1;
                if (n.corner_rel[c] == REL_HALFSIZE) n.has_fine = 1;
            }
        return n;
    }

    // Split every leaf whose face or corner neighbour region is covered by a
    // leaf more than one level coarser, until none is (the unique coarsest
    // 2:1-balanced refinement).
    void balance() {
        for (;;) {
            std::vector<char> split(leaves.size(), 0);
            bool any = false;
            for (size_t p = 0; p < leaves.size(); ++p) {
                const Leaf& l = leaves[p];
                const int32_t h = width(l.level);
                for (int dj = -1; dj <= 1; ++dj)
                    for (int di = -1; di <= 1; ++di) {
                        if (!di && !dj) continue;
                        const int32_t px = di < 0 ? l.x - 1 : (di > 0 ? l.x + h : l.x);
                        const int32_t py = dj < 0 ? l.y - 1 : (dj > 0 ? l.y + h : l.y);
                        const int a = locate(px, py);
                        if (a >= 0 && leaves[a].level < l.level - 1) { split[a] = 1; any = true; }
                    }
            }
            if (!any) return;
            std::vector<Leaf> nl;
            nl.reserve(leaves.size() + 3 * leaves.size() / 4);
            for (size_t p = 0; p < leaves.size(); ++p) {
                const Leaf& l = leaves[p];
                if (!split[p]) { nl.push_back(l); continue; }
                const int32_t hh = width(l.level + 1);
                for (int k = 0; k < 4; ++k) nl.push_back(make(l.level + 1, l.x + (k & 1) * hh, l.y + (k >> 1) * hh));
            }
            leaves.swap(nl);  // children replace their parent in place: order stays Morton
        }
    }
};

}  // namespace fcb
