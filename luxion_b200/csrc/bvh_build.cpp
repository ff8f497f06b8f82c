// bvh_build.cpp -- host builder: binned-SAH binary tree collapsed into compressed 8-wide nodes.
//
// Binary stage: top-down, 32 bins per axis over the centroid bounds of the node, cost
// SA(L)*nL + SA(R)*nR (the reference uses 16 bins and 1 + nL/n*SA(L) + nR/n*SA(R),
// src/mesh/bvh_build.cu:12,167-169 -- the constant and scale do not change the argmin; its
// 15% median fallback, :278-294, is replaced by an object-median split when binning cannot
// separate the centroids). Leaves hold one primitive.
// Collapse stage: each 8-wide node takes its binary node's two children and repeatedly opens
// the child of largest surface area until 8 slots are used; subtrees of at most
// kMaxLeafPrims primitives become leaf slots. Slots are assigned by child-centroid octant, boxes are
// quantised outward.

#include "bvh8.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <deque>

namespace lux {
namespace {

struct Box {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    double area() const {
        double d[3];
        for (int a = 0; a < 3; ++a) d[a] = std::max(0.0, double(hi[a]) - double(lo[a]));
        return 2.0 * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
};

struct BNode {
    Box box;
    int left = -1, right = -1;  // binary children (-1 for a leaf)
    int begin = 0, count = 0;   // primitive range in the order array
};

struct Binary {
    std::vector<BNode> nodes;
    std::vector<uint32_t> order;
};

constexpr int kBins = 32;

// One primitive of the binary build: its box, its centroid and its index, kept in a packed
// array that is partitioned in place, so every pass over a node's range reads memory in order.
struct PrimRec {
    float lo[3], hi[3], c[3];
    uint32_t id;
};

int bin_of(float c, float lo, double k1) {
    int b = int((double(c) - lo) * k1);
    return std::min(kBins - 1, std::max(0, b));
}

void build_binary(const float* boxes, int n, Binary& B) {
    B.nodes.clear();
    B.order.resize(n);
    std::vector<PrimRec> rec(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) {
        PrimRec& r = rec[size_t(i)];
        for (int a = 0; a < 3; ++a) {
            r.lo[a] = boxes[size_t(i) * 6 + a];
            r.hi[a] = boxes[size_t(i) * 6 + 3 + a];
            r.c[a] = 0.5f * (r.lo[a] + r.hi[a]);
        }
        r.id = uint32_t(i);
    }
    B.nodes.reserve(size_t(2 * n));
    B.nodes.push_back(BNode());
    B.nodes[0].begin = 0;
    B.nodes[0].count = n;
    std::vector<int> work{0};
    while (!work.empty()) {
        int ni = work.back();
        work.pop_back();
        BNode nd = B.nodes[ni];
        PrimRec* r0 = rec.data() + nd.begin;
        PrimRec* r1 = r0 + nd.count;
        Box cb;
        for (const PrimRec* r = r0; r < r1; ++r) {
            for (int a = 0; a < 3; ++a) {
                nd.box.lo[a] = std::min(nd.box.lo[a], r->lo[a]);
                nd.box.hi[a] = std::max(nd.box.hi[a], r->hi[a]);
            }
            cb.grow(r->c);
        }
        if (nd.count <= 1) {
            B.nodes[ni] = nd;
            continue;
        }
        if (nd.count == 2) {
            // Two primitives land in the first and last bins of every axis their centroids
            // span, every such split costs the same, and the first axis wins: the smaller
            // centroid on it goes left. Coincident centroids split the range in half.
            for (int a = 0; a < 3; ++a) {
                if (!(double(cb.hi[a]) - double(cb.lo[a]) > 0.0)) continue;
                if (r0[1].c[a] < r0[0].c[a]) std::swap(r0[0], r0[1]);
                break;
            }
            int l = int(B.nodes.size());
            B.nodes.push_back(BNode());
            B.nodes.push_back(BNode());
            nd.left = l;
            nd.right = l + 1;
            B.nodes[l].begin = nd.begin;
            B.nodes[l].count = 1;
            B.nodes[l + 1].begin = nd.begin + 1;
            B.nodes[l + 1].count = 1;
            B.nodes[ni] = nd;
            work.push_back(l);
            work.push_back(l + 1);
            continue;
        }
        // Bin all three axes in one pass; an axis whose centroids coincide takes no part. A bin's
        // box is written on its first primitive, and only non-empty bins enter the sweep: a run of
        // empty bins leaves both sides of a split unchanged, so the split after the last non-empty
        // bin on the left is the lowest-index one of equal cost.
        bool live[3];
        double k1[3];
        for (int a = 0; a < 3; ++a) {
            double ext = double(cb.hi[a]) - double(cb.lo[a]);
            live[a] = ext > 0.0;
            k1[a] = live[a] ? kBins / ext : 0.0;
        }
        struct BinBox {
            float lo[3], hi[3];
        };
        BinBox bb[3][kBins];
        int bc[3][kBins] = {};
        for (const PrimRec* r = r0; r < r1; ++r) {
            for (int a = 0; a < 3; ++a) {
                if (!live[a]) continue;
                int b = bin_of(r->c[a], cb.lo[a], k1[a]);
                BinBox& x = bb[a][b];
                if (bc[a][b]++ == 0) {
                    for (int d = 0; d < 3; ++d) {
                        x.lo[d] = r->lo[d];
                        x.hi[d] = r->hi[d];
                    }
                } else {
                    for (int d = 0; d < 3; ++d) {
                        x.lo[d] = std::min(x.lo[d], r->lo[d]);
                        x.hi[d] = std::max(x.hi[d], r->hi[d]);
                    }
                }
            }
        }
        int best_axis = -1, best_split = -1;
        double best_cost = DBL_MAX;
        for (int a = 0; a < 3; ++a) {
            if (!live[a]) continue;
            int nb = 0, idx[kBins];
            for (int b = 0; b < kBins; ++b)
                if (bc[a][b] != 0) idx[nb++] = b;
            double ra[kBins];
            int rc[kBins];
            Box acc;
            int cnt = 0;
            for (int j = nb - 1; j > 0; --j) {
                const BinBox& x = bb[a][idx[j]];
                acc.grow(x.lo);
                acc.grow(x.hi);
                cnt += bc[a][idx[j]];
                ra[j] = acc.area();
                rc[j] = cnt;
            }
            Box lacc;
            int lcnt = 0;
            for (int j = 0; j < nb - 1; ++j) {
                const BinBox& x = bb[a][idx[j]];
                lacc.grow(x.lo);
                lacc.grow(x.hi);
                lcnt += bc[a][idx[j]];
                double c = lacc.area() * lcnt + ra[j + 1] * rc[j + 1];
                if (c < best_cost) {
                    best_cost = c;
                    best_axis = a;
                    best_split = idx[j];
                }
            }
        }
        int mid;
        if (best_axis >= 0) {
            const int a = best_axis;
            const float lo = cb.lo[a];
            const double k = k1[a];
            // stable, so the order inside each side (which the two-primitive and coincident-centroid
            // cases below depend on) is the input order: the device build reproduces it exactly
            PrimRec* it = std::stable_partition(r0, r1, [&](const PrimRec& r) { return bin_of(r.c[a], lo, k) <= best_split; });
            mid = nd.begin + int(it - r0);
        } else {
            mid = nd.begin + nd.count / 2;  // coincident centroids: split the range in half
        }
        if (mid <= nd.begin || mid >= nd.begin + nd.count) mid = nd.begin + nd.count / 2;
        int l = int(B.nodes.size());
        B.nodes.push_back(BNode());
        B.nodes.push_back(BNode());
        nd.left = l;
        nd.right = l + 1;
        B.nodes[l].begin = nd.begin;
        B.nodes[l].count = mid - nd.begin;
        B.nodes[l + 1].begin = mid;
        B.nodes[l + 1].count = nd.begin + nd.count - mid;
        B.nodes[ni] = nd;
        work.push_back(l);
        work.push_back(l + 1);
    }
    for (int i = 0; i < n; ++i) B.order[size_t(i)] = rec[size_t(i)].id;
}

// ceil(log2(x)) for x > 0, exactly: x = m * 2^k with m in [0.5, 1) (frexp is exact), and
// log2(x) is k - 1 when m is 0.5, else strictly between k - 1 and k.
int ceil_log2(double x) {
    int k = 0;
    const double m = std::frexp(x, &k);
    return m == 0.5 ? k - 1 : k;
}

// Quantise the child boxes of one 8-wide node. The node box is first widened by a relative
// 1e-4 of its largest extent (plus 1e-7 of its coordinate magnitude), at least 1.27 % of a
// quantisation step on every axis, and every child plane is rounded outward by a further 1 %
// of a step. Either margin dominates the rounding error of the device slab test: at most
// 2^-9 of a step beyond a relative 2^-17 of the plane distance, which the device widens.
void encode_node(BVH8Node& N, const Box& nb, const Box* cbox, const bool* used) {
    double mext = 0.0, mabs = 0.0;
    for (int a = 0; a < 3; ++a) {
        mext = std::max(mext, double(nb.hi[a]) - double(nb.lo[a]));
        mabs = std::max(mabs, std::max(std::fabs(double(nb.lo[a])), std::fabs(double(nb.hi[a]))));
    }
    const double pad = 1e-4 * mext + 1e-7 * mabs + 1e-30;
    double hi_d[3];
    for (int a = 0; a < 3; ++a) {
        double lo_d = double(nb.lo[a]) - pad;
        hi_d[a] = double(nb.hi[a]) + pad;
        float pf = float(lo_d);
        if (double(pf) > lo_d) pf = std::nextafter(pf, -FLT_MAX);
        N.p[a] = pf;
    }
    for (int a = 0; a < 3; ++a) {
        double ext = hi_d[a] - double(N.p[a]);
        int e = -126;
        if (ext > 0.0) e = ceil_log2(ext / 255.0);
        e = std::max(-126, std::min(127, e));
        // make sure 255 steps cover the extent after the exponent rounding
        while (std::ldexp(255.0, e) < ext && e < 127) ++e;
        N.e[a] = uint8_t(e + 127);
    }
    uint8_t* qlo[3] = {N.qlox, N.qloy, N.qloz};
    uint8_t* qhi[3] = {N.qhix, N.qhiy, N.qhiz};
    for (int s = 0; s < 8; ++s) {
        for (int a = 0; a < 3; ++a) {
            if (!used[s]) {
                qlo[a][s] = 0xff;
                qhi[a][s] = 0x00;
                continue;
            }
            double scale = std::ldexp(1.0, int(N.e[a]) - 127);
            double lo = std::floor((double(cbox[s].lo[a]) - double(N.p[a])) / scale - 0.01);
            double hi = std::ceil((double(cbox[s].hi[a]) - double(N.p[a])) / scale + 0.01);
            qlo[a][s] = uint8_t(std::max(0.0, std::min(255.0, lo)));
            qhi[a][s] = uint8_t(std::max(0.0, std::min(255.0, hi)));
        }
    }
}

}  // namespace

void build_bvh8(const float* boxes, int n, BVH8Build& out) {
    out.nodes.clear();
    out.prim_order.clear();
    out.depth = 0;
    out.sah_cost = 0.0;
    if (n <= 0) return;
    Binary B;
    build_binary(boxes, n, B);
    struct Item {
        int bnode;
        int out_index;
        int level;
    };
    std::deque<Item> q;
    out.nodes.push_back(BVH8Node());
    q.push_back({0, 0, 1});
    const double root_area = std::max(1e-30, B.nodes[0].box.area());
    while (!q.empty()) {
        Item it = q.front();
        q.pop_front();
        out.depth = std::max(out.depth, it.level);
        const BNode& bn = B.nodes[it.bnode];
        // gather up to 8 children
        int ch[8];
        int nch = 0;
        if (bn.left < 0 || bn.count <= kMaxLeafPrims) {
            ch[nch++] = it.bnode;  // the whole node is one leaf slot
        } else {
            ch[nch++] = bn.left;
            ch[nch++] = bn.right;
            while (nch < 8) {
                int pick = -1;
                double pa = -1.0;
                for (int k = 0; k < nch; ++k) {
                    const BNode& c = B.nodes[ch[k]];
                    if (c.left < 0 || c.count <= kMaxLeafPrims) continue;
                    double a = c.box.area();
                    if (a > pa) {
                        pa = a;
                        pick = k;
                    }
                }
                if (pick < 0) break;
                int c = ch[pick];
                ch[pick] = B.nodes[c].left;
                ch[nch++] = B.nodes[c].right;
            }
        }
        // Slot assignment by centroid octant around the node centre: child c in slot s costs
        // the centroid offset projected on the octant's direction; pairs are taken cheapest
        // first (ties by child, then slot), skipping a pair whose child or slot is taken.
        float ctr[3];
        for (int a = 0; a < 3; ++a) ctr[a] = 0.5f * (bn.box.lo[a] + bn.box.hi[a]);
        int slot_of[8];
        bool slot_used[8] = {false};
        {
            double cost[8][8];
            for (int k = 0; k < nch; ++k) {
                const Box& b = B.nodes[ch[k]].box;
                double d[3];
                for (int a = 0; a < 3; ++a) d[a] = 0.5 * (double(b.lo[a]) + double(b.hi[a])) - ctr[a];
                for (int s = 0; s < 8; ++s) {
                    double c = 0;
                    for (int a = 0; a < 3; ++a) c += ((s >> a) & 1) ? -d[a] : d[a];
                    cost[k][s] = c;
                }
            }
            bool cdone[8] = {false};
            for (int round = 0; round < nch; ++round) {
                int bc = -1, bs = -1;
                double bcost = 0.0;
                for (int k = 0; k < nch; ++k) {
                    if (cdone[k]) continue;
                    for (int s = 0; s < 8; ++s) {
                        if (slot_used[s]) continue;
                        if (bc < 0 || cost[k][s] < bcost) {
                            bcost = cost[k][s];
                            bc = k;
                            bs = s;
                        }
                    }
                }
                cdone[bc] = true;
                slot_used[bs] = true;
                slot_of[bc] = bs;
            }
        }
        BVH8Node N;
        std::memset(&N, 0, sizeof(N));
        Box cbox[8];
        int child_at_slot[8];
        for (int s = 0; s < 8; ++s) child_at_slot[s] = -1;
        for (int k = 0; k < nch; ++k) {
            child_at_slot[slot_of[k]] = ch[k];
            cbox[slot_of[k]] = B.nodes[ch[k]].box;
        }
        encode_node(N, bn.box, cbox, slot_used);
        N.child_base = uint32_t(out.nodes.size());
        N.tri_base = uint32_t(out.prim_order.size());
        for (int s = 0; s < 8; ++s) {
            int c = child_at_slot[s];
            if (c < 0) continue;
            const BNode& cn = B.nodes[c];
            out.sah_cost += cn.box.area() / root_area;
            if (cn.left < 0 || cn.count <= kMaxLeafPrims) {
                // one record per leaf slot, in slot order: the record is the slot's rank
                for (int k = cn.begin; k < cn.begin + cn.count; ++k) out.prim_order.push_back(B.order[k]);
                N.meta[0] = uint8_t(N.meta[0] | (1u << s));
            } else {
                N.imask |= uint8_t(1u << s);
                out.nodes.push_back(BVH8Node());
                q.push_back({c, int(out.nodes.size()) - 1, it.level + 1});
            }
        }
        out.nodes[it.out_index] = N;
    }
}

}  // namespace lux
