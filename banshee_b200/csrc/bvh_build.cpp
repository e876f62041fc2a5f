// Binned-SAH builder + collapse to 4-wide nodes (see bvh_build.h).
//
// Determinism: each binary subtree with m triangles owns the node-index range
// [base, base + 2m - 1), so parallel recursion produces the same tree as the
// serial one, and the wide tree is emitted in a fixed depth-first order.
#include "bvh_build.h"
#include "qnode.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <thread>

namespace bg {
namespace {

struct Box {
    float lo[3], hi[3];
    void clear() {
        for (int k = 0; k < 3; ++k) { lo[k] = FLT_MAX; hi[k] = -FLT_MAX; }
    }
    void grow(const float* l, const float* h) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], l[k]); hi[k] = std::max(hi[k], h[k]); }
    }
    void grow(const Box& b) { grow(b.lo, b.hi); }
    void grow_pt(const float* p) { grow(p, p); }
    float area() const {
        float e0 = hi[0] - lo[0], e1 = hi[1] - lo[1], e2 = hi[2] - lo[2];
        if (e0 < 0 || e1 < 0 || e2 < 0) return 0.f;
        return 2.f * (e0 * e1 + e0 * e2 + e1 * e2);
    }
};

struct BNode {
    Box box;
    int32_t left = -1, right = -1;   // binary children (node indices)
    int32_t start = 0, count = 0;    // count > 0: leaf
};

struct Bin {
    Box box, cbox;
    int32_t count;
};

class Builder {
public:
    Builder(const float* lo, const float* hi, int64_t n, const BuildParams& p)
        : n_(n), p_(p), tlo_(3 * n), thi_(3 * n), cen_(3 * n), idx_(n), nodes_(2 * n) {
        for (int64_t i = 0; i < n; ++i) {
            bool ok = true;
            for (int k = 0; k < 3; ++k) ok = ok && std::isfinite(lo[3 * i + k]) && std::isfinite(hi[3 * i + k]);
            for (int k = 0; k < 3; ++k) {
                tlo_[3 * i + k] = ok ? lo[3 * i + k] : 0.f;
                thi_[3 * i + k] = ok ? hi[3 * i + k] : 0.f;
                cen_[3 * i + k] = 0.5f * (tlo_[3 * i + k] + thi_[3 * i + k]);
            }
            idx_[i] = int32_t(i);
        }
        int hw = p.threads > 0 ? p.threads : int(std::thread::hardware_concurrency());
        spare_threads_ = std::max(0, std::min(hw, 64) - 1);
    }

    void run() {
        Box box, cbox;
        box.clear(); cbox.clear();
        for (int64_t i = 0; i < n_; ++i) { box.grow(&tlo_[3 * i], &thi_[3 * i]); cbox.grow_pt(&cen_[3 * i]); }
        build(0, 0, n_, box, cbox);
    }

    BuildResult collapse() {
        BuildResult r;
        r.order = idx_;
        if (p_.wide4) {
            r.nodes.reserve(size_t(n_ / 2 + 16));
            if (nodes_[0].count > 0) {           // whole scene is one leaf
                WideNode4 w = empty_node();
                set_child(w, 0, nodes_[0]);
                w.child[0] = encode_leaf(nodes_[0].start, nodes_[0].count);
                r.nodes.push_back(w);
                r.max_depth = 1; r.max_stack = 1; r.nleaves = 1;
            } else {
                emit(r, 0, 1, 0);
            }
        }
        if (p_.wide8) {
            r.nodes8.reserve(size_t(n_ / 6 + 16));
            if (nodes_[0].count > 0) {
                int32_t kids[1] = {0};
                r.nodes8.push_back(QNode8{});
                int32_t code = encode_leaf(nodes_[0].start, nodes_[0].count);
                if (!fill_qnode(r.nodes8[0], kids, &code, 1)) q8_failed_ = true;
                r.max_depth8 = 1; r.max_stack8 = 1;
            } else {
                emit8(r, 0, 1, 0);
                run_q8_jobs(r);
            }
        }
        return r;
    }

private:
    static WideNode4 empty_node() {
        WideNode4 w;
        for (int i = 0; i < 4; ++i) {
            w.lox[i] = w.loy[i] = w.loz[i] = FLT_MAX;
            w.hix[i] = w.hiy[i] = w.hiz[i] = -FLT_MAX;
            w.child[i] = kEmptyChild;
            w.pad[i] = 0;
        }
        return w;
    }
    static void set_child(WideNode4& w, int i, const BNode& b) {
        w.lox[i] = b.box.lo[0]; w.hix[i] = b.box.hi[0];
        w.loy[i] = b.box.lo[1]; w.hiy[i] = b.box.hi[1];
        w.loz[i] = b.box.lo[2]; w.hiz[i] = b.box.hi[2];
    }

    int emit(BuildResult& r, int32_t b, int depth, int stack_acc) {
        int32_t kids[4] = {nodes_[b].left, nodes_[b].right, -1, -1};
        int nk = 2;
        while (nk < 4) {
            int best = -1;
            float ba = -1.f;
            for (int i = 0; i < nk; ++i) {
                const BNode& c = nodes_[kids[i]];
                if (c.count == 0 && c.box.area() > ba) { ba = c.box.area(); best = i; }
            }
            if (best < 0) break;
            int32_t l = nodes_[kids[best]].left, rr = nodes_[kids[best]].right;
            kids[best] = l;
            kids[nk++] = rr;
        }
        int me = int(r.nodes.size());
        r.nodes.push_back(empty_node());
        r.max_depth = std::max(r.max_depth, depth);
        int stack_here = stack_acc + (nk - 1);
        r.max_stack = std::max(r.max_stack, stack_here);
        for (int i = 0; i < nk; ++i) {
            const BNode& c = nodes_[kids[i]];
            int32_t code;
            if (c.count > 0) {
                code = encode_leaf(c.start, c.count);
                ++r.nleaves;
            } else {
                code = emit(r, kids[i], depth + 1, stack_here);
            }
            WideNode4& w = r.nodes[me];
            set_child(w, i, c);
            w.child[i] = code;
        }
        return me;
    }

    // 8-wide collapse: open the largest-area internal child until 8 children.
    int emit8(BuildResult& r, int32_t b, int depth, int stack_acc) {
        int32_t kids[8] = {nodes_[b].left, nodes_[b].right, -1, -1, -1, -1, -1, -1};
        int nk = 2;
        while (nk < 8) {
            int best = -1;
            float ba = -1.f;
            for (int i = 0; i < nk; ++i) {
                const BNode& c = nodes_[kids[i]];
                if (c.count == 0 && c.box.area() > ba) { ba = c.box.area(); best = i; }
            }
            if (best < 0) break;
            int32_t l = nodes_[kids[best]].left, rr = nodes_[kids[best]].right;
            kids[best] = l;
            kids[nk++] = rr;
        }
        int me = int(r.nodes8.size());
        r.nodes8.push_back(QNode8{});
        r.max_depth8 = std::max(r.max_depth8, depth);
        int stack_here = stack_acc + (nk - 1);
        r.max_stack8 = std::max(r.max_stack8, stack_here);
        int32_t codes[8];
        for (int i = 0; i < nk; ++i) {
            const BNode& c = nodes_[kids[i]];
            codes[i] = c.count > 0 ? encode_leaf(c.start, c.count) : emit8(r, kids[i], depth + 1, stack_here);
        }
        Q8Job job;
        job.node = me;
        job.nk = nk;
        for (int i = 0; i < nk; ++i) { job.kids[i] = kids[i]; job.codes[i] = codes[i]; }
        q8_jobs_.push_back(job);
        return me;
    }

    struct Q8Job {
        int32_t node, nk;
        int32_t kids[8], codes[8];
    };
    std::vector<Q8Job> q8_jobs_;

    // quantise every recorded 8-wide node (independent per node) on the host's cores
    void run_q8_jobs(BuildResult& r) {
        const int64_t n = int64_t(q8_jobs_.size());
        const int hw = std::max(1, std::min(64, int(std::thread::hardware_concurrency())));
        const int nt = int(std::min<int64_t>(hw, std::max<int64_t>(1, n / 4096)));
        std::atomic<bool> failed{false};
        auto work = [&](int64_t b, int64_t e) {
            bool f = false;
            for (int64_t i = b; i < e; ++i) {
                const Q8Job& j = q8_jobs_[size_t(i)];
                f = !fill_qnode(r.nodes8[size_t(j.node)], j.kids, j.codes, j.nk) || f;
            }
            if (f) failed = true;
        };
        if (nt <= 1) {
            work(0, n);
        } else {
            std::vector<std::thread> th;
            const int64_t chunk = (n + nt - 1) / nt;
            for (int k = 0; k < nt; ++k) {
                const int64_t b = k * chunk, e = std::min(n, b + chunk);
                if (b < e) th.emplace_back(work, b, e);
            }
            for (auto& t : th) t.join();
        }
        if (failed) q8_failed_ = true;
        q8_jobs_.clear();
        q8_jobs_.shrink_to_fit();
    }

    // Quantises one recorded 8-wide node (qnode.h); false when a plane cannot
    // be made conservative (coordinates too large)
    bool fill_qnode(QNode8& q, const int32_t* kids, const int32_t* codes, int nk) const {
        float kb[8][6];
        for (int i = 0; i < nk; ++i)
            for (int a = 0; a < 3; ++a) {
                kb[i][a] = nodes_[kids[i]].box.lo[a];
                kb[i][3 + a] = nodes_[kids[i]].box.hi[a];
            }
        return fill_qnode8(q, kb, codes, nk);
    }

    void make_leaf(int64_t nodeidx, int64_t begin, int64_t end, const Box& box) {
        BNode& nd = nodes_[nodeidx];
        nd.box = box;
        nd.start = int32_t(begin);
        nd.count = int32_t(end - begin);
    }

    void build(int64_t nodeidx, int64_t begin, int64_t end, const Box& box, const Box& cbox) {
        const int64_t m = end - begin;
        const int max_leaf = p_.max_leaf;
        if (m <= 1) { make_leaf(nodeidx, begin, end, box); return; }

        int best_axis = -1, best_bin = -1;
        float best_cost = FLT_MAX;
        Box bl, br, cbl, cbr;
        int64_t nl_best = 0;
        const int B = p_.bins;
        // per-thread scratch, reused by every node this thread splits (bins are
        // consumed before the recursion)
        thread_local std::vector<Bin> bins;
        thread_local std::vector<float> rarea;
        thread_local std::vector<int64_t> rcount;
        bins.resize(size_t(3 * B));
        rarea.resize(size_t(B));
        rcount.resize(size_t(B));
        float inv_area = box.area() > 0.f ? 1.f / box.area() : 0.f;
        // large nodes (the top of the tree, where few subtrees run in parallel yet)
        // bin their triangles in chunks on the host's cores and merge the bins;
        // bin contents are unions and counts, so the result is order-independent
        const int64_t kParBin = 262144;
        int nbt = 1;
        if (m >= kParBin) {
            const int hw = std::max(1, std::min(32, int(std::thread::hardware_concurrency())));
            nbt = int(std::min<int64_t>(hw, m / 65536));
        }
        for (int axis = 0; axis < 3; ++axis) {
            float ext = cbox.hi[axis] - cbox.lo[axis];
            if (!(ext > 0.f)) continue;
            float scale = float(B) / ext;
            Bin* bb = &bins[size_t(axis * B)];
            for (int i = 0; i < B; ++i) { bb[i].box.clear(); bb[i].cbox.clear(); bb[i].count = 0; }
            auto bin_range = [&](int64_t kb, int64_t ke, Bin* out) {
                for (int64_t k = kb; k < ke; ++k) {
                    int32_t t = idx_[k];
                    int bi = std::min(B - 1, std::max(0, int((cen_[3 * t + axis] - cbox.lo[axis]) * scale)));
                    out[bi].box.grow(&tlo_[3 * t], &thi_[3 * t]);
                    out[bi].cbox.grow_pt(&cen_[3 * t]);
                    ++out[bi].count;
                }
            };
            if (nbt <= 1) {
                bin_range(begin, end, bb);
            } else {
                std::vector<Bin> part(size_t(nbt) * B);
                for (Bin& x : part) { x.box.clear(); x.cbox.clear(); x.count = 0; }
                std::vector<std::thread> th;
                const int64_t chunk = (m + nbt - 1) / nbt;
                for (int k = 0; k < nbt; ++k) {
                    const int64_t b = begin + k * chunk, e = std::min(end, b + chunk);
                    if (b < e) th.emplace_back(bin_range, b, e, &part[size_t(k) * B]);
                }
                for (auto& t : th) t.join();
                for (int k = 0; k < nbt; ++k)
                    for (int i = 0; i < B; ++i) {
                        const Bin& x = part[size_t(k) * B + i];
                        bb[i].box.grow(x.box);
                        bb[i].cbox.grow(x.cbox);
                        bb[i].count += x.count;
                    }
            }
            Box acc; acc.clear();
            int64_t cnt = 0;
            for (int i = B - 1; i > 0; --i) {
                acc.grow(bb[i].box); cnt += bb[i].count;
                rarea[i] = acc.area(); rcount[i] = cnt;
            }
            acc.clear(); cnt = 0;
            for (int i = 0; i < B - 1; ++i) {
                acc.grow(bb[i].box); cnt += bb[i].count;
                if (cnt == 0 || rcount[i + 1] == 0) continue;
                float cost = p_.cost_node + (float(cnt) * acc.area() + float(rcount[i + 1]) * rarea[i + 1]) * inv_area;
                if (cost < best_cost) { best_cost = cost; best_axis = axis; best_bin = i; nl_best = cnt; }
            }
        }
        if (m <= max_leaf && float(m) <= best_cost) { make_leaf(nodeidx, begin, end, box); return; }

        int64_t mid;
        if (best_axis < 0) {                      // all centroids coincide: split the range
            if (m <= max_leaf) { make_leaf(nodeidx, begin, end, box); return; }
            mid = begin + m / 2;
            bl.clear(); br.clear(); cbl.clear(); cbr.clear();
            for (int64_t k = begin; k < mid; ++k) { int t = idx_[k]; bl.grow(&tlo_[3 * t], &thi_[3 * t]); cbl.grow_pt(&cen_[3 * t]); }
            for (int64_t k = mid; k < end; ++k) { int t = idx_[k]; br.grow(&tlo_[3 * t], &thi_[3 * t]); cbr.grow_pt(&cen_[3 * t]); }
        } else {
            const int axis = best_axis;
            const float lo = cbox.lo[axis];
            const float scale = float(B) / (cbox.hi[axis] - cbox.lo[axis]);
            Bin* bb = &bins[size_t(axis * B)];
            bl.clear(); br.clear(); cbl.clear(); cbr.clear();
            for (int i = 0; i < B; ++i) {
                if (i <= best_bin) { bl.grow(bb[i].box); cbl.grow(bb[i].cbox); }
                else { br.grow(bb[i].box); cbr.grow(bb[i].cbox); }
            }
            int32_t* first = idx_.data() + begin;
            int32_t* last = idx_.data() + end;
            int32_t* pm = std::partition(first, last, [&](int32_t t) {
                int bi = std::min(B - 1, std::max(0, int((cen_[3 * t + axis] - lo) * scale)));
                return bi <= best_bin;
            });
            mid = begin + (pm - first);
            (void)nl_best;
        }
        BNode& nd = nodes_[nodeidx];
        nd.box = box;
        nd.count = 0;
        const int64_t left = nodeidx + 1;
        const int64_t right = nodeidx + 2 * (mid - begin);
        nd.left = int32_t(left);
        nd.right = int32_t(right);
        bool spawn = m > 65536 && take_thread();
        if (spawn) {
            std::thread th([&, left, begin, mid]() { build(left, begin, mid, bl, cbl); });
            build(right, mid, end, br, cbr);
            th.join();
            spare_threads_.fetch_add(1);
        } else {
            build(left, begin, mid, bl, cbl);
            build(right, mid, end, br, cbr);
        }
    }

    bool take_thread() {
        int v = spare_threads_.load();
        while (v > 0) {
            if (spare_threads_.compare_exchange_weak(v, v - 1)) return true;
        }
        return false;
    }

    int64_t n_;
    BuildParams p_;
    std::vector<float> tlo_, thi_, cen_;
    std::vector<int32_t> idx_;
    std::vector<BNode> nodes_;
    std::atomic<int> spare_threads_{0};

public:
    mutable bool q8_failed_ = false;
};

}  // namespace

// Smallest grid step 2^e (e in [-120, kQMaxExp]) with an origin k * 2^e <= L,
// |k| <= 2^23 - 257 and (k + 255) * 2^e >= H.  All arithmetic is exact in
// double: L, H are floats, k is an integer below 2^24, the steps are powers of
// two.  e <= kQMaxExp keeps o2 = (k - 2^23) * 2^e finite; returns kQMaxExp + 1
// when no such step exists (node coordinates beyond ~1e33).
int qnode_axis(float L, float H, double* k) { return qnode_axis_exact(L, H, k); }

BuildResult build_wide_bvh(const float* lo, const float* hi, int64_t n, const BuildParams& p) {
    Builder b(lo, hi, n, p);
    b.run();
    BuildResult r = b.collapse();
    if (b.q8_failed_) {              // coordinates too large to quantise: 4-wide only
        r.nodes8.clear();
        r.max_depth8 = r.max_stack8 = 0;
    }
    return r;
}

}  // namespace bg
