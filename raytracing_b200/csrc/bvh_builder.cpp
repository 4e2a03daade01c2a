// Binned SAH builder (Wald, "On fast Construction of SAH-based Bounding Volume Hierarchies", RT 2007): primitives
// are binned by their box centroids on each axis, the split of least surface-area cost is taken, and recursion stops
// at a leaf when a leaf is cheaper than any split (or the range is down to one primitive).
#include "bvh_builder.h"

#include <algorithm>
#include <cmath>
#include <future>
#include <limits>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>

namespace rtb
{
float round_down(double x)
{
    const auto r = static_cast<float>(x);
    return static_cast<double>(r) <= x ? r : std::nextafter(r, -std::numeric_limits<float>::infinity());
}

float round_up(double x)
{
    const auto r = static_cast<float>(x);
    return static_cast<double>(r) >= x ? r : std::nextafter(r, std::numeric_limits<float>::infinity());
}

namespace
{
constexpr double inf = std::numeric_limits<double>::infinity();
constexpr int max_bins = 256;
// Ranges of at least this many primitives split their two subtrees across threads
constexpr int parallel_min = 1 << 14;

struct box
{
    double lo[3] = {inf, inf, inf};
    double hi[3] = {-inf, -inf, -inf};
    void grow(const box& b)
    {
        for (int a = 0; a < 3; ++a)
        {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const double* l, const double* h)
    {
        for (int a = 0; a < 3; ++a)
        {
            lo[a] = std::min(lo[a], l[a]);
            hi[a] = std::max(hi[a], h[a]);
        }
    }
    double area() const
    {
        const double dx = std::max(0.0, hi[0] - lo[0]);
        const double dy = std::max(0.0, hi[1] - lo[1]);
        const double dz = std::max(0.0, hi[2] - lo[2]);
        return 2 * (dx * dy + dy * dz + dz * dx);
    }
};

// A primitive as the builder moves it: its box, centroid, kind and source index in one 80-byte record, so that the
// passes over a range read memory in order and a partition moves the records themselves
struct item
{
    double lo[3];
    double hi[3];
    double c[3];
    int32_t kind;
    int32_t source;
};

// A subtree built on its own: nodes numbered from 0 and each kind's leaf order from 0, spliced into its parent's
// arrays where a depth-first build would have written it
struct fragment
{
    std::vector<bvh_node> nodes;
    std::vector<int32_t> order[3];
    int32_t depth = 0;
    int64_t leaves = 0;
};

// The SAH's best binned split of a range: axis and last bin of the left side (axis -1: none), and its cost
struct sah_split
{
    int axis = -1;
    int bin = -1;
    double cost = inf;
};

inline int bin_of(double c, double lo, double scale, int bins)
{
    return std::min(bins - 1, static_cast<int>((c - lo) * scale));
}

// The same choice for a range of at most sparse_max primitives, over its occupied bins only (a tree's many small
// ranges would spend more on sweeping every bin than on binning). The dense sweep's candidates between two occupied
// bins all cut the range in the same place at the same cost, so the first of them, the left side's last occupied bin,
// is the one that can win; the same boxes are merged into the same unions, so the costs compare the same and the
// split is the dense sweep's bit for bit.
constexpr int sparse_max = 32;

sah_split choose_sparse_sah_split(const item* first, int n, const box& centroids, int bins)
{
    sah_split best;
    for (int axis = 0; axis < 3; ++axis)
    {
        const double lo = centroids.lo[axis];
        const double extent = centroids.hi[axis] - lo;
        if (!(extent > 0))
        {
            continue;
        }
        const double scale = bins / extent;
        // the occupied bins in increasing order, each with its box and count (an insertion into a short sorted list)
        int key[sparse_max];
        box group[sparse_max];
        int count[sparse_max];
        int groups = 0;
        for (int i = 0; i < n; ++i)
        {
            const int b = bin_of(first[i].c[axis], lo, scale, bins);
            int g = groups;
            while (g > 0 && key[g - 1] > b)
            {
                --g;
            }
            if (g > 0 && key[g - 1] == b)
            {
                --g;
            }
            else
            {
                for (int j = groups; j > g; --j)
                {
                    key[j] = key[j - 1];
                    group[j] = group[j - 1];
                    count[j] = count[j - 1];
                }
                key[g] = b;
                group[g] = box{};
                count[g] = 0;
                ++groups;
            }
            group[g].grow(first[i].lo, first[i].hi);
            ++count[g];
        }
        double right_area[sparse_max];
        int right_count[sparse_max];
        box acc;
        int total = 0;
        for (int g = groups - 1; g > 0; --g)
        {
            acc.grow(group[g]);
            total += count[g];
            right_area[g] = acc.area();
            right_count[g] = total;
        }
        acc = box{};
        total = 0;
        for (int g = 0; g + 1 < groups; ++g)
        {
            acc.grow(group[g]);
            total += count[g];
            const double cost = acc.area() * total + right_area[g + 1] * right_count[g + 1];
            if (cost < best.cost)
            {
                best = {axis, key[g], cost};
            }
        }
    }
    return best;
}

// Every axis with a nonzero centroid extent binned in one pass over the range; the cost sweeps as before, axis by
// axis and bin by bin, the first strictly cheapest split winning
sah_split choose_sah_split(const item* first, int n, const box& centroids, int bins)
{
    // Only the `bins` entries of an axis in use are set up (small ranges, most of a tree, would pay more for clearing
    // every bin than for binning)
    struct bin
    {
        double lo[3], hi[3];
        int count;
    };
    bin bin_box[3][max_bins];
    double scale[3] = {0, 0, 0};
    bool binned[3] = {false, false, false};
    for (int axis = 0; axis < 3; ++axis)
    {
        const double extent = centroids.hi[axis] - centroids.lo[axis];
        if (extent > 0)
        {
            binned[axis] = true;
            scale[axis] = bins / extent;
            for (int b = 0; b < bins; ++b)
            {
                bin_box[axis][b] = {{inf, inf, inf}, {-inf, -inf, -inf}, 0};
            }
        }
    }
    for (int i = 0; i < n; ++i)
    {
        const item& it = first[i];
        for (int axis = 0; axis < 3; ++axis)
        {
            if (binned[axis])
            {
                bin& into = bin_box[axis][bin_of(it.c[axis], centroids.lo[axis], scale[axis], bins)];
                for (int a = 0; a < 3; ++a)
                {
                    into.lo[a] = std::min(into.lo[a], it.lo[a]);
                    into.hi[a] = std::max(into.hi[a], it.hi[a]);
                }
                ++into.count;
            }
        }
    }
    sah_split best;
    double right_area[max_bins];
    int right_count[max_bins];
    for (int axis = 0; axis < 3; ++axis)
    {
        if (!binned[axis])
        {
            continue;
        }
        box acc;
        int count = 0;
        for (int b = bins - 1; b > 0; --b)
        {
            acc.grow(bin_box[axis][b].lo, bin_box[axis][b].hi);
            count += bin_box[axis][b].count;
            right_area[b] = acc.area();
            right_count[b] = count;
        }
        acc = box{};
        count = 0;
        for (int b = 0; b < bins - 1; ++b)
        {
            acc.grow(bin_box[axis][b].lo, bin_box[axis][b].hi);
            count += bin_box[axis][b].count;
            const int rc = right_count[b + 1];
            if (count == 0 || rc == 0)
            {
                continue;
            }
            const double cost = acc.area() * count + right_area[b + 1] * rc;
            if (cost < best.cost)
            {
                best = {axis, b, cost};
            }
        }
    }
    return best;
}

class builder
{
public:
    builder(const std::vector<build_prim>& prims, const bvh_options& options) : options_(options), items_(prims.size())
    {
        for (size_t i = 0; i < prims.size(); ++i)
        {
            item& it = items_[i];
            for (int a = 0; a < 3; ++a)
            {
                it.lo[a] = prims[i].lo[a];
                it.hi[a] = prims[i].hi[a];
                it.c[a] = 0.5 * (prims[i].lo[a] + prims[i].hi[a]);
            }
            it.kind = prims[i].kind;
            it.source = prims[i].source;
        }
        // Threads for the subtrees: each split of a large range hands one side to a new thread, to this depth
        const unsigned threads = options.threads > 0 ? static_cast<unsigned>(options.threads)
                                                     : std::max(1u, std::thread::hardware_concurrency());
        while ((1u << spawn_levels_) < std::min(threads, 64u))
        {
            ++spawn_levels_;
        }
    }

    void run(bvh_result& out)
    {
        const int n = static_cast<int>(items_.size());
        if (n == 0)
        {
            return;
        }
        box bounds;
        fragment tree;
        const int32_t root = build(0, n, 1, bounds, false, tree, spawn_levels_);
        out.nodes = std::move(tree.nodes);
        for (int k = 0; k < 3; ++k)
        {
            out.order[k] = std::move(tree.order[k]);
        }
        out.depth = tree.depth;
        out.leaves = tree.leaves;
        if (root < 0)
        {
            // A scene that is one leaf: a root node whose second child is the empty leaf, boxed at +infinity so that
            // no ray enters it
            bvh_node node{};
            set_child(node, 0, root, bounds);
            box far;
            for (int a = 0; a < 3; ++a)
            {
                far.lo[a] = far.hi[a] = inf;
            }
            set_child(node, 1, leaf_link(0, 0, 0), far);
            out.nodes.insert(out.nodes.begin(), node);
        }
    }

private:
    const bvh_options& options_;
    std::vector<item> items_;
    int spawn_levels_ = 0;

    static void set_child(bvh_node& node, int c, int32_t link, const box& b)
    {
        node.x[2 * c] = round_down(b.lo[0]);
        node.x[2 * c + 1] = round_up(b.hi[0]);
        node.y[2 * c] = round_down(b.lo[1]);
        node.y[2 * c + 1] = round_up(b.hi[1]);
        node.z[2 * c] = round_down(b.lo[2]);
        node.z[2 * c + 1] = round_up(b.hi[2]);
        node.link[c] = link;
    }

    static void check_leaf_start(size_t start)
    {
        if (start >= (size_t{1} << (31 - leaf_start_shift)))
        {
            throw std::runtime_error("too many primitives of one kind for the leaf encoding (2^26)");
        }
    }

    int32_t make_leaf(int begin, int end, fragment& out) const
    {
        const int32_t kind = items_[static_cast<size_t>(begin)].kind;
        std::vector<int32_t>& order = out.order[kind];
        const size_t start = order.size();
        check_leaf_start(start);
        for (int i = begin; i < end; ++i)
        {
            order.push_back(items_[static_cast<size_t>(i)].source);
        }
        ++out.leaves;
        return leaf_link(static_cast<int32_t>(start), end - begin, kind);
    }

    // `f` (a subtree built on its own, whose root is `link`) appended to `out`: its nodes after out's, its leaves after
    // out's leaves of each kind; returns the root's link in out's numbering
    static int32_t splice(fragment& out, const fragment& f, int32_t link)
    {
        const auto base = static_cast<int32_t>(out.nodes.size());
        size_t offset[3];
        for (int k = 0; k < 3; ++k)
        {
            offset[k] = out.order[k].size();
        }
        const auto moved = [&](int32_t l) {
            if (l >= 0)
            {
                return l + base;
            }
            const int32_t kind = leaf_kind(l);
            const size_t start = static_cast<size_t>(leaf_start(l)) + offset[kind];
            check_leaf_start(start);
            return leaf_link(static_cast<int32_t>(start), leaf_count(l), kind);
        };
        out.nodes.reserve(out.nodes.size() + f.nodes.size());
        for (bvh_node node : f.nodes)
        {
            node.link[0] = moved(node.link[0]);
            node.link[1] = moved(node.link[1]);
            out.nodes.push_back(node);
        }
        for (int k = 0; k < 3; ++k)
        {
            out.order[k].insert(out.order[k].end(), f.order[k].begin(), f.order[k].end());
        }
        out.depth = std::max(out.depth, f.depth);
        out.leaves += f.leaves;
        return moved(link);
    }

    // ceil(log2(n)) for n >= 1
    static int ceil_log2(int n)
    {
        int levels = 0;
        while ((int64_t{1} << levels) < n)
        {
            ++levels;
        }
        return levels;
    }

    // The object median on the longest axis of the centroids' box (the reference's only split, bvh.ixx:53-73 and
    // bvh.cuh:425-432, there on where the boxes start): the range sorted by (centroid, kind, source), a total order,
    // so the tree does not depend on the sort's implementation, and cut in the middle
    int median_split(int begin, int end, const box& centroids)
    {
        int axis = 0;
        for (int a = 1; a < 3; ++a)
        {
            if (centroids.hi[a] - centroids.lo[a] > centroids.hi[axis] - centroids.lo[axis])
            {
                axis = a;
            }
        }
        std::sort(items_.begin() + begin, items_.begin() + end, [axis](const item& p, const item& q) {
            if (p.c[axis] != q.c[axis])
            {
                return p.c[axis] < q.c[axis];
            }
            return p.kind != q.kind ? p.kind < q.kind : p.source < q.source;
        });
        return begin + (end - begin) / 2;
    }

    // Returns the subtree's link in `out`: an inner node's index, or a leaf. `median`: the subtree is cut at object
    // medians. The SAH can peel one primitive a level off some inputs (centroids spaced geometrically: 400 spheres at
    // 1.5^i make a chain deeper than the traversal stack), so a subtree whose median cuts would only just fit the
    // stack from here takes them all the way down: halving n primitives takes ceil(log2 n) levels and a leaf-sized
    // range of two or three kinds at most two more, so no leaf lies deeper than max_bvh_depth. Trees of the usual
    // scenes (the 1.31M-triangle mesh is 24 levels deep) never come near that point and are pure SAH. `spawn`: levels
    // below this one that may still hand a subtree to a new thread; the tree is the same whichever threads build it.
    int32_t build(int begin, int end, int depth, box& bounds, bool median, fragment& out, int spawn)
    {
        bounds = box{};
        box centroids;
        bool one_kind = true;
        const int32_t first_kind = items_[static_cast<size_t>(begin)].kind;
        for (int i = begin; i < end; ++i)
        {
            const item& it = items_[static_cast<size_t>(i)];
            bounds.grow(it.lo, it.hi);
            centroids.grow(it.c, it.c);
            one_kind = one_kind && it.kind == first_kind;
        }
        out.depth = std::max(out.depth, depth);
        const int n = end - begin;
        const int max_leaf = std::clamp(options_.max_leaf_size, 1, max_leaf_size);
        if (n == 1)
        {
            return make_leaf(begin, end, out);
        }

        int split = -1;
        median = median || depth + ceil_log2(n) + 2 >= max_bvh_depth;
        if (!one_kind && n <= max_leaf)
        {
            // Few enough for one leaf but of several kinds: split off the first kind (stable, as bvh.cuh:404-410)
            auto middle = std::stable_partition(items_.begin() + begin, items_.begin() + end,
                                                [&](const item& it) { return it.kind == first_kind; });
            split = static_cast<int>(middle - items_.begin());
        }
        else if (median)
        {
            if (one_kind && n <= max_leaf)
            {
                return make_leaf(begin, end, out);
            }
            split = median_split(begin, end, centroids);
        }
        else
        {
            const int bins = std::clamp(options_.bins, 2, max_bins);
            const sah_split best = n <= sparse_max ? choose_sparse_sah_split(items_.data() + begin, n, centroids, bins)
                                                   : choose_sah_split(items_.data() + begin, n, centroids, bins);
            const double parent_area = bounds.area();
            const double split_cost =
                best.axis >= 0 && parent_area > 0 ? options_.node_cost + best.cost / parent_area : inf;
            if (one_kind && n <= max_leaf && static_cast<double>(n) <= split_cost)
            {
                return make_leaf(begin, end, out);
            }
            if (best.axis >= 0)
            {
                const int axis = best.axis;
                const double lo = centroids.lo[axis];
                const double scale = bins / (centroids.hi[axis] - lo);
                auto middle = std::partition(items_.begin() + begin, items_.begin() + end, [&](const item& it) {
                    return bin_of(it.c[axis], lo, scale, bins) <= best.bin;
                });
                split = static_cast<int>(middle - items_.begin());
            }
            if (split <= begin || split >= end)
            {
                // All centroids in one place: halve the range by index
                split = begin + n / 2;
            }
        }
        if (depth + 1 > max_bvh_depth)
        {
            throw std::runtime_error("the BVH is deeper than the traversal stack (" + std::to_string(max_bvh_depth) +
                                     " levels)");
        }
        const auto index = static_cast<int32_t>(out.nodes.size());
        out.nodes.push_back(bvh_node{});
        box left_box;
        box right_box;
        int32_t left = 0;
        int32_t right = 0;
        if (spawn > 0 && n >= parallel_min)
        {
            // The left subtree on another thread, the right on this one, each into a fragment of its own, spliced in
            // the depth-first order: the same nodes, links and leaf order as one thread's build
            fragment left_part;
            fragment right_part;
            std::future<int32_t> pending;
            try
            {
                pending = std::async(std::launch::async, [&] {
                    return build(begin, split, depth + 1, left_box, median, left_part, spawn - 1);
                });
            }
            catch (const std::system_error&)
            {
                // no thread to be had: this one builds both sides, into the same fragments
            }
            int32_t left_root = 0;
            if (!pending.valid())
            {
                left_root = build(begin, split, depth + 1, left_box, median, left_part, 0);
            }
            int32_t right_root = 0;
            try
            {
                right_root = build(split, end, depth + 1, right_box, median, right_part, pending.valid() ? spawn - 1 : 0);
            }
            catch (...)
            {
                if (pending.valid())
                {
                    pending.wait();
                }
                throw;
            }
            if (pending.valid())
            {
                left_root = pending.get();
            }
            left = splice(out, left_part, left_root);
            right = splice(out, right_part, right_root);
        }
        else
        {
            left = build(begin, split, depth + 1, left_box, median, out, spawn);
            right = build(split, end, depth + 1, right_box, median, out, spawn);
        }
        bvh_node& node = out.nodes[static_cast<size_t>(index)];
        set_child(node, 0, left, left_box);
        set_child(node, 1, right, right_box);
        return index;
    }
};
} // namespace

bvh_result build_bvh(std::vector<build_prim> prims, const bvh_options& options)
{
    bvh_result out;
    builder b(prims, options);
    prims.clear();
    prims.shrink_to_fit();
    b.run(out);
    return out;
}

namespace
{
// A child of a binary node: its box and link
struct wide_child
{
    float lo[3], hi[3];
    int32_t link;
};

wide_child child_of(const bvh_node& n, int c)
{
    return {{n.x[2 * c], n.y[2 * c], n.z[2 * c]}, {n.x[2 * c + 1], n.y[2 * c + 1], n.z[2 * c + 1]}, n.link[c]};
}

double area(const wide_child& c)
{
    const double dx = c.hi[0] - c.lo[0], dy = c.hi[1] - c.lo[1], dz = c.hi[2] - c.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

int32_t collapse(const std::vector<bvh_node>& nodes, int32_t index, std::vector<bvh4_node>& out, int32_t level,
                 int32_t& depth)
{
    depth = std::max(depth, level);
    std::vector<wide_child> kids = {child_of(nodes[static_cast<size_t>(index)], 0),
                                    child_of(nodes[static_cast<size_t>(index)], 1)};
    while (kids.size() < 4)
    {
        int best = -1;
        for (int k = 0; k < static_cast<int>(kids.size()); ++k)
        {
            if (kids[static_cast<size_t>(k)].link >= 0 && (best < 0 || area(kids[static_cast<size_t>(k)]) >
                                                                           area(kids[static_cast<size_t>(best)])))
            {
                best = k;
            }
        }
        if (best < 0)
        {
            break; // only leaves left
        }
        const bvh_node& n = nodes[static_cast<size_t>(kids[static_cast<size_t>(best)].link)];
        kids[static_cast<size_t>(best)] = child_of(n, 0);
        kids.insert(kids.begin() + best + 1, child_of(n, 1));
    }
    const auto self = static_cast<int32_t>(out.size());
    out.emplace_back();
    int32_t links[4] = {traversal_done_link, traversal_done_link, traversal_done_link, traversal_done_link};
    for (size_t k = 0; k < kids.size(); ++k)
    {
        links[k] = kids[k].link >= 0 ? collapse(nodes, kids[k].link, out, level + 1, depth) : kids[k].link;
    }
    bvh4_node& w = out[static_cast<size_t>(self)];
    for (int k = 0; k < 4; ++k)
    {
        const bool used = k < static_cast<int>(kids.size());
        const wide_child c = used ? kids[static_cast<size_t>(k)] : wide_child{{0, 0, 0}, {0, 0, 0}, 0};
        w.lo_x[k] = c.lo[0];
        w.hi_x[k] = c.hi[0];
        w.lo_y[k] = c.lo[1];
        w.hi_y[k] = c.hi[1];
        w.lo_z[k] = c.lo[2];
        w.hi_z[k] = c.hi[2];
        w.link[k] = links[k];
        w.pad[k] = 0;
    }
    return self;
}
} // namespace

int32_t collapse_bvh4(const std::vector<bvh_node>& nodes, std::vector<bvh4_node>& out)
{
    out.clear();
    int32_t depth = 0;
    if (!nodes.empty())
    {
        collapse(nodes, 0, out, 1, depth);
    }
    return depth;
}
} // namespace rtb
