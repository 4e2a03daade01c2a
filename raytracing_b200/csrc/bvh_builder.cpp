// Binned SAH builder (Wald, "On fast Construction of SAH-based Bounding Volume Hierarchies", RT 2007): primitives
// are binned by their box centroids on each axis, the split of least surface-area cost is taken, and recursion stops
// at a leaf when a leaf is cheaper than any split (or the range is down to one primitive).
#include "bvh_builder.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>

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
    void grow(const double* p)
    {
        for (int a = 0; a < 3; ++a)
        {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
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

class builder
{
public:
    builder(std::vector<build_prim>& prims, const bvh_options& options, bvh_result& out)
        : prims_(prims), options_(options), out_(out), index_(prims.size()), centroid_(prims.size() * 3),
          bin_of_(prims.size())
    {
        for (size_t i = 0; i < prims.size(); ++i)
        {
            index_[i] = static_cast<int32_t>(i);
            for (int a = 0; a < 3; ++a)
            {
                centroid_[3 * i + a] = 0.5 * (prims[i].lo[a] + prims[i].hi[a]);
            }
        }
    }

    void run()
    {
        const int n = static_cast<int>(prims_.size());
        if (n == 0)
        {
            return;
        }
        box bounds;
        const int32_t root = build(0, n, 1, bounds);
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
            out_.nodes.insert(out_.nodes.begin(), node);
        }
    }

private:
    std::vector<build_prim>& prims_;
    const bvh_options& options_;
    bvh_result& out_;
    std::vector<int32_t> index_;
    std::vector<double> centroid_;
    std::vector<int32_t> bin_of_;

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

    box prim_box(int32_t i) const
    {
        box b;
        for (int a = 0; a < 3; ++a)
        {
            b.lo[a] = prims_[static_cast<size_t>(i)].lo[a];
            b.hi[a] = prims_[static_cast<size_t>(i)].hi[a];
        }
        return b;
    }

    int32_t make_leaf(int begin, int end)
    {
        const int32_t kind = prims_[static_cast<size_t>(index_[static_cast<size_t>(begin)])].kind;
        std::vector<int32_t>& order = out_.order[kind];
        const auto start = static_cast<int32_t>(order.size());
        if (start >= (1 << (31 - leaf_start_shift)))
        {
            throw std::runtime_error("too many primitives of one kind for the leaf encoding (2^26)");
        }
        for (int i = begin; i < end; ++i)
        {
            order.push_back(prims_[static_cast<size_t>(index_[static_cast<size_t>(i)])].source);
        }
        ++out_.leaves;
        return leaf_link(start, end - begin, kind);
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
    // bvh.cuh:425-432, there on where the boxes start): the range sorted by (centroid, index), a total order, so the
    // tree does not depend on the sort's implementation, and cut in the middle
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
        std::sort(index_.begin() + begin, index_.begin() + end, [&](int32_t p, int32_t q) {
            const double cp = centroid_[3 * static_cast<size_t>(p) + static_cast<size_t>(axis)];
            const double cq = centroid_[3 * static_cast<size_t>(q) + static_cast<size_t>(axis)];
            return cp < cq || (cp == cq && p < q);
        });
        return begin + (end - begin) / 2;
    }

    // Returns the subtree's link: an inner node's index, or a leaf. `median`: the subtree is cut at object medians.
    // The SAH can peel one primitive a level off some inputs (centroids spaced geometrically: 400 spheres at 1.5^i
    // make a chain deeper than the traversal stack), so a subtree whose median cuts would only just fit the stack
    // from here takes them all the way down: halving n primitives takes ceil(log2 n) levels and a leaf-sized range of
    // two or three kinds at most two more, so no leaf lies deeper than max_bvh_depth. Trees of the usual scenes (the
    // 1.31M-triangle mesh is 24 levels deep) never come near that point and are pure SAH.
    int32_t build(int begin, int end, int depth, box& bounds, bool median = false)
    {
        bounds = box{};
        box centroids;
        bool one_kind = true;
        const int32_t first_kind = prims_[static_cast<size_t>(index_[static_cast<size_t>(begin)])].kind;
        for (int i = begin; i < end; ++i)
        {
            const int32_t p = index_[static_cast<size_t>(i)];
            bounds.grow(prim_box(p));
            centroids.grow(&centroid_[3 * static_cast<size_t>(p)]);
            one_kind = one_kind && prims_[static_cast<size_t>(p)].kind == first_kind;
        }
        out_.depth = std::max(out_.depth, depth);
        const int n = end - begin;
        const int max_leaf = std::clamp(options_.max_leaf_size, 1, max_leaf_size);
        if (n == 1)
        {
            return make_leaf(begin, end);
        }

        int split = -1;
        median = median || depth + ceil_log2(n) + 2 >= max_bvh_depth;
        if (!one_kind && n <= max_leaf)
        {
            // Few enough for one leaf but of several kinds: split off the first kind (stable, as bvh.cuh:404-410)
            auto middle = std::stable_partition(index_.begin() + begin, index_.begin() + end, [&](int32_t p) {
                return prims_[static_cast<size_t>(p)].kind == first_kind;
            });
            split = static_cast<int>(middle - index_.begin());
        }
        else if (median)
        {
            if (one_kind && n <= max_leaf)
            {
                return make_leaf(begin, end);
            }
            split = median_split(begin, end, centroids);
        }
        else
        {
            double best_cost = inf;
            int best_axis = -1;
            int best_bin = -1;
            const int bins = std::clamp(options_.bins, 2, 256);
            std::vector<box> bin_box(static_cast<size_t>(bins));
            std::vector<int> bin_count(static_cast<size_t>(bins));
            std::vector<double> right_area(static_cast<size_t>(bins));
            std::vector<int> right_count(static_cast<size_t>(bins));
            for (int axis = 0; axis < 3; ++axis)
            {
                const double lo = centroids.lo[axis];
                const double extent = centroids.hi[axis] - lo;
                if (!(extent > 0))
                {
                    continue;
                }
                std::fill(bin_box.begin(), bin_box.end(), box{});
                std::fill(bin_count.begin(), bin_count.end(), 0);
                const double scale = bins / extent;
                for (int i = begin; i < end; ++i)
                {
                    const int32_t p = index_[static_cast<size_t>(i)];
                    const int b = std::min(bins - 1, static_cast<int>((centroid_[3 * static_cast<size_t>(p) + axis] - lo) * scale));
                    bin_box[static_cast<size_t>(b)].grow(prim_box(p));
                    ++bin_count[static_cast<size_t>(b)];
                }
                box acc;
                int count = 0;
                for (int b = bins - 1; b > 0; --b)
                {
                    acc.grow(bin_box[static_cast<size_t>(b)]);
                    count += bin_count[static_cast<size_t>(b)];
                    right_area[static_cast<size_t>(b)] = acc.area();
                    right_count[static_cast<size_t>(b)] = count;
                }
                acc = box{};
                count = 0;
                for (int b = 0; b < bins - 1; ++b)
                {
                    acc.grow(bin_box[static_cast<size_t>(b)]);
                    count += bin_count[static_cast<size_t>(b)];
                    const int rc = right_count[static_cast<size_t>(b + 1)];
                    if (count == 0 || rc == 0)
                    {
                        continue;
                    }
                    const double cost = acc.area() * count + right_area[static_cast<size_t>(b + 1)] * rc;
                    if (cost < best_cost)
                    {
                        best_cost = cost;
                        best_axis = axis;
                        best_bin = b;
                    }
                }
            }
            const double parent_area = bounds.area();
            const double split_cost =
                best_axis >= 0 && parent_area > 0 ? options_.node_cost + best_cost / parent_area : inf;
            if (one_kind && n <= max_leaf && static_cast<double>(n) <= split_cost)
            {
                return make_leaf(begin, end);
            }
            if (best_axis >= 0)
            {
                const double lo = centroids.lo[best_axis];
                const double scale = bins / (centroids.hi[best_axis] - lo);
                auto middle = std::partition(index_.begin() + begin, index_.begin() + end, [&](int32_t p) {
                    const int b = std::min(bins - 1, static_cast<int>((centroid_[3 * static_cast<size_t>(p) + best_axis] - lo) * scale));
                    return b <= best_bin;
                });
                split = static_cast<int>(middle - index_.begin());
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
        const auto index = static_cast<int32_t>(out_.nodes.size());
        out_.nodes.push_back(bvh_node{});
        box left_box;
        box right_box;
        const int32_t left = build(begin, split, depth + 1, left_box, median);
        const int32_t right = build(split, end, depth + 1, right_box, median);
        bvh_node& node = out_.nodes[static_cast<size_t>(index)];
        set_child(node, 0, left, left_box);
        set_child(node, 1, right, right_box);
        return index;
    }
};
} // namespace

bvh_result build_bvh(std::vector<build_prim> prims, const bvh_options& options)
{
    bvh_result out;
    builder b(prims, options, out);
    b.run();
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
