"""The tree collapsed four wide (the wavefront's walk), checked on the host against the binary tree it came from.

`collapse_bvh4` (raytracing_b200/csrc/bvh_builder.cpp) is compiled here with g++ together with the binary builder and
a small driver; on random scenes of spheres, quads and triangles (SAH trees of 4 to 4096 primitives):

* every leaf of the binary tree is a child of exactly one wide node, with the binary tree's own box for it (so both
  walks test the same boxes and reach the same primitives);
* every inner binary node is either a wide node or was absorbed into its parent, and each wide node has two to four
  used slots, unused slots linked to nothing (traversal_done) and never hit;
* the wide tree is no deeper than the binary one and fits the wide walk's stack (three entries a level).
"""
import shutil
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
CSRC = REPO / "raytracing_b200" / "csrc"

DRIVER = r"""
#include <cstdio>
#include <map>
#include <random>
#include <vector>
#include "bvh_builder.h"
using namespace rtb;

static int check(int count, int seed, int leaf)
{
    std::mt19937 g(seed);
    std::uniform_real_distribution<double> u(-10.0, 10.0), r(0.01, 0.8);
    std::vector<build_prim> prims;
    for (int i = 0; i < count; ++i)
    {
        build_prim p{};
        const double c[3] = {u(g), u(g), u(g)}, e = r(g);
        for (int a = 0; a < 3; ++a) { p.lo[a] = c[a] - e; p.hi[a] = c[a] + e * (a == 1 ? 0.5 : 1.0); }
        p.kind = i % 3 == 0 ? kind_triangle : (i % 3 == 1 ? kind_sphere : kind_quad);
        p.source = i;
        prims.push_back(p);
    }
    bvh_options o;
    o.max_leaf_size = leaf;
    const bvh_result tree = build_bvh(prims, o);
    std::vector<bvh4_node> wide;
    const int depth4 = collapse_bvh4(tree.nodes, wide);
    // the binary tree's leaves with their boxes (from the parent's per-axis layout)
    std::map<int, std::vector<float>> binary_leaves;
    std::vector<int> stack = {0};
    while (!stack.empty())
    {
        const bvh_node& n = tree.nodes[stack.back()];
        stack.pop_back();
        for (int c = 0; c < 2; ++c)
        {
            if (n.link[c] >= 0) { stack.push_back(n.link[c]); continue; }
            binary_leaves[n.link[c]] = {n.x[2 * c], n.x[2 * c + 1], n.y[2 * c], n.y[2 * c + 1], n.z[2 * c], n.z[2 * c + 1]};
        }
    }
    std::map<int, std::vector<float>> wide_leaves;
    int inner = 0, duplicates = 0, bad_slots = 0, bad_boxes = 0;
    stack = {0};
    while (!stack.empty())
    {
        const bvh4_node& w = wide[stack.back()];
        stack.pop_back();
        ++inner;
        int used = 0;
        for (int k = 0; k < 4; ++k)
        {
            const int l = w.link[k];
            if (l == traversal_done_link) { continue; }
            ++used;
            if (l >= 0) { stack.push_back(l); continue; }
            if (wide_leaves.count(l)) { ++duplicates; }
            wide_leaves[l] = {w.lo_x[k], w.hi_x[k], w.lo_y[k], w.hi_y[k], w.lo_z[k], w.hi_z[k]};
        }
        for (int k = used; k < 4; ++k) { bad_slots += w.link[k] != traversal_done_link; }
        bad_slots += used < 2 || used > 4;
    }
    for (const auto& [l, b] : binary_leaves)
    {
        const auto it = wide_leaves.find(l);
        bad_boxes += it == wide_leaves.end() || it->second != b;
    }
    std::printf("%d %d %d %zu %zu %d %d %d %d %zu\n", count, tree.depth, depth4, binary_leaves.size(), wide_leaves.size(),
                duplicates, bad_slots, bad_boxes, inner, wide.size());
    return duplicates + bad_slots + bad_boxes + (binary_leaves.size() != wide_leaves.size()) +
           (depth4 > tree.depth) + (inner != static_cast<int>(wide.size()));
}

int main()
{
    int failures = 0;
    const int counts[] = {4, 17, 100, 1000, 4096};
    for (int count : counts)
    {
        for (int seed = 1; seed <= 3; ++seed)
        {
            failures += check(count, seed, count % 2 ? 1 : 4);
        }
    }
    return failures == 0 ? 0 : 1;
}
"""


def _cuda_include():
    for root in ("/usr/local/cuda/include", "/usr/local/cuda/targets/x86_64-linux/include"):
        if (Path(root) / "vector_types.h").exists():
            return root
    return None


@pytest.mark.skipif(shutil.which("g++") is None or _cuda_include() is None, reason="needs g++ and the CUDA headers")
def test_wide_tree_keeps_every_leaf_and_box(tmp_path):
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    subprocess.run(["g++", "-std=c++20", "-O1", "-I", str(CSRC), "-I", str(REPO / "include"), "-I", _cuda_include(),
                    str(src), str(CSRC / "bvh_builder.cpp"), "-o", str(exe)], check=True)
    run = subprocess.run([str(exe)], capture_output=True, text=True)
    lines = [list(map(int, line.split())) for line in run.stdout.split("\n") if line.strip()]
    assert run.returncode == 0, run.stdout
    assert len(lines) == 15
    for count, depth, depth4, binary_leaves, wide_leaves, dup, bad_slots, bad_boxes, inner, nodes in lines:
        assert binary_leaves == wide_leaves and dup == bad_slots == bad_boxes == 0
        assert 1 <= depth4 <= depth and 3 * depth4 <= 96  # the wide walk's stack: three entries a level
        assert inner == nodes
