// Test infrastructure, not product: the reference's own device traversal, closest_hit (src/gpu/bvh.cuh:576-706), run
// on given rays over the reference's own BVH (build_bvh, bvh.cuh:215-444, with the leaf size renderer.cu:81-82 and
// :1122-1126 picks), so that the first-hit parity test can compare three answers for the same rays: this library's
// kernel, the reference's device code and the oracle's double search. Compiled into oracle/_ref/libref_gpu.so by
// oracle/build_ref.py with the reference's headers from its source tree; nothing in the product links it.
#include "bvh.cuh" // the reference's headers, from its source tree
#include "renderer.h"

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "ref_scene_convert.h"
#include "rt_b200.h"

namespace
{
// renderer.cu:81-82: one primitive per leaf, except a scene of at most 8 shapes, which is one leaf
constexpr int reference_leaf_size = 1;
constexpr int reference_small_scene_shapes = 8;

__global__ void reference_closest_hits_kernel(gpu::bvh_view<float> tree, const float* origins, const float* directions,
                                              int64_t count, int32_t* ids, float* ts)
{
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count)
    {
        return;
    }
    gpu::ray<float> r;
    r.origin = {origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]};
    r.direction = {directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]};
    r.time = 0;
    // A camera ray starts on no surface: from = -1, not inward (camera.cuh:444-457)
    const gpu::bvh_hit<float> hit = gpu::closest_hit<float, gpu::kernel_kind::all_books>(tree, r, -1, false);
    ids[i] = hit.index;
    ts[i] = hit.t;
}

struct device_buffer
{
    void* p = nullptr;
    ~device_buffer()
    {
        if (p)
        {
            cudaFree(p);
        }
    }
};

void check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
    {
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
    }
}

template <typename T>
T* upload(device_buffer& b, const std::vector<T>& v)
{
    if (v.empty())
    {
        return nullptr;
    }
    check(cudaMalloc(&b.p, v.size() * sizeof(T)), "allocating device memory");
    check(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "copying to the device");
    return static_cast<T*>(b.p);
}

void copy_error(const char* what, char* error, int error_size)
{
    if (error && error_size > 0)
    {
        std::strncpy(error, what, static_cast<size_t>(error_size) - 1);
        error[error_size - 1] = '\0';
    }
}
} // namespace

extern "C" {

// The reference's closest hit of each ray (host arrays of 3 floats per ray), in SOURCE index space: spheres
// 0..S-1, quads S..S+Q-1 (bvh::sphere_ids / quad_ids undo the tree's leaf order, bvh.cuh:81-98), -1 for a miss; and
// its t. Scenes with triangle meshes are refused (the reference traces triangles only through OptiX).
int ref_gpu_closest_hits(const rt_scene_desc* scene, const float* origins, const float* directions, int64_t count,
                         int32_t* ids, float* ts, char* error, int32_t error_size)
{
    try
    {
        if (scene->mesh_count > 0)
        {
            copy_error("the reference traces triangle meshes only through OptiX", error, error_size);
            return 1;
        }
        const gpu::scene_desc s = ref_convert::to_ref(*scene);
        const size_t shapes = s.spheres.size() + s.quads.size();
        const int leaf = shapes <= static_cast<size_t>(reference_small_scene_shapes) ? reference_small_scene_shapes
                                                                                    : reference_leaf_size;
        const gpu::bvh<float> tree = gpu::build_bvh<float>(s.spheres, s.quads, leaf);
        // global id -> source index
        std::vector<int32_t> source(s.spheres.size() + s.quads.size(), -1);
        for (size_t k = 0; k < tree.sphere_ids.size(); ++k)
        {
            source[static_cast<size_t>(tree.sphere_ids[k])] = static_cast<int32_t>(k);
        }
        for (size_t k = 0; k < tree.quad_ids.size(); ++k)
        {
            source[static_cast<size_t>(tree.quad_ids[k])] = static_cast<int32_t>(s.spheres.size() + k);
        }
        device_buffer nodes, spheres, moving, quads, o, d, id_out, t_out;
        gpu::bvh_view<float> view{};
        view.nodes = upload(nodes, tree.nodes);
        view.node_count = static_cast<int>(tree.nodes.size());
        view.spheres = upload(spheres, tree.spheres);
        view.moving_spheres = upload(moving, tree.moving_spheres);
        view.moving_base = tree.moving_base;
        view.quads = upload(quads, tree.quads);
        view.quad_base = tree.quad_base;
        if (count > 0)
        {
            check(cudaMalloc(&o.p, static_cast<size_t>(count) * 3 * sizeof(float)), "allocating device memory");
            check(cudaMalloc(&d.p, static_cast<size_t>(count) * 3 * sizeof(float)), "allocating device memory");
            check(cudaMalloc(&id_out.p, static_cast<size_t>(count) * sizeof(int32_t)), "allocating device memory");
            check(cudaMalloc(&t_out.p, static_cast<size_t>(count) * sizeof(float)), "allocating device memory");
            check(cudaMemcpy(o.p, origins, static_cast<size_t>(count) * 3 * sizeof(float), cudaMemcpyHostToDevice),
                  "copying the rays");
            check(cudaMemcpy(d.p, directions, static_cast<size_t>(count) * 3 * sizeof(float),
                             cudaMemcpyHostToDevice),
                  "copying the rays");
            const int block = 128;
            const auto grid = static_cast<unsigned>((count + block - 1) / block);
            reference_closest_hits_kernel<<<grid, block>>>(view, static_cast<const float*>(o.p),
                                                           static_cast<const float*>(d.p), count,
                                                           static_cast<int32_t*>(id_out.p), static_cast<float*>(t_out.p));
            check(cudaGetLastError(), "launching the reference's closest_hit");
            check(cudaMemcpy(ids, id_out.p, static_cast<size_t>(count) * sizeof(int32_t), cudaMemcpyDeviceToHost),
                  "copying the hits");
            check(cudaMemcpy(ts, t_out.p, static_cast<size_t>(count) * sizeof(float), cudaMemcpyDeviceToHost),
                  "copying the hits");
        }
        for (int64_t i = 0; i < count; ++i)
        {
            if (ids[i] >= 0)
            {
                ids[i] = source[static_cast<size_t>(ids[i])];
            }
        }
        return 0;
    }
    catch (const std::exception& e)
    {
        copy_error(e.what(), error, error_size);
        return 1;
    }
}
}
