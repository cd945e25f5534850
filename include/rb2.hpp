/*
 * rb2.hpp -- header-only C++ classes over the C ABI that keep the reference's
 * names and signatures, so host code written against renderbox2's
 * acceleration-structure and tracer classes compiles against librb2:
 *
 *   Platform                    accelerators/sbvh/platform.h:78-90
 *   Mesh, Scene::add_mesh       core/mesh.h:45-62, core/scene.cpp:83-123
 *   BVH(Scene*, Platform, BuildParams)          accelerators/sbvh/bvh.h:83-115
 *   CudaBvh(const BVH&, BVHLayout) / (file, ok) accelerators/sbvh/cudabvh.h:76-98
 *   Ray, RayBuffer              core/primitives.h:145-208, core/buffer.h:114-118
 *   IntersectionBuffer          core/intersection.h:63-80 (field names kept,
 *                               including m_geomteric_normal)
 *   CudaTracer(const CudaBvh&, allocator) / trace(...) / get_bvh()
 *                               accelerators/sbvh/cudatracer.h:67-101
 *
 * Differences: failures throw std::runtime_error with rb2_last_error() text
 * (the reference printed and asserted); every object owns its memory (no
 * MemoryAllocator; the allocator argument is accepted and ignored); SceneBuffer
 * wraps the device scene handle made by Scene::gpu_prepare; trace() returns
 * its CUDA-event time in milliseconds.
 */
#pragma once

#include "rb2.h"
#include "rb2_render.h"

#include <cuda_runtime.h>
#include <vector_types.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace renderbox2 {

using GIndexType = uint32_t;
using GIndexVec3Type = uint3;

inline void rb2_throw_if(int rc)
{
    if (rc != RB2_OK) throw std::runtime_error(std::string("librb2: ") + rb2_last_error());
}

enum class BVHLayout { BVHLayout_Compact, BVHLayout_Compact2, BVHLayout_Max };

class Platform {
public:
    Platform()
        : m_name("Default"), m_sah_node_cost(1.f), m_sah_triangle_cost(1.f), m_node_batch_size(1),
          m_tri_batch_size(1), m_min_leaf_size(1), m_max_leaf_size(0x7FFFFFF)
    {
    }
    std::string m_name;
    float m_sah_node_cost;
    float m_sah_triangle_cost;
    int m_node_batch_size;
    int m_tri_batch_size;
    int m_min_leaf_size;
    int m_max_leaf_size;
};

// The fields Scene::add_mesh and the trace read; indices are scene-global, as
// the reference's readers produce them.
struct Mesh {
    std::string m_name;
    std::vector<float3> m_vertices;
    std::vector<GIndexVec3Type> m_vtx_indices;
    std::vector<uint32_t> m_mat_ids;
};

struct SceneBuffer {
    rb2_scene_dev* m_scene;
    GIndexType m_size;
    uint32_t m_num_lights;
};

class Scene {
public:
    Scene() = default;
    template <class Allocator>
    explicit Scene(Allocator&) {}
    ~Scene() { if (m_dev) rb2_scene_destroy(m_dev); }
    Scene(const Scene&) = delete;
    Scene& operator=(const Scene&) = delete;

    void add_mesh(const Mesh& M, bool is_emissive = false)
    {
        const GIndexType base = (GIndexType)h_vtx_indices.size();
        h_vertices.insert(h_vertices.end(), M.m_vertices.begin(), M.m_vertices.end());
        h_vtx_indices.insert(h_vtx_indices.end(), M.m_vtx_indices.begin(), M.m_vtx_indices.end());
        for (size_t i = 0; i < M.m_vtx_indices.size(); i++)
            h_tri_material_ids.push_back(i < M.m_mat_ids.size() ? M.m_mat_ids[i] : 0u);
        if (is_emissive)
            for (size_t j = 0; j < M.m_vtx_indices.size(); j++) h_light_ids.push_back(base + (GIndexType)j);
    }

    GIndexType get_num_triangles() const { return (GIndexType)h_vtx_indices.size(); }
    GIndexType get_num_vertices() const { return (GIndexType)h_vertices.size(); }
    uint32_t get_num_lights() const { return (uint32_t)h_light_ids.size(); }
    const float3* get_tri_vertices() const { return h_vertices.data(); }
    const GIndexVec3Type* get_tri_vtx_indices() const { return h_vtx_indices.data(); }
    const uint32_t* get_tri_material_ids() const { return h_tri_material_ids.data(); }
    const GIndexType* get_light_ids_to_primitive_ids() const { return h_light_ids.data(); }

    // Scene::gpu_prepare (core/scene.cpp:166-339) for the Lambertian +
    // diffuse-area-light subset: per-material albedo / emission (rgb, may be
    // empty for the defaults).  Lights are the triangles whose material emits.
    void gpu_prepare(const std::vector<float3>& albedo = {}, const std::vector<float3>& emission = {})
    {
        if (m_dev) { rb2_scene_destroy(m_dev); m_dev = nullptr; }
        uint32_t n_mat = 1;
        for (uint32_t m : h_tri_material_ids) n_mat = m + 1 > n_mat ? m + 1 : n_mat;
        if (albedo.size() > n_mat) n_mat = (uint32_t)albedo.size();
        if (emission.size() > n_mat) n_mat = (uint32_t)emission.size();
        std::vector<float> a, e;
        if (!albedo.empty()) { a.assign(3 * (size_t)n_mat, 0.5f); std::memcpy(a.data(), albedo.data(), 12 * albedo.size()); }
        if (!emission.empty()) { e.assign(3 * (size_t)n_mat, 0.0f); std::memcpy(e.data(), emission.data(), 12 * emission.size()); }
        rb2_throw_if(rb2_scene_create(reinterpret_cast<const float*>(h_vertices.data()), get_num_vertices(),
                                      reinterpret_cast<const uint32_t*>(h_vtx_indices.data()), get_num_triangles(),
                                      h_tri_material_ids.data(), n_mat, a.empty() ? nullptr : a.data(),
                                      e.empty() ? nullptr : e.data(), &m_dev));
    }
    SceneBuffer gpu_get_buffer() const
    {
        if (!m_dev) throw std::runtime_error("Scene::gpu_get_buffer before gpu_prepare");
        return SceneBuffer{m_dev, get_num_triangles(), get_num_lights()};
    }

private:
    std::vector<float3> h_vertices;
    std::vector<GIndexVec3Type> h_vtx_indices;
    std::vector<uint32_t> h_tri_material_ids;
    std::vector<GIndexType> h_light_ids;
    rb2_scene_dev* m_dev = nullptr;
};

class BVH {
public:
    struct Stats {
        float m_sah_cost = 0.f;
        GIndexType m_num_leaf_nodes = 0;
        GIndexType m_num_child_nodes = 0;
        GIndexType m_num_tris = 0;
    };
    struct BuildParams {
        Stats* m_stats = nullptr;
        bool m_enable_prints = true;
        float m_split_alpha = 1.0e-5f;
    };

    BVH(Scene* scene, const Platform& platform, const BuildParams& params) : m_scene(scene), m_platform(platform)
    {
        rb2_build_params p;
        rb2_throw_if(rb2_build_params_default(&p));
        p.sah_node_cost = platform.m_sah_node_cost;
        p.sah_triangle_cost = platform.m_sah_triangle_cost;
        p.min_leaf_size = (uint32_t)platform.m_min_leaf_size;
        p.max_leaf_size = (uint32_t)platform.m_max_leaf_size;
        p.split_alpha = params.m_split_alpha;
        rb2_throw_if(rb2_bvh_build(reinterpret_cast<const float*>(scene->get_tri_vertices()), scene->get_num_vertices(),
                                   reinterpret_cast<const uint32_t*>(scene->get_tri_vtx_indices()),
                                   scene->get_num_triangles(), &p, &m_bvh));
        if (params.m_stats) {
            rb2_bvh_counts c;
            rb2_throw_if(rb2_bvh_counts_get(m_bvh, &c));
            params.m_stats->m_sah_cost = c.sah;
            params.m_stats->m_num_leaf_nodes = c.n_leaves;
            params.m_stats->m_num_child_nodes = c.n_inner;
            params.m_stats->m_num_tris = c.n_tri_refs;
        }
    }
    ~BVH() { rb2_host_bvh_free(m_bvh); }
    BVH(const BVH&) = delete;
    BVH& operator=(const BVH&) = delete;

    Scene* get_scene() const { return m_scene; }
    const Platform& get_platform() const { return m_platform; }
    const rb2_host_bvh* handle() const { return m_bvh; }

private:
    Scene* m_scene;
    Platform m_platform;
    rb2_host_bvh* m_bvh = nullptr;
};

class CudaBvh {
public:
    CudaBvh(const BVH& bvh, BVHLayout layout) : m_layout(layout)
    {
        if (layout != BVHLayout::BVHLayout_Compact2) throw std::runtime_error("only BVHLayout_Compact2 is produced");
        copy_from(bvh.handle());
    }
    CudaBvh(const std::string& filename, bool& isLoadedProperly) : m_layout(BVHLayout::BVHLayout_Compact2)
    {
        rb2_host_bvh* b = nullptr;
        isLoadedProperly = rb2_bvh_load(filename.c_str(), &b) == RB2_OK;
        if (isLoadedProperly) { copy_from(b); rb2_host_bvh_free(b); }
    }

    // Writes the reference's text cache format (cudabvh.cpp:176-214).
    void serialize(const std::string& filename)
    {
        rb2_host_bvh* b = to_host();
        const int rc = rb2_bvh_save_text(b, filename.c_str());
        rb2_host_bvh_free(b);
        rb2_throw_if(rc);
    }

    const std::vector<uint4>& get_node_buffer() const { return m_nodes; }
    const std::vector<uint4>& get_tri_woop_buffer() const { return m_tri_woop; }
    const std::vector<GIndexType>& get_tri_index_buffer() const { return m_tri_index; }
    BVHLayout get_layout() const { return m_layout; }

    // Validated host BVH of these buffers (caller frees with rb2_host_bvh_free).
    rb2_host_bvh* to_host() const
    {
        rb2_host_bvh* b = nullptr;
        rb2_throw_if(rb2_bvh_from_buffers(reinterpret_cast<const uint32_t*>(m_nodes.data()), m_nodes.size(),
                                          reinterpret_cast<const uint32_t*>(m_tri_woop.data()), m_tri_woop.size(),
                                          m_tri_index.data(), m_tri_index.size(), &b));
        return b;
    }

private:
    void copy_from(const rb2_host_bvh* b)
    {
        rb2_bvh_counts c;
        rb2_throw_if(rb2_bvh_counts_get(b, &c));
        m_nodes.resize(c.n_nodes_u4);
        m_tri_woop.resize(c.n_woop_u4);
        m_tri_index.resize(c.n_triidx);
        std::memcpy(m_nodes.data(), rb2_bvh_nodes(b), 16 * c.n_nodes_u4);
        std::memcpy(m_tri_woop.data(), rb2_bvh_woop(b), 16 * c.n_woop_u4);
        std::memcpy(m_tri_index.data(), rb2_bvh_triidx(b), 4 * c.n_triidx);
    }
    BVHLayout m_layout;
    std::vector<uint4> m_nodes;
    std::vector<uint4> m_tri_woop;
    std::vector<GIndexType> m_tri_index;
};

struct Ray {
    float4 m_origin;     // origin.xyz, tmin
    float4 m_direction;  // direction.xyz, tmax
};

struct RayBuffer {
    Ray* m_data;
    GIndexType m_size;
};

struct IntersectionBuffer {
    float* m_position[3];
    float* m_geomteric_normal[3];
    float* m_shading_normal[3];
    float* m_tangent[3];              // not written by trace
    float* m_bitangent[3];            // not written by trace
    float* m_incoming_direction[3];
    float2* m_uv;
    GIndexType* m_primitive_id;
    uint32_t* m_primitive_material_id;
    uint8_t* m_front;
    uint8_t* m_intersected;
    float* m_epsilon;
    uint32_t* m_depth;                // not written by trace
    float4* m_contribution;           // not written by trace
    GIndexType m_size;
};

class CudaTracer {
public:
    explicit CudaTracer(const CudaBvh& bvh)
    {
        rb2_host_bvh* b = bvh.to_host();
        const int rc = rb2_tracer_create(b, &m_tracer);
        rb2_host_bvh_free(b);
        rb2_throw_if(rc);
    }
    template <class Allocator>
    CudaTracer(const CudaBvh& bvh, Allocator&) : CudaTracer(bvh) {}
    ~CudaTracer() { rb2_tracer_destroy(m_tracer); }
    CudaTracer(const CudaTracer&) = delete;
    CudaTracer& operator=(const CudaTracer&) = delete;

    // Traces rb.m_size rays on the legacy default stream and waits for them;
    // fills isects as the reference's bulk kernel does.  Returns milliseconds.
    float trace(const RayBuffer& rb, IntersectionBuffer& isects, SceneBuffer& scene_data, uint8_t* stencil,
                bool any_hit = true)
    {
        rb2_isect_buffer o;
        for (int k = 0; k < 3; k++) {
            o.position[k] = isects.m_position[k];
            o.geometric_normal[k] = isects.m_geomteric_normal[k];
            o.shading_normal[k] = isects.m_shading_normal[k];
            o.incoming_direction[k] = isects.m_incoming_direction[k];
        }
        o.uv = reinterpret_cast<float*>(isects.m_uv);
        o.primitive_id = isects.m_primitive_id;
        o.primitive_material_id = isects.m_primitive_material_id;
        o.front = isects.m_front;
        o.intersected = isects.m_intersected;
        o.epsilon = isects.m_epsilon;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, 0);
        const int rc = rb2_trace_isect(m_tracer, scene_data.m_scene, reinterpret_cast<const float*>(rb.m_data),
                                       rb.m_size, any_hit ? 1 : 0, stencil, &o, nullptr);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        rb2_throw_if(rc);
        uint32_t status = 0;
        rb2_throw_if(rb2_tracer_status(m_tracer, &status, nullptr));
        if (status) throw std::runtime_error("librb2: device status word set");
        return ms;
    }

    // Device view of the BVH for kernels calling rb2::trace_ray (rb2_device.cuh).
    rb2_dev_bvh get_bvh() const
    {
        rb2_dev_bvh d;
        rb2_throw_if(rb2_tracer_dev_bvh(m_tracer, &d));
        return d;
    }
    rb2_tracer* handle() const { return m_tracer; }

private:
    rb2_tracer* m_tracer = nullptr;
};

}  // namespace renderbox2
