// Host-only use of the reference-named C++ classes (rb2.hpp): a scene of two
// meshes, BVH(Scene*, Platform, BuildParams), CudaBvh(bvh, Compact2), the
// getters, serialize() to the reference's text cache and CudaBvh(file, ok).
// Prints one line of counts and FNV-1a hashes of the buffers.
#include "rb2.hpp"

#include <cstdio>
#include <cstdlib>

using namespace renderbox2;

static uint64_t fnv(const void* p, size_t n, uint64_t h = 1469598103934665603ull)
{
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ull; }
    return h;
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    const int g = 24;  // grid of g x g cells -> 2 g^2 triangles
    Mesh ground;
    for (int z = 0; z <= g; z++)
        for (int x = 0; x <= g; x++)
            ground.m_vertices.push_back(make_float3(x / (float)g, 0.05f * ((x * 7 + z * 3) % 5) / 4.0f, z / (float)g));
    for (int z = 0; z < g; z++)
        for (int x = 0; x < g; x++) {
            const uint32_t a = z * (g + 1) + x, b = a + 1, c = a + g + 1, d = c + 1;
            ground.m_vtx_indices.push_back(make_uint3(a, c, b));
            ground.m_vtx_indices.push_back(make_uint3(b, c, d));
        }
    Mesh light;
    const uint32_t base = (uint32_t)ground.m_vertices.size();
    light.m_vertices = {make_float3(0.4f, 0.9f, 0.4f), make_float3(0.6f, 0.9f, 0.4f), make_float3(0.4f, 0.9f, 0.6f),
                        make_float3(0.6f, 0.9f, 0.6f)};
    light.m_vtx_indices = {make_uint3(base, base + 2, base + 1), make_uint3(base + 1, base + 2, base + 3)};
    light.m_mat_ids = {1, 1};
    Scene scene;
    scene.add_mesh(ground);
    scene.add_mesh(light, true);

    BVH::Stats stats;
    BVH::BuildParams params;
    params.m_stats = &stats;
    BVH bvh(&scene, Platform(), params);
    CudaBvh cb(bvh, BVHLayout::BVHLayout_Compact2);
    cb.serialize(argv[1]);
    bool ok = false;
    CudaBvh loaded(argv[1], ok);
    if (!ok) { std::printf("load failed\n"); return 1; }
    const bool same = loaded.get_node_buffer().size() == cb.get_node_buffer().size() &&
                      fnv(loaded.get_node_buffer().data(), 16 * loaded.get_node_buffer().size()) ==
                          fnv(cb.get_node_buffer().data(), 16 * cb.get_node_buffer().size()) &&
                      fnv(loaded.get_tri_woop_buffer().data(), 16 * loaded.get_tri_woop_buffer().size()) ==
                          fnv(cb.get_tri_woop_buffer().data(), 16 * cb.get_tri_woop_buffer().size());
    bool threw = false;
    try {
        CudaBvh bad(bvh, BVHLayout::BVHLayout_Compact);
    } catch (const std::runtime_error&) {
        threw = true;
    }
    std::printf("tris %u lights %u nodes %zu woop %zu triidx %zu leaves %u sah %.6f roundtrip %d threw %d "
                "hash %016llx %016llx\n",
                scene.get_num_triangles(), scene.get_num_lights(), cb.get_node_buffer().size(),
                cb.get_tri_woop_buffer().size(), cb.get_tri_index_buffer().size(), stats.m_num_leaf_nodes,
                stats.m_sah_cost, same ? 1 : 0, threw ? 1 : 0,
                (unsigned long long)fnv(cb.get_node_buffer().data(), 16 * cb.get_node_buffer().size()),
                (unsigned long long)fnv(cb.get_tri_woop_buffer().data(), 16 * cb.get_tri_woop_buffer().size()));
    return 0;
}
