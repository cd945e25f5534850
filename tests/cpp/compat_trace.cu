// Device-side use of the public headers from a user's own CUDA code:
// rb2.hpp's CudaTracer::trace(RayBuffer, IntersectionBuffer&, SceneBuffer&,
// stencil, any_hit) and a user kernel calling the header-only rb2::trace_ray
// (rb2_device.cuh) with CudaTracer::get_bvh() and the scene's device view.
// Prints one line: rays, hits, and mismatch counts between the two paths.
#include "rb2.hpp"
#include "rb2_device.cuh"

#include <cstdio>
#include <vector>

using namespace renderbox2;

__global__ void user_kernel(rb2_dev_bvh bvh, rb2_dev_scene scene, const Ray* rays, uint32_t n, uint32_t* prim,
                            uint8_t* hit, float* px)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rb2::Intersection is;
    const bool h = rb2::trace_ray(rays[i].m_origin, rays[i].m_direction, false, &is, bvh, scene);
    hit[i] = h ? 1 : 0;
    prim[i] = h ? is.primitive_id : 0xFFFFFFFFu;
    px[i] = h ? is.position.x : 0.0f;
}

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { std::printf("cuda %s\n", cudaGetErrorString(e_)); return 1; } } while (0)

int main()
{
    const int g = 64;
    Mesh ground;
    for (int z = 0; z <= g; z++)
        for (int x = 0; x <= g; x++)
            ground.m_vertices.push_back(make_float3(x / (float)g, 0.1f * (((x * 13 + z * 7) % 11) / 10.0f), z / (float)g));
    for (int z = 0; z < g; z++)
        for (int x = 0; x < g; x++) {
            const uint32_t a = z * (g + 1) + x, b = a + 1, c = a + g + 1, d = c + 1;
            ground.m_vtx_indices.push_back(make_uint3(a, c, b));
            ground.m_vtx_indices.push_back(make_uint3(b, c, d));
            ground.m_mat_ids.push_back((x + z) % 3);
            ground.m_mat_ids.push_back((x + z) % 3);
        }
    Scene scene;
    scene.add_mesh(ground);
    scene.gpu_prepare();
    BVH bvh(&scene, Platform(), BVH::BuildParams());
    CudaBvh cb(bvh, BVHLayout::BVHLayout_Compact2);
    CudaTracer tracer(cb);

    const uint32_t n = 100000;
    std::vector<Ray> h_rays(n);
    uint64_t s = 12345;
    auto rnd = [&]() { s = s * 6364136223846793005ull + 1442695040888963407ull; return (float)((s >> 40) & 0xFFFFFF) / 16777216.0f; };
    for (uint32_t i = 0; i < n; i++) {
        const float ox = rnd() * 1.2f - 0.1f, oz = rnd() * 1.2f - 0.1f;
        const float dx = rnd() - 0.5f, dz = rnd() - 0.5f;
        h_rays[i].m_origin = make_float4(ox, 0.5f, oz, 0.0f);
        h_rays[i].m_direction = make_float4(dx, -1.0f, dz, i % 5 == 0 ? 0.2f : 1e30f);
    }
    Ray* d_rays;
    CK(cudaMalloc(&d_rays, n * sizeof(Ray)));
    CK(cudaMemcpy(d_rays, h_rays.data(), n * sizeof(Ray), cudaMemcpyHostToDevice));
    IntersectionBuffer ib{};
    std::vector<void*> allocs;
    auto dalloc = [&](size_t bytes) { void* p = nullptr; cudaMalloc(&p, bytes); cudaMemset(p, 0xFF, bytes); allocs.push_back(p); return p; };
    for (int k = 0; k < 3; k++) {
        ib.m_position[k] = (float*)dalloc(4 * n);
        ib.m_geomteric_normal[k] = (float*)dalloc(4 * n);
        ib.m_shading_normal[k] = (float*)dalloc(4 * n);
        ib.m_incoming_direction[k] = (float*)dalloc(4 * n);
    }
    ib.m_uv = (float2*)dalloc(8 * n);
    ib.m_primitive_id = (GIndexType*)dalloc(4 * n);
    ib.m_primitive_material_id = (uint32_t*)dalloc(4 * n);
    ib.m_front = (uint8_t*)dalloc(n);
    ib.m_intersected = (uint8_t*)dalloc(n);
    ib.m_epsilon = (float*)dalloc(4 * n);
    ib.m_size = n;
    RayBuffer rb{d_rays, n};
    SceneBuffer sb = scene.gpu_get_buffer();
    const float ms = tracer.trace(rb, ib, sb, nullptr, false);

    uint32_t* d_prim; uint8_t* d_hit; float* d_px;
    CK(cudaMalloc(&d_prim, 4 * n)); CK(cudaMalloc(&d_hit, n)); CK(cudaMalloc(&d_px, 4 * n));
    rb2_dev_scene dsc;
    rb2_throw_if(rb2_scene_dev_view(sb.m_scene, &dsc));
    user_kernel<<<(n + 127) / 128, 128>>>(tracer.get_bvh(), dsc, d_rays, n, d_prim, d_hit, d_px);
    CK(cudaDeviceSynchronize());

    std::vector<uint32_t> p1(n), p2(n); std::vector<uint8_t> h1(n), h2(n); std::vector<float> x1(n), x2(n);
    CK(cudaMemcpy(p1.data(), ib.m_primitive_id, 4 * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h1.data(), ib.m_intersected, n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(x1.data(), ib.m_position[0], 4 * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(p2.data(), d_prim, 4 * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h2.data(), d_hit, n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(x2.data(), d_px, 4 * n, cudaMemcpyDeviceToHost));
    uint32_t hits = 0, bad_hit = 0, bad_prim = 0, bad_pos = 0;
    for (uint32_t i = 0; i < n; i++) {
        hits += h1[i];
        bad_hit += h1[i] != h2[i];
        if (h1[i] && h2[i]) {
            if (p1[i] != p2[i]) bad_prim++;
            else if (x1[i] != x2[i]) bad_pos++;
        }
    }
    std::printf("rays %u hits %u bad_hit %u bad_prim %u bad_pos %u ms %.3f\n", n, hits, bad_hit, bad_prim, bad_pos, ms);
    for (void* p : allocs) cudaFree(p);
    cudaFree(d_rays); cudaFree(d_prim); cudaFree(d_hit); cudaFree(d_px);
    return 0;
}
