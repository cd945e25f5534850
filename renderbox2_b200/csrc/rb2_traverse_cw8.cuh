// Persistent traversal of the compressed 8-wide layout (RB2_NODE_ORDER_CW8,
// node format in rb2_cw8.cpp), after Ylitie, Karras and Laine, "Efficient
// Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs" (HPG 2017).
//
// Per lane: a node group (child_base of a visited node and a mask of its hit
// inner children, bits 24-31 in octant-permuted order, the node's inner-child
// mask in bits 0-7), a triangle group (tri_base, the node's triangle mask and
// the hit triangles among its bits) and a stack of node groups.  A node test
// yields an 8-bit mask of hit slots; two table lookups turn it into both
// groups (instead of the paper's per-child meta-byte decoding).  The warp walks nodes
// until every busy lane holds triangles (the counterpart of the binary
// kernel's postponed leaf) or too few lanes still want nodes, then tests
// triangles, then refills lanes from the
// ray source as the binary kernel does (same RaySource policy, same dynamic
// fetch).  Triangles are the binary layout's Woop rows with the same test
// arithmetic, so an accepted hit has the same t, u, v bits; boxes are
// conservative, so the closest hit equals the binary traversal's except for
// exact ties in t.
#pragma once

#include "rb2_traverse.cuh"

namespace rb2dev {

// Node groups on the stack: at most one per wide level.  The host refuses a
// layout deeper than this (rb2_tracer_set_node_order).
constexpr int kStackSizeCw8 = 72;
constexpr uint32_t kCw8NodeWords = 20;

// Two quantized planes (bytes 2h and 2h + 1 of w) as floats 32768 + q: each
// byte is moved into bits 8-15 of the float 32768 (0x47000000), whose unit in
// the last place there is 1, so one byte permute yields the plane exactly.
// The 32768 cells are folded into the per-node slab offset (the layout widens
// every box by 2^-14 of its node for that offset's rounding).
constexpr float kCw8PlaneBias = 32768.0f;
__device__ __forceinline__ float cw8_plane(uint32_t w, int b)
{
    return __uint_as_float(__byte_perm(w, 0x47000000u, 0x7504u | ((uint32_t)b << 4)));
}
__device__ __forceinline__ float2 cw8_planes(uint32_t w, int h)
{
    return make_float2(cw8_plane(w, 2 * h), cw8_plane(w, 2 * h + 1));
}

// Two IEEE single-precision FMAs in one paired instruction (sm_100 f32x2).
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
    unsigned long long ra, rb, rc, rd;
    asm("mov.b64 %0, {%1, %2};" : "=l"(ra) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(rb) : "f"(b.x), "f"(b.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(rc) : "f"(c.x), "f"(c.y));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(rd) : "l"(ra), "l"(rb), "l"(rc));
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(rd));
    return r;
}

// Woop test of one triangle (the binary leaf loop's arithmetic); updates
// hitT / hitIndex and returns true when it accepts.
__device__ __forceinline__ bool cw8_triangle(Lane& L, int triAddr)
{
    const float4* wp = L.woop + triAddr;
    const float4 v00 = __ldg(wp + 0);
    const float4 v11 = __ldg(wp + 1);
    const float4 v22 = __ldg(wp + 2);
    const float Oz = __fmaf_rn(-L.oz, v00.z, __fmaf_rn(-L.oy, v00.y, __fmaf_rn(-L.ox, v00.x, v00.w)));
    const float Dz = __fmaf_rn(L.dz, v00.z, __fmaf_rn(L.dy, v00.y, __fmul_rn(L.dx, v00.x)));
    const float t = __fmul_rn(Oz, __frcp_rn(Dz));  // IEEE 1 / Dz, as __fdiv_rn(1, Dz)
    if (!(t > L.tmin && t < L.hitT)) return false;
    const float Ox = __fmaf_rn(L.oz, v11.z, __fmaf_rn(L.oy, v11.y, __fmaf_rn(L.ox, v11.x, v11.w)));
    const float Dx = __fmaf_rn(L.dz, v11.z, __fmaf_rn(L.dy, v11.y, __fmul_rn(L.dx, v11.x)));
    const float u = __fmaf_rn(t, Dx, Ox);
    if (!(u >= 0.0f)) return false;
    const float Oy = __fmaf_rn(L.oz, v22.z, __fmaf_rn(L.oy, v22.y, __fmaf_rn(L.ox, v22.x, v22.w)));
    const float Dy = __fmaf_rn(L.dz, v22.z, __fmaf_rn(L.dy, v22.y, __fmul_rn(L.dx, v22.x)));
    const float v = __fmaf_rn(t, Dy, Oy);
    if (!(v >= 0.0f && __fadd_rn(u, v) <= 1.0f)) return false;
    L.hitT = t;
    L.hitIndex = triAddr;
    return true;
}

// kOodSlab: form a node's slab offsets from the ray's precomputed o * idir
// (one FMA per axis) instead of (plane - o) * idir.  The boxes' margin covers
// the rounding of either form.  The integrators' kernels take it (fewer
// instructions, no added spills); in the batched job kernel it adds spills
// and costs more than it saves, so that kernel keeps the subtraction.
//
// node_threshold: a node phase also ends, so that pending triangle groups are
// tested, once fewer than this many lanes still want nodes while some lane
// holds triangles (0 or 1: only when no lane wants nodes).  Testing triangles
// earlier shortens the lanes' hit distances sooner and keeps more lanes busy
// in the node phases; a lane's own order of node visits and triangle tests is
// unchanged, so results do not depend on it.
template <class Source, bool kOodSlab = false>
__device__ __forceinline__ void persistent_trace_cw8(Source& src, uint32_t fetch_threshold, uint32_t node_threshold,
                                                     unsigned int* status)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    uint2 stack[kStackSizeCw8];
    int sp = 0;
    Lane L;
    L.hitIndex = -1;
    uint32_t ng_base = 0, ng_bits = 0, tg_base = 0, tg_bits = 0, tg_mask = 0;
    uint32_t tg2_base = 0, tg2_bits = 0, tg2_mask = 0;  // a second pending triangle group
    uint32_t oct_inv = 0;  // 7 xor the ray's direction octant (set when a ray is fetched)
    bool has_ray = false, retired = false;

    // Tables shared by the block: s_perm[o][m] moves bit s of an 8-bit slot
    // mask to bit s ^ o (inner children in ray-octant order); s_spread[m]
    // moves bit s to bit 3s (a slot's three triangle bits).
    __shared__ uint8_t s_perm[8 * 256];
    __shared__ uint32_t s_spread[256];
    for (uint32_t i = threadIdx.x; i < 8u * 256u; i += blockDim.x) {
        const uint32_t o = i >> 8, m = i & 255u;
        uint32_t r = 0;
        for (uint32_t s = 0; s < 8; s++) r |= ((m >> s) & 1u) << (s ^ o);
        s_perm[i] = (uint8_t)r;
    }
    for (uint32_t m = threadIdx.x; m < 256u; m += blockDim.x) {
        uint32_t r = 0;
        for (uint32_t s = 0; s < 8; s++) r |= ((m >> s) & 1u) << (3 * s);
        s_spread[m] = r;
    }
    __syncthreads();

    for (;;) {
        // ---- refill: lanes without a ray claim the next slots from the queue.
        const bool need = !has_ray && !retired;
        const unsigned needm = __ballot_sync(kFull, need);
        if (needm) {
            const int leader = __ffs(needm) - 1;
            unsigned long long b1 = 0, b2 = 0;
            unsigned n1 = 0;
            if ((int)lane == leader) src.claim((unsigned)__popc(needm), b1, n1, b2);
            b1 = __shfl_sync(kFull, b1, leader);
            b2 = __shfl_sync(kFull, b2, leader);
            n1 = __shfl_sync(kFull, n1, leader);
            if (need) {
                const unsigned rank = (unsigned)__popc(needm & lt_mask);
                const unsigned long long slot = rank < n1 ? b1 + rank : b2 + (rank - n1);
                const int r = src.fetch(slot, L);
                if (r == 0) {
                    retired = true;
                } else if (r > 0) {
                    sp = 0;
                    ng_base = 0;             // the root: node 0, reached through bit 31
                    ng_bits = 0x80000000u;   // with an empty inner-child mask
                    tg_bits = 0;
                    tg2_bits = 0;
                    oct_inv = 7u ^ ((__float_as_uint(L.idx) >> 31) | ((__float_as_uint(L.idy) >> 31) << 1) |
                                    ((__float_as_uint(L.idz) >> 31) << 2));
                    has_ray = true;
                }
            }
        }
        if (__all_sync(kFull, retired)) break;

        while (__any_sync(kFull, has_ray)) {
            // ---- nodes, until every busy lane holds triangles or is done, or
            //      fewer than node_threshold lanes want nodes while some lane
            //      holds triangles.
            for (;;) {
                const bool in = has_ray && tg2_bits == 0 && (ng_bits > 0x00FFFFFFu || sp > 0);
                const unsigned inm = __ballot_sync(kFull, in);
                if (inm == 0) break;
                if ((unsigned)__popc(inm) < node_threshold && __any_sync(kFull, has_ray && tg_bits != 0)) break;
                if (in) {
                    if (ng_bits <= 0x00FFFFFFu) {
                        --sp;
                        ng_base = stack[sp].x;
                        ng_bits = stack[sp].y;
                    }
                    const uint32_t k = 31u - (uint32_t)__clz(ng_bits);
                    ng_bits &= ~(1u << k);
                    const uint32_t slot = (k - 24u) ^ oct_inv;
                    const uint32_t node = ng_base + (uint32_t)__popc(ng_bits & ((1u << slot) - 1u));
                    bool ok = true;
                    if (ng_bits > 0x00FFFFFFu) {
                        if (sp >= kStackSizeCw8) {
                            // Unreachable for layouts whose depth was validated; a corrupt
                            // layout abandons the ray and reports it.
                            atomicOr(status, kStatusStack);
                            ok = false;
                        } else {
                            stack[sp].x = ng_base;
                            stack[sp].y = ng_bits;
                            ++sp;
                        }
                    }
                    if (!ok) {
                        L.hitIndex = -1;
                        ng_bits = 0;
                        sp = 0;
                    } else {
                        const float4* np = L.nodes + (size_t)node * (kCw8NodeWords / 4);
                        const float4 h0 = __ldg(np + 0), h1 = __ldg(np + 1);
                        const float4 qx = __ldg(np + 2), qy = __ldg(np + 3), qz = __ldg(np + 4);
                        const uint32_t ew = __float_as_uint(h0.w);
                        const float sx = __fmul_rn(__uint_as_float((ew & 0xFFu) << 23), L.idx);
                        const float sy = __fmul_rn(__uint_as_float(((ew >> 8) & 0xFFu) << 23), L.idy);
                        const float sz = __fmul_rn(__uint_as_float(((ew >> 16) & 0xFFu) << 23), L.idz);
                        // Slab offsets less the plane bias (planes arrive as 32768 + q cells).
                        float ax, ay, az;
                        if constexpr (kOodSlab) {
                            ax = __fmaf_rn(-kCw8PlaneBias, sx, __fmaf_rn(h0.x, L.idx, -L.oodx));
                            ay = __fmaf_rn(-kCw8PlaneBias, sy, __fmaf_rn(h0.y, L.idy, -L.oody));
                            az = __fmaf_rn(-kCw8PlaneBias, sz, __fmaf_rn(h0.z, L.idz, -L.oodz));
                        } else {
                            ax = __fmaf_rn(-kCw8PlaneBias, sx, __fmul_rn(__fsub_rn(h0.x, L.ox), L.idx));
                            ay = __fmaf_rn(-kCw8PlaneBias, sy, __fmul_rn(__fsub_rn(h0.y, L.oy), L.idy));
                            az = __fmaf_rn(-kCw8PlaneBias, sz, __fmul_rn(__fsub_rn(h0.z, L.oz), L.idz));
                        }
                        // Near and far plane words per axis (the high plane is near for a
                        // negative direction), children 0-3 in the first word, 4-7 in the second.
                        const bool rx = L.idx < 0.0f, ry = L.idy < 0.0f, rz = L.idz < 0.0f;
                        const uint32_t nx0 = __float_as_uint(rx ? qx.z : qx.x), nx1 = __float_as_uint(rx ? qx.w : qx.y);
                        const uint32_t fx0 = __float_as_uint(rx ? qx.x : qx.z), fx1 = __float_as_uint(rx ? qx.y : qx.w);
                        const uint32_t ny0 = __float_as_uint(ry ? qy.z : qy.x), ny1 = __float_as_uint(ry ? qy.w : qy.y);
                        const uint32_t fy0 = __float_as_uint(ry ? qy.x : qy.z), fy1 = __float_as_uint(ry ? qy.y : qy.w);
                        const uint32_t nz0 = __float_as_uint(rz ? qz.z : qz.x), nz1 = __float_as_uint(rz ? qz.w : qz.y);
                        const uint32_t fz0 = __float_as_uint(rz ? qz.x : qz.z), fz1 = __float_as_uint(rz ? qz.y : qz.w);
                        uint32_t hm = 0;  // slots whose box the ray enters
                        const float2 sx2 = make_float2(sx, sx), sy2 = make_float2(sy, sy), sz2 = make_float2(sz, sz);
                        const float2 ax2 = make_float2(ax, ax), ay2 = make_float2(ay, ay), az2 = make_float2(az, az);
#pragma unroll
                        for (int s = 0; s < 8; s += 2) {
                            const int w = s >> 2, hh = (s >> 1) & 1;
                            const float2 nx = cw8_planes(w ? nx1 : nx0, hh), fx = cw8_planes(w ? fx1 : fx0, hh);
                            const float2 ny = cw8_planes(w ? ny1 : ny0, hh), fy = cw8_planes(w ? fy1 : fy0, hh);
                            const float2 nz = cw8_planes(w ? nz1 : nz0, hh), fz = cw8_planes(w ? fz1 : fz0, hh);
                            // Slab distances of the two children, one paired FMA per plane.
                            const float2 tnx2 = fma2(nx, sx2, ax2), tfx2 = fma2(fx, sx2, ax2);
                            const float2 tny2 = fma2(ny, sy2, ay2), tfy2 = fma2(fy, sy2, ay2);
                            const float2 tnz2 = fma2(nz, sz2, az2), tfz2 = fma2(fz, sz2, az2);
#pragma unroll
                            for (int e = 0; e < 2; e++) {
                                const float tnx = e ? tnx2.y : tnx2.x, tfx = e ? tfx2.y : tfx2.x;
                                const float tny = e ? tny2.y : tny2.x, tfy = e ? tfy2.y : tfy2.x;
                                const float tnz = e ? tnz2.y : tnz2.x, tfz = e ? tfz2.y : tfz2.x;
                                const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, L.tmin));
                                const float tf = fminf(fminf(tfx, tfy), fminf(tfz, L.hitT));
                                if (tn <= tf) hm |= 1u << (s + e);
                            }
                        }
                        // Hit inner slots, octant-permuted, into bits 24-31 (above the
                        // node's inner-child mask); hit leaf slots' triangles from the
                        // node's triangle mask (inner and empty slots have no bits there).
                        const uint32_t imask = ew >> 24;
                        ng_base = __float_as_uint(h1.x);
                        ng_bits = ((uint32_t)s_perm[(oct_inv << 8) | (hm & imask)] << 24) | imask;
                        const uint32_t tmask = __float_as_uint(h1.z), tbits = (s_spread[hm] * 7u) & tmask;
                        if (tbits) {
                            if (tg_bits == 0) {
                                tg_base = __float_as_uint(h1.y); tg_mask = tmask; tg_bits = tbits;
                            } else {
                                tg2_base = __float_as_uint(h1.y); tg2_mask = tmask; tg2_bits = tbits;
                            }
                        }
                    }
                }
            }

            // ---- triangles of the current group, then finish lanes with no work left.
            if (has_ray) {
                for (;;) {
                    if (tg_bits == 0) {
                        if (tg2_bits == 0) break;
                        tg_base = tg2_base; tg_mask = tg2_mask; tg_bits = tg2_bits; tg2_bits = 0;
                    }
                    const int i = __ffs(tg_bits) - 1;
                    tg_bits &= tg_bits - 1u;
                    // Triangle bit i is the node's (mask bits below i)-th triangle.
                    const uint32_t tri = tg_base + (uint32_t)__popc(tg_mask & ((1u << i) - 1u));
                    if (cw8_triangle(L, 3 * (int)tri) && L.mode() != kClosest) {
                        tg_bits = 0;
                        tg2_bits = 0;
                        ng_bits = 0;
                        sp = 0;
                    }
                }
                if (ng_bits <= 0x00FFFFFFu && sp == 0) {
                    src.finish(L);
                    has_ray = false;
                }
            }
            // Dynamic fetch (kepler_dynamic_fetch.h:308-310).
            if ((unsigned)__popc(__ballot_sync(kFull, has_ray)) < fetch_threshold) break;
        }
    }
}

}  // namespace rb2dev
