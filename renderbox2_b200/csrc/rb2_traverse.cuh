// Persistent while-while traversal body shared by every launch flavour
// (single tracer, batched job table, integrator queues).
//
// Semantics follow the reference's Aila-Laine persistent kernel
// (accelerators/sbvh/kepler_dynamic_fetch.h:67-363) and single-ray trace_ray
// (accelerators/sbvh/cuda_tracer_functions.cu:42-279); arithmetic is pinned
// to the CPU oracle's (oracle/rb2_oracle.c) with __fmaf_rn / __fmul_rn /
// __fdiv_rn so results are bit-identical.
//
// A RaySource policy supplies rays and consumes results:
//   void claim(unsigned count, u64& b1, unsigned& n1, u64& b2)
//        warp leader reserves `count` slots: ranks [0, n1) get b1 + rank,
//        ranks [n1, count) get b2 + (rank - n1)
//   int fetch(u64 slot, Lane& L)   1: ray loaded; 0: slot past the end (lane
//                                  retires); -1: ray consumed by the source
//                                  (masked ray, result already written)
//   void finish(const Lane& L)     write the result of a finished ray
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rb2dev {

constexpr int kSentinel = 0x76543210;
constexpr int kStackSize = 64;
// 4-wide node layout (tracer layout RB2_NODE_ORDER_WIDE4): a binary Compact2
// tree collapsed so each node holds up to four child boxes, 128 bytes:
// float4 lo.x[4], hi.x[4], lo.y[4], hi.y[4], lo.z[4], hi.z[4], int4 child[4],
// one unused float4.  Children keep the Compact2 encoding (inner = float4
// offset of the wide node, leaf = ~Woop offset); kWideEmpty marks an unused
// slot.  A wide node pushes up to three children, so its stack is deeper.
constexpr int kWideEmpty = 0x7FFFFFFF;
constexpr int kStackSizeWide = 192;
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kStatusStack = 1u;

enum Mode : uint32_t { kClosest = 0, kAny = 1, kOcclusion = 2 };

// Node layouts of the traversal kernel variants.
enum Layout : int { kLayoutBinary = 0, kLayoutWide4 = 1, kLayoutCw8 = 2 };

// Node-phase threshold of persistent_trace / persistent_trace_cw8 for a launch
// configuration that leaves it 0: the fastest measured on the batching
// workload for each layout.
__host__ __device__ constexpr uint32_t default_node_threshold(int layout)
{
    return layout == kLayoutCw8 ? 12u : 8u;
}

constexpr uint32_t kJobMask = 0x3FFFFFFFu;          // job index bits of Lane::tag
constexpr uint64_t kMaxJobRays = 0xFFFFFFFFull;     // rays per job (Lane::ray is 32-bit)

// Per-lane traversal state.  Kept small on purpose: every register here is
// live across the whole loop, and the kernel is latency-bound, so fewer
// registers mean more resident warps (48 registers: 40 warps per SM).  The
// triangle-index buffer is not carried (sources pass it to hit_record), u, v
// are recomputed once at the end from the accepted triangle (hit_uv), and the
// mode shares a word with the job index.
struct Lane {
    // BVH of the ray's scene
    const float4* nodes;
    const float4* woop;
    // ray
    float ox, oy, oz, dx, dy, dz, idx, idy, idz, oodx, oody, oodz, tmin;
    // state
    float hitT;
    int nodeAddr, leafAddr, hitIndex;
    uint32_t tag;       // Mode << 30 | source-defined job index
    uint32_t ray;       // source-defined index of the ray within its job

    __device__ __forceinline__ uint32_t mode() const { return tag >> 30; }
    __device__ __forceinline__ uint32_t job() const { return tag & kJobMask; }
    __device__ __forceinline__ void set_tag(uint32_t mode, uint32_t job) { tag = (mode << 30) | (job & kJobMask); }
};

// One 32-byte read-only load (sm_100 256-bit ld.global.nc.v8); `p` must be
// 32-byte aligned.
__device__ __forceinline__ void ldg_v8(const float4* p, float4& a, float4& b)
{
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}

// A 64-byte Compact2 node as four 128-bit read-only loads.  (Two 256-bit
// ld.global.nc.v8 loads halve the L1 sector lookups but measured 1-2 %
// slower at the tuned register budget: the kernel is bound by L2 latency
// with 40 resident warps per SM, not by L1 throughput.)
__device__ __forceinline__ void load_node(const float4* np, float4& n0xy, float4& n1xy, float4& nz, float4& cn)
{
    n0xy = __ldg(np + 0);
    n1xy = __ldg(np + 1);
    nz = __ldg(np + 2);
    cn = __ldg(np + 3);
}

__device__ __forceinline__ float fmin_s(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmax_s(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float imin_f(float a, float b) { return __int_as_float(min(__float_as_int(a), __float_as_int(b))); }
__device__ __forceinline__ float imax_f(float a, float b) { return __int_as_float(max(__float_as_int(a), __float_as_int(b))); }

__device__ __forceinline__ float span_begin(float a0, float a1, float b0, float b1, float c0, float c1, float d)
{
    return imax_f(imax_f(fmin_s(a0, a1), fmin_s(b0, b1)), imax_f(imin_f(c0, c1), d));
}
__device__ __forceinline__ float span_end(float a0, float a1, float b0, float b1, float c0, float c1, float d)
{
    return imin_f(imin_f(fmax_s(a0, a1), fmax_s(b0, b1)), imin_f(imax_f(c0, c1), d));
}

__device__ __forceinline__ float safe_rcp(float d)
{
    const float ooeps = 0x1p-80f;
    return __fdiv_rn(1.0f, fabsf(d) > ooeps ? d : copysignf(ooeps, d));
}

// Ray set-up (cuda_tracer_functions.cu:68-89).
__device__ __forceinline__ void setup_ray(Lane& L, float4 o4, float4 d4)
{
    L.ox = o4.x; L.oy = o4.y; L.oz = o4.z; L.tmin = o4.w;
    L.dx = d4.x; L.dy = d4.y; L.dz = d4.z; L.hitT = d4.w;
    L.idx = safe_rcp(L.dx); L.idy = safe_rcp(L.dy); L.idz = safe_rcp(L.dz);
    L.oodx = __fmul_rn(L.ox, L.idx); L.oody = __fmul_rn(L.oy, L.idy); L.oodz = __fmul_rn(L.oz, L.idz);
    L.leafAddr = 0;
    L.nodeAddr = 0;
    L.hitIndex = -1;
}

// One child slot of a wide node: the same slab and span arithmetic as the
// binary node test, so a child passes here exactly when it passes there.
__device__ __forceinline__ void wide_span(const Lane& L, float lox, float hix, float loy, float hiy, float loz, float hiz,
                                          float& cmin, float& cmax)
{
    const float a0 = __fmaf_rn(lox, L.idx, -L.oodx), a1 = __fmaf_rn(hix, L.idx, -L.oodx);
    const float b0 = __fmaf_rn(loy, L.idy, -L.oody), b1 = __fmaf_rn(hiy, L.idy, -L.oody);
    const float c0 = __fmaf_rn(loz, L.idz, -L.oodz), c1 = __fmaf_rn(hiz, L.idz, -L.oodz);
    cmin = span_begin(a0, a1, b0, b1, c0, c1, L.tmin);
    cmax = span_end(a0, a1, b0, b1, c0, c1, L.hitT);
}

// Orders (key, child) pairs so key[0] is the smallest.
__device__ __forceinline__ void cswap(float& ka, int& ca, float& kb, int& cb)
{
    if (kb < ka) {
        const float tk = ka; ka = kb; kb = tk;
        const int tc = ca; ca = cb; cb = tc;
    }
}

// node_threshold: the node phase also ends, so that postponed leaves are
// tested, once fewer than this many lanes still traverse nodes while some lane
// holds a leaf (0 or 1: only when no lane is left searching for one).
template <class Source, bool WIDE = false>
__device__ __forceinline__ void persistent_trace(Source& src, uint32_t fetch_threshold, uint32_t node_threshold,
                                                 unsigned int* status)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    constexpr int kStack = WIDE ? kStackSizeWide : kStackSize;
    int stack[kStack + 2];
    int sp = 0;
    Lane L;
    L.nodeAddr = kSentinel;
    L.leafAddr = 0;
    L.hitIndex = -1;
    bool has_ray = false, retired = false;

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
                    stack[0] = kSentinel;
                    sp = 0;
                    has_ray = true;
                }
            }
        }
        if (__all_sync(kFull, retired)) break;

        // ---- traversal until too few lanes are busy.
        while (__any_sync(kFull, has_ray)) {
            // Inner nodes until every busy lane has postponed a leaf, or fewer
            // than node_threshold lanes still traverse while some lane holds one.
            for (;;) {
                const bool in = has_ray && (unsigned)L.nodeAddr < (unsigned)kSentinel;
                if (!__any_sync(kFull, in)) break;
                if (in && !WIDE) {
                    const float4* np = L.nodes + L.nodeAddr;
                    float4 n0xy, n1xy, nz, cn;
                    load_node(np, n0xy, n1xy, nz, cn);
                    int c0 = __float_as_int(cn.x), c1 = __float_as_int(cn.y);

                    const float c0lox = __fmaf_rn(n0xy.x, L.idx, -L.oodx);
                    const float c0hix = __fmaf_rn(n0xy.y, L.idx, -L.oodx);
                    const float c0loy = __fmaf_rn(n0xy.z, L.idy, -L.oody);
                    const float c0hiy = __fmaf_rn(n0xy.w, L.idy, -L.oody);
                    const float c0loz = __fmaf_rn(nz.x, L.idz, -L.oodz);
                    const float c0hiz = __fmaf_rn(nz.y, L.idz, -L.oodz);
                    const float c1loz = __fmaf_rn(nz.z, L.idz, -L.oodz);
                    const float c1hiz = __fmaf_rn(nz.w, L.idz, -L.oodz);
                    const float c0min = span_begin(c0lox, c0hix, c0loy, c0hiy, c0loz, c0hiz, L.tmin);
                    const float c0max = span_end(c0lox, c0hix, c0loy, c0hiy, c0loz, c0hiz, L.hitT);
                    const float c1lox = __fmaf_rn(n1xy.x, L.idx, -L.oodx);
                    const float c1hix = __fmaf_rn(n1xy.y, L.idx, -L.oodx);
                    const float c1loy = __fmaf_rn(n1xy.z, L.idy, -L.oody);
                    const float c1hiy = __fmaf_rn(n1xy.w, L.idy, -L.oody);
                    const float c1min = span_begin(c1lox, c1hix, c1loy, c1hiy, c1loz, c1hiz, L.tmin);
                    const float c1max = span_end(c1lox, c1hix, c1loy, c1hiy, c1loz, c1hiz, L.hitT);

                    const bool swp = c1min < c0min;
                    const bool t0 = c0max >= c0min;
                    const bool t1 = c1max >= c1min;
                    if (!t0 && !t1) {
                        L.nodeAddr = stack[sp--];
                    } else {
                        L.nodeAddr = t0 ? c0 : c1;
                        if (t0 && t1) {
                            if (swp) { const int tmp = L.nodeAddr; L.nodeAddr = c1; c1 = tmp; }
                            if (sp >= kStackSize) {
                                // Unreachable for validated trees (depth <= 64); a
                                // corrupt tree abandons the ray and reports it.
                                atomicOr(status, kStatusStack);
                                L.nodeAddr = kSentinel;
                                L.leafAddr = 0;
                                L.hitIndex = -1;
                            } else {
                                stack[++sp] = c1;
                            }
                        }
                    }
                    if (L.nodeAddr < 0 && L.leafAddr >= 0) {
                        L.leafAddr = L.nodeAddr;
                        L.nodeAddr = stack[sp--];
                    }
                }
                if (WIDE && in) {
                    const float4* np = L.nodes + L.nodeAddr;
                    // A wide node is 128-byte aligned: three 256-bit loads for the
                    // boxes, one 128-bit load for the children.  (Measured: four
                    // 256-bit loads of per-child records were slower, and seven
                    // 128-bit loads slower still.)
                    float4 lx, hx, ly, hy, lz, hz;
                    ldg_v8(np + 0, lx, hx);
                    ldg_v8(np + 2, ly, hy);
                    ldg_v8(np + 4, lz, hz);
                    const int4 ch = __ldg(reinterpret_cast<const int4*>(np + 6));
                    float k0, k1, k2, k3, m;
                    wide_span(L, lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, k0, m);
                    if (!(ch.x != kWideEmpty && m >= k0)) k0 = __int_as_float(0x7f800000);
                    wide_span(L, lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, k1, m);
                    if (!(ch.y != kWideEmpty && m >= k1)) k1 = __int_as_float(0x7f800000);
                    wide_span(L, lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, k2, m);
                    if (!(ch.z != kWideEmpty && m >= k2)) k2 = __int_as_float(0x7f800000);
                    wide_span(L, lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, k3, m);
                    if (!(ch.w != kWideEmpty && m >= k3)) k3 = __int_as_float(0x7f800000);
                    const int hits = (k0 != __int_as_float(0x7f800000)) + (k1 != __int_as_float(0x7f800000)) +
                                     (k2 != __int_as_float(0x7f800000)) + (k3 != __int_as_float(0x7f800000));
                    int c0 = ch.x, c1 = ch.y, c2 = ch.z, c3 = ch.w;
                    // Five compare-exchanges sort four keys (nearest entry first).
                    cswap(k0, c0, k1, c1);
                    cswap(k2, c2, k3, c3);
                    cswap(k0, c0, k2, c2);
                    cswap(k1, c1, k3, c3);
                    cswap(k1, c1, k2, c2);
                    if (hits == 0) {
                        L.nodeAddr = stack[sp--];
                    } else if (sp + hits - 1 > kStack) {
                        // Unreachable for trees whose wide depth was validated; a
                        // corrupt tree abandons the ray and reports it.
                        atomicOr(status, kStatusStack);
                        L.nodeAddr = kSentinel;
                        L.leafAddr = 0;
                        L.hitIndex = -1;
                    } else {
                        // Farther children first, so the next nearest pops first.
                        if (hits > 3) stack[++sp] = c3;
                        if (hits > 2) stack[++sp] = c2;
                        if (hits > 1) stack[++sp] = c1;
                        L.nodeAddr = c0;
                    }
                    if (L.nodeAddr < 0 && L.leafAddr >= 0) {
                        L.leafAddr = L.nodeAddr;
                        L.nodeAddr = stack[sp--];
                    }
                }
                if (!__any_sync(kFull, in && L.leafAddr >= 0)) break;
                if ((unsigned)__popc(__ballot_sync(kFull, has_ray && (unsigned)L.nodeAddr < (unsigned)kSentinel)) <
                        node_threshold &&
                    __any_sync(kFull, has_ray && L.leafAddr < 0))
                    break;
            }

            // Postponed leaves.
            if (has_ray) {
                while (L.leafAddr < 0) {
                    for (int triAddr = ~L.leafAddr;; triAddr += 3) {
                        const float4* wp = L.woop + triAddr;
                        const float4 v00 = __ldg(wp + 0);
                        const float4 v11 = __ldg(wp + 1);
                        const float4 v22 = __ldg(wp + 2);
                        if (__float_as_int(v00.x) == (int)0x80000000) break;

                        const float Oz = __fmaf_rn(-L.oz, v00.z, __fmaf_rn(-L.oy, v00.y, __fmaf_rn(-L.ox, v00.x, v00.w)));
                        const float Dz = __fmaf_rn(L.dz, v00.z, __fmaf_rn(L.dy, v00.y, __fmul_rn(L.dx, v00.x)));
                        const float t = __fmul_rn(Oz, __frcp_rn(Dz));  // IEEE 1 / Dz, as __fdiv_rn(1, Dz)
                        if (t > L.tmin && t < L.hitT) {
                            const float Ox = __fmaf_rn(L.oz, v11.z, __fmaf_rn(L.oy, v11.y, __fmaf_rn(L.ox, v11.x, v11.w)));
                            const float Dx = __fmaf_rn(L.dz, v11.z, __fmaf_rn(L.dy, v11.y, __fmul_rn(L.dx, v11.x)));
                            const float u = __fmaf_rn(t, Dx, Ox);
                            if (u >= 0.0f) {
                                const float Oy = __fmaf_rn(L.oz, v22.z, __fmaf_rn(L.oy, v22.y, __fmaf_rn(L.ox, v22.x, v22.w)));
                                const float Dy = __fmaf_rn(L.dz, v22.z, __fmaf_rn(L.dy, v22.y, __fmul_rn(L.dx, v22.x)));
                                const float v = __fmaf_rn(t, Dy, Oy);
                                if (v >= 0.0f && __fadd_rn(u, v) <= 1.0f) {
                                    L.hitT = t;
                                    L.hitIndex = triAddr;
                                    if (L.mode() != kClosest) {
                                        L.nodeAddr = kSentinel;
                                        break;
                                    }
                                }
                            }
                        }
                    }
                    L.leafAddr = L.nodeAddr;
                    if (L.nodeAddr < 0) L.nodeAddr = stack[sp--];
                }
                if (L.nodeAddr == kSentinel) {
                    src.finish(L);
                    has_ray = false;
                }
            }
            // Dynamic fetch (kepler_dynamic_fetch.h:308-310).
            if ((unsigned)__popc(__ballot_sync(kFull, has_ray)) < fetch_threshold) break;
        }
    }
}

// u, v of the accepted triangle, recomputed with the leaf loop's exact
// operations at t = hitT (the accepted t), so the bits equal those of the
// test that accepted it.  Valid only when hitIndex >= 0.
__device__ __forceinline__ float2 hit_uv(const Lane& L)
{
    const float4 v11 = __ldg(L.woop + L.hitIndex + 1), v22 = __ldg(L.woop + L.hitIndex + 2);
    const float Ox = __fmaf_rn(L.oz, v11.z, __fmaf_rn(L.oy, v11.y, __fmaf_rn(L.ox, v11.x, v11.w)));
    const float Dx = __fmaf_rn(L.dz, v11.z, __fmaf_rn(L.dy, v11.y, __fmul_rn(L.dx, v11.x)));
    const float Oy = __fmaf_rn(L.oz, v22.z, __fmaf_rn(L.oy, v22.y, __fmaf_rn(L.ox, v22.x, v22.w)));
    const float Dy = __fmaf_rn(L.dz, v22.z, __fmaf_rn(L.dy, v22.y, __fmul_rn(L.dx, v22.x)));
    return make_float2(__fmaf_rn(L.hitT, Dx, Ox), __fmaf_rn(L.hitT, Dy, Oy));
}

// Result record shared by all sources: prim (original triangle id, -1 miss), t, u, v.
__device__ __forceinline__ int4 hit_record(const Lane& L, const uint32_t* triidx)
{
    if (L.hitIndex < 0) return make_int4(-1, __float_as_int(L.hitT), 0, 0);
    const float2 uv = hit_uv(L);
    return make_int4((int)__ldg(triidx + L.hitIndex), __float_as_int(L.hitT), __float_as_int(uv.x),
                     __float_as_int(uv.y));
}

}  // namespace rb2dev
