// phx_kernels.cuh : device-side scene description, closest-hit traversal and the per-photon
// bounce loop shared by the plain, batched and adjoint kernels.
#pragma once
#include "phx_pod.h"
#include "phx_vec.cuh"
#include "phx_csg.cuh"
#include "phx_physics.cuh"

#define PHX_BVH_STACK 48
// phx_visit_node orders the hit children with a sorting network on integer keys (0: insertion
// sort on the distances)
#ifndef PHX_VISIT_SORTNET
#define PHX_VISIT_SORTNET 1
#endif
// leaf steps are taken when leaf-ready lanes x this weight >= node-ready lanes (or no node work is left)
#ifndef PHX_TRACE_LEAF_WEIGHT
#define PHX_TRACE_LEAF_WEIGHT 1
#endif

struct PhxScene {
    const phx_bvh4_node* bvh;   // root at 0
    const phx_leaf* leaves;
    const phx_leaf* globals;    // leaves tested first by every ray (boxes spanning much of the scene)
    const float4* leaf_sph;     // world bounding sphere (centre, radius) of each hierarchy leaf
    const float4* global_sph;   // and of each global leaf
    const float4* inst_inv;     // (num_inst*4) rows of the world->object 4x4 (row-vector convention)
    PhxCsgCtx csg;
    float4 cull;                // ball no hierarchy leaf reaches: centre xyz, radius^2 (0: none)
    int num_global;
    int num_leaf;               // hierarchy leaves (stack ranges from here on address the global leaves)
    int bvh_empty;              // no hierarchy leaves
    int empty;                  // no leaves at all
};

struct PhxBest {
    float t;
    int4 L;                     // leaf (inst, node_offset, gp_bd, ii_id); L.x < 0 : none
    float4 isect;
    float lposcost;
};

// IS program of CSGOptiX/CSGOptiX7.cu:896-967 for one (instance, prim) leaf: object-frame
// intersect_prim, keep the closest hit and its lposcost
// Can the ray segment (tmin, tmax) meet the ball (centre, radius)?  The radius is padded on the
// host beyond FP32 error, so a false answer never hides a hit of the leaf inside the ball.
PHX_D bool phx_ball_overlaps(const float4 b, const float3& o, const float3& d, float tmin, float tmax)
{
    const float3 oc = make_float3(b.x - o.x, b.y - o.y, b.z - o.z);
    const float dd = dot(d, d);
    const float tc = dot(oc, d) / dd;
    const float3 q = oc - tc * d;
    if (dot(q, q) > b.w * b.w) return false;
    const float h = b.w * rsqrtf(dd);
    return tc + h >= tmin && tc - h <= tmax;
}

template <int CV>
PHX_D void phx_test_leaf(const PhxScene& S, const int4 L, const float4 ball, const float3& o, const float3& d, float tmin, PhxBest& B,
                         unsigned& status)
{
    if (!phx_ball_overlaps(ball, o, d, tmin, B.t)) return;
    const float4* q = S.inst_inv + 4 * L.x;
    float4 m[4] = { __ldg(q + 0), __ldg(q + 1), __ldg(q + 2), __ldg(q + 3) };
    const float3 lo = xform_row(m, o, 1.f);
    const float3 ld = xform_row(m, d, 0.f);
    float4 is;
    const bool valid = intersect_prim<CV>(is, S.csg, L.y, tmin, lo, ld, status);
    // OptiX's interval rule: a report outside [tmin, tmax] is ignored (a convexpolyhedron wholly
    // behind the ray reports valid with t = 0, CSG/csg_intersect_leaf_convexpolyhedron.h:85-101)
    if (valid && is.w >= tmin && is.w < B.t) {
        B.t = is.w;
        B.L = L;
        B.isect = is;
        const float3 lpos = lo + is.w * ld;
        B.lposcost = lpos.z / sqrtf(dot(lpos, lpos));
    }
}

// Visit BVH4 node ni: slab-test its four children against [tmin, tmax] and push the hit ones
// (inner nodes and leaf ranges) far-to-near, so that the nearest is taken next.
PHX_D void phx_visit_node(const PhxScene& S, int ni, const float3& inv, const float3& oi, float tmin, float tmax, int2* stk,
                          int& sp, unsigned& status)
{
    const float4* nf = reinterpret_cast<const float4*>(S.bvh + ni);
    const float4 lx = __ldg(nf + 0), hx = __ldg(nf + 1), ly = __ldg(nf + 2), hy = __ldg(nf + 3);
    const float4 lz = __ldg(nf + 4), hz = __ldg(nf + 5);
    const int4 ch = __ldg(reinterpret_cast<const int4*>(nf + 6));
    const float lxa[4] = { lx.x, lx.y, lx.z, lx.w }, hxa[4] = { hx.x, hx.y, hx.z, hx.w };
    const float lya[4] = { ly.x, ly.y, ly.z, ly.w }, hya[4] = { hy.x, hy.y, hy.z, hy.w };
    const float lza[4] = { lz.x, lz.y, lz.z, lz.w }, hza[4] = { hz.x, hz.y, hz.z, hz.w };
    const int cha[4] = { ch.x, ch.y, ch.z, ch.w };
    float tn[4];
    int hitmask = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float tx0 = fmaf(lxa[c], inv.x, oi.x), tx1 = fmaf(hxa[c], inv.x, oi.x);
        const float ty0 = fmaf(lya[c], inv.y, oi.y), ty1 = fmaf(hya[c], inv.y, oi.y);
        const float tz0 = fmaf(lza[c], inv.z, oi.z), tz1 = fmaf(hza[c], inv.z, oi.z);
        const float tnear = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
        const float tfar = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
        // slab arithmetic slack: boxes are padded on the host, and a relative slack here
        tn[c] = tnear;
        if (cha[c] != 0 && tnear <= tfar * 1.00001f + 1e-4f) hitmask |= 1 << c;
    }
#if PHX_VISIT_SORTNET
    // order by a 4-key sorting network: key = the near distance's magnitude bits with the child
    // slot in the two low bits, all ones for a missed child (sorts last).  For tnear >= 0 the bits
    // order like the floats; the pushed distance itself is the exact tnear.
    unsigned k0, k1, k2, k3;
    {
        unsigned kk[4];
#pragma unroll
        for (int c = 0; c < 4; c++)
            kk[c] = (hitmask >> c) & 1 ? ((__float_as_uint(tn[c]) & 0x7ffffffcu) | (unsigned)c) : 0xffffffffu;
        k0 = kk[0]; k1 = kk[1]; k2 = kk[2]; k3 = kk[3];
    }
    unsigned t;
    t = min(k0, k1); k1 = max(k0, k1); k0 = t;
    t = min(k2, k3); k3 = max(k2, k3); k2 = t;
    t = min(k0, k2); k2 = max(k0, k2); k0 = t;
    t = min(k1, k3); k3 = max(k1, k3); k1 = t;
    t = min(k1, k2); k2 = max(k1, k2); k1 = t;
    const unsigned ks[4] = { k0, k1, k2, k3 };
#pragma unroll
    for (int j = 3; j >= 0; j--) {
        const unsigned key = ks[j];
        if (key == 0xffffffffu) continue;
        if (sp >= PHX_BVH_STACK) { status |= PHX_STATUS_BVH_STACK; continue; }
        const unsigned c = key & 3u;
        stk[sp] = make_int2(c == 0u ? cha[0] : c == 1u ? cha[1] : c == 2u ? cha[2] : cha[3],
                            __float_as_int(c == 0u ? tn[0] : c == 1u ? tn[1] : c == 2u ? tn[2] : tn[3]));
        sp++;
    }
#else
    int order[4] = { 0, 1, 2, 3 };
#pragma unroll
    for (int i = 1; i < 4; i++)
#pragma unroll
        for (int j = i; j > 0; j--) {
            if (tn[order[j]] < tn[order[j - 1]]) { int t = order[j]; order[j] = order[j - 1]; order[j - 1] = t; }
        }
#pragma unroll
    for (int k = 3; k >= 0; k--) {
        const int c = order[k];
        if (!(hitmask & (1 << c))) continue;
        if (sp >= PHX_BVH_STACK) { status |= PHX_STATUS_BVH_STACK; continue; }
        stk[sp] = make_int2(cha[c], __float_as_int(tn[c])); sp++;
    }
#endif
}

// ray set-up shared by both traversal loops: reciprocal direction (zero components nudged) and
// the slab offsets
PHX_D void phx_ray_slabs(const float3& o, const float3& d, float3& inv, float3& oi)
{
    const float3 dd = make_float3(fabsf(d.x) < 1e-30f ? copysignf(1e-30f, d.x) : d.x,
                                  fabsf(d.y) < 1e-30f ? copysignf(1e-30f, d.y) : d.y,
                                  fabsf(d.z) < 1e-30f ? copysignf(1e-30f, d.z) : d.z);
    inv = make_float3(1.f / dd.x, 1.f / dd.y, 1.f / dd.z);
    oi = make_float3(-o.x * inv.x, -o.y * inv.y, -o.z * inv.z);
}

// The segment [tmin, t] lies inside the ball no hierarchy leaf reaches: skip the hierarchy.
PHX_D bool phx_culled(const PhxScene& S, const float3& o, const float3& d, float tmin, float t)
{
    if (!(S.cull.w > 0.f)) return false;
    const float3 c = make_float3(S.cull.x, S.cull.y, S.cull.z);
    const float3 p0 = o + tmin * d - c;
    const float3 p1 = o + t * d - c;
    return dot(p0, p0) < S.cull.w && dot(p1, p1) < S.cull.w;
}

// PRD of a closest hit (CH program CSGOptiX/CSGOptiX7.cu:776-874), or of a miss
PHX_D void phx_best_prd(const PhxScene& S, const PhxBest& B, PhxPRD& prd)
{
    if (B.L.x < 0) {
        prd.gp_bd = 0xffffffffu;
        prd.ii_id = 0xffffffffu;
        prd.normal = make_float3(0.f, 0.f, 0.f);
        prd.distance = 0.f;
        prd.lposcost = 0.f;
        return;
    }
    const float4* q = S.inst_inv + 4 * B.L.x;
    float4 m[4] = { __ldg(q + 0), __ldg(q + 1), __ldg(q + 2), __ldg(q + 3) };
    prd.normal = xform_col(m, make_float3(B.isect.x, B.isect.y, B.isect.z), 0.f);
    prd.distance = B.t;
    prd.lposcost = B.lposcost;
    prd.gp_bd = (unsigned)B.L.z;
    prd.ii_id = (unsigned)B.L.w;
}

// Closest hit over all (instance, prim) leaves: restates optixTrace over the IAS with the
// IS program CSGOptiX/CSGOptiX7.cu:896-967 (object-frame intersect_prim, lposcost) and the
// CH program :776-874 (object->world normal, iindex<<16|identity, globalPrimIdx<<16|boundary).
// The global leaves are tested first, then the hierarchy is traversed unless the segment
// [tmin, closest so far] lies inside the ball no hierarchy leaf reaches.
// Returns false for a miss (prd boundary 0xffff).
template <int CV>
PHX_D bool phx_trace(const PhxScene& S, const float3& o, const float3& d, float tmin, float tmax, PhxPRD& prd, unsigned& status)
{
    prd.gp_bd = 0xffffffffu;
    prd.ii_id = 0xffffffffu;
    prd.normal = make_float3(0.f, 0.f, 0.f);
    prd.distance = 0.f;
    prd.lposcost = 0.f;
    if (S.empty) return false;
    PhxBest B;
    B.t = tmax;
    B.L = make_int4(-1, 0, 0, 0);
    B.isect = make_float4(0.f, 0.f, 0.f, 0.f);
    B.lposcost = 0.f;
    for (int g = 0; g < S.num_global; g++)
        phx_test_leaf<CV>(S, __ldg(reinterpret_cast<const int4*>(S.globals + g)), __ldg(S.global_sph + g), o, d, tmin, B, status);
    if (!S.bvh_empty && !phx_culled(S, o, d, tmin, B.t)) {
        float3 inv, oi;
        phx_ray_slabs(o, d, inv, oi);
        int2 stk[PHX_BVH_STACK];     // node or leaf range, near distance bits
        int sp = 0;
        stk[sp] = make_int2(0, __float_as_int(tmin)); sp++;
        // Each step the lanes of the warp that traverse together vote: either the lanes whose next
        // entry is an inner node visit it, or the lanes whose next entry is a leaf range test it.
        // Every lane still takes its own entries in its own near-first order; the vote only
        // gathers the expensive leaf tests into steps where many lanes run them.
        const unsigned mask = __activemask();
        for (;;) {
            while (sp > 0 && __int_as_float(stk[sp - 1].y) > B.t) sp--;
            const bool leaf_top = sp > 0 && stk[sp - 1].x < 0;
            const unsigned want_leaf = __ballot_sync(mask, leaf_top);
            const unsigned want_node = __ballot_sync(mask, sp > 0 && !leaf_top);
            if (!(want_leaf | want_node)) break;
            const bool leaf_step = want_node == 0u || __popc(want_leaf) * PHX_TRACE_LEAF_WEIGHT >= __popc(want_node);
            if (sp == 0 || leaf_top != leaf_step) continue;
            sp--;
            const int ni = stk[sp].x;
            if (leaf_step) {
                const int enc = -ni - 1;
                const int first = enc >> 3;
                const int count = (enc & 7) + 1;
                for (int li = first; li < first + count; li++)
                    phx_test_leaf<CV>(S, __ldg(reinterpret_cast<const int4*>(S.leaves + li)), __ldg(S.leaf_sph + li), o, d, tmin,
                                          B, status);
                continue;
            }
            phx_visit_node(S, ni, inv, oi, tmin, B.t, stk, sp, status);
        }
    }
    phx_best_prd(S, B, prd);
    return B.L.x >= 0;
}

struct PhxLoopCfg {
    int max_bounce;
    float max_time;
    float tmin, tmin0, tmax;
    unsigned eps0_mask;
};

PHX_D void seq_add_nibble(unsigned long long* seqhis, unsigned long long* seqbnd, unsigned slot, unsigned flag, unsigned boundary)
{
    const unsigned iseq = slot / 16u;
    const unsigned shift = 4u * (slot - iseq * 16u);
    if (iseq < 2u) {
        const unsigned long long f = (unsigned long long)(__ffs((int)flag) & 0xf);
        const unsigned long long b = (unsigned long long)(boundary & 0xfu);
        if (iseq == 0u) { seqhis[0] |= f << shift; seqbnd[0] |= b << shift; }
        else            { seqhis[1] |= f << shift; seqbnd[1] |= b << shift; }
    }
}

// The bounce loop of CSGOptiX/CSGOptiX7.cu:432-530 with sctx::point/end seq recording
// (sysrap/sctx.h:134-185, sysrap/sseq.h:174-184) always on.
template <int CV>
PHX_D void phx_bounce_loop(PhxPhoton& p, curandStateXORWOW& rng, const PhxScene& S, const PhxProps& P, const PhxLoopCfg& C,
                           unsigned long long* seqhis, unsigned long long* seqbnd, unsigned& status)
{
    int bounce = 0;
    seq_add_nibble(seqhis, seqbnd, 0u, p.flag(), p.boundary());
    while (bounce < C.max_bounce && p.time < C.max_time) {
        const float tmin = (p.obf & C.eps0_mask) ? C.tmin0 : C.tmin;
        PhxPRD prd;
        phx_trace<CV>(S, p.pos, p.mom, tmin, C.tmax, prd, status);
        if (prd.boundary() == 0xffffu) break;
        prd.normal = normalize(prd.normal);
        const int command = propagate(p, rng, prd, P, status);
        bounce++;
        seq_add_nibble(seqhis, seqbnd, (unsigned)bounce, p.flag(), p.boundary());
        if (command == PHX_BREAK) break;
    }
}

// genstep of photon idx: the last g with off[g] <= idx (empty gensteps are skipped)
PHX_D int phx_find_genstep(const long long* off, int G, long long idx)
{
    int lo = 0, hi = G;   // off[lo] <= idx < off[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(off + mid) <= idx) lo = mid; else hi = mid;
    }
    return lo;
}

// Advance a loaded XORWOW state by n steps with a precomputed jump matrix M (= T^n, see
// phx_rngjump.h): v <- M v over GF(2), d <- d + 362437 n.  Same state as skipahead(n).
PHX_D void phx_rng_jump(curandStateXORWOW& s, const uint32_t* __restrict__ M, unsigned long long n)
{
    uint32_t o0 = 0u, o1 = 0u, o2 = 0u, o3 = 0u, o4 = 0u;
    const uint32_t in[5] = { s.v[0], s.v[1], s.v[2], s.v[3], s.v[4] };
#pragma unroll 1
    for (int w = 0; w < 5; w++) {
        const uint32_t x = in[w];
        const uint32_t* colw = M + (size_t)(32 * w) * 8;
#pragma unroll 8
        for (int b = 0; b < 32; b++) {
            const uint32_t m = 0u - ((x >> b) & 1u);
            const uint4 a = __ldg(reinterpret_cast<const uint4*>(colw + 8 * b));
            const uint32_t e4 = __ldg(colw + 8 * b + 4);
            o0 ^= a.x & m; o1 ^= a.y & m; o2 ^= a.z & m; o3 ^= a.w & m; o4 ^= e4 & m;
        }
    }
    s.v[0] = o0; s.v[1] = o1; s.v[2] = o2; s.v[3] = o3; s.v[4] = o4;
    s.d += (unsigned int)((362437ull * n) & 0xffffffffull);
}

// v <- M v through the 4-bit group tables of M (k_jump_nibbles): 40 lookups instead of 160 column
// steps, the same XOR of the same columns, so the same state as phx_rng_jump and skipahead(n)
PHX_D void phx_rng_jump4(curandStateXORWOW& s, const uint32_t* __restrict__ T, unsigned long long n)
{
    uint32_t o0 = 0u, o1 = 0u, o2 = 0u, o3 = 0u, o4 = 0u;
    const uint32_t in[5] = { s.v[0], s.v[1], s.v[2], s.v[3], s.v[4] };
#pragma unroll 1
    for (int w = 0; w < 5; w++) {
        const uint32_t x = in[w];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const uint32_t* e = T + (size_t)((8 * w + q) * 16 + ((x >> (4 * q)) & 15u)) * PHX_JUMP_COLW;
            const uint4 a = __ldg(reinterpret_cast<const uint4*>(e));
            const uint32_t e4 = __ldg(e + 4);
            o0 ^= a.x; o1 ^= a.y; o2 ^= a.z; o3 ^= a.w; o4 ^= e4;
        }
    }
    s.v[0] = o0; s.v[1] = o1; s.v[2] = o2; s.v[3] = o3; s.v[4] = o4;
    s.d += (unsigned int)((362437ull * n) & 0xffffffffull);
}

// the 4-bit group tables of jump matrix blockIdx.y of M (one per genstep in batched calls):
// thread t builds entry (t / 16, t % 16)
__global__ void k_jump_nibbles(const uint32_t* __restrict__ M, uint32_t* T)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= PHX_JUMP_BITS / 4 * 16) return;
    M += (size_t)blockIdx.y * PHX_JUMP_MATW;
    T += (size_t)blockIdx.y * PHX_JUMP_NIBW;
    const int g = t >> 4, k = t & 15;
    uint32_t o[5] = { 0u, 0u, 0u, 0u, 0u };
    for (int b = 0; b < 4; b++) {
        if (!((k >> b) & 1)) continue;
        const uint32_t* col = M + (size_t)(4 * g + b) * PHX_JUMP_COLW;
        for (int q = 0; q < 5; q++) o[q] ^= col[q];
    }
    uint32_t* dst = T + (size_t)t * PHX_JUMP_COLW;
    for (int q = 0; q < 5; q++) dst[q] = o[q];
    dst[5] = dst[6] = dst[7] = 0u;
}

// one event jump matrix per entry: entry i uses event ev[i] (or `single` when ev is null);
// thread c composes column c of prod_k P_k^(bit k of event)
__global__ void k_jump_build(const int* ev, unsigned long long single, const uint32_t* __restrict__ P, uint32_t* out)
{
    const int c = threadIdx.x;
    if (c >= 160) return;
    const unsigned long long e = ev ? (unsigned long long)(unsigned)ev[blockIdx.x] : single;
    uint32_t v[5] = { 0u, 0u, 0u, 0u, 0u };
    v[c >> 5] = 1u << (c & 31);
    for (int k = 0; k < 32; k++) {
        if (!((e >> k) & 1ull)) continue;
        const uint32_t* Pk = P + (size_t)k * 160 * 8;
        uint32_t o[5] = { 0u, 0u, 0u, 0u, 0u };
        for (int bit = 0; bit < 160; bit++) {
            if ((v[bit >> 5] >> (bit & 31)) & 1u)
                for (int q = 0; q < 5; q++) o[q] ^= Pk[bit * 8 + q];
        }
        for (int q = 0; q < 5; q++) v[q] = o[q];
    }
    uint32_t* dst = out + (size_t)blockIdx.x * 160 * 8 + c * 8;
    for (int q = 0; q < 5; q++) dst[q] = v[q];
    dst[5] = dst[6] = dst[7] = 0u;
}

PHX_D void phx_load_rng(curandStateXORWOW& s, const uint32_t* rng, long long slots, long long slot)
{
    s.d = __ldg(rng + slot);
    s.v[0] = __ldg(rng + slots * 1 + slot);
    s.v[1] = __ldg(rng + slots * 2 + slot);
    s.v[2] = __ldg(rng + slots * 3 + slot);
    s.v[3] = __ldg(rng + slots * 4 + slot);
    s.v[4] = __ldg(rng + slots * 5 + slot);
    s.boxmuller_flag = 0;
    s.boxmuller_flag_double = 0;
    s.boxmuller_extra = 0.f;
    s.boxmuller_extra_double = 0.0;
}

PHX_D void phx_store_photon(phx_photon* out, const PhxPhoton& p)
{
    float4* o = reinterpret_cast<float4*>(out);
    o[0] = make_float4(p.pos.x, p.pos.y, p.pos.z, p.time);
    o[1] = make_float4(p.mom.x, p.mom.y, p.mom.z, __uint_as_float(p.hitcount_iindex));
    o[2] = make_float4(p.pol.x, p.pol.y, p.pol.z, p.wavelength);
    o[3] = make_float4(__uint_as_float(p.obf), __uint_as_float(p.identity), __uint_as_float(p.index), __uint_as_float(p.flagmask));
}
