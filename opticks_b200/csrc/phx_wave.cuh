// phx_wave.cuh : wavefront form of the photon loop — closest-hit search and physics as separate
// kernels over a pool of in-flight paths held in HBM.
//
// The one-kernel loop (phx_persist.cuh) keeps every path in registers, so the whole bounce —
// traversal, CSG, generation, propagate, bookkeeping — is compiled as one function whose register
// count (about 200) leaves ten warps per SM to hide the latency of the traversal's dependent
// loads.  Here a round is two launches:
//   k_wave_trace  reads ray origin/direction of every live path, runs phx_trace and writes the PRD
//                 (a lean kernel: 168 registers, 12 warps per SM, against about 200 and 10)
//   k_wave_shade  reads the path and its PRD, runs propagate / seq nibble / finish exactly as the
//                 one-kernel loop does, and appends live slots to the next round's list and
//                 finished slots to a free list
//   k_wave_fill   (only when the event has more photons than slots) gives every free slot the next
//                 photon from the queue: whole warps take consecutive photons of one genstep, so
//                 generation runs coherently instead of in the few lanes that just finished
// Path state is 128 B per slot (sphoton, the XORWOW words, bounce, event, seqhis/seqbnd) plus a
// 32 B PRD; the extra HBM traffic is about 0.4 KB per bounce against microseconds of traversal.
// Every photon consumes its random numbers in the same order as in the one-kernel loop, so
// photons, seq and hits are bit-identical to it.
//
// The host drives rounds until the live count reaches zero (read back every few rounds); the
// number of rounds is bounded by (N / pool + 1) * (max_bounce + 1).
#pragma once
#include "phx_persist.cuh"

struct PhxWaveSlot {          // 128 B
    float4 q0, q1, q2, q3;    // sphoton
    uint4 ra;                 // xorwow d, v0, v1, v2
    uint4 rb;                 // xorwow v3, v4, bounce, event
    ulonglong2 his, bnd;      // seqhis[2], seqbnd[2]
};

struct PhxWavePrd {           // 32 B
    float4 nd;                // normal.xyz, distance
    uint4 lgi;                // lposcost bits, gp_bd, ii_id, 0
};

struct WaveArgs {
    PersistArgs A;            // scene, physics, gensteps, outputs, queue, status
    PhxWaveSlot* slot;
    PhxWavePrd* prd;
    long long* sidx;          // photon index per slot
    const uint32_t* act_in;   // live slots of this round
    uint32_t* act_out;        // live slots of the next round
    const unsigned* n_in;
    unsigned* n_out;
    float4* score;            // ADJ: 8 float4 (the 32 score terms) per slot
    uint32_t* free_list;      // slots freed by this round's physics (refilled by k_wave_fill)
    unsigned* n_free;
    unsigned* trace_ctr;      // rays of this round handed to warps (k_wave_trace_df); zeroed by the kernel before
    long long pool;           // slots (init only)
    uint32_t* live_bits;      // refill rounds: live slots as bits, turned into the next list in slot
                              // order by k_wave_act (null: live slots are appended to act_out)
    int refill_idle;          // k_wave_trace_df: idle lanes a warp waits for before taking new rays
};

// The slot's first 32 B sector (position, time, direction, q1.w) is all the closest-hit kernel
// needs: bit 31 of the stored q1.w carries the choice of tmin (the last flag against the epsilon0
// mask), and the photon's own bit 31 of q1.w rides in bit 30 of the bounce word.  `first`: the
// slot takes a new photon (its index is written once).
// the slot's eight 16 B chunks of a path (PhxWaveSlot order)
PHX_D void wave_pack(const WaveArgs& W, const PhxLane& L, float4 (&c)[8])
{
    const PhxPhoton& p = L.p;
    const unsigned eps0 = (p.obf & W.A.C.eps0_mask) ? 0x80000000u : 0u;
    c[0] = make_float4(p.pos.x, p.pos.y, p.pos.z, p.time);
    c[1] = make_float4(p.mom.x, p.mom.y, p.mom.z, __uint_as_float((p.hitcount_iindex & 0x7fffffffu) | eps0));
    c[2] = make_float4(p.pol.x, p.pol.y, p.pol.z, p.wavelength);
    c[3] = make_float4(__uint_as_float(p.obf), __uint_as_float(p.identity), __uint_as_float(p.index), __uint_as_float(p.flagmask));
    c[4] = make_float4(__uint_as_float(L.rng.d), __uint_as_float(L.rng.v[0]), __uint_as_float(L.rng.v[1]), __uint_as_float(L.rng.v[2]));
    c[5] = make_float4(__uint_as_float(L.rng.v[3]), __uint_as_float(L.rng.v[4]),
                       __uint_as_float((unsigned)L.bounce | ((p.hitcount_iindex >> 1) & 0x40000000u)), __uint_as_float((unsigned)L.ev));
    c[6] = make_float4(__uint_as_float((unsigned)L.seqhis[0]), __uint_as_float((unsigned)(L.seqhis[0] >> 32)),
                       __uint_as_float((unsigned)L.seqhis[1]), __uint_as_float((unsigned)(L.seqhis[1] >> 32)));
    c[7] = make_float4(__uint_as_float((unsigned)L.seqbnd[0]), __uint_as_float((unsigned)(L.seqbnd[0] >> 32)),
                       __uint_as_float((unsigned)L.seqbnd[1]), __uint_as_float((unsigned)(L.seqbnd[1] >> 32)));
}

// the tmin of a slot's next closest hit, from its first sector
PHX_D float wave_tmin(const WaveArgs& W, const float4& q1)
{
    return (__float_as_uint(q1.w) & 0x80000000u) ? W.A.C.tmin0 : W.A.C.tmin;
}

// a path from its slot's eight 16 B chunks
PHX_D void wave_unpack(const float4 (&c)[8], PhxLane& L)
{
    PhxPhoton& p = L.p;
    p.pos = make_float3(c[0].x, c[0].y, c[0].z); p.time = c[0].w;
    p.mom = make_float3(c[1].x, c[1].y, c[1].z);
    p.pol = make_float3(c[2].x, c[2].y, c[2].z); p.wavelength = c[2].w;
    p.obf = __float_as_uint(c[3].x); p.identity = __float_as_uint(c[3].y);
    p.index = __float_as_uint(c[3].z); p.flagmask = __float_as_uint(c[3].w);
    L.rng.d = __float_as_uint(c[4].x); L.rng.v[0] = __float_as_uint(c[4].y);
    L.rng.v[1] = __float_as_uint(c[4].z); L.rng.v[2] = __float_as_uint(c[4].w);
    L.rng.v[3] = __float_as_uint(c[5].x); L.rng.v[4] = __float_as_uint(c[5].y);
    L.rng.boxmuller_flag = 0; L.rng.boxmuller_flag_double = 0;
    L.rng.boxmuller_extra = 0.f; L.rng.boxmuller_extra_double = 0.0;
    const unsigned bz = __float_as_uint(c[5].z);
    L.bounce = (int)(bz & 0x3fffffffu); L.ev = (int)__float_as_uint(c[5].w);
    p.hitcount_iindex = (__float_as_uint(c[1].w) & 0x7fffffffu) | ((bz & 0x40000000u) << 1);
    L.seqhis[0] = (unsigned long long)__float_as_uint(c[6].x) | ((unsigned long long)__float_as_uint(c[6].y) << 32);
    L.seqhis[1] = (unsigned long long)__float_as_uint(c[6].z) | ((unsigned long long)__float_as_uint(c[6].w) << 32);
    L.seqbnd[0] = (unsigned long long)__float_as_uint(c[7].x) | ((unsigned long long)__float_as_uint(c[7].y) << 32);
    L.seqbnd[1] = (unsigned long long)__float_as_uint(c[7].z) | ((unsigned long long)__float_as_uint(c[7].w) << 32);
}

PHX_D void wave_load(const WaveArgs& W, uint32_t s, PhxLane& L)
{
    const float4* o = reinterpret_cast<const float4*>(W.slot + s);
    float4 c[8];
#pragma unroll
    for (int k = 0; k < 8; k++) c[k] = o[k];
    wave_unpack(c, L);
    L.idx = W.sidx[s];
}

// Slots of a whole warp moved through shared memory (`st`: 256 float4 of the warp's own): lane j
// moves 16 B chunk j & 7 of the slot of lane 4k + (j >> 3), so one instruction reads or writes
// four whole 128 B slots where per-lane accesses touch 16 B of 32 different slots.  Chunk c of
// lane l's slot sits at st[8l + (c ^ (l & 7))], which keeps both sides free of bank conflicts.
// Warp-collective; `take` selects the lanes whose slots move.
PHX_D void wave_gather(const WaveArgs& W, float4* st, uint32_t s, bool take)
{
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned c = lane & 7u;
    const unsigned m = __ballot_sync(FULL, take);
    const float4* src = reinterpret_cast<const float4*>(W.slot);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const unsigned l = 4u * (unsigned)k + (lane >> 3);
        const uint32_t sl = __shfl_sync(FULL, s, (int)l);
        if ((m >> l) & 1u) st[8u * l + (c ^ (l & 7u))] = src[(size_t)sl * 8u + c];
    }
    __syncwarp();
}

PHX_D void wave_scatter(const WaveArgs& W, float4* st, uint32_t s, bool take)
{
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned c = lane & 7u;
    const unsigned m = __ballot_sync(FULL, take);
    __syncwarp();
    float4* dst = reinterpret_cast<float4*>(W.slot);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const unsigned l = 4u * (unsigned)k + (lane >> 3);
        const uint32_t sl = __shfl_sync(FULL, s, (int)l);
        if ((m >> l) & 1u) dst[(size_t)sl * 8u + c] = st[8u * l + (c ^ (l & 7u))];
    }
    __syncwarp();
}

// this lane's slot chunks in the warp's staging area
PHX_D void wave_stage_get(const float4* st, float4 (&c)[8])
{
    const unsigned lane = threadIdx.x & 31u;
#pragma unroll
    for (int k = 0; k < 8; k++) c[k] = st[8u * lane + ((unsigned)k ^ (lane & 7u))];
}

PHX_D void wave_stage_put(float4* st, const float4 (&c)[8])
{
    const unsigned lane = threadIdx.x & 31u;
#pragma unroll
    for (int k = 0; k < 8; k++) st[8u * lane + ((unsigned)k ^ (lane & 7u))] = c[k];
}

// the 32 score terms and the refraction tangent (pos, mom, pol) of a path: PHX_WAVE_SCORE_F4 float4
#define PHX_WAVE_SCORE_F4 11
PHX_D void wave_store_score(const WaveArgs& W, uint32_t s, const PhxScore* sc)
{
    float4* o = W.score + PHX_WAVE_SCORE_F4 * (size_t)s;
#pragma unroll
    for (int k = 0; k < 8; k++)
        o[k] = make_float4(PHX_SG(*sc, 4 * k), PHX_SG(*sc, 4 * k + 1), PHX_SG(*sc, 4 * k + 2), PHX_SG(*sc, 4 * k + 3));
    o[8] = make_float4(sc->tpos.x, sc->tpos.y, sc->tpos.z, sc->tdir.x);
    o[9] = make_float4(sc->tdir.y, sc->tdir.z, sc->tpol.x, sc->tpol.y);
    o[10] = make_float4(sc->tpol.z, 0.f, 0.f, 0.f);
}

PHX_D void wave_load_score(const WaveArgs& W, uint32_t s, PhxScore* sc)
{
    const float4* o = W.score + PHX_WAVE_SCORE_F4 * (size_t)s;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const float4 v = o[k];
        PHX_SG(*sc, 4 * k) = v.x; PHX_SG(*sc, 4 * k + 1) = v.y; PHX_SG(*sc, 4 * k + 2) = v.z; PHX_SG(*sc, 4 * k + 3) = v.w;
    }
    const float4 a = o[8], b = o[9], c = o[10];
    sc->tpos = make_float3(a.x, a.y, a.z);
    sc->tdir = make_float3(a.w, b.x, b.y);
    sc->tpol = make_float3(b.z, b.w, c.x);
}

PHX_D void wave_score_setup(PhxScore& score, const PersistArgs& A)
{
    score_setup(score, A);
}

// The slot kernels move whole warps of slots through shared memory (wave_gather / wave_scatter).
// this warp's staging area: 256 float4 (the slot kernels run 128-thread blocks)
PHX_D float4* wave_stage_area()
{
    __shared__ float4 stage[128 * 8];
    return stage + 256u * (threadIdx.x >> 5);
}

// a live path back into its slot (`first`: the slot took a new photon).  Warp-collective.
PHX_D void wave_put(const WaveArgs& W, float4* st, uint32_t s, const PhxLane& L, bool live, bool first)
{
    if (live) {
        float4 c[8];
        wave_pack(W, L, c);
        wave_stage_put(st, c);
        if (first) W.sidx[s] = L.idx;
    }
    wave_scatter(W, st, s, live);
}

// a path may take another bounce (the loop condition of CSGOptiX/CSGOptiX7.cu:477)
PHX_D bool wave_can_trace(const PhxLane& L, const PersistArgs& A)
{
    return L.bounce < A.C.max_bounce && L.p.time < A.C.max_time;
}

// warp-aggregated append of slot s to a list (the next round's live list, or the free list)
PHX_D void wave_push(uint32_t* list, unsigned* count, bool keep, uint32_t s)
{
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned m = __ballot_sync(FULL, keep);
    if (!m) return;
    const unsigned leader = __ffs(m) - 1u;
    unsigned base = 0u;
    if (lane == leader) base = atomicAdd(count, (unsigned)__popc(m));
    base = __shfl_sync(FULL, base, leader);
    if (keep) list[base + __popc(m & ((1u << lane) - 1u))] = s;
}

PHX_D void wave_append(const WaveArgs& W, bool keep, uint32_t s)
{
    if (W.live_bits) {
        if (keep) atomicOr(W.live_bits + (s >> 5), 1u << (s & 31u));
    } else {
        wave_push(W.act_out, W.n_out, keep, s);
    }
}

// The next round's live list in slot order, from the live bits of a refill round (offsets by
// k_word_scan / k_block_scan over the same words); the bits are cleared for the round after.
// A refilled pool is nearly full, so slot order makes the next round's slot reads and writes
// almost sequential, where appends in finishing order scatter them over the pool.
__global__ void k_wave_act(uint32_t* bits, long long nword, const uint32_t* wordoff, const uint32_t* blocksum,
                           const long long* total, uint32_t* act, unsigned* n)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) *n = (unsigned)*total;
    const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;     // one word per thread
    if (w >= nword) return;
    uint32_t b = bits[w];
    if (!b) return;
    bits[w] = 0u;
    uint32_t* o = act + (long long)blocksum[w >> 8] + wordoff[w];
    const uint32_t s0 = (uint32_t)(w << 5);
    for (int k = 0; b != 0u && k < 32; k++) {
        const int lane = __ffs(b) - 1;
        *o++ = s0 + (uint32_t)lane;
        b &= b - 1u;
    }
}

// Lanes in `need` take new photons from the queue until each has a path that can be traced
// (photons that cannot take a first bounce are finished at once) or the queue is empty.
// Returns true in the lanes that hold a live path.  Warp-collective.
template <int CV, bool ADJ = false>
PHX_D bool wave_refill(PhxLane& L, const PersistArgs& A, bool need, unsigned& status, PhxScore* sc = nullptr,
                       const uint32_t* planes = nullptr)
{
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    bool live = false;
    for (int guard = 0; guard < 64; guard++) {
        const unsigned m = __ballot_sync(FULL, need);
        if (!m) break;
        unsigned long long base = 0ull;
        if (lane == (unsigned)(__ffs(m) - 1)) base = atomicAdd(A.queue, (unsigned long long)__popc(m));
        base = __shfl_sync(FULL, base, __ffs(m) - 1);
        if ((long long)base >= A.N) break;                  // queue exhausted for every lane
        if (need) {
            const long long idx = (long long)base + __popc(m & ((1u << lane) - 1u));
            if (idx >= A.N) {
                need = false;
            } else {
                persist_start<CV, ADJ>(L, A, idx, status, sc, planes);
                if (wave_can_trace(L, A)) { live = true; need = false; }
                else persist_finish<CV, ADJ>(L, A, sc);
            }
        }
    }
    return live;
}

// the generating kernels' copy of a single-event jump table (block-collective; null when the call
// advances its states some other way)
PHX_D const uint32_t* wave_jump_planes(const PersistArgs& A)
{
    __shared__ uint32_t planes[5 * PHX_JUMP_PLANE];
    if (!A.jump4 || A.gs_event || A.ev_rng || A.event_index == 0ull) return nullptr;
    phx_jump_planes_load(planes, A.jump4);
    __syncthreads();
    return planes;
}

// resident 128-thread blocks per SM asked for the generating kernels (k_wave_init, k_wave_fill;
// not the adjoint forms)
#ifndef PHX_WAVE_FILL_MINB
#define PHX_WAVE_FILL_MINB 6
#endif

// fill the pool: every slot takes photons until it holds a live path or the queue is empty
template <int CV, bool ADJ = false>
__global__ void __launch_bounds__(128, ADJ ? 1 : PHX_WAVE_FILL_MINB) k_wave_init(WaveArgs W)
{
    unsigned status = 0;
    PhxLane L;
    PhxScore score;
    if (ADJ) wave_score_setup(score, W.A);
    float4* st = wave_stage_area();
    const uint32_t* planes = wave_jump_planes(W.A);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < W.pool; base += stride) {
        const long long s = base + (threadIdx.x & 31);
        const bool live = wave_refill<CV, ADJ>(L, W.A, s < W.pool, status, ADJ ? &score : nullptr, planes);
        wave_put(W, st, (uint32_t)s, L, live, true);
        if (ADJ && live) wave_store_score(W, (uint32_t)s, &score);
        wave_append(W, live, (uint32_t)s);
    }
    if (status) atomicOr(W.A.status, status);
}

// closest hit of every live path (CSGOptiX/CSGOptiX7.cu:477-490: tmin by the last flag, optixTrace)
// resident 128-thread blocks per SM asked of the compiler for the closest-hit kernel (caps its
// registers: 3 -> 168 registers, 12 warps per SM, no spills; 4 -> 128 with spills, measured slower)
#ifndef PHX_WAVE_TRACE_MINB
#define PHX_WAVE_TRACE_MINB 3
#endif

template <int CV>
__global__ void __launch_bounds__(128, PHX_WAVE_TRACE_MINB) k_wave_trace(WaveArgs W)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) { *W.n_out = 0u; *W.n_free = 0u; }   // the launches after this one append
    const unsigned n = *W.n_in;
    unsigned status = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)n; i += stride) {
        const uint32_t s = W.act_in[i];
        const PhxWaveSlot* o = W.slot + s;
        const float4 q0 = o->q0, q1 = o->q1;
        const float tmin = wave_tmin(W, q1);
        const PhxPRD prd = phx_trace_step<CV>(W.A.S, make_float3(q0.x, q0.y, q0.z), make_float3(q1.x, q1.y, q1.z), tmin,
                                                  W.A.C.tmax, status);
        W.prd[s].nd = make_float4(prd.normal.x, prd.normal.y, prd.normal.z, prd.distance);
        W.prd[s].lgi = make_uint4(__float_as_uint(prd.lposcost), prd.gp_bd, prd.ii_id, 0u);
    }
    if (status) atomicOr(W.A.status, status);
}

// The closest-hit round with persistent warps that refill finished lanes: each warp takes the
// round's rays 32 indices at a time (one atomic per 32 rays), and whenever lanes of the warp have
// finished their ray they start the next ones of the window, so the warp keeps stepping with
// most lanes busy instead of waiting for its slowest ray.  A ray starts by testing the global
// leaves, then (unless the cull ball holds the whole segment) walks the hierarchy from its own
// stack, in the same order and with the same arithmetic as phx_trace: the PRDs are the same as
// the plain kernel's.
#ifndef PHX_WAVE_TRACE_DF
#define PHX_WAVE_TRACE_DF 1
#endif
template <int CV>
__global__ void __launch_bounds__(128, PHX_WAVE_TRACE_MINB) k_wave_trace_df(WaveArgs W)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) { *W.n_out = 0u; *W.n_free = 0u; }   // the launches after this one append
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    const unsigned n = *W.n_in;
    const PhxScene& S = W.A.S;
    unsigned status = 0;
    unsigned wnext = 0u, wend = 0u;       // this warp's unassigned ray indices [wnext, wend)
    bool drained = false;                 // the round's rays are all handed out
    bool has = false;                     // this lane holds a ray
    uint32_t s = 0u;
    float3 o = make_float3(0.f, 0.f, 0.f), d = o, inv = o, oi = o;
    float tmin = 0.f;
    PhxBest B;
    B.t = 0.f; B.L = make_int4(-1, 0, 0, 0); B.isect = make_float4(0.f, 0.f, 0.f, 0.f); B.lposcost = 0.f;
    int2 stk[PHX_BVH_STACK];         // node or leaf range, near distance bits
    int sp = 0;
    for (;;) {
        // hand new rays to the idle lanes (at most a window and a fresh window per step)
        unsigned idle = __ballot_sync(FULL, !has);
        // idle lanes a warp waits for before it takes new rays (32: only when the whole warp is done)
        if (__popc(idle) < W.refill_idle) idle = 0u;
        for (int pass = 0; pass < 2 && idle != 0u && !drained; pass++) {
            if (wnext >= wend) {
                unsigned b = 0u;
                if (lane == 0u) b = atomicAdd(W.trace_ctr, 32u);
                b = __shfl_sync(FULL, b, 0);
                if (b >= n) { drained = true; break; }
                wnext = b;
                wend = min(b + 32u, n);
            }
            const unsigned take = min((unsigned)__popc(idle), wend - wnext);
            const unsigned rank = __popc(idle & below);
            if (!has && rank < take) {
                s = W.act_in[wnext + rank];
                const PhxWaveSlot* ps = W.slot + s;
                const float4 q0 = ps->q0, q1 = ps->q1;
                tmin = wave_tmin(W, q1);
                o = make_float3(q0.x, q0.y, q0.z);
                d = make_float3(q1.x, q1.y, q1.z);
                phx_ray_slabs(o, d, inv, oi);
                B.t = W.A.C.tmax; B.L = make_int4(-1, 0, 0, 0); B.isect = make_float4(0.f, 0.f, 0.f, 0.f); B.lposcost = 0.f;
                sp = 0;
                // the global leaves first, then the hierarchy unless the cull ball holds the segment
                for (int g = 0; g < S.num_global; g++)
                    phx_test_leaf<CV>(S, __ldg(reinterpret_cast<const int4*>(S.globals + g)), __ldg(S.global_sph + g), o, d, tmin, B,
                                      status);
                if (!S.bvh_empty && !phx_culled(S, o, d, tmin, B.t)) { stk[0] = make_int2(0, __float_as_int(tmin)); sp = 1; }
                has = true;
            }
            wnext += take;
            idle = __ballot_sync(FULL, !has);
        }
        // finish the rays whose stacks are empty
        if (has) {
            while (sp > 0 && __int_as_float(stk[sp - 1].y) > B.t) sp--;
            if (sp == 0) {
                PhxPRD prd;
                phx_best_prd(S, B, prd);
                W.prd[s].nd = make_float4(prd.normal.x, prd.normal.y, prd.normal.z, prd.distance);
                W.prd[s].lgi = make_uint4(__float_as_uint(prd.lposcost), prd.gp_bd, prd.ii_id, 0u);
                has = false;
            }
        }
        const bool leaf_top = has && stk[sp - 1].x < 0;
        const unsigned want_leaf = __ballot_sync(FULL, leaf_top);
        const unsigned want_node = __ballot_sync(FULL, has && !leaf_top);
        if (!(want_leaf | want_node)) {
            if (drained) break;
            continue;
        }
        // one step: the lanes whose next entry is a leaf range, or those whose next entry is a node
        const bool leaf_step = want_node == 0u || __popc(want_leaf) * PHX_TRACE_LEAF_WEIGHT >= __popc(want_node);
        if (!has || leaf_top != leaf_step) continue;
        sp--;
        const int ni = stk[sp].x;
        if (leaf_step) {
            const int enc = -ni - 1;
            const int first = enc >> 3;
            const int count = (enc & 7) + 1;
            for (int li = first; li < first + count; li++)
                phx_test_leaf<CV>(S, __ldg(reinterpret_cast<const int4*>(S.leaves + li)), __ldg(S.leaf_sph + li), o, d, tmin, B, status);
        } else {
            phx_visit_node(S, ni, inv, oi, tmin, B.t, stk, sp, status);
        }
    }
    if (status) atomicOr(W.A.status, status);
}

// The last live paths of a call, once few remain and no photons wait in the queue: persistent
// warps run them to the end with the one-kernel loop's step (persist_step: the shared closest-hit
// and physics code), so a long chain no longer costs two launches per bounce.  A lane whose path
// ends takes the next one of the list at once (one atomic per warp on the round's ray counter,
// which the physics kernel left at zero), so the lanes of a warp do not wait for its longest path.
// Photons, seq and hits are the same as the rounds would give.
template <int CV, bool ADJ = false>
__global__ void __launch_bounds__(128) k_wave_tail(WaveArgs W)
{
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned n = *W.n_in;
    unsigned status = 0;
    PhxLane L;
    PhxScore score;
    if (ADJ) wave_score_setup(score, W.A);
    bool has = false, drained = false;
    for (;;) {
        const unsigned idle = drained ? 0u : __ballot_sync(FULL, !has);
        if (idle) {
            const unsigned leader = __ffs(idle) - 1u;
            unsigned base = 0u;
            if (lane == leader) base = atomicAdd(W.trace_ctr, (unsigned)__popc(idle));
            base = __shfl_sync(FULL, base, (int)leader);
            if (base >= n) drained = true;
            if (!has) {
                const unsigned k = base + __popc(idle & ((1u << lane) - 1u));
                if (k < n) {
                    const uint32_t s = W.act_in[k];
                    wave_load(W, s, L);
                    if (ADJ) wave_load_score(W, s, &score);
                    has = true;
                }
            }
        }
        if (!__any_sync(FULL, has)) break;
        // persist_step ends a path within max_bounce steps
        if (has && persist_step<CV, ADJ>(L, W.A, status, ADJ ? &score : nullptr)) {
            persist_finish<CV, ADJ>(L, W.A, ADJ ? &score : nullptr);
            has = false;
        }
    }
    if (status) atomicOr(W.A.status, status);
}

// physics of every live path after its closest hit (CSGOptiX/CSGOptiX7.cu:491-509), finishing
// and refilling slots; live slots go to the next round's list
// resident 128-thread blocks per SM asked for the physics kernel (its loads of path state are
// latency-bound, so occupancy matters more than registers); the adjoint form carries the score
// terms as well and is left to the compiler
#ifndef PHX_WAVE_SHADE_MINB
#define PHX_WAVE_SHADE_MINB 7
#endif
#ifndef PHX_WAVE_SHADE_ADJ_MINB
#define PHX_WAVE_SHADE_ADJ_MINB 1
#endif

// the physics of one path whose slot is in the warp's staging area; true when it goes on
template <int CV, bool ADJ>
PHX_D bool wave_shade_path(const WaveArgs& W, const float4* st, uint32_t s, const float4 nd, const uint4 lgi, PhxLane& L,
                           PhxScore* sc, unsigned& status)
{
    float4 c[8];
    wave_stage_get(st, c);
    wave_unpack(c, L);                   // the photon index is read only when the path finishes
    if (ADJ) wave_load_score(W, s, sc);
    PhxPRD prd;
    prd.normal = make_float3(nd.x, nd.y, nd.z);
    prd.distance = nd.w;
    prd.lposcost = __uint_as_float(lgi.x);
    prd.gp_bd = lgi.y;
    prd.ii_id = lgi.z;
    bool done = true;
    if (prd.boundary() != 0xffffu) {
        int command;
        if (ADJ) {
            prd.normal = normalize(prd.normal);
            command = propagate<true>(L.p, L.rng, prd, W.A.P, status, sc);
        } else {
            command = phx_propagate_step(L.p, L.rng, prd, W.A.P, status);
        }
        L.bounce++;
        seq_add_nibble(L.seqhis, L.seqbnd, (unsigned)L.bounce, L.p.flag(), L.p.boundary());
        done = command == PHX_BREAK || !wave_can_trace(L, W.A);
    }
    if (done) {
        L.idx = W.sidx[s];
        persist_finish<CV, ADJ>(L, W.A, sc);
    }
    return !done;
}

template <int CV, bool ADJ = false>
__global__ void __launch_bounds__(128, ADJ ? PHX_WAVE_SHADE_ADJ_MINB : PHX_WAVE_SHADE_MINB) k_wave_shade(WaveArgs W)
{
    if (blockIdx.x == 0 && threadIdx.x == 0 && W.trace_ctr) *W.trace_ctr = 0u;   // for the next round's closest-hit kernel
    const unsigned n = *W.n_in;
    unsigned status = 0;
    PhxLane L;
    PhxScore score;
    if (ADJ) wave_score_setup(score, W.A);
    const unsigned lane = threadIdx.x & 31u;
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
    float4* st = wave_stage_area();
    for (; base < (long long)n; base += stride) {
        const long long i = base + lane;
        const bool valid = i < (long long)n;
        const uint32_t s = valid ? W.act_in[i] : 0u;
        float4 nd = make_float4(0.f, 0.f, 0.f, 0.f);
        uint4 lgi = make_uint4(0u, 0u, 0u, 0u);
        if (valid) { nd = W.prd[s].nd; lgi = W.prd[s].lgi; }     // in flight with the slot reads
        wave_gather(W, st, s, valid);
        const bool live = valid && wave_shade_path<CV, ADJ>(W, st, s, nd, lgi, L, ADJ ? &score : nullptr, status);
        wave_put(W, st, s, L, live, false);
        if (ADJ && live) wave_store_score(W, s, &score);
        wave_append(W, live, s);
        wave_push(W.free_list, W.n_free, valid && !live, s);
    }
    if (status) atomicOr(W.A.status, status);
}

// new photons from the queue into the slots freed this round (warp-coherent generation)
template <int CV, bool ADJ = false>
__global__ void __launch_bounds__(128, ADJ ? 1 : PHX_WAVE_FILL_MINB) k_wave_fill(WaveArgs W)
{
    const unsigned n = *W.n_free;
    // the whole block leaves or stays (other blocks move the queue head meanwhile)
    __shared__ int drained;
    if (threadIdx.x == 0) drained = (long long)*W.A.queue >= W.A.N;
    __syncthreads();
    if (drained) return;
    unsigned status = 0;
    PhxLane L;
    PhxScore score;
    if (ADJ) wave_score_setup(score, W.A);
    float4* st = wave_stage_area();
    const uint32_t* planes = wave_jump_planes(W.A);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < (long long)n; base += stride) {
        const long long i = base + (threadIdx.x & 31);
        const bool valid = i < (long long)n;
        const uint32_t s = valid ? W.free_list[i] : 0u;
        const bool live = wave_refill<CV, ADJ>(L, W.A, valid, status, ADJ ? &score : nullptr, planes);
        wave_put(W, st, s, L, live, true);
        if (ADJ && live) wave_store_score(W, s, &score);
        wave_append(W, live, s);
    }
    if (status) atomicOr(W.A.status, status);
}
