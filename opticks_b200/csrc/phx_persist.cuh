// phx_persist.cuh : persistent-thread photon kernel with a device work queue.
//
// Many events of uneven size (or one large event) are flattened into one photon index space.
// Each warp takes chunks of photon indices from a global counter; a lane whose photon finishes
// is refilled with the next index from the warp's chunk every `regroup` bounces, so lanes do
// not idle until the longest photon of their warp ends (the divergence of a one-thread-per-photon
// launch).  Photon j of genstep g belongs to event ev[g]; its RNG slot is its index within the
// event and its stream is advanced by skipahead(event * skip), exactly as a separate launch of
// that event would do (qudarap/qrng.h:85-90 with photon_slot_offset, CSGOptiX/CSGOptiX7.cu:441),
// so batched results are identical to the per-event loop.
//
// There are no waits: the queue is a monotonic atomic counter, loops are bounded by the number
// of photons, and each photon's bounce count is bounded by max_bounce.
#pragma once
#include "phx_kernels.cuh"

struct PersistArgs {
    PhxScene S;
    PhxProps P;
    PhxLoopCfg C;
    const float4* gs;
    const long long* gs_off;        // (G+1) photon offsets of the gensteps
    int G;
    long long N;
    long long photon_offset;        // single-event mode: absolute index of photon 0
    unsigned long long event_index; // single-event mode: event index
    const int* gs_event;            // batched mode: event index of each genstep (non-decreasing), or null
    const long long* ev_start;      // batched mode: photon offset of the first photon of each genstep's event
    unsigned long long skip;
    unsigned long long seed, rng_offset;   // curand_init arguments for photons beyond the prepared slots
    const uint32_t* rng;
    long long rng_slots;
    const uint32_t* jump;           // event jump matrices: one (single event) or one per genstep (batched)
    const uint32_t* jump4;          // the 4-bit group tables of those matrices (same indexing), or null
    const uint32_t* ev_rng;         // optional: XORWOW states already advanced to each photon's event
    long long ev_rng_n;             //   (six planes of ev_rng_n words, by photon index; k_rng_event)
    phx_photon* photon;
    phx_seq* seq;
    uint32_t* hitword;              // zeroed before launch; bits set with atomicOr
    unsigned hit_mask;
    unsigned* status;
    unsigned long long* queue;      // work counter, zeroed before launch
    int regroup;                    // bounces between refills
    int chunk;                      // queue grab per warp, in units of 32 photons
    unsigned* ev_left;              // optional: photons left per event (batched), for completion times
    unsigned long long* ev_done_ns; // optional: globaltimer when the event's last photon finished
    int num_event;
    // adjoint (ADJ kernels): per-sensor hit counts and score sums, (num_sensor) and (num_sensor, 32)
    double* adj_hits;
    double* adj_grad;
    int num_sensor;
    unsigned adj_mat;
    float adj_nm0, adj_nms, adj_wl_lo, adj_binw;
    int adj_pathwise;               // carry the refraction tangent (d/d n terms beyond the Fresnel score)
    const int* adj_prim_node;       // root node of each prim, for the tangent's probe intersections
};

// the block's shared score area (32 terms x PHX_SCORE_LANES threads, 16 KB), this thread's column
PHX_D float* score_area()
{
    __shared__ float sg[32 * PHX_SCORE_LANES];
    return sg + threadIdx.x;
}

// the adjoint accumulator's constant fields for one kernel
PHX_D void score_setup(PhxScore& score, const PersistArgs& A)
{
    score.g = score_area();
    score.mat = A.adj_mat; score.nm0 = A.adj_nm0; score.nms = A.adj_nms;
    score.wl_lo = A.adj_wl_lo; score.binw = A.adj_binw;
    score.pathwise = A.adj_pathwise;
    score.csg = A.S.csg;
    score.inst_inv = A.S.inst_inv;
    score.prim_node = A.adj_prim_node;
    score.tmin = A.C.tmin; score.tmin0 = A.C.tmin0; score.eps0_mask = A.C.eps0_mask;
    score_tangent_reset(score);
}

PHX_D unsigned long long phx_globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// One compiled copy of the closest-hit search and of the physics step, called by the one-kernel
// loop and by the wavefront kernels: with fast-math contraction decided per inlining context,
// sharing the code is what keeps the two forms bit-identical.
#ifndef PHX_STEP_OUTLINE_TRACE
#define PHX_STEP_OUTLINE_TRACE 0
#endif
#ifndef PHX_STEP_OUTLINE_PROP
#define PHX_STEP_OUTLINE_PROP 1
#endif
#if PHX_STEP_OUTLINE_TRACE
#define PHX_STEPFN_T __device__ __noinline__
#else
#define PHX_STEPFN_T __device__ __forceinline__
#endif
#if PHX_STEP_OUTLINE_PROP
#define PHX_STEPFN_P __device__ __noinline__
#else
#define PHX_STEPFN_P __device__ __forceinline__
#endif

template <int CV>
PHX_STEPFN_T PhxPRD phx_trace_step(const PhxScene S, const float3 o, const float3 d, const float tmin, const float tmax,
                                 unsigned& status)
{
    PhxPRD prd;
    phx_trace<CV>(S, o, d, tmin, tmax, prd, status);
    return prd;
}

// the PRD normal is normalised here (CSGOptiX/CSGOptiX7.cu:491-498) as part of the shared step
#ifndef PHX_PROP_IO
#define PHX_PROP_IO 1
#endif
#if PHX_PROP_IO
// The photon and its RNG state go in and come back by value: the out-of-line step then takes no
// address of the caller's copies, which stay in registers (by reference they live in local
// memory for the whole caller).  Every caller shares this one compiled step.
struct PhxStepIO {
    PhxPhoton p;
    curandStateXORWOW rng;
    unsigned status;
    int command;
};
PHX_STEPFN_P PhxStepIO phx_propagate_io(PhxStepIO io, PhxPRD prd, const PhxProps P)
{
    prd.normal = normalize(prd.normal);
    io.command = propagate<false>(io.p, io.rng, prd, P, io.status, nullptr);
    return io;
}

PHX_D int phx_propagate_step(PhxPhoton& p, curandStateXORWOW& rng, PhxPRD prd, const PhxProps& P, unsigned& status)
{
    PhxStepIO io;
    io.p = p;
    io.rng = rng;
    io.status = 0u;
    io.command = 0;
    io = phx_propagate_io(io, prd, P);
    p = io.p;
    rng = io.rng;
    status |= io.status;
    return io.command;
}
#else
PHX_STEPFN_P int phx_propagate_step(PhxPhoton& p, curandStateXORWOW& rng, PhxPRD prd, const PhxProps P, unsigned& status)
{
    prd.normal = normalize(prd.normal);
    return propagate<false>(p, rng, prd, P, status, nullptr);
}
#endif

struct PhxLane {
    PhxPhoton p;
    curandStateXORWOW rng;
    unsigned long long seqhis[2], seqbnd[2];
    long long idx;
    int bounce;
    int ev;
};

// the 4-bit group tables of a single-event jump matrix staged in shared memory as five word planes
// (plane w holds word w of every entry), so a warp's 32 lookups in one group read 16 consecutive
// words of each plane: no bank conflicts.  The same entries are XOR-ed as by phx_rng_jump4.
#define PHX_JUMP_PLANE (PHX_JUMP_BITS / 4 * 16)
PHX_D void phx_jump_planes_load(uint32_t* P, const uint32_t* __restrict__ T)
{
    for (int i = threadIdx.x; i < 5 * PHX_JUMP_PLANE; i += blockDim.x) {
        const int w = i / PHX_JUMP_PLANE, e = i - w * PHX_JUMP_PLANE;
        P[i] = __ldg(T + (size_t)e * PHX_JUMP_COLW + w);
    }
}

PHX_D void phx_rng_jump4_planes(curandStateXORWOW& s, const uint32_t* P, unsigned long long n)
{
    uint32_t o0 = 0u, o1 = 0u, o2 = 0u, o3 = 0u, o4 = 0u;
    const uint32_t in[5] = { s.v[0], s.v[1], s.v[2], s.v[3], s.v[4] };
#pragma unroll 1
    for (int w = 0; w < 5; w++) {
        const uint32_t x = in[w];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int e = (8 * w + q) * 16 + (int)((x >> (4 * q)) & 15u);
            o0 ^= P[e]; o1 ^= P[PHX_JUMP_PLANE + e]; o2 ^= P[2 * PHX_JUMP_PLANE + e];
            o3 ^= P[3 * PHX_JUMP_PLANE + e]; o4 ^= P[4 * PHX_JUMP_PLANE + e];
        }
    }
    s.v[0] = o0; s.v[1] = o1; s.v[2] = o2; s.v[3] = o3; s.v[4] = o4;
    s.d += (unsigned int)((362437ull * n) & 0xffffffffull);
}

// the XORWOW state of RNG slot `slot` advanced by skipahead(event * skip) (qudarap/qrng.h:85-90);
// `planes`: the single-event group tables staged in shared memory, or null
PHX_D void phx_event_rng(curandStateXORWOW& s, const PersistArgs& A, int gi, long long slot, unsigned long long ev, unsigned& status,
                         const uint32_t* planes = nullptr)
{
    if (slot < A.rng_slots) {
        phx_load_rng(s, A.rng, A.rng_slots, slot);
    } else {
        // same state as a prepared slot, computed on the fly (slower; flagged)
        status |= PHX_STATUS_RNG_RANGE;
        curand_init(A.seed, (unsigned long long)slot, A.rng_offset, &s);
    }
    if (ev > 0ull) {
        if (planes) phx_rng_jump4_planes(s, planes, A.skip * ev);
        else if (A.jump4) phx_rng_jump4(s, A.jump4 + (A.gs_event ? (size_t)gi * PHX_JUMP_NIBW : 0), A.skip * ev);
        else if (A.jump) phx_rng_jump(s, A.jump + (A.gs_event ? (size_t)gi * PHX_JUMP_MATW : 0), A.skip * ev);
        else skipahead(A.skip * ev, &s);
    }
}

template <int CV, bool ADJ>
PHX_D void persist_start(PhxLane& L, const PersistArgs& A, long long idx, unsigned& status, PhxScore* sc,
                         const uint32_t* planes = nullptr)
{
    if (ADJ) {
#pragma unroll
        for (int k = 0; k < 32; k++) PHX_SG(*sc, k) = 0.f;
        score_tangent_reset(*sc);
    }
    const int gi = phx_find_genstep(A.gs_off, A.G, idx);
    const float4* g = A.gs + 6 * gi;     // read in place: a local copy would live in local memory
    long long slot;
    unsigned long long ev;
    if (A.gs_event) {
        ev = (unsigned long long)__ldg(A.gs_event + gi);
        slot = idx - __ldg(A.ev_start + gi);
    } else {
        ev = A.event_index;
        slot = A.photon_offset + idx;
    }
    if (A.ev_rng) {
        phx_load_rng(L.rng, A.ev_rng, A.ev_rng_n, idx);
    } else {
        phx_event_rng(L.rng, A, gi, slot, ev, status, planes);
    }
    memset(&L.p, 0, sizeof(L.p));
    generate_photon(L.p, L.rng, g, (unsigned long long)slot, A.P, status);
    L.seqhis[0] = L.seqhis[1] = L.seqbnd[0] = L.seqbnd[1] = 0ull;
    seq_add_nibble(L.seqhis, L.seqbnd, 0u, L.p.flag(), L.p.boundary());
    L.idx = idx;
    L.bounce = 0;
    L.ev = (int)ev;
}

template <int CV, bool ADJ>
PHX_D void persist_finish(PhxLane& L, const PersistArgs& A, const PhxScore* sc)
{
    const long long idx = L.idx;
    if (ADJ && (L.p.flagmask & A.hit_mask) == A.hit_mask) {
        // estimator of d E[hits_s] / d theta : sum over hits on s of the path score
        const unsigned id = L.p.identity & 0xffffffu;
        if (id > 0u && (int)(id - 1u) < A.num_sensor) {
            const unsigned s = id - 1u;
            atomicAdd(A.adj_hits + s, 1.0);
            for (int k = 0; k < 32; k++)
                if (PHX_SG(*sc, k) != 0.f) atomicAdd(A.adj_grad + (size_t)s * 32 + k, (double)PHX_SG(*sc, k));
        }
    }
    if (A.photon) phx_store_photon(A.photon + idx, L.p);
    if (A.seq) {
        ulonglong2* s = reinterpret_cast<ulonglong2*>(A.seq + idx);
        s[0] = make_ulonglong2(L.seqhis[0], L.seqhis[1]);
        s[1] = make_ulonglong2(L.seqbnd[0], L.seqbnd[1]);
    }
    if (A.hitword && (L.p.flagmask & A.hit_mask) == A.hit_mask) atomicOr(A.hitword + (idx >> 5), 1u << (idx & 31));
    if (A.ev_left) {
        // one atomic per event among the lanes finishing together; the lane whose subtraction
        // empties the count stamps the event's completion time
        const int e = A.gs_event ? L.ev : 0;
        if (e >= 0 && e < A.num_event) {
            const unsigned peers = __match_any_sync(__activemask(), e);
            const unsigned n = (unsigned)__popc(peers);
            if ((int)(threadIdx.x & 31u) == __ffs(peers) - 1 && atomicSub(A.ev_left + e, n) == n)
                A.ev_done_ns[e] = phx_globaltimer();
        }
    }
}

// one bounce of CSGOptiX/CSGOptiX7.cu:477-509; returns true when the photon is finished
template <int CV, bool ADJ>
PHX_D bool persist_step(PhxLane& L, const PersistArgs& A, unsigned& status, PhxScore* sc)
{
    if (!(L.bounce < A.C.max_bounce && L.p.time < A.C.max_time)) return true;
    const float tmin = (L.p.obf & A.C.eps0_mask) ? A.C.tmin0 : A.C.tmin;
    PhxPRD prd;
    if (ADJ) phx_trace<CV>(A.S, L.p.pos, L.p.mom, tmin, A.C.tmax, prd, status);
    else prd = phx_trace_step<CV>(A.S, L.p.pos, L.p.mom, tmin, A.C.tmax, status);
    if (prd.boundary() == 0xffffu) return true;
    int command;
    if (ADJ) {
        prd.normal = normalize(prd.normal);
        command = propagate<ADJ>(L.p, L.rng, prd, A.P, status, sc);
    } else {
        command = phx_propagate_step(L.p, L.rng, prd, A.P, status);
    }
    L.bounce++;
    seq_add_nibble(L.seqhis, L.seqbnd, (unsigned)L.bounce, L.p.flag(), L.p.boundary());
    return command == PHX_BREAK;
}

// Minimum resident warps per SM asked of the compiler (caps registers per thread); 0 leaves the
// register count to the compiler.
#ifndef PHX_PERSIST_MIN_WARPS
#define PHX_PERSIST_MIN_WARPS 0
#endif
#define PHX_PERSIST_MINB(BLOCK) ((PHX_PERSIST_MIN_WARPS * 32 / (BLOCK)) > 0 ? (PHX_PERSIST_MIN_WARPS * 32 / (BLOCK)) : 1)

template <int CV, int BLOCK, bool ADJ = false>
__global__ void __launch_bounds__(BLOCK, PHX_PERSIST_MINB(BLOCK)) k_sim_persistent(PersistArgs A)
{
    static_assert(!ADJ || BLOCK <= PHX_SCORE_LANES, "score-carrying blocks hold at most PHX_SCORE_LANES threads");
    PhxScore score;
    if (ADJ) score_setup(score, A);
    PhxScore* sc = ADJ ? &score : nullptr;
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lanes_below = (1u << lane) - 1u;
    const long long grab = 32ll * (long long)(A.chunk > 0 ? A.chunk : 1);
    const int regroup = A.regroup > 0 ? A.regroup : 1;
    long long wnext = 0, wend = 0;   // warp-uniform pool of photon indices
    bool exhausted = false;
    bool active = false;
    unsigned status = 0;
    PhxLane L;
    for (;;) {
        unsigned need = __ballot_sync(FULL, !active);
        while (need && !exhausted) {
            if (wnext >= wend) {
                unsigned long long base = 0ull;
                if (lane == 0) base = atomicAdd(A.queue, (unsigned long long)grab);
                base = __shfl_sync(FULL, base, 0);
                if ((long long)base >= A.N) { exhausted = true; break; }
                wnext = (long long)base;
                wend = min(wnext + grab, A.N);
            }
            const long long avail = wend - wnext;
            unsigned take = need;
            if ((long long)__popc(take) > avail) {
                // keep the lowest `avail` requesting lanes
                unsigned t = 0u, m = need;
                for (long long k = 0; k < avail; k++) { const unsigned b = m & (0u - m); t |= b; m ^= b; }
                take = t;
            }
            if ((take >> lane) & 1u) {
                persist_start<CV, ADJ>(L, A, wnext + __popc(take & lanes_below), status, sc);
                active = true;
            }
            wnext += __popc(take);
            need &= ~take;
        }
        if (!__any_sync(FULL, active)) break;
        for (int k = 0; k < regroup; k++) {
            if (active && persist_step<CV, ADJ>(L, A, status, sc)) {
                persist_finish<CV, ADJ>(L, A, sc);
                active = false;
            }
        }
    }
    if (status) atomicOr(A.status, status);
}

// per genstep: photon offset of the first photon of its event (gs_event non-decreasing)
__global__ void k_event_starts(const int* gs_event, const long long* gs_off, int G, long long* ev_start)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const int ev = gs_event[g];
    int lo = 0, hi = g;   // first index with gs_event == ev
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (gs_event[mid] < ev) lo = mid + 1; else hi = mid;
    }
    ev_start[g] = gs_off[lo];
}

// photons per event (for completion times): ev_left[e] = sum of genstep counts of event e
__global__ void k_event_counts(const int* gs_event, const long long* gs_off, int G, unsigned* ev_left, int num_event)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const int ev = gs_event[g];
    if (ev >= 0 && ev < num_event) atomicAdd(ev_left + ev, (unsigned)(gs_off[g + 1] - gs_off[g]));
}

// largest photon count of one event (the RNG slots a batched launch needs)
__global__ void k_event_max(const long long* gs_off, const long long* ev_start, int G, unsigned long long* out)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    atomicMax(out, (unsigned long long)(gs_off[g + 1] - ev_start[g]));
}

__global__ void k_stamp(unsigned long long* t)
{
    *t = phx_globaltimer();
}

// Event-advanced XORWOW state of every photon of the call, by photon index, ahead of the loop:
// consecutive photons share their genstep and jump matrix, so the 160-column GF(2) product runs
// with whole warps here instead of in the few lanes that start a photon at a time in the loop.
__global__ void k_rng_event(PersistArgs A, uint32_t* out, long long n)
{
    unsigned status = 0;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int gi = phx_find_genstep(A.gs_off, A.G, idx);
        long long slot;
        unsigned long long ev;
        if (A.gs_event) {
            ev = (unsigned long long)__ldg(A.gs_event + gi);
            slot = idx - __ldg(A.ev_start + gi);
        } else {
            ev = A.event_index;
            slot = A.photon_offset + idx;
        }
        curandStateXORWOW s;
        phx_event_rng(s, A, gi, slot, ev, status);
        out[idx] = s.d;
        out[n * 1 + idx] = s.v[0];
        out[n * 2 + idx] = s.v[1];
        out[n * 3 + idx] = s.v[2];
        out[n * 4 + idx] = s.v[3];
        out[n * 5 + idx] = s.v[4];
    }
    if (status) atomicOr(A.status, status);
}
