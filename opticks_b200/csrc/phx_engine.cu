// phx_engine.cu : kernels and the C ABI of the photon engine (include/phox.h).
//
// Data layout in HBM (one engine per device):
//   node/itra/plan      CSGFoundry arrays, uploaded unchanged (float4 rows)
//   bvh, leaves         4-wide BVH over (instance, prim) leaves, built on the host (phx_bvh.cc)
//   inst_inv            world->object transform per instance (4 float4 rows)
//   bnd texture         float4 (num_wl x num_bnd*8), hardware linear filter like qudarap/QBnd.cc:155
//   icdf texture        float  (4096 x 3), hardware linear filter like qudarap/QScint.cc:104
//   rng                 cuRAND XORWOW state per photon slot, SoA of six u32 words (24 B/slot)
//   photon, seq, hit    sphoton (64 B), sseq (32 B), sphoton per hit
//   hitword             one bit per photon (hit mask ballot), scanned to compact hits in order
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <cstdio>
#include <cstring>
#include <cstdarg>
#include <cmath>
#include <string>
#include <vector>
#include <algorithm>

#include "phox.h"
#include "phx_pod.h"
#include "phx_bvh.h"
#include "phx_kernels.cuh"
#include "phx_persist.cuh"
#include "phx_wave.cuh"
#include "phx_rngjump.h"

// ------------------------------------------------------------------ error plumbing
static thread_local std::string g_last_error;
static int phx_fail(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}
#define PHX_CU(call)                                                                         \
    do {                                                                                     \
        cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess)                                                               \
            return phx_fail(-2, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); \
    } while (0)

// ------------------------------------------------------------------ engine state
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t want)
    {
        if (want <= n && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr; n = 0;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(want, 1) * sizeof(T));
        if (e == cudaSuccess) n = want;
        return e;
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
};

#include "phx_merge.cuh"

// scratch of the hit merge (grow-only, per engine)
struct PhxMergeWs {
    DevBuf<uint32_t> sel, tcount, val0, val1, head, tsum, hist, pmin, gor, gsum, hin, hout;
    DevBuf<unsigned long long> key0, key1, amin, key_or;
    DevBuf<long long> total;
    void release()
    {
        sel.release(); tcount.release(); val0.release(); val1.release(); head.release(); tsum.release(); hist.release();
        pmin.release(); gor.release(); gsum.release(); hin.release(); hout.release();
        key0.release(); key1.release(); amin.release(); key_or.release(); total.release();
    }
};

struct PhxBatchCall {
    const float* gs; const int32_t* ev; int G; long long N; int block, chunk, regroup, num_event;
    uint64_t* done; float* photon; uint64_t* seq; float* hit; long long hcap; uint32_t* sensor; cudaStream_t st;
    bool operator==(const PhxBatchCall& o) const { return memcmp(this, &o, sizeof(*this)) == 0; }
};

struct phx_engine {
    int device = 0;
    phx_config cfg;
    cudaStream_t stream = nullptr;
    // geometry
    DevBuf<float4> node, itra, plan, inst_inv;
    PhxCsgCtx csg = { nullptr, nullptr, nullptr };
    DevBuf<phx_bvh4_node> bvh;
    DevBuf<phx_leaf> leaves, globals;
    DevBuf<float4> leaf_sph, global_sph;   // world bounding sphere per leaf (centre, radius)
    int num_global = 0;
    float cull[4] = { 0.f, 0.f, 0.f, 0.f };
    int num_node = 0, num_prim = 0, num_inst = 0, num_leaf = 0, bvh_depth = 0;
    bool has_full = false;    // a list node or a leaf beyond sphere/zsphere/cylinder/box3/torus: full CSG variant
    int last_tail = 0;        // the last wavefront call finished its paths in one tail kernel
    long long last_wave_launches = 0;   // kernel launches of the last wavefront loop
    std::vector<int> prim_node_offset;
    // physics
    cudaArray_t bnd_arr = nullptr, icdf_arr = nullptr, planck_arr = nullptr;
    cudaTextureObject_t bnd_tex = 0, icdf_tex = 0, planck_tex = 0;
    DevBuf<uint4> optical;
    DevBuf<float4> input_own;              // input photons copied from the host
    const float4* input_photon = nullptr;  // the input photons in use (input_own or a caller's buffer)
    long long num_input_photon = 0;
    float nm0 = 60.f, nms = 1.f;
    unsigned nx = 0, ny = 0, hd_factor = 20;
    int num_bnd = 0;
    std::vector<float> bnd_host;   // kept for the adjoint (property re-tabulation)
    std::vector<uint32_t> optical_host;
    cudaArray_t adj_arr = nullptr;
    cudaTextureObject_t adj_tex = 0;
    float* adj_tab_h = nullptr;    // pinned staging of the adjoint's re-tabulated property table
    cudaEvent_t adj_up = nullptr;  // recorded after its upload
    int num_wl = 0;
    // rng
    DevBuf<uint32_t> rng;
    long long rng_slots = 0;
    // scratch
    DevBuf<float4> gs;
    DevBuf<long long> gs_off;
    DevBuf<int> gs_event;
    DevBuf<int> prim_node_d;              // root node of each prim
    DevBuf<phx_photon> photon;
    DevBuf<phx_seq> seq;
    DevBuf<phx_photon> hit;
    DevBuf<uint32_t> hitword, wordoff, blocksum, sensor;
    DevBuf<long long> counters;   // [0] num_hit, [1] queue head, [3] largest event
    DevBuf<long long> ev_start;
    DevBuf<unsigned> ev_left;
    DevBuf<uint32_t> jump_pow, jump_tab;   // P_k = T^(skip 2^k) and per-call event jump matrices
    DevBuf<uint32_t> jump4;                // 4-bit group tables of a single-event jump matrix
    DevBuf<uint32_t> ev_rng;               // per-call event-advanced XORWOW states (k_rng_event)
    cudaGraphExec_t batch_exec = nullptr;   // cached batched launch sequence (use_graph)
    PhxBatchCall batch_call;
#define PHX_BATCH_BUFS 20
    const void* batch_bufs[PHX_BATCH_BUFS] = {};
    unsigned long long batch_launch = 0;     // launch_key of the captured graph
    DevBuf<unsigned> status;
    unsigned* h_pinned = nullptr;  // 16 words of pinned readback
    PhxMergeWs merge;
    // wavefront pool (kernel_mode 2)
    DevBuf<PhxWaveSlot> wslot;
    DevBuf<PhxWavePrd> wprd;
    DevBuf<long long> wsidx;
    DevBuf<uint32_t> wact0, wact1, wfree;
    DevBuf<uint32_t> wlive, wlive_off, wlive_blk;    // refill rounds: live bits, their word and block offsets
    DevBuf<long long> wlive_tot;
    DevBuf<float4> wscore;                          // adjoint score terms per slot
    DevBuf<unsigned> wcnt;
    long long last_launches = 0, last_rounds = 0;   // of the last plain simulate call
    int last_graph = 0;                             // the last batched call replayed a CUDA graph
};

static PhxScene scene_of(const phx_engine* e, int polish)
{
    PhxScene S;
    S.bvh = e->bvh.p;
    S.leaves = e->leaves.p;
    S.inst_inv = e->inst_inv.p;
    S.csg = e->csg;
    (void)polish;
    S.globals = e->globals.p;
    S.leaf_sph = e->leaf_sph.p;
    S.global_sph = e->global_sph.p;
    S.num_global = e->num_global;
    S.num_leaf = e->num_leaf;
    S.cull = make_float4(e->cull[0], e->cull[1], e->cull[2], e->cull[3]);
    S.bvh_empty = e->num_leaf == 0;
    S.empty = e->num_leaf == 0 && e->num_global == 0;
    return S;
}

static PhxProps props_of(const phx_engine* e)
{
    PhxProps P;
    P.bnd_tex = e->bnd_tex;
    P.optical = e->optical.p;
    P.nm0 = e->nm0;
    P.nms = e->nms;
    P.nx = e->nx;
    P.ny = e->ny;
    P.icdf_tex = e->icdf_tex;
    P.hd_factor = e->hd_factor;
    P.planck_tex = e->planck_tex;
    P.input_photon = e->input_photon;
    P.num_input_photon = e->num_input_photon;
    return P;
}

static PhxLoopCfg loop_of(const phx_engine* e)
{
    PhxLoopCfg C;
    C.max_bounce = e->cfg.max_bounce;
    C.max_time = e->cfg.max_time;
    C.tmin = e->cfg.propagate_epsilon;
    C.tmin0 = e->cfg.propagate_epsilon0;
    C.tmax = 1000000.f;
    C.eps0_mask = e->cfg.epsilon0_mask;
    return C;
}

// ------------------------------------------------------------------ kernels
// curand_init(seed, subsequence=slot, offset) per photon slot : qudarap/QCurandState.cu:22-27
__global__ void k_rng_init(unsigned long long seed, unsigned long long offset, long long first, long long count, long long slots, uint32_t* rng)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    long long slot = first + i;
    curandStateXORWOW s;
    curand_init(seed, (unsigned long long)slot, offset, &s);
    rng[slot] = s.d;
    rng[slots * 1 + slot] = s.v[0];
    rng[slots * 2 + slot] = s.v[1];
    rng[slots * 3 + slot] = s.v[2];
    rng[slots * 4 + slot] = s.v[3];
    rng[slots * 5 + slot] = s.v[4];
}

// exclusive scan of genstep photon counts (quad6 q0.w) into off[G+1] : replaces the
// thrust reduce + iexpand seed buffer of qudarap/QEvt.cu:180-230 (photons find their genstep by
// binary search over off, so no per-photon seed array is written or read)
__global__ void k_genstep_offsets(const float4* gs, int G, long long* off)
{
    __shared__ long long warp_tot[32];
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < G; base += blockDim.x) {
        int g = base + threadIdx.x;
        long long v = g < G ? (long long)__float_as_int(gs[6 * g].w) : 0;
        if (v < 0) v = 0;
        long long x = v;
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) { long long y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        if (lane == 31) warp_tot[wid] = x;
        __syncthreads();
        if (wid == 0) {
            long long t = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) { long long y = __shfl_up_sync(0xffffffffu, t, o); if (lane >= o) t += y; }
            warp_tot[lane] = t;
        }
        __syncthreads();
        long long incl = x + (wid > 0 ? warp_tot[wid - 1] : 0) + carry;
        if (g < G) off[g + 1] = incl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) off[0] = 0;
}

struct SimArgs {
    PhxScene S;
    PhxProps P;
    PhxLoopCfg C;
    const float4* gs;
    const long long* gs_off;
    int G;
    long long N;
    long long photon_offset;
    unsigned long long event_index;
    unsigned long long skip;
    const uint32_t* rng;
    long long rng_slots;
    const uint32_t* jump;      // event jump matrix (phx_rngjump.h) or null for cuRAND skipahead
    const uint32_t* jump4;     // its 4-bit group tables, or null
    phx_photon* photon;
    phx_seq* seq;
    uint32_t* hitword;
    unsigned hit_mask;
    unsigned* status;
};

// one thread per photon : CSGOptiX/CSGOptiX7.cu:432-530 simulate()
#ifndef PHX_SIM_BLOCK
#define PHX_SIM_BLOCK 64
#endif
#ifndef PHX_SIM_MINB
#define PHX_SIM_MINB 8
#endif
template <int CV>
__global__ void __launch_bounds__(PHX_SIM_BLOCK, PHX_SIM_MINB) k_simulate(SimArgs a)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned status = 0;
    bool is_hit = false;
    if (idx < a.N) {
        const int gi = phx_find_genstep(a.gs_off, a.G, idx);
        const float4* g = a.gs + 6 * gi;
        const long long photon_idx = a.photon_offset + idx;
        curandStateXORWOW rng;
        if (photon_idx < a.rng_slots) {
            phx_load_rng(rng, a.rng, a.rng_slots, photon_idx);
        } else {
            status |= PHX_STATUS_RNG_RANGE;
            curand_init(0ull, (unsigned long long)photon_idx, 0ull, &rng);
        }
        if (a.event_index > 0ull) {
            if (a.jump4) phx_rng_jump4(rng, a.jump4, a.skip * a.event_index);
            else if (a.jump) phx_rng_jump(rng, a.jump, a.skip * a.event_index);
            else skipahead(a.skip * a.event_index, &rng);
        }
        PhxPhoton p;
        memset(&p, 0, sizeof(p));
        generate_photon(p, rng, g, (unsigned long long)photon_idx, a.P, status);
        unsigned long long seqhis[2] = { 0ull, 0ull }, seqbnd[2] = { 0ull, 0ull };
        phx_bounce_loop<CV>(p, rng, a.S, a.P, a.C, seqhis, seqbnd, status);
        if (a.photon) phx_store_photon(a.photon + idx, p);
        if (a.seq) {
            ulonglong2* s = reinterpret_cast<ulonglong2*>(a.seq + idx);
            s[0] = make_ulonglong2(seqhis[0], seqhis[1]);
            s[1] = make_ulonglong2(seqbnd[0], seqbnd[1]);
        }
        is_hit = (p.flagmask & a.hit_mask) == a.hit_mask;
    }
    const unsigned word = __ballot_sync(0xffffffffu, is_hit);
    if (a.hitword && (threadIdx.x & 31) == 0 && idx < a.N) a.hitword[idx >> 5] = word;
    if (status) atomicOr(a.status, status);
}

// per-word exclusive popcount offsets within blocks of 256 words, block totals
__global__ void k_word_scan(const uint32_t* word, long long nword, uint32_t* wordoff, uint32_t* blocksum)
{
    __shared__ uint32_t wt[8];
    const long long w = (long long)blockIdx.x * 256 + threadIdx.x;
    uint32_t c = w < nword ? __popc(word[w]) : 0u;
    uint32_t x = c;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) wt[wid] = x;
    __syncthreads();
    uint32_t before = 0;
    for (int k = 0; k < wid; k++) before += wt[k];
    if (w < nword) wordoff[w] = before + x - c;
    if (threadIdx.x == 255) blocksum[blockIdx.x] = before + x;
}

// exclusive scan of block totals in place, total into *total
__global__ void k_block_scan(uint32_t* blocksum, int nblock, long long* total)
{
    __shared__ uint32_t wt[32];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nblock; base += blockDim.x) {
        int b = base + threadIdx.x;
        uint32_t v = b < nblock ? blocksum[b] : 0u;
        uint32_t x = v;
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        if (lane == 31) wt[wid] = x;
        __syncthreads();
        if (wid == 0) {
            uint32_t t = lane < (int)(blockDim.x >> 5) ? wt[lane] : 0u;
            for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xffffffffu, t, o); if (lane >= o) t += y; }
            wt[lane] = t;
        }
        __syncthreads();
        unsigned long long incl = (unsigned long long)x + (wid > 0 ? wt[wid - 1] : 0u) + carry;
        if (b < nblock) blocksum[b] = (uint32_t)(incl - v);
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = (long long)carry;
}

// warp w handles hit word w : ordered copy of the selected photons (QEvt::gatherHit with
// SU::copy_if sphoton_selector, qudarap/QEvt.cc:934-985, sysrap/SU.cu:139-166) plus the
// per-sensor tally (identity-1).
__global__ void k_compact(const phx_photon* photon, long long N, const uint32_t* word, const uint32_t* wordoff,
                          const uint32_t* blocksum, phx_photon* hit, long long hit_capacity,
                          uint32_t* sensor, int num_sensor, unsigned* status)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= N) return;
    const long long w = idx >> 5;
    const uint32_t bits = word[w];
    const int lane = threadIdx.x & 31;
    if (!((bits >> lane) & 1u)) return;
    const uint32_t rank = __popc(bits & ((1u << lane) - 1u));
    const long long dst = (long long)blocksum[w >> 8] + wordoff[w] + rank;
    const float4* src = reinterpret_cast<const float4*>(photon + idx);
    const float4 q0 = src[0], q1 = src[1], q2 = src[2], q3 = src[3];
    if (hit) {
        if (dst < hit_capacity) {
            float4* o = reinterpret_cast<float4*>(hit + dst);
            o[0] = q0; o[1] = q1; o[2] = q2; o[3] = q3;
        } else {
            atomicOr(status, (unsigned)PHX_STATUS_HIT_OVERFLOW);
        }
    }
    if (sensor) {
        const unsigned id = __float_as_uint(q3.y) & 0xffffffu;
        if (id > 0u && (int)(id - 1u) < num_sensor) atomicAdd(sensor + (id - 1u), 1u);
    }
}

// CSGScan : one thread per ray, SoA rays
template <int CV>
__global__ void k_csg_scan(PhxCsgCtx csg, int root, float t_min, const float* rays, long long n, float4* out, unsigned* status)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 o = make_float3(__ldg(rays + i), __ldg(rays + n + i), __ldg(rays + 2 * n + i));
    const float3 d = make_float3(__ldg(rays + 3 * n + i), __ldg(rays + 4 * n + i), __ldg(rays + 5 * n + i));
    unsigned st = 0;
    float4 is;
    const bool valid = intersect_prim<CV>(is, csg, root, t_min, o, d, st);
    out[i] = valid ? is : make_float4(0.f, 0.f, 0.f, 0.f);
    if (st) atomicOr(status, st);
}

// The trace step of simtrace (CSGOptiX/CSGOptiX7.cu:563-603 calls trace(), :112-218): the closest
// hit of arbitrary rays over the whole geometry, one thread per ray (SoA rays), written as the
// reference's quad2 PRD (sysrap/squad.h:180-245): q0 normal.xyz (world, unnormalised), t;
// q1 lposcost, 0, iindex<<16|identity, globalPrimIdx<<16|boundary (0xffffffff words: a miss)
template <int CV>
__global__ void k_trace_rays(PhxScene S, const float* rays, long long n, float t_min, float t_max, float4* prd_out, unsigned* status)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 o = make_float3(__ldg(rays + i), __ldg(rays + n + i), __ldg(rays + 2 * n + i));
    const float3 d = make_float3(__ldg(rays + 3 * n + i), __ldg(rays + 4 * n + i), __ldg(rays + 5 * n + i));
    unsigned st = 0;
    PhxPRD prd;
    phx_trace<CV>(S, o, d, t_min, t_max, prd, st);
    prd_out[2 * i] = make_float4(prd.normal.x, prd.normal.y, prd.normal.z, prd.distance);
    prd_out[2 * i + 1] = make_float4(prd.lposcost, 0.f, __uint_as_float(prd.ii_id), __uint_as_float(prd.gp_bd));
    if (st) atomicOr(status, st);
}

// QSim::rng_sequence : uniforms of each photon slot after the event skipahead
__global__ void k_rng_sequence(const uint32_t* rng, long long slots, unsigned long long skip, long long first, long long n, int K, float* out)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    curandStateXORWOW s;
    phx_load_rng(s, rng, slots, first + j);
    if (skip) skipahead(skip, &s);
    for (int k = 0; k < K; k++) out[j * K + k] = curand_uniform(&s);
}

// ------------------------------------------------------------------ host helpers
static double det3(const double m[3][3])
{
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) + m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

// inverse of a row-vector affine 4x4 (rows 0..2 linear, row 3 translation), .w column ignored
static bool invert_affine(const float* q, float* out)
{
    double a[3][3];
    for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) a[r][c] = q[4 * r + c];
    double det = det3(a);
    if (!(std::fabs(det) > 0.0)) return false;
    double inv[3][3];
    inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    double t[3] = { q[12], q[13], q[14] };
    double ti[3];
    for (int c = 0; c < 3; c++) ti[c] = -(t[0] * inv[0][c] + t[1] * inv[1][c] + t[2] * inv[2][c]);
    for (int r = 0; r < 3; r++) { for (int c = 0; c < 3; c++) out[4 * r + c] = (float)inv[r][c]; out[4 * r + 3] = 0.f; }
    out[12] = (float)ti[0]; out[13] = (float)ti[1]; out[14] = (float)ti[2]; out[15] = 1.f;
    return true;
}

// ------------------------------------------------------------------ leaf bounding spheres
// A conservative sphere around each (instance, prim) leaf lets the traversal reject a leaf with
// one ray-sphere test before it loads the instance transform and walks the CSG tree.  The prim's
// sphere is the smaller of the sphere around its box and one composed over its CSG tree (leaf
// spheres, enclosing sphere for union, the smaller operand for intersection, A for A - B;
// complemented leaves are unbounded).
struct PhxSph { double c[3]; double r; };

static const double PHX_SPH_INF = 1e300;

static PhxSph sph_union(const PhxSph& a, const PhxSph& b)
{
    if (a.r >= PHX_SPH_INF || b.r >= PHX_SPH_INF) return { { 0, 0, 0 }, PHX_SPH_INF };
    double dv[3] = { b.c[0] - a.c[0], b.c[1] - a.c[1], b.c[2] - a.c[2] };
    const double d = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    if (d + b.r <= a.r) return a;
    if (d + a.r <= b.r) return b;
    const double r = 0.5 * (d + a.r + b.r);
    PhxSph s;
    for (int k = 0; k < 3; k++) s.c[k] = a.c[k] + dv[k] / d * (r - a.r);
    s.r = r;
    return s;
}

// largest stretch of the 3x3 linear part of a row-vector affine matrix (power iteration on M^T M)
static double max_scale(const double* m)
{
    double v[3] = { 0.577, 0.577, 0.577 }, lam = 0.0;
    for (int it = 0; it < 64; it++) {
        double w[3], u[3];
        for (int c = 0; c < 3; c++) w[c] = v[0] * m[0 * 4 + c] + v[1] * m[1 * 4 + c] + v[2] * m[2 * 4 + c];
        for (int r = 0; r < 3; r++) u[r] = m[r * 4 + 0] * w[0] + m[r * 4 + 1] * w[1] + m[r * 4 + 2] * w[2];
        const double n = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        if (!(n > 0.0)) return 0.0;
        lam = n;
        for (int k = 0; k < 3; k++) v[k] = u[k] / n;
    }
    return std::sqrt(lam) * (1.0 + 1e-9);
}

static PhxSph sph_transform(const PhxSph& s, const double* m)
{
    if (s.r >= PHX_SPH_INF) return s;
    PhxSph o;
    for (int c = 0; c < 3; c++) o.c[c] = s.c[0] * m[0 * 4 + c] + s.c[1] * m[1 * 4 + c] + s.c[2] * m[2 * 4 + c] + m[3 * 4 + c];
    o.r = s.r * max_scale(m);
    return o;
}

// sphere of node i (level order) of the complete tree rooted at node offset no, in the prim frame
static PhxSph node_sphere(const phx_geometry* geo, int no, int i, int num)
{
    const PhxSph inf = { { 0, 0, 0 }, PHX_SPH_INF };
    if (i >= num || no + i >= geo->num_node) return inf;
    const float* q = geo->node + 16 * (size_t)(no + i);
    uint32_t tc, tw;
    memcpy(&tc, q + 14, 4);
    memcpy(&tw, q + 15, 4);
    if (tc == PHX_CSG_UNION || tc == PHX_CSG_INTERSECTION || tc == PHX_CSG_DIFFERENCE) {
        const PhxSph a = node_sphere(geo, no, 2 * i + 1, num), b = node_sphere(geo, no, 2 * i + 2, num);
        if (tc == PHX_CSG_UNION) return sph_union(a, b);
        if (tc == PHX_CSG_INTERSECTION) return a.r <= b.r ? a : b;
        return a;
    }
    if (tw & 0x80000000u) return inf;   // complemented leaf
    PhxSph s = inf;
    switch (tc) {
        case PHX_CSG_SPHERE:
        case PHX_CSG_ZSPHERE:
            s = { { q[0], q[1], q[2] }, std::fabs((double)q[3]) };
            break;
        case PHX_CSG_CYLINDER: {
            const double r = q[3], z1 = q[4], z2 = q[5];
            s = { { 0, 0, 0.5 * (z1 + z2) }, std::sqrt(r * r + 0.25 * (z2 - z1) * (z2 - z1)) };   // axis on local z
            break;
        }
        case PHX_CSG_BOX3:
            s = { { 0, 0, 0 }, 0.5 * std::sqrt((double)q[0] * q[0] + (double)q[1] * q[1] + (double)q[2] * q[2]) };
            break;
        case PHX_CSG_TORUS:
            s = { { 0, 0, 0 }, std::fabs((double)q[2]) + std::fabs((double)q[1]) };
            break;
        case PHX_CSG_CONE: {
            const double r = std::max(std::fabs((double)q[0]), std::fabs((double)q[2])), h = 0.5 * ((double)q[3] - q[1]);
            s = { { 0, 0, 0.5 * ((double)q[1] + q[3]) }, std::sqrt(r * r + h * h) };
            break;
        }
        case PHX_CSG_HYPERBOLOID: {
            const double r0 = q[0], zf = q[1], z1 = q[2], z2 = q[3];
            const double zm = std::max(std::fabs(z1), std::fabs(z2)) / zf, h = 0.5 * (z2 - z1);
            s = { { 0, 0, 0.5 * (z1 + z2) }, std::sqrt(r0 * r0 * (zm * zm + 1.0) + h * h) };
            break;
        }
        case PHX_CSG_DISC: {
            const double r = q[3], h = 0.5 * ((double)q[5] - q[4]);
            s = { { q[0], q[1], 0.5 * ((double)q[4] + q[5]) }, std::sqrt(r * r + h * h) };
            break;
        }
        default:
            return inf;
    }
    const uint32_t g = tw & 0x7fffffffu;
    if (g > 0) {
        if ((int)g > geo->num_itra || !geo->itra) return inf;
        float fwd[16];
        if (!invert_affine(geo->itra + 16 * (size_t)(g - 1), fwd)) return inf;
        double m[16];
        for (int k = 0; k < 16; k++) m[k] = fwd[k];
        s = sph_transform(s, m);
    }
    return s;
}

// Every node a prim's intersector can reach, checked on the host so that no device read leaves
// the node, itra or plan tables: the tree's complete binary range (root subNum), list sub-node
// ranges, leaf gtransformIdx and convexpolyhedron plane ranges.  Returns nullptr or the problem.
static const char* check_leaf_node(const phx_geometry* geo, int ni)
{
    const float* q = geo->node + 16 * (size_t)ni;
    uint32_t tc, tw;
    memcpy(&tc, q + 14, 4);
    memcpy(&tw, q + 15, 4);
    const uint32_t g = tw & 0x7fffffffu;
    if (g > 0 && ((int64_t)g > geo->num_itra || !geo->itra)) return "leaf gtransformIdx beyond the itra table";
    if (tc == PHX_CSG_CONVEXPOLYHEDRON) {
        uint32_t idx, num;
        memcpy(&idx, q + 0, 4);
        memcpy(&num, q + 1, 4);
        if ((int64_t)idx + (int64_t)num > (int64_t)std::max(0, geo->num_plan) || (num > 0 && !geo->plan))
            return "convexpolyhedron planes beyond the plan table";
    }
    return nullptr;
}

static const char* check_list_node(const phx_geometry* geo, int ni, int root)
{
    const float* q = geo->node + 16 * (size_t)ni;
    uint32_t num, off;
    memcpy(&num, q + 0, 4);
    memcpy(&off, q + 1, 4);
    if ((int64_t)root + (int64_t)off + (int64_t)num > geo->num_node) return "list sub-nodes beyond the node table";
    for (uint32_t i = 0; i < num; i++) {
        const char* m = check_leaf_node(geo, root + (int)(off + i));
        if (m) return m;
    }
    return nullptr;
}

static const char* check_prim_nodes(const phx_geometry* geo, int root)
{
    uint32_t tc;
    memcpy(&tc, geo->node + 16 * (size_t)root + 14, 4);
    if (tc >= PHX_CSG_LEAF) return check_leaf_node(geo, root);
    if (tc >= PHX_CSG_CONTIGUOUS && tc <= PHX_CSG_OVERLAP) return check_list_node(geo, root, root);
    if (tc >= PHX_CSG_NODE) return nullptr;   // no intersector: always a miss
    uint32_t num;
    memcpy(&num, geo->node + 16 * (size_t)root, 4);    // subNum: complete binary tree size
    if (num < 1 || num > 65535u || ((num + 1) & num) != 0) return "tree subNum is not 2^h - 1 (h 1..16)";
    if ((int64_t)root + (int64_t)num > geo->num_node) return "tree nodes beyond the node table";
    for (uint32_t i = 0; i < num; i++) {
        const int ni = root + (int)i;
        uint32_t t;
        memcpy(&t, geo->node + 16 * (size_t)ni + 14, 4);
        const char* m = t >= PHX_CSG_LEAF ? check_leaf_node(geo, ni)
                      : t >= PHX_CSG_CONTIGUOUS && t <= PHX_CSG_OVERLAP ? check_list_node(geo, ni, root) : nullptr;
        if (m) return m;
    }
    return nullptr;
}

// prim-frame sphere: the smaller of the box sphere and the tree sphere
static PhxSph prim_sphere(const phx_geometry* geo, int p)
{
    const float* pr = geo->prim + 16 * (size_t)p;
    int32_t nn, no;
    memcpy(&nn, pr + 0, 4);
    memcpy(&no, pr + 1, 4);
    PhxSph b;
    double h2 = 0.0;
    for (int k = 0; k < 3; k++) {
        b.c[k] = 0.5 * ((double)pr[8 + k] + (double)pr[11 + k]);
        const double h = 0.5 * ((double)pr[11 + k] - (double)pr[8 + k]);
        h2 += h * h;
    }
    b.r = std::sqrt(h2);
    const PhxSph t = node_sphere(geo, no, 0, std::max(1, nn));
    return t.r < b.r ? t : b;
}

// World box of node i of a prim's tree under the instance matrix `inst` (row-vector, object ->
// world), tighter than the corner box of the prim's box: each leaf's own bounds (the exact box of a
// sphere, and of a cylinder's disc swept along its axis, under an affine map; the corner box of a
// box3 and of a zsphere's z slab, the zsphere's clipped to its sphere's) through its node transform
// and the instance, combined as the operators combine point sets (union: union; intersection:
// overlap; difference: the first operand).  false: a complemented or unhandled leaf, or an empty
// overlap; the caller keeps the prim's box then.
struct PhxBox {
    double lo[3], hi[3];
};

static void mat_mul_rows(const double* a, const double* b, double* o)   // o = a b (4x4)
{
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) o[r * 4 + c] = a[r * 4 + 0] * b[0 * 4 + c] + a[r * 4 + 1] * b[1 * 4 + c] + a[r * 4 + 2] * b[2 * 4 + c] + a[r * 4 + 3] * b[3 * 4 + c];
}

static void box_of_corners(const double* lo, const double* hi, const double* m, PhxBox& b)
{
    for (int k = 0; k < 3; k++) { b.lo[k] = 1e300; b.hi[k] = -1e300; }
    for (int i = 0; i < 8; i++) {
        const double p[3] = { (i & 1) ? hi[0] : lo[0], (i & 2) ? hi[1] : lo[1], (i & 4) ? hi[2] : lo[2] };
        for (int k = 0; k < 3; k++) {
            const double w = p[0] * m[0 * 4 + k] + p[1] * m[1 * 4 + k] + p[2] * m[2 * 4 + k] + m[3 * 4 + k];
            b.lo[k] = std::min(b.lo[k], w);
            b.hi[k] = std::max(b.hi[k], w);
        }
    }
}

static bool node_box(const phx_geometry* geo, int no, int i, int num, const double* inst, PhxBox& out)
{
    if (i >= num || no + i >= geo->num_node) return false;
    const float* q = geo->node + 16 * (size_t)(no + i);
    uint32_t tc, tw;
    memcpy(&tc, q + 14, 4);
    memcpy(&tw, q + 15, 4);
    if (tc == PHX_CSG_UNION || tc == PHX_CSG_INTERSECTION || tc == PHX_CSG_DIFFERENCE) {
        PhxBox a, b;
        if (!node_box(geo, no, 2 * i + 1, num, inst, a)) return false;
        if (tc == PHX_CSG_DIFFERENCE) { out = a; return true; }
        if (!node_box(geo, no, 2 * i + 2, num, inst, b)) return false;
        for (int k = 0; k < 3; k++) {
            out.lo[k] = tc == PHX_CSG_UNION ? std::min(a.lo[k], b.lo[k]) : std::max(a.lo[k], b.lo[k]);
            out.hi[k] = tc == PHX_CSG_UNION ? std::max(a.hi[k], b.hi[k]) : std::min(a.hi[k], b.hi[k]);
            if (!(out.lo[k] <= out.hi[k])) return false;
        }
        return true;
    }
    if (tw & 0x80000000u) return false;
    double m[16];
    const uint32_t g = tw & 0x7fffffffu;
    if (g > 0) {
        if ((int)g > geo->num_itra || !geo->itra) return false;
        float fwd[16];
        if (!invert_affine(geo->itra + 16 * (size_t)(g - 1), fwd)) return false;
        double f[16];
        for (int k = 0; k < 16; k++) f[k] = fwd[k];
        mat_mul_rows(f, inst, m);
    } else {
        memcpy(m, inst, sizeof(m));
    }
    // half extent along world axis k of a unit ball / unit disc in the local xy plane
    double ball[3], disc[3];
    for (int k = 0; k < 3; k++) {
        disc[k] = std::sqrt(m[0 * 4 + k] * m[0 * 4 + k] + m[1 * 4 + k] * m[1 * 4 + k]);
        ball[k] = std::sqrt(disc[k] * disc[k] + m[2 * 4 + k] * m[2 * 4 + k]);
    }
    auto at = [&](double x, double y, double z, int k) { return x * m[0 * 4 + k] + y * m[1 * 4 + k] + z * m[2 * 4 + k] + m[3 * 4 + k]; };
    switch (tc) {
        case PHX_CSG_SPHERE:
        case PHX_CSG_ZSPHERE: {
            const double r = std::fabs((double)q[3]);
            for (int k = 0; k < 3; k++) {
                const double c = at(q[0], q[1], q[2], k);
                out.lo[k] = c - r * ball[k];
                out.hi[k] = c + r * ball[k];
            }
            if (tc == PHX_CSG_ZSPHERE) {
                const double lo[3] = { q[0] - r, q[1] - r, q[2] + std::min(q[4], q[5]) };
                const double hi[3] = { q[0] + r, q[1] + r, q[2] + std::max(q[4], q[5]) };
                PhxBox s;
                box_of_corners(lo, hi, m, s);
                for (int k = 0; k < 3; k++) {
                    out.lo[k] = std::max(out.lo[k], s.lo[k]);
                    out.hi[k] = std::min(out.hi[k], s.hi[k]);
                    if (!(out.lo[k] <= out.hi[k])) return false;
                }
            }
            return true;
        }
        case PHX_CSG_CYLINDER: {
            const double r = std::fabs((double)q[3]);
            for (int k = 0; k < 3; k++) {
                const double c1 = at(0.0, 0.0, q[4], k), c2 = at(0.0, 0.0, q[5], k);
                out.lo[k] = std::min(c1, c2) - r * disc[k];
                out.hi[k] = std::max(c1, c2) + r * disc[k];
            }
            return true;
        }
        case PHX_CSG_BOX3: {
            const double lo[3] = { -0.5 * std::fabs((double)q[0]), -0.5 * std::fabs((double)q[1]), -0.5 * std::fabs((double)q[2]) };
            const double hi[3] = { -lo[0], -lo[1], -lo[2] };
            box_of_corners(lo, hi, m, out);
            return true;
        }
        default:
            return false;
    }
}

// QPlanck's table (qudarap/QPlanck.cc:36-48): sblackbody<double>(4096, 4096, 6500 K, 80 nm, 800 nm)
// narrowed to float.  Planck's law sampled at 4096 wavelengths (sysrap/sblackbody.h:77-116), its
// trapezoid integral normalised by the last value (NP::trapz, NP::divide_by_last), inverted at
// y = j / 4096 by the first bin with y0 <= y < y1 and linear interpolation (NP::MakeICDF with
// hd_factor 0, NP::pdomain), in double as the reference does.
extern "C" int phx_planck_icdf(float* out, int n)
{
    if (!out || n < PHX_PLANCK_N) return phx_fail(-1, "phx_planck_icdf: need %d floats", PHX_PLANCK_N);
    const int ni = 4096, nu = PHX_PLANCK_N;
    const double temp_K = 6500.0, nm0 = 80.0, nm1 = 800.0;
    const double h = 6.62606957e-34, c = 299792458.0, k = 1.3806488e-23;
    const double a = 2.0 * h * c * c, b = h * c / k;
    std::vector<double> x((size_t)ni), y((size_t)ni);
    for (int i = 0; i < ni; i++) {
        x[i] = nm0 + (nm1 - nm0) * double(i) / double(ni - 1);
        const double wlm = x[i] * 1e-9;
        y[i] = (a * std::pow(wlm, -5.0)) / (std::exp(b / (wlm * temp_K)) - 1.0);
    }
    std::vector<double> cdf((size_t)ni);
    cdf[0] = 0.0;
    for (int i = 0; i < ni - 1; i++) cdf[i + 1] = cdf[i] + (x[i + 1] - x[i]) * (y[i] + y[i + 1]) * 0.5;
    const double last = cdf[ni - 1];
    if (last != 0.0) for (int i = 0; i < ni; i++) cdf[i] /= last;
    for (int j = 0; j < nu; j++) {
        const double yv = double(j) / double(nu);
        double xv = x[0];
        if (yv <= cdf[0]) xv = x[0];
        else if (yv >= cdf[ni - 1]) xv = x[ni - 1];
        else {
            for (int i = 0; i < ni - 1; i++) {
                const double y0 = cdf[i], y1 = cdf[i + 1], dy = y1 - y0;
                if (y0 <= yv && yv < y1) {
                    xv = x[i];
                    if (dy > 0.0) xv += (yv - y0) * (x[i + 1] - x[i]) / dy;
                    break;
                }
            }
        }
        out[j] = static_cast<float>(xv);
    }
    return 0;
}

static int make_texture_f4(cudaArray_t& arr, cudaTextureObject_t& tex, const float* data, int width, int height)
{
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float4>();
    PHX_CU(cudaMallocArray(&arr, &ch, width, height));
    PHX_CU(cudaMemcpy2DToArray(arr, 0, 0, data, width * sizeof(float4), width * sizeof(float4), height, cudaMemcpyHostToDevice));
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    PHX_CU(cudaCreateTextureObject(&tex, &rd, &td, nullptr));
    return 0;
}

static int make_texture_f1(cudaArray_t& arr, cudaTextureObject_t& tex, const float* data, int width, int height)
{
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
    PHX_CU(cudaMallocArray(&arr, &ch, width, height));
    PHX_CU(cudaMemcpy2DToArray(arr, 0, 0, data, width * sizeof(float), width * sizeof(float), height, cudaMemcpyHostToDevice));
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    PHX_CU(cudaCreateTextureObject(&tex, &rd, &td, nullptr));
    return 0;
}

static int ensure_rng(phx_engine* e, long long want)
{
    if (want <= e->rng_slots) return 0;
    long long slots = std::max<long long>(want, e->rng_slots * 2);
    DevBuf<uint32_t> nb;
    PHX_CU(nb.ensure((size_t)slots * 6));
    if (e->rng_slots > 0) {
        for (int k = 0; k < 6; k++)
            PHX_CU(cudaMemcpyAsync(nb.p + (size_t)k * slots, e->rng.p + (size_t)k * e->rng_slots, e->rng_slots * sizeof(uint32_t), cudaMemcpyDeviceToDevice, e->stream));
    }
    long long first = e->rng_slots, count = slots - e->rng_slots;
    const int B = 256;
    k_rng_init<<<(unsigned)((count + B - 1) / B), B, 0, e->stream>>>(e->cfg.seed, e->cfg.offset, first, count, slots, nb.p);
    PHX_CU(cudaGetLastError());
    PHX_CU(cudaStreamSynchronize(e->stream));
    e->rng.release();
    e->rng = nb;
    e->rng_slots = slots;
    return 0;
}

// ------------------------------------------------------------------ C ABI
extern "C" {

const char* phx_version(void) { return "phox 0.1 sm_100a"; }
const char* phx_last_error(void) { return g_last_error.c_str(); }

void phx_config_default(phx_config* c)
{
    memset(c, 0, sizeof(*c));
    c->seed = 0;
    c->offset = 0;
    c->skipahead_event_offset = 100000;
    c->max_photon = 1000000;
    c->max_bounce = 31;
    c->max_time = 1.e27f;
    c->propagate_epsilon = 0.05f;
    c->propagate_epsilon0 = 0.05f;
    c->epsilon0_mask = PHX_TORCH | PHX_CERENKOV | PHX_SCINTILLATION | PHX_BULK_SCATTER | PHX_BULK_REEMIT;
    c->hit_mask = PHX_SURFACE_DETECT;
    c->root_polish = 0;
    c->num_sensor = 0;
    c->kernel_mode = 2;
    c->block = 64;
    c->regroup = 1;
    c->chunk = 1;
    c->use_graph = 1;
    c->wave_pool = 0;
    c->wave_refill = 12;
    c->wave_rounds = 2;
    c->wave_tail = 1 << 18;
    c->adj_wave_rounds = 12;
}

// the launch-shape fields a captured batched graph depends on, packed into one word
static unsigned long long launch_key(const phx_engine* e)
{
    const phx_config& c = e->cfg;
    return (unsigned long long)(c.kernel_mode & 3) | ((unsigned long long)(c.wave_refill & 63) << 2) |
           ((unsigned long long)(c.wave_rounds & 0x1fff) << 8) | ((unsigned long long)(c.wave_tail & 0xffffffffll) << 21) |
           ((unsigned long long)(c.use_graph & 1) << 53);
}

// the launch-shape fields of a config, checked (they change no result, only how work is launched)
static int check_launch_config(const phx_config* c)
{
    if (c->kernel_mode < 0 || c->kernel_mode > 2) return phx_fail(-1, "kernel_mode %d not in 0..2", c->kernel_mode);
    if (c->wave_refill < 1 || c->wave_refill > 32) return phx_fail(-1, "wave_refill %d not in 1..32", c->wave_refill);
    if (c->wave_rounds < 0 || c->wave_rounds > 4096) return phx_fail(-1, "wave_rounds %d not in 0..4096", c->wave_rounds);
    if (c->wave_tail < 0) return phx_fail(-1, "wave_tail %lld is negative", (long long)c->wave_tail);
    if (c->adj_wave_rounds < 0 || c->adj_wave_rounds > 4096)
        return phx_fail(-1, "adj_wave_rounds %d not in 0..4096", c->adj_wave_rounds);
    return 0;
}

int64_t phx_count_photons(const float* gensteps, int32_t num_genstep)
{
    int64_t n = 0;
    for (int g = 0; g < num_genstep; g++) {
        int32_t v;
        memcpy(&v, gensteps + 24 * g + 3, 4);
        if (v > 0) n += v;
    }
    return n;
}

int phx_destroy(phx_engine* e)
{
    if (!e) return 0;
    cudaSetDevice(e->device);
    if (e->bnd_tex) cudaDestroyTextureObject(e->bnd_tex);
    if (e->adj_tex) cudaDestroyTextureObject(e->adj_tex);
    if (e->adj_arr) cudaFreeArray(e->adj_arr);
    if (e->adj_up) cudaEventDestroy(e->adj_up);
    if (e->adj_tab_h) cudaFreeHost(e->adj_tab_h);
    if (e->icdf_tex) cudaDestroyTextureObject(e->icdf_tex);
    if (e->bnd_arr) cudaFreeArray(e->bnd_arr);
    if (e->icdf_arr) cudaFreeArray(e->icdf_arr);
    if (e->planck_tex) cudaDestroyTextureObject(e->planck_tex);
    if (e->planck_arr) cudaFreeArray(e->planck_arr);
    e->node.release(); e->itra.release(); e->plan.release(); e->inst_inv.release(); e->prim_node_d.release();
    e->bvh.release(); e->leaves.release(); e->globals.release(); e->leaf_sph.release(); e->global_sph.release(); e->optical.release(); e->rng.release();
    e->gs.release(); e->gs_off.release(); e->gs_event.release(); e->photon.release(); e->seq.release();
    e->hit.release(); e->hitword.release(); e->wordoff.release(); e->blocksum.release(); e->sensor.release();
    e->counters.release(); e->status.release(); e->ev_start.release(); e->ev_left.release();
    e->jump_pow.release(); e->jump_tab.release(); e->jump4.release(); e->ev_rng.release();
    e->merge.release();
    e->wslot.release(); e->wprd.release(); e->wsidx.release(); e->wact0.release(); e->wact1.release(); e->wfree.release(); e->wscore.release(); e->wcnt.release();
    e->wlive.release(); e->wlive_off.release(); e->wlive_blk.release(); e->wlive_tot.release();
    if (e->batch_exec) cudaGraphExecDestroy(e->batch_exec);
    if (e->h_pinned) cudaFreeHost(e->h_pinned);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return 0;
}

int phx_set_launch_config(phx_engine* e, const phx_config* cfg)
{
    if (!e || !cfg) return phx_fail(-1, "phx_set_launch_config: null argument");
    int rc = check_launch_config(cfg);
    if (rc) return rc;
    e->cfg.kernel_mode = cfg->kernel_mode;
    e->cfg.block = cfg->block;
    e->cfg.regroup = cfg->regroup;
    e->cfg.chunk = cfg->chunk;
    e->cfg.use_graph = cfg->use_graph;
    e->cfg.wave_refill = cfg->wave_refill;
    e->cfg.wave_rounds = cfg->wave_rounds;
    e->cfg.wave_tail = cfg->wave_tail;
    e->cfg.wave_pool = cfg->wave_pool;
    e->cfg.adj_wave_rounds = cfg->adj_wave_rounds;
    return 0;
}

int phx_trim(phx_engine* e, int64_t* bytes_released)
{
    if (!e) return phx_fail(-1, "phx_trim: null engine");
    PHX_CU(cudaSetDevice(e->device));
    PHX_CU(cudaStreamSynchronize(e->stream));
    PHX_CU(cudaDeviceSynchronize());   // calls on caller streams may still use the buffers
    int64_t b = 0;
    auto rel = [&b](auto& buf) { b += (int64_t)(buf.n * sizeof(*buf.p)); buf.release(); };
    rel(e->wslot); rel(e->wprd); rel(e->wsidx); rel(e->wact0); rel(e->wact1); rel(e->wfree); rel(e->wscore); rel(e->wcnt);
    rel(e->wlive); rel(e->wlive_off); rel(e->wlive_blk); rel(e->wlive_tot);
    rel(e->ev_rng); rel(e->photon); rel(e->seq); rel(e->hit); rel(e->hitword); rel(e->wordoff);
    e->merge.release();
    if (e->batch_exec) { cudaGraphExecDestroy(e->batch_exec); e->batch_exec = nullptr; }
    if (bytes_released) *bytes_released = b;
    return 0;
}

int phx_create(const phx_geometry* geo, const phx_physics* phys, const phx_config* cfg_in, int device, phx_engine** out)
{
    if (!geo || !phys || !out) return phx_fail(-1, "phx_create: null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return phx_fail(-3, "phx_create: no CUDA device");
    if (device < 0 || device >= ndev) return phx_fail(-1, "phx_create: device %d out of range (%d devices)", device, ndev);
    phx_engine* e = new phx_engine();
    e->device = device;
    if (cfg_in) e->cfg = *cfg_in; else phx_config_default(&e->cfg);
    int rc = check_launch_config(&e->cfg);
    if (rc) { delete e; return rc; }
#define PHX_TRY(x) do { rc = (x); if (rc) { phx_destroy(e); return rc; } } while (0)
#define PHX_TRYCU(call) do { cudaError_t _e = (call); if (_e != cudaSuccess) { rc = phx_fail(-2, "%s failed: %s", #call, cudaGetErrorString(_e)); phx_destroy(e); return rc; } } while (0)
    PHX_TRYCU(cudaSetDevice(device));
    PHX_TRYCU(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    PHX_TRYCU(cudaMallocHost(&e->h_pinned, 64 * sizeof(unsigned)));

    // ---- geometry
    if (geo->num_node <= 0 || !geo->node) { phx_destroy(e); return phx_fail(-1, "phx_create: no CSGNode"); }
    e->num_node = geo->num_node;
    e->num_prim = geo->num_prim;
    e->num_inst = geo->num_inst;
    PHX_TRYCU(e->node.ensure((size_t)geo->num_node * 4));
    PHX_TRYCU(cudaMemcpy(e->node.p, geo->node, (size_t)geo->num_node * 64, cudaMemcpyHostToDevice));
    PHX_TRYCU(e->itra.ensure((size_t)std::max(1, geo->num_itra) * 4));
    if (geo->num_itra > 0) PHX_TRYCU(cudaMemcpy(e->itra.p, geo->itra, (size_t)geo->num_itra * 64, cudaMemcpyHostToDevice));
    PHX_TRYCU(e->plan.ensure((size_t)std::max(1, geo->num_plan)));
    if (geo->num_plan > 0) PHX_TRYCU(cudaMemcpy(e->plan.p, geo->plan, (size_t)geo->num_plan * 16, cudaMemcpyHostToDevice));
    e->csg.node = e->node.p;
    e->csg.itra = e->itra.p;
    e->csg.plan = e->plan.p;

    e->prim_node_offset.resize(geo->num_prim);
    for (int p = 0; p < geo->num_prim; p++) {
        int32_t no;
        memcpy(&no, geo->prim + 16 * p + 1, 4);
        e->prim_node_offset[p] = no;
        int32_t nn;
        memcpy(&nn, geo->prim + 16 * p + 0, 4);
        if (no < 0 || no + std::max(nn, 1) > geo->num_node) { phx_destroy(e); return phx_fail(-1, "phx_create: prim %d node range out of bounds", p); }
        if (const char* m = check_prim_nodes(geo, no)) { phx_destroy(e); return phx_fail(-1, "phx_create: prim %d: %s", p, m); }
    }
    if (geo->num_prim > 0) {   // root node per prim on the device (the adjoint's probe intersections)
        PHX_TRYCU(e->prim_node_d.ensure((size_t)geo->num_prim));
        PHX_TRYCU(cudaMemcpy(e->prim_node_d.p, e->prim_node_offset.data(), sizeof(int) * (size_t)geo->num_prim, cudaMemcpyHostToDevice));
    }
    for (int i = 0; i < geo->num_node && !e->has_full; i++) {
        uint32_t tc;
        memcpy(&tc, geo->node + 16 * (size_t)i + 14, 4);
        e->has_full = !phx_csg_base_typecode(tc);
    }
    std::vector<float> inv((size_t)std::max(1, geo->num_inst) * 16, 0.f);
    std::vector<PhxLeafInput> leaves;
    std::vector<PhxSph> psph((size_t)std::max(1, geo->num_prim));
    for (int p = 0; p < geo->num_prim; p++) psph[p] = prim_sphere(geo, p);
    for (int i = 0; i < geo->num_inst; i++) {
        const float* q = geo->inst + 16 * i;
        float m[16];
        memcpy(m, q, sizeof(m));
        m[3] = m[7] = m[11] = 0.f; m[15] = 1.f;   // clear identity info in the .w column
        if (!invert_affine(m, &inv[16 * (size_t)i])) { phx_destroy(e); return phx_fail(-1, "phx_create: instance %d transform is singular", i); }
        int32_t gas_idx, sensor_id1;
        memcpy(&gas_idx, q + 7, 4);
        memcpy(&sensor_id1, q + 11, 4);
        if (gas_idx < 0 || gas_idx >= geo->num_solid) { phx_destroy(e); return phx_fail(-1, "phx_create: instance %d gas_idx %d out of range", i, gas_idx); }
        const int32_t* so = geo->solid + 12 * gas_idx;
        const int numPrim = so[4], primOffset = so[5];
        for (int p = primOffset; p < primOffset + numPrim; p++) {
            if (p < 0 || p >= geo->num_prim) { phx_destroy(e); return phx_fail(-1, "phx_create: solid %d prim %d out of range", gas_idx, p); }
            const float* pr = geo->prim + 16 * p;
            PhxLeafInput L;
            L.bbox[0] = pr[8]; L.bbox[1] = pr[9]; L.bbox[2] = pr[10];
            L.bbox[3] = pr[11]; L.bbox[4] = pr[12]; L.bbox[5] = pr[13];
            memcpy(L.xform, m, sizeof(m));
            {
                double md[16];
                for (int k = 0; k < 16; k++) md[k] = m[k];
                int32_t nn, no;
                memcpy(&nn, pr + 0, 4);
                memcpy(&no, pr + 1, 4);
                PhxBox tb;
                L.has_wbox = node_box(geo, no, 0, std::max(1, nn), md, tb) ? 1 : 0;
                for (int k = 0; k < 3; k++) { L.wbox[k] = L.has_wbox ? tb.lo[k] : 0.0; L.wbox[3 + k] = L.has_wbox ? tb.hi[k] : 0.0; }
                const PhxSph w = sph_transform(psph[p], md);
                const double cn = std::sqrt(w.c[0] * w.c[0] + w.c[1] * w.c[1] + w.c[2] * w.c[2]);
                // pad: relative, plus absolute for FP32 rays at these coordinates (never excludes a hit)
                const double r = w.r >= PHX_SPH_INF ? 3e38 : w.r * (1.0 + 1e-4) + 1e-5 * (cn + w.r) + 0.5;
                L.sphere[0] = (float)w.c[0]; L.sphere[1] = (float)w.c[1]; L.sphere[2] = (float)w.c[2];
                L.sphere[3] = (float)std::min(r, 3e38);
            }
            int32_t gpi;
            memcpy(&gpi, pr + 15, 4);
            const int no = e->prim_node_offset[p];
            uint32_t boundary;
            memcpy(&boundary, geo->node + 16 * no + 6, 4);
            L.leaf.inst = i;
            L.leaf.node_offset = no;
            L.leaf.gp_bd = ((uint32_t)(gpi & 0xffff) << 16) | (boundary & 0xffffu);
            L.leaf.ii_id = ((uint32_t)(i & 0xffff) << 16) | ((uint32_t)sensor_id1 & 0xffffu);
            leaves.push_back(L);
        }
    }
    PhxBvh4Result bv;
    if (phx_build_bvh4(leaves, bv) != 0) { phx_destroy(e); return phx_fail(-1, "phx_create: BVH build failed"); }
    e->num_leaf = (int)bv.leaves.size();
    e->bvh_depth = bv.max_depth;
    if (3 * (bv.max_depth + 1) + 4 > PHX_BVH_STACK) { phx_destroy(e); return phx_fail(-1, "phx_create: BVH depth %d exceeds traversal stack", bv.max_depth); }
    PHX_TRYCU(e->bvh.ensure(std::max<size_t>(1, bv.nodes.size())));
    if (!bv.nodes.empty()) PHX_TRYCU(cudaMemcpy(e->bvh.p, bv.nodes.data(), bv.nodes.size() * sizeof(phx_bvh4_node), cudaMemcpyHostToDevice));
    PHX_TRYCU(e->leaves.ensure(std::max<size_t>(1, bv.leaves.size())));
    if (!bv.leaves.empty()) PHX_TRYCU(cudaMemcpy(e->leaves.p, bv.leaves.data(), bv.leaves.size() * sizeof(phx_leaf), cudaMemcpyHostToDevice));
    PHX_TRYCU(e->leaf_sph.ensure(std::max<size_t>(1, bv.leaf_sphere.size() / 4)));
    if (!bv.leaf_sphere.empty()) PHX_TRYCU(cudaMemcpy(e->leaf_sph.p, bv.leaf_sphere.data(), bv.leaf_sphere.size() * sizeof(float), cudaMemcpyHostToDevice));
    PHX_TRYCU(e->global_sph.ensure(std::max<size_t>(1, bv.global_sphere.size() / 4)));
    if (!bv.global_sphere.empty()) PHX_TRYCU(cudaMemcpy(e->global_sph.p, bv.global_sphere.data(), bv.global_sphere.size() * sizeof(float), cudaMemcpyHostToDevice));
    e->num_global = (int)bv.globals.size();
    memcpy(e->cull, bv.cull, sizeof(e->cull));
    PHX_TRYCU(e->globals.ensure(std::max<size_t>(1, bv.globals.size())));
    if (!bv.globals.empty()) PHX_TRYCU(cudaMemcpy(e->globals.p, bv.globals.data(), bv.globals.size() * sizeof(phx_leaf), cudaMemcpyHostToDevice));
    PHX_TRYCU(e->inst_inv.ensure(inv.size() / 4));
    PHX_TRYCU(cudaMemcpy(e->inst_inv.p, inv.data(), inv.size() * sizeof(float), cudaMemcpyHostToDevice));

    // ---- physics
    if (!phys->bnd || phys->num_bnd <= 0 || phys->num_wl <= 1 || !phys->optical) { phx_destroy(e); return phx_fail(-1, "phx_create: bnd/optical missing"); }
    e->num_bnd = phys->num_bnd;
    e->num_wl = phys->num_wl;
    e->nx = (unsigned)phys->num_wl;
    e->ny = (unsigned)phys->num_bnd * 8u;
    e->nm0 = phys->wl_low;
    e->nms = phys->wl_step;
    e->bnd_host.assign(phys->bnd, phys->bnd + (size_t)phys->num_bnd * 8 * phys->num_wl * 4);
    PHX_TRY(make_texture_f4(e->bnd_arr, e->bnd_tex, phys->bnd, (int)e->nx, (int)e->ny));
    PHX_TRYCU(e->optical.ensure((size_t)phys->num_bnd * 4));
    PHX_TRYCU(cudaMemcpy(e->optical.p, phys->optical, (size_t)phys->num_bnd * 4 * 16, cudaMemcpyHostToDevice));
    e->optical_host.assign(phys->optical, phys->optical + (size_t)phys->num_bnd * 16);
    if (phys->icdf && phys->icdf_width > 1 && phys->icdf_layers > 0) {
        e->hd_factor = (unsigned)phys->hd_factor;
        PHX_TRY(make_texture_f1(e->icdf_arr, e->icdf_tex, phys->icdf, phys->icdf_width, phys->icdf_layers));
    } else {
        e->hd_factor = 0xffffffffu;  // no scintillator table : reemission wavelength 0
        float dummy[4] = { 0.f, 0.f, 0.f, 0.f };
        PHX_TRY(make_texture_f1(e->icdf_arr, e->icdf_tex, dummy, 2, 2));
    }
    {
        // black-body wavelengths for torch photons without a wavelength (QPlanck)
        float table[PHX_PLANCK_N];
        phx_planck_icdf(table, PHX_PLANCK_N);
        PHX_TRY(make_texture_f1(e->planck_arr, e->planck_tex, table, PHX_PLANCK_N, 1));
    }
    // ---- rng + small buffers
    {
        const std::vector<uint32_t> pw = phx_jump_powers(e->cfg.skipahead_event_offset);
        PHX_TRYCU(e->jump_pow.ensure(pw.size()));
        PHX_TRYCU(cudaMemcpy(e->jump_pow.p, pw.data(), pw.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
        PHX_TRYCU(e->jump_tab.ensure(PHX_JUMP_MATW));
    }
    PHX_TRYCU(e->status.ensure(4));
    PHX_TRYCU(e->counters.ensure(8));
    PHX_TRY(ensure_rng(e, std::max<long long>(1, e->cfg.max_photon)));
    PHX_TRYCU(cudaStreamSynchronize(e->stream));
#undef PHX_TRY
#undef PHX_TRYCU
    *out = e;
    return 0;
}

}  // extern "C"

static PersistArgs persist_args_from(const phx_engine* e, const SimArgs& a)
{
    PersistArgs A;
    memset(&A, 0, sizeof(A));
    A.seed = e->cfg.seed;
    A.rng_offset = e->cfg.offset;
    A.S = a.S; A.P = a.P; A.C = a.C;
    A.gs = a.gs; A.gs_off = a.gs_off; A.G = a.G; A.N = a.N;
    A.photon_offset = a.photon_offset; A.event_index = a.event_index;
    A.gs_event = nullptr; A.ev_start = nullptr;
    A.skip = a.skip; A.rng = a.rng; A.rng_slots = a.rng_slots; A.jump = a.jump; A.jump4 = a.jump4;
    A.photon = a.photon; A.seq = a.seq; A.hitword = a.hitword; A.hit_mask = a.hit_mask; A.status = a.status;
    A.regroup = 1; A.chunk = 1;
    return A;
}

// grid = SMs x resident blocks of the chosen block size (one wave of persistent blocks)
template <int CV, int BLOCK, bool ADJ = false>
static int launch_persistent_t(phx_engine* e, const PersistArgs& A, cudaStream_t st)
{
    // occupancy is queried once per (device, kernel) so graph capture sees only the launch
    static int cached_sms[128] = {}, cached_per_sm[128] = {};
    int dev = e->device;
    if (dev < 0 || dev >= 128) return phx_fail(-1, "device ordinal %d out of range", dev);
    if (!cached_sms[dev]) {
        int sms = 0, per_sm = 0;
        PHX_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        PHX_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sim_persistent<CV, BLOCK, ADJ>, BLOCK, 0));
        cached_per_sm[dev] = per_sm;
        cached_sms[dev] = sms;
    }
    const int sms = cached_sms[dev], per_sm = cached_per_sm[dev];
    const long long want = (A.N + BLOCK - 1) / BLOCK;
    const long long grid = std::max<long long>(1, std::min<long long>((long long)sms * std::max(1, per_sm), want));
    k_sim_persistent<CV, BLOCK, ADJ><<<(unsigned)grid, BLOCK, 0, st>>>(A);
    PHX_CU(cudaGetLastError());
    return 0;
}

// the CSG variant (PHX_CV_*) of an engine: root polish from the config, the full set of leaves
// and list nodes when the geometry uses any of them
static int cv_of(const phx_engine* e, bool polish)
{
    return (polish ? PHX_CV_POLISH : 0) | (e->has_full ? PHX_CV_FULL : 0);
}

// `return EXPR` with the compile-time constant CVK set to the runtime variant cv
#define PHX_CV_RETURN(cv, EXPR)                               \
    switch (cv) {                                             \
        case 1: { constexpr int CVK = 1; return EXPR; }       \
        case 2: { constexpr int CVK = 2; return EXPR; }       \
        case 3: { constexpr int CVK = 3; return EXPR; }       \
        default: { constexpr int CVK = 0; return EXPR; }      \
    }

template <int BLOCK, bool ADJ = false>
static int launch_persistent_b(phx_engine* e, const PersistArgs& A, int cv, cudaStream_t st)
{
    PHX_CV_RETURN(cv, (launch_persistent_t<CVK, BLOCK, ADJ>(e, A, st)));
}

static int launch_persistent(phx_engine* e, const PersistArgs& A, int block, cudaStream_t st)
{
    const int cv = cv_of(e, e->cfg.root_polish != 0);
    switch (block) {
        case 32:  return launch_persistent_b<32>(e, A, cv, st);
        case 64:  return launch_persistent_b<64>(e, A, cv, st);
        case 256: return launch_persistent_b<256>(e, A, cv, st);
        case 128:
        default:  return launch_persistent_b<128>(e, A, cv, st);
    }
}

// Wavefront form (phx_wave.cuh): fill a pool of paths, then rounds of trace + shade launches, then
// the tail kernel for the paths still live.  When every photon of the call fits in the pool the
// schedule is fixed (phx_config.wave_rounds rounds, 2 by default: the rounds that carry every path
// through the scintillator and acrylic, where the wavefront's coherent launches pay; the longer,
// divergent chains after them run faster in the tail kernel's registers than through the pool;
// adjoint passes take phx_config.adj_wave_rounds, 12 by default), with no host read, so the call can
// be captured into a graph.  Otherwise (refill, or wave_rounds 0) the
// live count is read back every PHX_WAVE_ROUNDS rounds and the tail kernel starts below
// wave_tail paths; that call synchronises the stream.
// Paths in flight: unless phx_config.wave_pool fixes the count, every photon of a call starts at
// once (generation in one coherent pass, no refill) as long as its slots fit in half of the device
// memory still free, and never fewer than PHX_WAVE_POOL slots start; a larger call refills slots
// as paths finish, with each refill round's live list rebuilt in slot order (k_wave_act).  4096
// uneven events in one batched call (338.9M photons) take 723 ms through 2^23 slots, 703 ms
// through 2^26, 655 ms through 2^28 and 652 ms with all of them in flight.  The engine keeps its
// slots for later calls (grow-only).
#ifndef PHX_WAVE_POOL
#define PHX_WAVE_POOL (1LL << 26)
#endif
#define PHX_WAVE_POOL_MAX (1LL << 31)   // slot indexes are 32-bit
#define PHX_WAVE_SLOT_BYTES (sizeof(PhxWaveSlot) + sizeof(PhxWavePrd) + sizeof(long long) + 3 * sizeof(uint32_t))

// path slots of a wavefront call over N photons (adj: with the score terms and tangent per slot)
static long long wave_pool_for(const phx_engine* e, long long N, bool adj)
{
    long long pool = e->cfg.wave_pool > 0 ? (long long)e->cfg.wave_pool : (long long)PHX_WAVE_POOL;
    if (e->cfg.wave_pool <= 0 && N > pool) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            const size_t per = PHX_WAVE_SLOT_BYTES + (adj ? PHX_WAVE_SCORE_F4 * sizeof(float4) : 0);
            const long long fit = (long long)e->wslot.n + (long long)(free_b / 2 / per);
            pool = std::max(pool, std::min(N, fit));
        }
    }
    return std::max<long long>(1, std::min(std::min(N, pool), PHX_WAVE_POOL_MAX));
}
// calls of at most this many photons get their event-advanced RNG states in one coherent pass
// ahead of the loop (24 B per photon of scratch); larger ones advance each state as it starts
#define PHX_EV_RNG_MAX (1LL << 26)
#ifndef PHX_WAVE_ROUNDS
#define PHX_WAVE_ROUNDS 4
#endif

template <typename K>
static int wave_grid(K kernel, int dev, int* cache)
{
    if (!cache[dev]) {
        int sms = 0, per_sm = 0;
        PHX_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        PHX_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0));
        cache[dev] = sms * std::max(1, per_sm);
    }
    return 0;
}

template <int CV, bool ADJ = false>
static int launch_wave_t(phx_engine* e, const PersistArgs& A, cudaStream_t st)
{
    static int g_init[128] = {}, g_trace[128] = {}, g_shade[128] = {}, g_fill[128] = {}, g_tail[128] = {};
    const int dev = e->device;
    if (dev < 0 || dev >= 128) return phx_fail(-1, "device ordinal %d out of range", dev);
    int rc;
    if ((rc = wave_grid(k_wave_init<CV, ADJ>, dev, g_init))) return rc;
#if PHX_WAVE_TRACE_DF
    if ((rc = wave_grid(k_wave_trace_df<CV>, dev, g_trace))) return rc;
#else
    if ((rc = wave_grid(k_wave_trace<CV>, dev, g_trace))) return rc;
#endif
    if ((rc = wave_grid(k_wave_shade<CV, ADJ>, dev, g_shade))) return rc;
    if ((rc = wave_grid(k_wave_fill<CV, ADJ>, dev, g_fill))) return rc;
    if ((rc = wave_grid(k_wave_tail<CV, ADJ>, dev, g_tail))) return rc;
    const long long N = A.N;
    const long long pool = wave_pool_for(e, N, ADJ);
    PHX_CU(e->wslot.ensure((size_t)pool)); PHX_CU(e->wprd.ensure((size_t)pool)); PHX_CU(e->wsidx.ensure((size_t)pool));
    PHX_CU(e->wact0.ensure((size_t)pool)); PHX_CU(e->wact1.ensure((size_t)pool)); PHX_CU(e->wcnt.ensure(4));
    const bool refill = N > pool;
    PHX_CU(e->wfree.ensure((size_t)pool));
    if (ADJ) PHX_CU(e->wscore.ensure((size_t)pool * PHX_WAVE_SCORE_F4));
    const long long nlw = (pool + 31) / 32, nlb = (nlw + 255) / 256;     // live-bit words, scan blocks
    if (refill) {
        PHX_CU(e->wlive.ensure((size_t)nlw)); PHX_CU(e->wlive_off.ensure((size_t)nlw));
        PHX_CU(e->wlive_blk.ensure((size_t)nlb)); PHX_CU(e->wlive_tot.ensure(1));
        PHX_CU(cudaMemsetAsync(e->wlive.p, 0, sizeof(uint32_t) * (size_t)nlw, st));
    }
    PHX_CU(cudaMemsetAsync(e->wcnt.p, 0, 4 * sizeof(unsigned), st));
    WaveArgs W;
    W.A = A;
    W.slot = e->wslot.p; W.prd = e->wprd.p; W.sidx = e->wsidx.p; W.pool = pool;
    uint32_t* act[2] = { e->wact0.p, e->wact1.p };
    unsigned* cnt[2] = { e->wcnt.p, e->wcnt.p + 1 };
    W.free_list = e->wfree.p;
    W.score = ADJ ? e->wscore.p : nullptr;
    W.n_free = e->wcnt.p + 2;
    W.trace_ctr = e->wcnt.p + 3;
    W.act_in = nullptr; W.n_in = nullptr; W.act_out = act[0]; W.n_out = cnt[0];
    W.live_bits = nullptr;
    W.refill_idle = e->cfg.wave_refill;
    const unsigned gi = (unsigned)std::min<long long>(g_init[dev], (pool + 127) / 128);
    k_wave_init<CV, ADJ><<<gi, 128, 0, st>>>(W);
    W.live_bits = refill ? e->wlive.p : nullptr;
    PHX_CU(cudaGetLastError());
    int cur = 0;
    const int rounds = ADJ ? e->cfg.adj_wave_rounds : e->cfg.wave_rounds;
    if (rounds > 0 && !refill) {
        // fixed schedule, no host read: wave_rounds rounds, then the tail kernel finishes whatever is
        // still live (it reads the count on the device; a grid-stride loop over any count), so the
        // whole call can be captured as a CUDA graph
        for (int r = 0; r < rounds; r++) {
            W.act_in = act[cur]; W.n_in = cnt[cur]; W.act_out = act[1 - cur]; W.n_out = cnt[1 - cur];
#if PHX_WAVE_TRACE_DF
            k_wave_trace_df<CV><<<(unsigned)g_trace[dev], 128, 0, st>>>(W);
#else
            k_wave_trace<CV><<<(unsigned)g_trace[dev], 128, 0, st>>>(W);
#endif
            k_wave_shade<CV, ADJ><<<(unsigned)g_shade[dev], 128, 0, st>>>(W);
            cur = 1 - cur;
        }
        W.act_in = act[cur]; W.n_in = cnt[cur];
        k_wave_tail<CV, ADJ><<<(unsigned)g_tail[dev], 128, 0, st>>>(W);
        PHX_CU(cudaGetLastError());
        e->last_rounds = rounds;
        e->last_tail = 1;
        e->last_wave_launches = 2 + 2LL * rounds;
        return 0;
    }
    const long long max_rounds = (N / pool + 1) * (long long)(A.C.max_bounce + 1) + 2 * PHX_WAVE_ROUNDS;
    e->last_rounds = 0;
    e->last_tail = 0;
    bool done = false;
    bool filling = refill;                          // photons still wait in the queue (as last read)
    long long nl = 1;                               // launches of this call (k_wave_init)
    for (long long r = 0; r < max_rounds && !done;) {
        for (int k = 0; k < PHX_WAVE_ROUNDS; k++, r++) {
            W.act_in = act[cur]; W.n_in = cnt[cur]; W.act_out = act[1 - cur]; W.n_out = cnt[1 - cur];
#if PHX_WAVE_TRACE_DF
            k_wave_trace_df<CV><<<(unsigned)g_trace[dev], 128, 0, st>>>(W);
#else
            k_wave_trace<CV><<<(unsigned)g_trace[dev], 128, 0, st>>>(W);
#endif
            k_wave_shade<CV, ADJ><<<(unsigned)g_shade[dev], 128, 0, st>>>(W);
            nl += 2;
            if (filling) {
                k_wave_fill<CV, ADJ><<<(unsigned)g_fill[dev], 128, 0, st>>>(W);
                k_word_scan<<<(unsigned)nlb, 256, 0, st>>>(e->wlive.p, nlw, e->wlive_off.p, e->wlive_blk.p);
                k_block_scan<<<1, 1024, 0, st>>>(e->wlive_blk.p, (int)nlb, e->wlive_tot.p);
                k_wave_act<<<(unsigned)((nlw + 255) / 256), 256, 0, st>>>(e->wlive.p, nlw, e->wlive_off.p, e->wlive_blk.p,
                                                                         e->wlive_tot.p, act[1 - cur], cnt[1 - cur]);
                nl += 4;
            }
            cur = 1 - cur;
        }
        PHX_CU(cudaGetLastError());
        PHX_CU(cudaMemcpyAsync(e->h_pinned + 40, cnt[cur], sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        if (refill) PHX_CU(cudaMemcpyAsync(e->h_pinned + 44, A.queue, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        PHX_CU(cudaStreamSynchronize(st));
        const unsigned live = e->h_pinned[40];
        done = live == 0u;
        e->last_rounds = r;
        bool queue_done = !refill;                  // every photon of the queue has been started
        if (refill) {
            unsigned long long head;
            memcpy(&head, e->h_pinned + 44, sizeof(head));
            queue_done = head >= (unsigned long long)N;
        }
        if (filling && queue_done) {
            // nothing left to start: the live list (in slot order now) shrinks by appends again
            filling = false;
            W.live_bits = nullptr;
        }
        if (!done && queue_done && (long long)live <= e->cfg.wave_tail) {
            // few paths left and none queued: finish them in one kernel
            W.act_in = act[cur]; W.n_in = cnt[cur];
            k_wave_tail<CV, ADJ><<<(unsigned)std::min<long long>(g_tail[dev], (live + 127) / 128), 128, 0, st>>>(W);
            PHX_CU(cudaGetLastError());
            e->last_tail = 1;
            nl += 1;
            done = true;
        }
    }
    e->last_wave_launches = nl;
    if (!done) return phx_fail(-5, "wavefront loop did not drain within %lld rounds", max_rounds);
    return 0;
}

template <bool ADJ = false>
static int launch_wave_cv(phx_engine* e, const PersistArgs& A, int cv, cudaStream_t st)
{
    PHX_CV_RETURN(cv, (launch_wave_t<CVK, ADJ>(e, A, st)));
}

static int launch_wave(phx_engine* e, const PersistArgs& A, cudaStream_t st)
{
    return launch_wave_cv(e, A, cv_of(e, e->cfg.root_polish != 0), st);
}

template <int CV>
static void launch_simulate_t(const SimArgs& a, long long N, cudaStream_t st)
{
    const int B = PHX_SIM_BLOCK;
    k_simulate<CV><<<(unsigned)((N + B - 1) / B), B, 0, st>>>(a);
}

static int launch_simulate(phx_engine* e, const SimArgs& a, long long N, cudaStream_t st)
{
    PHX_CV_RETURN(cv_of(e, e->cfg.root_polish != 0), (launch_simulate_t<CVK>(a, N, st), 0));
}

template <int CV>
static void launch_scan_t(const PhxCsgCtx& csg, int root, float t_min, const float* d_rays, long long n, float4* out, unsigned* status,
                          cudaStream_t st)
{
    const int B = 128;
    k_csg_scan<CV><<<(unsigned)((n + B - 1) / B), B, 0, st>>>(csg, root, t_min, d_rays, n, out, status);
}

template <int CV>
static void launch_trace_t(const PhxScene& S, const float* d_rays, long long n, float t_min, float t_max, float4* out, unsigned* status,
                           cudaStream_t st)
{
    const int B = 128;
    k_trace_rays<CV><<<(unsigned)((n + B - 1) / B), B, 0, st>>>(S, d_rays, n, t_min, t_max, out, status);
}

static int launch_trace(phx_engine* e, const float* d_rays, long long n, float t_min, float t_max, float4* out, cudaStream_t st)
{
    const PhxScene S = scene_of(e, e->cfg.root_polish);
    PHX_CV_RETURN(cv_of(e, e->cfg.root_polish != 0), (launch_trace_t<CVK>(S, d_rays, n, t_min, t_max, out, e->status.p, st), 0));
}

extern "C" {

// device buffers of one plain simulate call (engine buffers, or the fixed no-alloc scratch)
struct PhxPlainBufs {
    long long* gs_off;
    uint32_t* hitword;
    uint32_t* wordoff;
    uint32_t* blocksum;
    long long* counters;   // [0] num_hit, [1] queue head
    unsigned* status;
    uint32_t* jump;        // one event jump matrix (PHX_JUMP_MATW words)
    uint32_t* jump4;       // its 4-bit group tables (PHX_JUMP_NIBW words), or null to use the matrix
};

// every device operation of one plain simulate call on st, then the D2H of num_hit/status
// into the engine's pinned words; the caller synchronises
static int plain_enqueue(phx_engine* e, const PhxPlainBufs& b, const float* d_gs, int G, long long N, int event_index,
                         long long photon_offset, phx_photon* photon, phx_seq* seq, phx_photon* hit, long long hcap,
                         uint32_t* sensor, bool want_hits, cudaStream_t st, bool wave_ok = false)
{
    const long long nword = (N + 31) / 32;
    PHX_CU(cudaMemsetAsync(b.status, 0, sizeof(unsigned), st));
    PHX_CU(cudaMemsetAsync(b.counters, 0, 2 * sizeof(long long), st));
    k_genstep_offsets<<<1, 1024, 0, st>>>(reinterpret_cast<const float4*>(d_gs), G, b.gs_off);
    if (event_index > 0) k_jump_build<<<1, 160, 0, st>>>(nullptr, (unsigned long long)event_index, e->jump_pow.p, b.jump);
    if (event_index > 0 && b.jump4) k_jump_nibbles<<<(PHX_JUMP_BITS / 4 * 16 + 127) / 128, 128, 0, st>>>(b.jump, b.jump4);
    PHX_CU(cudaGetLastError());
    SimArgs a;
    a.S = scene_of(e, e->cfg.root_polish);
    a.P = props_of(e);
    a.C = loop_of(e);
    a.gs = reinterpret_cast<const float4*>(d_gs);
    a.gs_off = b.gs_off;
    a.G = G;
    a.N = N;
    a.photon_offset = photon_offset;
    a.event_index = (unsigned long long)event_index;
    a.skip = e->cfg.skipahead_event_offset;
    a.rng = e->rng.p;
    a.rng_slots = e->rng_slots;
    a.jump = event_index > 0 ? b.jump : nullptr;
    a.jump4 = event_index > 0 ? b.jump4 : nullptr;
    a.photon = photon;
    a.seq = seq;
    a.hitword = want_hits ? b.hitword : nullptr;
    a.hit_mask = e->cfg.hit_mask;
    a.status = b.status;
    if (N > 0 && (e->cfg.kernel_mode == 1 || e->cfg.kernel_mode == 2)) {
        // persistent threads with per-lane refill (phx_persist.cuh), or the wavefront rounds
        // (phx_wave.cuh); hit bits are OR-ed in
        if (want_hits) PHX_CU(cudaMemsetAsync(b.hitword, 0, sizeof(uint32_t) * (size_t)nword, st));
        PersistArgs A = persist_args_from(e, a);
        A.queue = reinterpret_cast<unsigned long long*>(b.counters + 1);
        A.regroup = e->cfg.regroup;
        A.chunk = e->cfg.chunk;
        const bool wave = e->cfg.kernel_mode == 2 && wave_ok;
        // the pre-pass pays off where photons start a few lanes at a time (persistent refill,
        // wavefront refill); when every photon starts in the wavefront's first kernel, whole
        // warps advance their states there
        if (wave_ok && event_index > 0 && N <= PHX_EV_RNG_MAX && !(wave && N <= wave_pool_for(e, N, false))) {
            PHX_CU(e->ev_rng.ensure((size_t)N * 6));
            k_rng_event<<<(unsigned)std::min<long long>((N + 255) / 256, 148LL * 16), 256, 0, st>>>(A, e->ev_rng.p, N);
            PHX_CU(cudaGetLastError());
            A.ev_rng = e->ev_rng.p;
            A.ev_rng_n = N;
        }
        e->last_rounds = 0;
        int rc = wave ? launch_wave(e, A, st) : launch_persistent(e, A, e->cfg.block, st);
        if (rc) return rc;
        e->last_launches = 1 + (event_index > 0 ? (b.jump4 ? 2 : 1) : 0) + (A.ev_rng ? 1 : 0) +
                           (wave ? e->last_wave_launches : 1) + (want_hits ? 3 : 0);
    } else if (N > 0) {
        launch_simulate(e, a, N, st);
        PHX_CU(cudaGetLastError());
        e->last_rounds = 0;
        e->last_launches = 1 + (event_index > 0 ? (b.jump4 ? 2 : 1) : 0) + 1 + (want_hits ? 3 : 0);
    }
    if (sensor) PHX_CU(cudaMemsetAsync(sensor, 0, sizeof(uint32_t) * std::max(0, e->cfg.num_sensor), st));
    if (want_hits && N > 0) {
        const long long nblock = (nword + 255) / 256;
        k_word_scan<<<(unsigned)nblock, 256, 0, st>>>(b.hitword, nword, b.wordoff, b.blocksum);
        k_block_scan<<<1, 1024, 0, st>>>(b.blocksum, (int)nblock, b.counters);
        k_compact<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(photon, N, b.hitword, b.wordoff, b.blocksum,
                                                              hit, hcap, sensor, e->cfg.num_sensor, b.status);
        PHX_CU(cudaGetLastError());
    }
    PHX_CU(cudaMemcpyAsync(e->h_pinned + 2, b.counters, sizeof(long long), cudaMemcpyDeviceToHost, st));
    PHX_CU(cudaMemcpyAsync(e->h_pinned, b.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    return 0;
}

// shared device path : gensteps already on device, engine-owned scratch grown on demand
static int simulate_device_impl(phx_engine* e, const float* d_gs, int G, long long N, int event_index, long long photon_offset,
                                phx_photon* d_photon, phx_seq* d_seq, phx_photon* d_hit, long long hit_capacity,
                                uint32_t* d_sensor, long long* num_hit, unsigned* status, cudaStream_t st)
{
    if (G < 0 || N < 0) return phx_fail(-1, "simulate: negative sizes");
    if (photon_offset < 0) return phx_fail(-1, "simulate: negative photon_offset");
    if (event_index < 0) return phx_fail(-1, "simulate: negative event index");
    int rc = ensure_rng(e, photon_offset + N);
    if (rc) return rc;
    const long long nword = (N + 31) / 32;
    const bool want_hits = d_hit != nullptr || d_sensor != nullptr;
    phx_photon* photon = d_photon;
    if (want_hits && !photon) { PHX_CU(e->photon.ensure((size_t)std::max<long long>(1, N))); photon = e->photon.p; }
    PHX_CU(e->gs_off.ensure((size_t)G + 1));
    PHX_CU(e->counters.ensure(8));
    PHX_CU(e->hitword.ensure((size_t)std::max<long long>(1, nword)));
    PHX_CU(e->wordoff.ensure((size_t)std::max<long long>(1, nword)));
    PHX_CU(e->blocksum.ensure((size_t)std::max<long long>(1, (nword + 255) / 256)));
    PHX_CU(e->jump_tab.ensure(PHX_JUMP_MATW));
    PHX_CU(e->jump4.ensure(PHX_JUMP_NIBW));
    PhxPlainBufs b = { e->gs_off.p, e->hitword.p, e->wordoff.p, e->blocksum.p, e->counters.p, e->status.p, e->jump_tab.p, e->jump4.p };
    rc = plain_enqueue(e, b, d_gs, G, N, event_index, photon_offset, photon, d_seq, d_hit, hit_capacity, d_sensor, want_hits, st,
                       true);
    if (rc) return rc;
    PHX_CU(cudaStreamSynchronize(st));
    long long nh = 0;
    if (want_hits && N > 0) memcpy(&nh, e->h_pinned + 2, sizeof(long long));
    *num_hit = nh;
    *status = e->h_pinned[0];
    return 0;
}

int phx_simulate_device(phx_engine* e, const float* d_gensteps, int32_t num_genstep, int64_t num_photon,
                        int32_t event_index, int64_t photon_offset, phx_outputs* d_out, void* stream)
{
    if (!e || !d_out) return phx_fail(-1, "phx_simulate_device: null argument");
    PHX_CU(cudaSetDevice(e->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : e->stream;
    long long nh = 0;
    unsigned status = 0;
    int rc = simulate_device_impl(e, d_gensteps, num_genstep, num_photon, event_index, photon_offset,
                                  reinterpret_cast<phx_photon*>(d_out->photon), reinterpret_cast<phx_seq*>(d_out->seq),
                                  reinterpret_cast<phx_photon*>(d_out->hit), d_out->hit_capacity, d_out->sensor_hits, &nh, &status, st);
    if (rc) return rc;
    d_out->num_photon = num_photon;
    d_out->num_hit = nh;
    d_out->status = status;
    return 0;
}

int phx_simulate(phx_engine* e, const float* gensteps, int32_t num_genstep, int32_t event_index, phx_outputs* out)
{
    if (!e || !out || (num_genstep > 0 && !gensteps)) return phx_fail(-1, "phx_simulate: null argument");
    PHX_CU(cudaSetDevice(e->device));
    cudaStream_t st = e->stream;
    const long long N = phx_count_photons(gensteps, num_genstep);
    PHX_CU(e->gs.ensure((size_t)std::max(1, num_genstep) * 6));
    if (num_genstep > 0) PHX_CU(cudaMemcpyAsync(e->gs.p, gensteps, (size_t)num_genstep * 96, cudaMemcpyHostToDevice, st));
    PHX_CU(e->photon.ensure((size_t)std::max<long long>(1, N)));
    if (out->seq) PHX_CU(e->seq.ensure((size_t)std::max<long long>(1, N)));
    if (out->hit) PHX_CU(e->hit.ensure((size_t)std::max<long long>(1, std::min<long long>(N, out->hit_capacity))));
    if (out->sensor_hits) PHX_CU(e->sensor.ensure((size_t)std::max(1, e->cfg.num_sensor)));
    long long nh = 0;
    unsigned status = 0;
    const long long hcap = std::min<long long>(N, out->hit_capacity);
    int rc = simulate_device_impl(e, reinterpret_cast<const float*>(e->gs.p), num_genstep, N, event_index, 0, e->photon.p,
                                  out->seq ? e->seq.p : nullptr, out->hit ? e->hit.p : nullptr, hcap,
                                  out->sensor_hits ? e->sensor.p : nullptr, &nh, &status, st);
    if (rc) return rc;
    if (out->photon && N > 0) PHX_CU(cudaMemcpyAsync(out->photon, e->photon.p, (size_t)N * 64, cudaMemcpyDeviceToHost, st));
    if (out->seq && N > 0) PHX_CU(cudaMemcpyAsync(out->seq, e->seq.p, (size_t)N * 32, cudaMemcpyDeviceToHost, st));
    if (out->hit && nh > 0) PHX_CU(cudaMemcpyAsync(out->hit, e->hit.p, (size_t)std::min(nh, hcap) * 64, cudaMemcpyDeviceToHost, st));
    if (out->sensor_hits && e->cfg.num_sensor > 0) PHX_CU(cudaMemcpyAsync(out->sensor_hits, e->sensor.p, (size_t)e->cfg.num_sensor * 4, cudaMemcpyDeviceToHost, st));
    PHX_CU(cudaStreamSynchronize(st));
    out->num_photon = N;
    out->num_hit = nh;
    out->status = status;
    return 0;
}

int phx_csg_scan_device(phx_engine* e, int32_t prim, float t_min, const float* d_rays, int64_t n, float* d_isect, int32_t polish, void* stream)
{
    if (!e || (n > 0 && (!d_rays || !d_isect))) return phx_fail(-1, "phx_csg_scan_device: null argument");
    if (prim < 0 || prim >= e->num_prim) return phx_fail(-1, "phx_csg_scan_device: prim %d out of range", prim);
    PHX_CU(cudaSetDevice(e->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : e->stream;
    PHX_CU(cudaMemsetAsync(e->status.p, 0, sizeof(unsigned), st));
    const PhxCsgCtx csg = e->csg;
    if (n > 0) {
        float4* out = reinterpret_cast<float4*>(d_isect);
        const int root = e->prim_node_offset[prim];
        switch (cv_of(e, polish != 0)) {
            case 1: launch_scan_t<1>(csg, root, t_min, d_rays, n, out, e->status.p, st); break;
            case 2: launch_scan_t<2>(csg, root, t_min, d_rays, n, out, e->status.p, st); break;
            case 3: launch_scan_t<3>(csg, root, t_min, d_rays, n, out, e->status.p, st); break;
            default: launch_scan_t<0>(csg, root, t_min, d_rays, n, out, e->status.p, st); break;
        }
        PHX_CU(cudaGetLastError());
    }
    return 0;
}

int phx_csg_scan(phx_engine* e, int32_t prim, float t_min, const float* rays, int64_t n, float* isect)
{
    if (!e || (n > 0 && (!rays || !isect))) return phx_fail(-1, "phx_csg_scan: null argument");
    PHX_CU(cudaSetDevice(e->device));
    cudaStream_t st = e->stream;
    float* d_r = nullptr;
    float* d_o = nullptr;
    PHX_CU(cudaMallocAsync(&d_r, std::max<int64_t>(1, n) * 24, st));
    PHX_CU(cudaMallocAsync(&d_o, std::max<int64_t>(1, n) * 16, st));
    if (n > 0) PHX_CU(cudaMemcpyAsync(d_r, rays, n * 24, cudaMemcpyHostToDevice, st));
    int rc = phx_csg_scan_device(e, prim, t_min, d_r, n, d_o, e->cfg.root_polish, st);
    if (!rc && n > 0) {
        cudaError_t ce = cudaMemcpyAsync(isect, d_o, n * 16, cudaMemcpyDeviceToHost, st);
        if (ce != cudaSuccess) rc = phx_fail(-2, "phx_csg_scan: copy back failed: %s", cudaGetErrorString(ce));
    }
    cudaFreeAsync(d_r, st);
    cudaFreeAsync(d_o, st);
    PHX_CU(cudaStreamSynchronize(st));
    return rc;
}

int phx_trace_device(phx_engine* e, const float* d_rays, int64_t n, float t_min, float t_max, float* d_prd, uint32_t* status,
                     void* stream)
{
    if (!e || (n > 0 && (!d_rays || !d_prd))) return phx_fail(-1, "phx_trace_device: null argument");
    if (!(t_max > t_min)) return phx_fail(-1, "phx_trace_device: t_max %g must exceed t_min %g", (double)t_max, (double)t_min);
    PHX_CU(cudaSetDevice(e->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : e->stream;
    PHX_CU(cudaMemsetAsync(e->status.p, 0, sizeof(unsigned), st));
    if (n > 0) launch_trace(e, d_rays, n, t_min, t_max, reinterpret_cast<float4*>(d_prd), st);
    PHX_CU(cudaGetLastError());
    if (status) {
        PHX_CU(cudaMemcpyAsync(e->h_pinned, e->status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        PHX_CU(cudaStreamSynchronize(st));
        *status = e->h_pinned[0];
    }
    return 0;
}

int phx_trace(phx_engine* e, const float* rays, int64_t n, float t_min, float t_max, float* prd, uint32_t* status)
{
    if (!e || (n > 0 && (!rays || !prd))) return phx_fail(-1, "phx_trace: null argument");
    PHX_CU(cudaSetDevice(e->device));
    cudaStream_t st = e->stream;
    float* d_r = nullptr;
    float* d_o = nullptr;
    PHX_CU(cudaMallocAsync(&d_r, std::max<int64_t>(1, n) * 24, st));
    PHX_CU(cudaMallocAsync(&d_o, std::max<int64_t>(1, n) * 32, st));
    if (n > 0) PHX_CU(cudaMemcpyAsync(d_r, rays, n * 24, cudaMemcpyHostToDevice, st));
    int rc = phx_trace_device(e, d_r, n, t_min, t_max, d_o, status, st);
    if (!rc && n > 0) {
        cudaError_t ce = cudaMemcpyAsync(prd, d_o, n * 32, cudaMemcpyDeviceToHost, st);
        if (ce != cudaSuccess) rc = phx_fail(-2, "phx_trace: copy back failed: %s", cudaGetErrorString(ce));
    }
    cudaFreeAsync(d_r, st);
    cudaFreeAsync(d_o, st);
    PHX_CU(cudaStreamSynchronize(st));
    return rc;
}

int phx_rng_sequence(phx_engine* e, int32_t event_index, int64_t photon_offset, int64_t num_photon, int32_t num_per_photon, float* out)
{
    if (!e || !out || num_photon < 0 || num_per_photon <= 0 || photon_offset < 0) return phx_fail(-1, "phx_rng_sequence: bad argument");
    PHX_CU(cudaSetDevice(e->device));
    int rc = ensure_rng(e, photon_offset + num_photon);
    if (rc) return rc;
    cudaStream_t st = e->stream;
    float* d_o = nullptr;
    size_t bytes = (size_t)std::max<int64_t>(1, num_photon) * num_per_photon * sizeof(float);
    PHX_CU(cudaMallocAsync(&d_o, bytes, st));
    if (num_photon > 0) {
        const int B = 128;
        k_rng_sequence<<<(unsigned)((num_photon + B - 1) / B), B, 0, st>>>(e->rng.p, e->rng_slots,
            e->cfg.skipahead_event_offset * (unsigned long long)event_index, photon_offset, num_photon, num_per_photon, d_o);
        PHX_CU(cudaGetLastError());
        PHX_CU(cudaMemcpyAsync(out, d_o, (size_t)num_photon * num_per_photon * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    cudaFreeAsync(d_o, st);
    PHX_CU(cudaStreamSynchronize(st));
    return 0;
}

// every device operation of one batched call, enqueued on st with no host synchronisation
// (capturable as a CUDA graph); buffers are sized before this is called
static int batched_enqueue(phx_engine* e, const PhxBatchCall& c, phx_photon* photon, bool want_hits)
{
    cudaStream_t st = c.st;
    const int G = c.G;
    const long long N = c.N;
    const long long nword = (N + 31) / 32;
    PHX_CU(cudaMemsetAsync(e->status.p, 0, sizeof(unsigned), st));
    PHX_CU(cudaMemsetAsync(e->counters.p, 0, 8 * sizeof(long long), st));
    k_genstep_offsets<<<1, 1024, 0, st>>>(reinterpret_cast<const float4*>(c.gs), G, e->gs_off.p);
    if (G > 0) {
        k_event_starts<<<(G + 255) / 256, 256, 0, st>>>(c.ev, e->gs_off.p, G, e->ev_start.p);
        k_jump_build<<<G, 160, 0, st>>>(c.ev, 0ull, e->jump_pow.p, e->jump_tab.p);
        k_jump_nibbles<<<dim3((PHX_JUMP_BITS / 4 * 16 + 127) / 128, (unsigned)G), 128, 0, st>>>(e->jump_tab.p, e->jump4.p);
    }
    PHX_CU(cudaGetLastError());
    if (want_hits) PHX_CU(cudaMemsetAsync(e->hitword.p, 0, sizeof(uint32_t) * (size_t)std::max<long long>(1, nword), st));
    if (c.done && c.num_event > 0) {
        PHX_CU(cudaMemsetAsync(e->ev_left.p, 0, sizeof(unsigned) * (size_t)c.num_event, st));
        PHX_CU(cudaMemsetAsync(c.done, 0, sizeof(uint64_t) * ((size_t)c.num_event + 1), st));
        if (G > 0) k_event_counts<<<(G + 255) / 256, 256, 0, st>>>(c.ev, e->gs_off.p, G, e->ev_left.p, c.num_event);
        k_stamp<<<1, 1, 0, st>>>(reinterpret_cast<unsigned long long*>(c.done) + c.num_event);
    }
    SimArgs a;
    a.S = scene_of(e, e->cfg.root_polish);
    a.P = props_of(e);
    a.C = loop_of(e);
    a.gs = reinterpret_cast<const float4*>(c.gs);
    a.gs_off = e->gs_off.p;
    a.G = G;
    a.N = N;
    a.photon_offset = 0;
    a.event_index = 0;
    a.skip = e->cfg.skipahead_event_offset;
    a.rng = e->rng.p;
    a.rng_slots = e->rng_slots;
    a.jump = e->jump_tab.p;
    a.jump4 = e->jump4.p;
    a.photon = photon;
    a.seq = reinterpret_cast<phx_seq*>(c.seq);
    a.hitword = want_hits ? e->hitword.p : nullptr;
    a.hit_mask = e->cfg.hit_mask;
    a.status = e->status.p;
    PersistArgs A = persist_args_from(e, a);
    A.gs_event = c.ev;
    A.ev_start = e->ev_start.p;
    A.queue = reinterpret_cast<unsigned long long*>(e->counters.p + 1);
    A.regroup = c.regroup;
    A.chunk = c.chunk;
    if (c.done && c.num_event > 0) {
        A.ev_left = e->ev_left.p;
        A.ev_done_ns = reinterpret_cast<unsigned long long*>(c.done);
        A.num_event = c.num_event;
    }
    if (N > 0 && e->ev_rng.n >= (size_t)N * 6) {
        k_rng_event<<<(unsigned)std::min<long long>((N + 255) / 256, 148LL * 16), 256, 0, st>>>(A, e->ev_rng.p, N);
        PHX_CU(cudaGetLastError());
        A.ev_rng = e->ev_rng.p;
        A.ev_rng_n = N;
    }
    if (N > 0) {
        int rc = e->cfg.kernel_mode == 2 ? launch_wave(e, A, st) : launch_persistent(e, A, c.block, st);
        if (rc) return rc;
    }
    if (want_hits && N > 0) {
        const long long nblock = (nword + 255) / 256;
        k_word_scan<<<(unsigned)nblock, 256, 0, st>>>(e->hitword.p, nword, e->wordoff.p, e->blocksum.p);
        k_block_scan<<<1, 1024, 0, st>>>(e->blocksum.p, (int)nblock, e->counters.p);
        if (c.sensor) PHX_CU(cudaMemsetAsync(c.sensor, 0, sizeof(uint32_t) * std::max(0, e->cfg.num_sensor), st));
        k_compact<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(photon, N, e->hitword.p, e->wordoff.p, e->blocksum.p,
                                                              reinterpret_cast<phx_photon*>(c.hit), c.hcap,
                                                              c.sensor, e->cfg.num_sensor, e->status.p);
        PHX_CU(cudaGetLastError());
    }
    PHX_CU(cudaMemcpyAsync(e->h_pinned + 2, e->counters.p, sizeof(long long), cudaMemcpyDeviceToHost, st));
    PHX_CU(cudaMemcpyAsync(e->h_pinned, e->status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    return 0;
}

int phx_simulate_batched_device(phx_engine* e, const float* d_gensteps, const int32_t* d_genstep_event,
                                int32_t num_genstep, int64_t num_photon, int32_t block, int32_t chunk,
                                int32_t regroup, int32_t num_event, uint64_t* d_event_done_ns,
                                phx_outputs* d_out, void* stream)
{
    if (!e || !d_out || (num_genstep > 0 && (!d_gensteps || !d_genstep_event)))
        return phx_fail(-1, "phx_simulate_batched_device: null argument");
    if (num_genstep < 0 || num_photon < 0 || num_event < 0) return phx_fail(-1, "phx_simulate_batched_device: negative size");
    PHX_CU(cudaSetDevice(e->device));
    PhxBatchCall c;
    memset(&c, 0, sizeof(c));
    c.gs = d_gensteps; c.ev = d_genstep_event; c.G = num_genstep; c.N = num_photon;
    c.block = block > 0 ? block : e->cfg.block;
    c.chunk = chunk > 0 ? chunk : e->cfg.chunk;
    c.regroup = regroup > 0 ? regroup : e->cfg.regroup;
    c.num_event = d_event_done_ns ? num_event : 0;
    c.done = d_event_done_ns;
    c.photon = d_out->photon; c.seq = d_out->seq; c.hit = d_out->hit; c.hcap = d_out->hit_capacity; c.sensor = d_out->sensor_hits;
    c.st = stream ? (cudaStream_t)stream : e->stream;
    const long long N = c.N;
    const long long nword = (N + 31) / 32;
    const bool want_hits = c.hit != nullptr || c.sensor != nullptr;
    // size every buffer first (no allocation may happen inside a captured sequence)
    PHX_CU(e->gs_off.ensure((size_t)c.G + 1));
    PHX_CU(e->ev_start.ensure((size_t)std::max(1, c.G)));
    PHX_CU(e->counters.ensure(8));
    phx_photon* photon = reinterpret_cast<phx_photon*>(c.photon);
    if (want_hits && !photon) { PHX_CU(e->photon.ensure((size_t)std::max<long long>(1, N))); photon = e->photon.p; }
    if (want_hits) {
        PHX_CU(e->hitword.ensure((size_t)std::max<long long>(1, nword)));
        PHX_CU(e->wordoff.ensure((size_t)std::max<long long>(1, nword)));
        PHX_CU(e->blocksum.ensure((size_t)std::max<long long>(1, (nword + 255) / 256)));
    }
    if (c.num_event > 0) PHX_CU(e->ev_left.ensure((size_t)c.num_event));
    if (N > 0 && N <= PHX_EV_RNG_MAX) PHX_CU(e->ev_rng.ensure((size_t)N * 6));
    PHX_CU(e->jump_tab.ensure((size_t)std::max(1, c.G) * PHX_JUMP_MATW));
    PHX_CU(e->jump4.ensure((size_t)std::max(1, c.G) * PHX_JUMP_NIBW));
    // the wavefront loop is capturable when its schedule is fixed (wave_rounds) and the pool holds
    // every photon of the call (no refill rounds, which the host drives)
    const bool wave_fixed = e->cfg.kernel_mode == 2 && e->cfg.wave_rounds > 0 && N > 0 && wave_pool_for(e, N, false) >= N;
    if (e->cfg.use_graph && (e->cfg.kernel_mode != 2 || wave_fixed)) {
        // the captured graph bakes in every engine buffer pointer: reuse it only if none moved
        if (wave_fixed) {   // size the path pool before the capture
            const long long pool = wave_pool_for(e, N, false);
            PHX_CU(e->wslot.ensure((size_t)pool)); PHX_CU(e->wprd.ensure((size_t)pool)); PHX_CU(e->wsidx.ensure((size_t)pool));
            PHX_CU(e->wact0.ensure((size_t)pool)); PHX_CU(e->wact1.ensure((size_t)pool)); PHX_CU(e->wcnt.ensure(4));
            PHX_CU(e->wfree.ensure((size_t)pool));
        }
        const void* bufs[PHX_BATCH_BUFS] = { e->hitword.p, e->wordoff.p, e->blocksum.p, e->gs_off.p, e->ev_start.p, e->ev_left.p,
                                             e->counters.p, e->status.p, e->photon.p, e->rng.p, e->jump_tab.p, e->ev_rng.p, e->jump4.p,
                                             e->wslot.p, e->wprd.p, e->wsidx.p, e->wact0.p, e->wact1.p, e->wcnt.p, e->wfree.p };
        const bool reuse = e->batch_exec && e->batch_call == c && e->batch_launch == launch_key(e) &&
                           memcmp(bufs, e->batch_bufs, sizeof(bufs)) == 0;
        if (!reuse) {
            if (e->batch_exec) { cudaGraphExecDestroy(e->batch_exec); e->batch_exec = nullptr; }
            cudaGraph_t graph = nullptr;
            PHX_CU(cudaStreamBeginCapture(c.st, cudaStreamCaptureModeRelaxed));
            int rc = batched_enqueue(e, c, photon, want_hits);
            cudaError_t ce = cudaStreamEndCapture(c.st, &graph);
            if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
            if (ce != cudaSuccess) return phx_fail(-2, "batched graph capture failed: %s", cudaGetErrorString(ce));
            ce = cudaGraphInstantiate(&e->batch_exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ce != cudaSuccess) { e->batch_exec = nullptr; return phx_fail(-2, "batched graph instantiate failed: %s", cudaGetErrorString(ce)); }
            e->batch_call = c;
            e->batch_launch = launch_key(e);
            memcpy(e->batch_bufs, bufs, sizeof(bufs));
        }
        PHX_CU(cudaGraphLaunch(e->batch_exec, c.st));
        e->last_graph = 1;
    } else {
        e->last_graph = 0;
        int rc = batched_enqueue(e, c, photon, want_hits);
        if (rc) return rc;
    }
    PHX_CU(cudaStreamSynchronize(c.st));
    long long nh = 0;
    if (want_hits && N > 0) memcpy(&nh, e->h_pinned + 2, sizeof(long long));
    d_out->num_photon = N;
    d_out->num_hit = nh;
    d_out->status = e->h_pinned[0];
    return 0;
}

int phx_adjoint_device(phx_engine* e, const float* d_gensteps, int32_t num_genstep, int64_t num_photon,
                       int32_t event_index, const float* theta, int32_t mat_line, float wl_lo, float wl_hi,
                       double* d_hits, double* d_grad, int32_t flags, void* stream)
{
    if (!e || !theta || !d_hits || !d_grad || (num_genstep > 0 && !d_gensteps)) return phx_fail(-1, "phx_adjoint_device: null argument");
    if (num_genstep < 0 || num_photon < 0 || event_index < 0) return phx_fail(-1, "phx_adjoint_device: negative size");
    if (mat_line < 0 || mat_line >= e->num_bnd * 4 || !(wl_hi > wl_lo)) return phx_fail(-1, "phx_adjoint_device: bad material line or bins");
    if (e->cfg.num_sensor <= 0) return phx_fail(-1, "phx_adjoint_device: the engine needs num_sensor > 0");
    for (int k = 0; k < 32; k++)
        if (!(theta[k] == theta[k])) return phx_fail(-1, "phx_adjoint_device: theta[%d] is NaN", k);
    PHX_CU(cudaSetDevice(e->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : e->stream;
    const uint32_t mat = e->optical_host[(size_t)mat_line * 4];
    if (mat == 0) return phx_fail(-1, "phx_adjoint_device: line %d is not a material line", mat_line);
    // re-tabulate every material line (omat/imat) of this material with theta, in 8 bins, into a
    // pinned staging copy of the table, once the previous call's upload from it has completed
    const float binw = (wl_hi - wl_lo) / 8.f;
    if (!e->adj_tab_h) {
        PHX_CU(cudaMallocHost((void**)&e->adj_tab_h, e->bnd_host.size() * sizeof(float)));
        PHX_CU(cudaEventCreateWithFlags(&e->adj_up, cudaEventDisableTiming));
    } else {
        PHX_CU(cudaEventSynchronize(e->adj_up));
    }
    float* const tab = e->adj_tab_h;
    memcpy(tab, e->bnd_host.data(), e->bnd_host.size() * sizeof(float));
    const int nwl = e->num_wl;
    for (int b = 0; b < e->num_bnd; b++)
        for (int j = 0; j < 4; j += 3) {
            if (e->optical_host[(size_t)(4 * b + j) * 4] != mat) continue;
            float* g0 = tab + (size_t)((b * 4 + j) * 2 + 0) * nwl * 4;
            float* g1 = tab + (size_t)((b * 4 + j) * 2 + 1) * nwl * 4;
            for (int i = 0; i < nwl; i++) {
                const float lam = e->nm0 + i * e->nms;
                if (!(lam >= wl_lo && lam < wl_hi)) continue;
                const int bin = std::min(7, (int)std::floor((lam - wl_lo) / binw));
                g0[4 * i + 0] = theta[24 + bin];
                g0[4 * i + 1] = theta[bin];
                g0[4 * i + 2] = theta[8 + bin];
                g0[4 * i + 3] = theta[16 + bin];
                g1[4 * i + 0] = 299.792458f / theta[24 + bin];
            }
        }
    if (!e->adj_arr) {
        int rc = make_texture_f4(e->adj_arr, e->adj_tex, tab, (int)e->nx, (int)e->ny);
        if (rc) return rc;
    } else {
        PHX_CU(cudaMemcpy2DToArrayAsync(e->adj_arr, 0, 0, tab, e->nx * sizeof(float4), e->nx * sizeof(float4), e->ny,
                                        cudaMemcpyHostToDevice, st));
    }
    PHX_CU(cudaEventRecord(e->adj_up, st));
    int rc = ensure_rng(e, num_photon);
    if (rc) return rc;
    const int G = num_genstep;
    const long long N = num_photon;
    PHX_CU(e->gs_off.ensure((size_t)G + 1));
    PHX_CU(e->counters.ensure(8));
    PHX_CU(e->jump_tab.ensure(PHX_JUMP_MATW));
    PHX_CU(cudaMemsetAsync(e->status.p, 0, sizeof(unsigned), st));
    PHX_CU(cudaMemsetAsync(e->counters.p, 0, 2 * sizeof(long long), st));
    PHX_CU(cudaMemsetAsync(d_hits, 0, sizeof(double) * (size_t)e->cfg.num_sensor, st));
    PHX_CU(cudaMemsetAsync(d_grad, 0, sizeof(double) * (size_t)e->cfg.num_sensor * 32, st));
    k_genstep_offsets<<<1, 1024, 0, st>>>(reinterpret_cast<const float4*>(d_gensteps), G, e->gs_off.p);
    PHX_CU(e->jump4.ensure(PHX_JUMP_NIBW));
    if (event_index > 0) {
        k_jump_build<<<1, 160, 0, st>>>(nullptr, (unsigned long long)event_index, e->jump_pow.p, e->jump_tab.p);
        k_jump_nibbles<<<(PHX_JUMP_BITS / 4 * 16 + 127) / 128, 128, 0, st>>>(e->jump_tab.p, e->jump4.p);
    }
    PHX_CU(cudaGetLastError());
    SimArgs a;
    a.S = scene_of(e, 0);
    a.P = props_of(e);
    a.P.bnd_tex = e->adj_tex;
    a.C = loop_of(e);
    a.gs = reinterpret_cast<const float4*>(d_gensteps);
    a.gs_off = e->gs_off.p;
    a.G = G;
    a.N = N;
    a.photon_offset = 0;
    a.event_index = (unsigned long long)event_index;
    a.skip = e->cfg.skipahead_event_offset;
    a.rng = e->rng.p;
    a.rng_slots = e->rng_slots;
    a.jump = event_index > 0 ? e->jump_tab.p : nullptr;
    a.jump4 = event_index > 0 ? e->jump4.p : nullptr;
    a.photon = nullptr;
    a.seq = nullptr;
    a.hitword = nullptr;
    a.hit_mask = e->cfg.hit_mask;
    a.status = e->status.p;
    PersistArgs A = persist_args_from(e, a);
    A.queue = reinterpret_cast<unsigned long long*>(e->counters.p + 1);
    A.regroup = e->cfg.regroup;
    A.chunk = e->cfg.chunk;
    A.adj_hits = d_hits;
    A.adj_grad = d_grad;
    A.num_sensor = e->cfg.num_sensor;
    A.adj_mat = mat;
    A.adj_nm0 = e->nm0;
    A.adj_nms = e->nms;
    A.adj_wl_lo = wl_lo;
    A.adj_binw = binw;
    A.adj_pathwise = (flags & PHX_ADJ_PATHWISE) ? 1 : 0;
    A.adj_prim_node = e->prim_node_d.p;
    if (N > 0) {
        const int cv = cv_of(e, false);
        rc = e->cfg.kernel_mode == 2 ? launch_wave_cv<true>(e, A, cv, st) : launch_persistent_b<64, true>(e, A, cv, st);
        if (rc) return rc;
    }
    PHX_CU(cudaMemcpyAsync(e->h_pinned, e->status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    PHX_CU(cudaStreamSynchronize(st));
    if (e->h_pinned[0] & ~(unsigned)PHX_STATUS_RNG_RANGE)
        return phx_fail(-5, "phx_adjoint_device: device status 0x%x", e->h_pinned[0]);
    return 0;
}

}  // extern "C"

// ------------------------------------------------------------------ allocation-free simulate
// Some callers cannot allocate device memory per call: a framework whose caching allocator owns
// every device byte, or a per-event loop that cannot afford the device-wide synchronisation that
// cudaMalloc/cudaFree may imply.  phx_simulate_device_noalloc serves them: its scratch (genstep
// offsets, hit bit words and their prefix sums, counters, status, the event jump matrix and its
// 4-bit group tables) lives in one fixed file-scope device array instead of engine buffers that
// grow on demand.  The array below is sized for PHX_NOALLOC_MAX_PHOTON photons and
// PHX_NOALLOC_MAX_GENSTEP gensteps per call (about 2.6 MB) and is held on every GPU that loads
// this library until the process exits.  The bounce loop is always the one-kernel form (the
// persistent work queue, or one thread per photon when kernel_mode is 0): the wavefront loop's
// path pool is sized per call and would need allocation.
#define PHX_NOALLOC_MAX_PHOTON (1ll << 23)
#define PHX_NOALLOC_MAX_GENSTEP 65536
#define PHX_NOALLOC_WORDS (PHX_NOALLOC_MAX_PHOTON / 32)
#define PHX_NOALLOC_BLOCKS (PHX_NOALLOC_WORDS / 256)

struct PhxNoAllocScratch {
    long long gs_off[PHX_NOALLOC_MAX_GENSTEP + 1];
    uint32_t hitword[PHX_NOALLOC_WORDS];
    uint32_t wordoff[PHX_NOALLOC_WORDS];
    uint32_t blocksum[PHX_NOALLOC_BLOCKS];
    long long counters[8];
    unsigned status[8];
    __align__(16) uint32_t jump[PHX_JUMP_MATW];
    __align__(16) uint32_t jump4[PHX_JUMP_NIBW];
};

static __device__ __align__(256) PhxNoAllocScratch g_phx_noalloc_scratch;

// In host code the symbol above is only a host-side stand-in, never a device address.  The
// device address is looked up once per device, with that device current, and cached.
#include <mutex>
static std::mutex g_phx_noalloc_mu;
static PhxNoAllocScratch* g_phx_noalloc_ptr[128] = {};

static int noalloc_scratch(int device, PhxNoAllocScratch** out)
{
    std::lock_guard<std::mutex> lock(g_phx_noalloc_mu);
    if (device < 0 || device >= 128) return phx_fail(-1, "phx_simulate_device_noalloc: device %d out of range", device);
    if (!g_phx_noalloc_ptr[device]) {
        void* p = nullptr;
        cudaError_t rc = cudaGetSymbolAddress(&p, g_phx_noalloc_scratch);
        if (rc != cudaSuccess || !p)
            return phx_fail(-2, "phx_simulate_device_noalloc: cudaGetSymbolAddress of the scratch array failed on device %d: %s",
                            device, cudaGetErrorString(rc));
        g_phx_noalloc_ptr[device] = static_cast<PhxNoAllocScratch*>(p);
    }
    *out = g_phx_noalloc_ptr[device];
    return 0;
}

extern "C" int phx_simulate_device_noalloc(phx_engine* e, const float* d_gensteps, int32_t num_genstep, int64_t num_photon,
                                           int32_t event_index, int64_t photon_offset, phx_outputs* d_out, void* stream)
{
    if (!e || !d_out) return phx_fail(-1, "phx_simulate_device_noalloc: null argument");
    if (num_genstep < 0 || num_photon < 0 || photon_offset < 0)
        return phx_fail(-1, "phx_simulate_device_noalloc: negative size or offset");
    if (num_genstep > PHX_NOALLOC_MAX_GENSTEP)
        return phx_fail(-4, "phx_simulate_device_noalloc: %d gensteps exceed the fixed scratch limit of %d per call",
                        num_genstep, PHX_NOALLOC_MAX_GENSTEP);
    if (event_index < 0) return phx_fail(-1, "phx_simulate_device_noalloc: negative event index");
    if (num_photon > PHX_NOALLOC_MAX_PHOTON)
        return phx_fail(-4, "phx_simulate_device_noalloc: %lld photons exceed the fixed scratch limit of %lld per call",
                        (long long)num_photon, (long long)PHX_NOALLOC_MAX_PHOTON);
    if (photon_offset + num_photon > e->rng_slots)
        return phx_fail(-4, "phx_simulate_device_noalloc: photons %lld..%lld need RNG slots the engine did not prepare (%lld); "
                        "create the engine with a larger max_photon", (long long)photon_offset,
                        (long long)(photon_offset + num_photon), e->rng_slots);
    const bool want_hits = d_out->hit != nullptr || d_out->sensor_hits != nullptr;
    if (want_hits && num_photon > 0 && !d_out->photon)
        return phx_fail(-1, "phx_simulate_device_noalloc: hit selection reads the photon output, pass d_out->photon");
    PHX_CU(cudaSetDevice(e->device));
    PhxNoAllocScratch* scr = nullptr;
    int rc = noalloc_scratch(e->device, &scr);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : e->stream;
    const long long N = num_photon;
    // phx_simulate_device's launch sequence in its one-kernel loop form (never the wavefront
    // rounds), on the fixed scratch
    PhxPlainBufs b = { scr->gs_off, scr->hitword, scr->wordoff, scr->blocksum, scr->counters, scr->status, scr->jump,
                       scr->jump4 };
    rc = plain_enqueue(e, b, d_gensteps, num_genstep, N, event_index, photon_offset, reinterpret_cast<phx_photon*>(d_out->photon),
                       reinterpret_cast<phx_seq*>(d_out->seq), reinterpret_cast<phx_photon*>(d_out->hit), d_out->hit_capacity,
                       d_out->sensor_hits, want_hits, st);
    if (rc) return rc;
    PHX_CU(cudaStreamSynchronize(st));
    long long nh = 0;
    if (want_hits && N > 0) memcpy(&nh, e->h_pinned + 2, sizeof(long long));
    d_out->num_photon = N;
    d_out->num_hit = nh;
    d_out->status = e->h_pinned[0];
    return 0;
}

// ------------------------------------------------------------------ hit merging
// exclusive scan of n u32 in place; the total goes to *d_total when given
static int merge_scan(PhxMergeWs& w, uint32_t* x, long long n, long long* d_total, cudaStream_t st)
{
    const long long nt = (n + PHX_MERGE_SCAN_TILE - 1) / PHX_MERGE_SCAN_TILE;
    PHX_CU(w.tsum.ensure((size_t)std::max(1LL, nt)));
    PHX_CU(w.total.ensure(2));
    k_scan_tile<<<(unsigned)nt, 256, 0, st>>>(x, n, w.tsum.p);
    k_block_scan<<<1, 1024, 0, st>>>(w.tsum.p, (int)nt, d_total ? d_total : w.total.p + 1);
    k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, n, w.tsum.p);
    PHX_CU(cudaGetLastError());
    return 0;
}

// read back a few bytes through the engine's pinned words (synchronises the stream)
static int merge_read(phx_engine* e, const void* d, size_t bytes, void* h, cudaStream_t st)
{
    PHX_CU(cudaMemcpyAsync(e->h_pinned + 48, d, bytes, cudaMemcpyDeviceToHost, st));
    PHX_CU(cudaStreamSynchronize(st));
    memcpy(h, e->h_pinned + 48, bytes);
    return 0;
}

template <int LITE>
static int merge_impl(phx_engine* e, const uint32_t* in, long long n, uint32_t mask, float tw, uint32_t* out, long long cap,
                      long long* num_out, cudaStream_t st)
{
    PhxMergeWs& w = e->merge;
    *num_out = 0;
    if (n == 0) return 0;
    long long m = n;
    const uint32_t* sel = nullptr;
    int rc;
    PHX_CU(w.total.ensure(2));
    if (mask != 0xffffffffu) {
        const long long nt = (n + PHX_MERGE_TILE - 1) / PHX_MERGE_TILE;
        PHX_CU(w.tcount.ensure((size_t)nt));
        PHX_CU(w.sel.ensure((size_t)n));
        k_merge_sel_count<LITE><<<(unsigned)nt, 256, 0, st>>>(in, n, mask, w.tcount.p);
        k_block_scan<<<1, 1024, 0, st>>>(w.tcount.p, (int)nt, w.total.p);
        k_merge_sel_write<LITE><<<(unsigned)nt, 256, 0, st>>>(in, n, mask, w.tcount.p, w.sel.p);
        PHX_CU(cudaGetLastError());
        if ((rc = merge_read(e, w.total.p, sizeof(long long), &m, st))) return rc;
        sel = w.sel.p;
    }
    if (m == 0) return 0;
    const int W = PhxRec<LITE>::W;
    const unsigned grid = (unsigned)std::min<long long>((m + 255) / 256, 148LL * 16);
    if (tw == 0.f) {                 // selection only, input order
        *num_out = m;
        if (m > cap) return phx_fail(-3, "phx_merge_hits: %lld records selected, out_capacity %lld", m, cap);
        k_merge_gather<LITE><<<(unsigned)std::min<long long>((m * W + 255) / 256, 148LL * 32), 256, 0, st>>>(in, sel, m, out);
        PHX_CU(cudaGetLastError());
        return 0;
    }
    PHX_CU(w.key0.ensure((size_t)m)); PHX_CU(w.key1.ensure((size_t)m));
    PHX_CU(w.val0.ensure((size_t)m)); PHX_CU(w.val1.ensure((size_t)m));
    PHX_CU(w.key_or.ensure(1));
    PHX_CU(cudaMemsetAsync(w.key_or.p, 0, sizeof(unsigned long long), st));
    k_merge_keys<LITE><<<grid, 256, 0, st>>>(in, sel, m, tw, w.key0.p, w.val0.p, w.key_or.p);
    PHX_CU(cudaGetLastError());
    unsigned long long kor = 0;
    if ((rc = merge_read(e, w.key_or.p, sizeof(kor), &kor, st))) return rc;
    // stable LSD radix passes over the key bytes that are non-zero somewhere
    const long long nt = (m + PHX_MERGE_TILE - 1) / PHX_MERGE_TILE;
    PHX_CU(w.hist.ensure((size_t)(256 * nt)));
    unsigned long long* kin = w.key0.p;
    unsigned long long* kout = w.key1.p;
    uint32_t* vin = w.val0.p;
    uint32_t* vout = w.val1.p;
    for (int b = 0; b < 8; b++) {
        if (((kor >> (8 * b)) & 0xffull) == 0ull) continue;
        k_radix_hist<<<(unsigned)nt, 256, 0, st>>>(kin, m, 8 * b, w.hist.p, (int)nt);
        if ((rc = merge_scan(w, w.hist.p, 256 * nt, nullptr, st))) return rc;
        k_radix_scatter<<<(unsigned)nt, 256, 0, st>>>(kin, vin, kout, vout, m, 8 * b, w.hist.p, (int)nt);
        PHX_CU(cudaGetLastError());
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    // groups
    PHX_CU(w.head.ensure((size_t)m));
    k_merge_heads<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(kin, m, w.head.p);
    if ((rc = merge_scan(w, w.head.p, m, w.total.p, st))) return rc;
    long long ng = 0;
    if ((rc = merge_read(e, w.total.p, sizeof(long long), &ng, st))) return rc;
    *num_out = ng;
    if (ng > cap) return phx_fail(-3, "phx_merge_hits: %lld merged records, out_capacity %lld", ng, cap);
    PHX_CU(w.amin.ensure((size_t)ng)); PHX_CU(w.pmin.ensure((size_t)ng));
    PHX_CU(w.gor.ensure((size_t)ng)); PHX_CU(w.gsum.ensure((size_t)ng));
    PHX_CU(cudaMemsetAsync(w.amin.p, 0xff, sizeof(unsigned long long) * ng, st));
    PHX_CU(cudaMemsetAsync(w.pmin.p, 0xff, sizeof(uint32_t) * ng, st));
    PHX_CU(cudaMemsetAsync(w.gor.p, 0, sizeof(uint32_t) * ng, st));
    PHX_CU(cudaMemsetAsync(w.gsum.p, 0, sizeof(uint32_t) * ng, st));
    k_merge_reduce<LITE><<<grid, 256, 0, st>>>(in, sel, kin, vin, w.head.p, m, w.amin.p, w.pmin.p, w.gor.p, w.gsum.p);
    k_merge_write<LITE><<<(unsigned)((ng + 255) / 256), 256, 0, st>>>(in, sel, ng, w.amin.p, w.pmin.p, w.gor.p, w.gsum.p, out);
    PHX_CU(cudaGetLastError());
    return 0;
}

static int merge_check(const char* fn, phx_engine* e, const void* in, int64_t n, int32_t lite, float tw)
{
    if (!e) return phx_fail(-1, "%s: null engine", fn);
    if (n < 0 || n > 0x7fffffffLL) return phx_fail(-1, "%s: num_in %lld outside [0, 2^31)", fn, (long long)n);
    if (n > 0 && !in) return phx_fail(-1, "%s: null input", fn);
    if (lite != 0 && lite != 1) return phx_fail(-1, "%s: record kind %d (0 sphoton, 1 sphotonlite)", fn, lite);
    if (!(tw >= 0.f)) return phx_fail(-1, "%s: time_window must be >= 0", fn);
    return 0;
}

int phx_merge_hits_device(phx_engine* e, const void* d_in, int64_t num_in, int32_t lite, uint32_t select_flagmask,
                          float time_window, void* d_out, int64_t out_capacity, int64_t* num_out, void* stream)
{
    int rc = merge_check("phx_merge_hits_device", e, d_in, num_in, lite, time_window);
    if (rc) return rc;
    if (out_capacity > 0 && !d_out) return phx_fail(-1, "phx_merge_hits_device: null output with out_capacity > 0");
    PHX_CU(cudaSetDevice(e->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : e->stream;
    long long no = 0;
    rc = lite ? merge_impl<1>(e, (const uint32_t*)d_in, num_in, select_flagmask, time_window, (uint32_t*)d_out, out_capacity, &no, st)
              : merge_impl<0>(e, (const uint32_t*)d_in, num_in, select_flagmask, time_window, (uint32_t*)d_out, out_capacity, &no, st);
    if (num_out) *num_out = no;
    return rc;
}

int phx_merge_hits(phx_engine* e, const void* in, int64_t num_in, int32_t lite, uint32_t select_flagmask, float time_window,
                   void* out, int64_t out_capacity, int64_t* num_out)
{
    int rc = merge_check("phx_merge_hits", e, in, num_in, lite, time_window);
    if (rc) return rc;
    PHX_CU(cudaSetDevice(e->device));
    cudaStream_t st = e->stream;
    const size_t rb = lite ? 16 : 64;
    PhxMergeWs& w = e->merge;
    PHX_CU(w.hin.ensure((size_t)std::max<int64_t>(1, num_in) * rb / 4));
    PHX_CU(w.hout.ensure((size_t)std::max<int64_t>(1, num_in) * rb / 4));
    if (num_in > 0) PHX_CU(cudaMemcpyAsync(w.hin.p, in, (size_t)num_in * rb, cudaMemcpyHostToDevice, st));
    long long no = 0;
    rc = lite ? merge_impl<1>(e, w.hin.p, num_in, select_flagmask, time_window, w.hout.p, num_in, &no, st)
              : merge_impl<0>(e, w.hin.p, num_in, select_flagmask, time_window, w.hout.p, num_in, &no, st);
    if (num_out) *num_out = no;
    if (rc) return rc;
    if (no > out_capacity) return phx_fail(-3, "phx_merge_hits: %lld merged records, out_capacity %lld", no, (long long)out_capacity);
    if (no > 0) {
        if (!out) return phx_fail(-1, "phx_merge_hits: null output");
        PHX_CU(cudaMemcpyAsync(out, w.hout.p, (size_t)no * rb, cudaMemcpyDeviceToHost, st));
    }
    PHX_CU(cudaStreamSynchronize(st));
    return 0;
}

// SEvt::setInputPhoton (sysrap/SEvt.cc:602-640) with QEvt's upload of the input photons
// (qudarap/QEvt.cc:540-560): INPUT_PHOTON gensteps copy photon[photon index] and set TORCH.
int phx_set_input_photon(phx_engine* e, const float* photon, int64_t num_photon)
{
    if (!e) return phx_fail(-1, "phx_set_input_photon: null engine");
    if (num_photon < 0 || (num_photon > 0 && !photon)) return phx_fail(-1, "phx_set_input_photon: bad array");
    PHX_CU(cudaSetDevice(e->device));
    e->input_photon = nullptr;
    e->num_input_photon = 0;
    if (num_photon == 0) { e->input_own.release(); return 0; }
    PHX_CU(e->input_own.ensure((size_t)num_photon * 4));
    PHX_CU(cudaMemcpy(e->input_own.p, photon, (size_t)num_photon * 64, cudaMemcpyHostToDevice));
    e->input_photon = e->input_own.p;
    e->num_input_photon = num_photon;
    return 0;
}

int phx_set_input_photon_device(phx_engine* e, const float* d_photon, int64_t num_photon)
{
    if (!e) return phx_fail(-1, "phx_set_input_photon_device: null engine");
    if (num_photon < 0 || (num_photon > 0 && !d_photon)) return phx_fail(-1, "phx_set_input_photon_device: bad array");
    if (((uintptr_t)d_photon & 15u) != 0u) return phx_fail(-1, "phx_set_input_photon_device: array not 16-byte aligned");
    e->input_own.release();
    e->input_photon = num_photon > 0 ? reinterpret_cast<const float4*>(d_photon) : nullptr;
    e->num_input_photon = num_photon;
    return 0;
}

int phx_last_call_stats(phx_engine* e, int64_t* kernel_launches, int64_t* wave_rounds, int32_t* graph)
{
    if (!e) return phx_fail(-1, "phx_last_call_stats: null engine");
    if (kernel_launches) *kernel_launches = e->last_launches;
    if (wave_rounds) *wave_rounds = e->last_rounds;
    if (graph) *graph = e->last_graph;
    return 0;
}
