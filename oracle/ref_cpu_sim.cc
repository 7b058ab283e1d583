// ref_cpu_sim.cc : TEST INFRASTRUCTURE ONLY — the reference's own simulate path compiled for the
// CPU, the CPU baseline of the bench.
//
// Built by oracle/Makefile (target `ref`) from the unmodified reference headers where they lie in
// the reference checkout (qudarap/qsim.h, sysrap/*.h, CSG/csg_intersect_*.h) with g++ and the
// reference's CPU mocking switches (MOCK_CURAND, MOCK_CUDA, MOCK_TEXTURE; qudarap/tests/
// QSim_MockTest.sh), into oracle/_ref/libref_cpu_sim.so.  The GLM and plog headers those sysrap
// headers name are replaced by declaration-only stand-ins (oracle/shim/).  As in ref_sim.cu the
// raygen loop of CSGOptiX/CSGOptiX7.cu:432-530 is restated with optixTrace replaced by a closest
// hit over (instance, prim) pairs calling the reference's intersect_prim (with a world-box cull of
// the pairs); generation, fill_state, propagate and the seq nibbles are the reference's code.
// Randoms: the reference's CPU generator (sysrap/srngcpu.h, mt19937_64), one per worker thread.
// Textures: the reference's mock (sysrap/s_mock_texture.h, nearest sample) for the float4
// boundary table; the scintillation ICDF is a float table, which that mock does not read, so this
// driver supplies tex2D<float> with the same nearest-sample rule.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>
#include "scuda.h"
#include "squad.h"
#include "sqat4.h"
#include "srngcpu.h"
using RNG = srngcpu;
#include "stexture.h"

MockTextureManager* MockTextureManager::INSTANCE = nullptr;

// float tables (the scintillation ICDF): ids from 1 << 20, nearest sample as MockTexture::lookup
struct FloatTex { std::vector<float> v; int width, height; };
static std::vector<FloatTex> g_ftex;
static const cudaTextureObject_t FTEX0 = 1u << 20;

template <> inline float tex2D<float>(cudaTextureObject_t t, float x, float y)
{
    const FloatTex& f = g_ftex[(size_t)(t - FTEX0)];
    int ix = int(x * float(f.width));
    int iy = int(y * float(f.height));
    ix = ix < 0 ? 0 : (ix >= f.width ? f.width - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= f.height ? f.height - 1 : iy);
    return f.v[(size_t)iy * f.width + ix];
}

#include "sphoton.h"
#include "sphotonlite.h"
#include "scerenkov.h"
#include "sstate.h"
#include "stag.h"
#include "sseq.h"
#include "srec.h"
#include "sevent.h"
#include "sctx.h"
#include "qsim.h"
#include "csg_intersect_leaf.h"
#include "csg_intersect_node.h"
#include "csg_intersect_tree.h"

struct CpuScene {
    const CSGNode* node;
    const float4* plan;
    const qat4* itra;
    const qat4* inst_inv;
    const int* pair_inst;
    const int* pair_node;
    const unsigned* pair_gpbd;
    const unsigned* pair_iiid;
    const float* pair_bbox;   // (num_pair, 6) world box lo, hi
    int num_pair;
};

// closest hit over the pairs with the IS/CH semantics of CSGOptiX/CSGOptiX7.cu:776-967
static void cpu_trace(const CpuScene& S, const float3& o, const float3& d, float tmin, float tmax, quad2* prd)
{
    float best = tmax;
    int bi = -1;
    float4 bis = make_float4(0.f, 0.f, 0.f, 0.f);
    float blc = 0.f;
    const float ix = 1.f / (d.x != 0.f ? d.x : 1e-30f), iy = 1.f / (d.y != 0.f ? d.y : 1e-30f), iz = 1.f / (d.z != 0.f ? d.z : 1e-30f);
    for (int k = 0; k < S.num_pair; k++) {
        const float* b = S.pair_bbox + 6 * k;
        float t0 = (b[0] - o.x) * ix, t1 = (b[3] - o.x) * ix;
        float lo = fminf(t0, t1), hi = fmaxf(t0, t1);
        t0 = (b[1] - o.y) * iy; t1 = (b[4] - o.y) * iy;
        lo = fmaxf(lo, fminf(t0, t1)); hi = fminf(hi, fmaxf(t0, t1));
        t0 = (b[2] - o.z) * iz; t1 = (b[5] - o.z) * iz;
        lo = fmaxf(lo, fminf(t0, t1)); hi = fminf(hi, fmaxf(t0, t1));
        if (hi < lo || hi < tmin || lo > best) continue;
        const qat4* m = S.inst_inv + S.pair_inst[k];
        float3 lo3 = m->right_multiply(o, 1.f);
        float3 ld3 = m->right_multiply(d, 0.f);
        float4 is = make_float4(0.f, 0.f, 0.f, 0.f);
        bool v = intersect_prim(is, S.node + S.pair_node[k], S.plan, S.itra, tmin, lo3, ld3, false);
        if (v && is.w >= tmin && is.w < best) {
            best = is.w; bi = k; bis = is;
            const float3 lpos = lo3 + is.w * ld3;
            blc = normalize_cost(lpos);
        }
    }
    if (bi < 0) {
        prd->q0.f = make_float4(0.f, 0.f, 0.f, 1.f);
        prd->set_iindex_identity_(0xffffffffu);
        prd->set_globalPrimIdx_boundary_(0xffffffffu);
        prd->set_lpos(0.f, 0.f);
        return;
    }
    const qat4* m = S.inst_inv + S.pair_inst[bi];
    float3 n = m->left_multiply(make_float3(bis.x, bis.y, bis.z), 0.f);
    prd->q0.f = make_float4(n.x, n.y, n.z, best);
    prd->set_iindex_identity_(S.pair_iiid[bi]);
    prd->set_globalPrimIdx_boundary_(S.pair_gpbd[bi]);
    prd->set_lpos(blc, 0.f);
}

// CSGOptiX/CSGOptiX7.cu:432-530 for photons [begin, end) of the event on one worker thread
static void cpu_simulate_range(qsim* sim, sevent* evt, const CpuScene& S, srngcpu& rng, long long begin, long long end,
                               float tmin, float tmin0, unsigned mask, float max_time, float* photon_out)
{
    for (long long idx = begin; idx < end; idx++) {
        const unsigned genstep_idx = evt->seed[idx];
        const quad6& gs = evt->genstep[genstep_idx];
        quad2 prd;
        prd.zero();
        sctx ctx = {};
        ctx.evt = evt;
        ctx.prd = &prd;
        ctx.idx = (unsigned)idx;
        ctx.pidx = (unsigned long long)idx;
        sim->generate_photon(ctx.p, rng, gs, (unsigned long long)idx, genstep_idx);
        int command = START;
        int bounce = 0;
        ctx.point(bounce);
        while (bounce < evt->max_bounce && ctx.p.time < max_time) {
            const float tm = (ctx.p.orient_boundary_flag & mask) ? tmin0 : tmin;
            cpu_trace(S, ctx.p.pos, ctx.p.mom, tm, 1000000.f, &prd);
            if (prd.boundary() == 0xffffu) break;
            float3* normal = prd.normal();
            *normal = normalize(*normal);
            ctx.trace(bounce);
            command = sim->propagate(bounce, rng, ctx);
            bounce++;
            ctx.point(bounce);
            if (command == BREAK) break;
        }
        ctx.end();
        if (photon_out) memcpy(photon_out + 16 * idx, &ctx.p, sizeof(sphoton));
    }
}

extern "C" int ref_cpu_sim_run(
    const float* node, const float* itra, const float* plan, const float* inst_inv,
    const int* pair_inst, const int* pair_node, const unsigned* pair_gpbd, const unsigned* pair_iiid, const float* pair_bbox, int npair,
    const float* bnd, int nb, int nwl, float nm0, float nms, const unsigned* optical,
    const float* icdf, int icdf_w, int icdf_h, int hd_factor,
    const float* gs, int G, long long N, int max_bounce, float max_time, float tmin, float tmin0, unsigned eps0mask,
    unsigned long long seed, int nthreads, float* photon_out, unsigned long long* seq_out, double* seconds)
{
    std::vector<unsigned> seed_h((size_t)(N > 0 ? N : 1));
    long long k = 0;
    for (int g = 0; g < G; g++) {
        int c; memcpy(&c, gs + 24 * g + 3, 4);
        for (int j = 0; j < c && k < N; j++) seed_h[(size_t)k++] = (unsigned)g;
    }
    if (k != N) return -1;
    CpuScene S;
    S.node = (const CSGNode*)node;
    S.plan = (const float4*)plan;
    S.itra = (const qat4*)itra;
    S.inst_inv = (const qat4*)inst_inv;
    S.pair_inst = pair_inst; S.pair_node = pair_node; S.pair_gpbd = pair_gpbd; S.pair_iiid = pair_iiid;
    S.pair_bbox = pair_bbox;
    S.num_pair = npair;

    // the boundary table as the reference's mock float4 texture: rows (num_bnd*4*2) of num_wl samples
    NP* bnd_np = NP::Make<float>(nb * 8, nwl, 4);
    memcpy(bnd_np->bytes(), bnd, sizeof(float) * (size_t)nb * 8 * nwl * 4);
    bnd_np->set_meta<float>("domain_low", nm0);
    bnd_np->set_meta<float>("domain_high", nm0 + nms * (nwl - 1));
    bnd_np->set_meta<float>("domain_step", nms);
    bnd_np->set_meta<float>("domain_range", nms * (nwl - 1));
    quad4 meta; memset(&meta, 0, sizeof(meta));
    meta.q0.u.x = (unsigned)nwl; meta.q0.u.y = (unsigned)(nb * 8);
    meta.q1.f.x = nm0; meta.q1.f.z = nms;
    qbnd bnd_h; memset(&bnd_h, 0, sizeof(bnd_h));
    bnd_h.boundary_tex = MockTextureManager::Add(bnd_np);
    bnd_h.boundary_meta = &meta;
    bnd_h.optical = (quad*)optical;
    qscint sc_h; memset(&sc_h, 0, sizeof(sc_h));
    if (icdf) {
        FloatTex f;
        f.v.assign(icdf, icdf + (size_t)icdf_w * icdf_h);
        f.width = icdf_w; f.height = icdf_h;
        g_ftex.push_back(f);
        sc_h.scint_tex = FTEX0 + (cudaTextureObject_t)(g_ftex.size() - 1);
    }
    sc_h.hd_factor = (unsigned)hd_factor;
    qbase base_h; base_h.pidx = 0xffffffffffffffffull;
    qcerenkov ck_h; memset(&ck_h, 0, sizeof(ck_h));
    ck_h.base = &base_h; ck_h.bnd = &bnd_h;

    sevent ev; memset(&ev, 0, sizeof(ev));
    ev.max_bounce = max_bounce;
    ev.max_seq = 1;
    ev.index = 0;
    ev.num_seed = (size_t)N;
    ev.num_photon = (size_t)N;
    ev.num_genstep = (size_t)G;
    ev.genstep = (quad6*)gs;
    ev.seed = (int*)seed_h.data();
    std::vector<sphoton> ph((size_t)(N > 0 ? N : 1));
    std::vector<sseq> sq((size_t)(N > 0 ? N : 1));
    memset(sq.data(), 0, sizeof(sseq) * sq.size());
    ev.photon = ph.data();
    ev.seq = sq.data();

    qsim sim_h;
    memset(&sim_h, 0, sizeof(sim_h));
    sim_h.base = &base_h; sim_h.evt = &ev; sim_h.bnd = &bnd_h; sim_h.cerenkov = &ck_h; sim_h.scint = &sc_h;

    const int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<long long> next(0);
    const long long chunk = 256;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; t++) {
        pool.emplace_back([&, t]() {
            srngcpu rng;
            rng.engine.seed(seed + 7919ull * (unsigned long long)t);
            for (;;) {
                const long long b = next.fetch_add(chunk);
                if (b >= N) break;
                cpu_simulate_range(&sim_h, &ev, S, rng, b, std::min(N, b + chunk), tmin, tmin0, eps0mask, max_time, photon_out);
            }
        });
    }
    for (auto& th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    if (seq_out && N > 0) memcpy(seq_out, sq.data(), sizeof(sseq) * (size_t)N);
    return nt;
}
