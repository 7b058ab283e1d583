// ref_sim.cu : TEST INFRASTRUCTURE ONLY — a driver that runs the reference's own device code.
//
// Compiled by oracle/Makefile (target `ref`) against the unmodified reference headers where
// they lie in the reference checkout (qudarap/qsim.h, sysrap/*.h, CSG/csg_intersect_*.h), with
// the reference's flags (-DRNG_XORWOW --use_fast_math, cmake/Modules/OpticksCUDAFlags.cmake:95,
// sysrap/CMakeLists.txt:902) and without PRODUCTION so sctx records seq.  The output goes to
// oracle/_ref/libref_sim.so.  OptiX is absent, so this driver restates the raygen simulate()
// of CSGOptiX/CSGOptiX7.cu:432-530 with optixTrace replaced by a brute-force closest-hit loop
// over (instance, prim) pairs that calls the reference's intersect_prim with the IS/CH
// semantics of CSGOptiX/CSGOptiX7.cu:776-967.  Everything physical (generation, fill_state,
// propagate, seq nibbles) is the reference's code.
#include <cstdio>
#include <cstring>
#include <vector>
#include "scuda.h"
#include "squad.h"
#include "sqat4.h"
#include "sphoton.h"
#include "sphotonlite.h"
#include "scerenkov.h"
#include "sstate.h"
#include "stag.h"
#include "sseq.h"
#include "srec.h"
#include "sevent.h"
#include "sctx.h"
#include <curand_kernel.h>
#include "qrng.h"
#include "qsim.h"
#include "qplanck.h"
#include "sblackbody.h"
#include "csg_intersect_leaf.h"
#include "csg_intersect_node.h"
#include "csg_intersect_tree.h"

struct RefScene {
    const CSGNode* node;
    const float4* plan;
    const qat4* itra;
    const qat4* inst_inv;
    const int* pair_inst;
    const int* pair_node;
    const unsigned* pair_gpbd;
    const unsigned* pair_iiid;
    int num_pair;
};

__device__ void ref_trace(const RefScene& S, const float3& o, const float3& d, float tmin, float tmax, quad2* prd)
{
    float best = tmax;
    int bi = -1;
    float4 bis = make_float4(0.f, 0.f, 0.f, 0.f);
    float blc = 0.f;
    for (int k = 0; k < S.num_pair; k++) {
        const qat4* m = S.inst_inv + S.pair_inst[k];
        float3 lo = m->right_multiply(o, 1.f);
        float3 ld = m->right_multiply(d, 0.f);
        float4 is = make_float4(0.f, 0.f, 0.f, 0.f);
        bool v = intersect_prim(is, S.node + S.pair_node[k], S.plan, S.itra, tmin, lo, ld, false);
        // OptiX ignores a reported intersection outside the ray's [tmin, tmax] interval; a leaf
        // can report valid with t = 0 (a convexpolyhedron wholly behind the ray leaves isect
        // unset, CSG/csg_intersect_leaf_convexpolyhedron.h:85-101), which that rule drops
        if (v && is.w >= tmin && is.w < best) {
            best = is.w; bi = k; bis = is;
            const float3 lpos = lo + is.w * ld;
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

__global__ void ref_simulate_k(qsim* sim, sevent* evt, RefScene S, float tmin, float tmin0, unsigned mask, float max_time)
{
    unsigned idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= evt->num_seed) return;
    unsigned genstep_idx = evt->seed[idx];
    const quad6& gs = evt->genstep[genstep_idx];
    unsigned long long photon_idx = idx;
    RNG rng;
    sim->rng->init(rng, sim->evt->index, photon_idx);
    quad2 prd;
    prd.zero();
    sctx ctx = {};
    ctx.evt = evt;
    ctx.prd = &prd;
    ctx.idx = idx;
    ctx.pidx = photon_idx;
    sim->generate_photon(ctx.p, rng, gs, photon_idx, genstep_idx);
    int command = START;
    int bounce = 0;
    ctx.point(bounce);
    while (bounce < evt->max_bounce && ctx.p.time < max_time) {
        float tm = (ctx.p.orient_boundary_flag & mask) ? tmin0 : tmin;
        ref_trace(S, ctx.p.pos, ctx.p.mom, tm, 1000000.f, &prd);
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
    evt->photon[idx] = ctx.p;
}

__global__ void ref_curand_init_k(unsigned long long seed, int n, XORWOW* states)
{
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    curand_init(seed, id, 0, states + id);
}

// reference CSG on the device for the scan comparison
__global__ void ref_scan_k(const CSGNode* node, const float4* plan, const qat4* itra, float tmin, const float* rays, long long n, float4* out)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 o = make_float3(rays[i], rays[n + i], rays[2 * n + i]);
    float3 d = make_float3(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]);
    float4 is = make_float4(0.f, 0.f, 0.f, 0.f);
    bool v = intersect_prim(is, node, plan, itra, tmin, o, d, false);
    out[i] = v ? is : make_float4(0.f, 0.f, 0.f, 0.f);
}

template <typename T>
static T* up(const T* h, size_t n)
{
    T* d = nullptr;
    cudaMalloc(&d, sizeof(T) * (n > 0 ? n : 1));
    if (n > 0) cudaMemcpy(d, h, sizeof(T) * n, cudaMemcpyHostToDevice);
    return d;
}

static cudaTextureObject_t tex_f4(const float* data, int w, int h, cudaArray_t* arr)
{
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float4>();
    cudaMallocArray(arr, &ch, w, h);
    cudaMemcpy2DToArray(*arr, 0, 0, data, w * sizeof(float4), w * sizeof(float4), h, cudaMemcpyHostToDevice);
    cudaResourceDesc rd; memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray; rd.res.array.array = *arr;
    cudaTextureDesc td; memset(&td, 0, sizeof(td));
    td.addressMode[0] = cudaAddressModeWrap; td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear; td.readMode = cudaReadModeElementType; td.normalizedCoords = 1;
    cudaTextureObject_t t = 0;
    cudaCreateTextureObject(&t, &rd, &td, nullptr);
    return t;
}

static cudaTextureObject_t tex_f1(const float* data, int w, int h, cudaArray_t* arr)
{
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
    cudaMallocArray(arr, &ch, w, h);
    cudaMemcpy2DToArray(*arr, 0, 0, data, w * sizeof(float), w * sizeof(float), h, cudaMemcpyHostToDevice);
    cudaResourceDesc rd; memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray; rd.res.array.array = *arr;
    cudaTextureDesc td; memset(&td, 0, sizeof(td));
    td.addressMode[0] = cudaAddressModeWrap; td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear; td.readMode = cudaReadModeElementType; td.normalizedCoords = 1;
    cudaTextureObject_t t = 0;
    cudaCreateTextureObject(&t, &rd, &td, nullptr);
    return t;
}

extern "C" int ref_sim_run(
    const float* node, int nn, const float* itra, int nt, const float* plan, int npl, const float* inst_inv, int ni,
    const int* pair_inst, const int* pair_node, const unsigned* pair_gpbd, const unsigned* pair_iiid, int npair,
    const float* bnd, int nb, int nwl, float nm0, float nms, const unsigned* optical,
    const float* icdf, int icdf_w, int icdf_h, int hd_factor,
    unsigned long long seed, unsigned long long skip, int event_index,
    const float* gs, int G, long long N,
    int max_bounce, float max_time, float tmin, float tmin0, unsigned eps0mask,
    float* photon_out, unsigned long long* seq_out, float* record_out, float* prd_out, int max_record,
    const float* input_photon, long long num_input)
{
    // record_out (N, max_record, 4, 4) sphoton per point and prd_out (N, max_record, 2, 4) quad2 per
    // trace, as the reference's sctx::point / sctx::trace write them; max_record >= max_bounce + 1
    if (record_out && max_record < max_bounce + 1) return -3;
    std::vector<int> seed_h((size_t)N);
    long long k = 0;
    for (int g = 0; g < G; g++) {
        int c; memcpy(&c, gs + 24 * g + 3, 4);
        for (int j = 0; j < c && k < N; j++) seed_h[(size_t)k++] = g;
    }
    if (k != N) return -1;

    RefScene S;
    S.node = up((const CSGNode*)node, (size_t)nn);
    S.plan = npl > 0 ? up((const float4*)plan, (size_t)npl) : nullptr;
    S.itra = up((const qat4*)itra, (size_t)nt);
    S.inst_inv = up((const qat4*)inst_inv, (size_t)ni);
    S.pair_inst = up(pair_inst, (size_t)npair);
    S.pair_node = up(pair_node, (size_t)npair);
    S.pair_gpbd = up(pair_gpbd, (size_t)npair);
    S.pair_iiid = up(pair_iiid, (size_t)npair);
    S.num_pair = npair;

    cudaArray_t a_bnd = nullptr, a_icdf = nullptr;
    cudaTextureObject_t t_bnd = tex_f4(bnd, nwl, nb * 8, &a_bnd);
    float zero4[4] = { 0, 0, 0, 0 };
    cudaTextureObject_t t_icdf = icdf ? tex_f1(icdf, icdf_w, icdf_h, &a_icdf) : tex_f1(zero4, 2, 2, &a_icdf);

    quad4 meta_h; memset(&meta_h, 0, sizeof(meta_h));
    meta_h.q0.u.x = (unsigned)nwl; meta_h.q0.u.y = (unsigned)(nb * 8);
    meta_h.q1.f.x = nm0; meta_h.q1.f.z = nms;
    quad4* meta_d = up(&meta_h, 1);

    qbnd bnd_h; memset(&bnd_h, 0, sizeof(bnd_h));
    bnd_h.boundary_tex = t_bnd;
    bnd_h.boundary_meta = meta_d;
    bnd_h.optical = up((const quad*)optical, (size_t)nb * 4);
    qbnd* bnd_d = up(&bnd_h, 1);

    qscint sc_h; memset(&sc_h, 0, sizeof(sc_h));
    sc_h.scint_tex = t_icdf;
    sc_h.hd_factor = (unsigned)hd_factor;
    qscint* sc_d = up(&sc_h, 1);

    // the Planck wavelength texture QPlanck builds (qudarap/QPlanck.cc:36-48): sblackbody<double>
    // narrowed to float, 4096 x 1, linear, normalized coordinates, wrap
    std::vector<float> planck_h(4096);
    {
        sblackbody<double> bb(4096, 4096, 6500., 80., 800., 1000);
        const double* v = bb.icdf->cvalues<double>();
        for (int i = 0; i < 4096; i++) planck_h[i] = static_cast<float>(v[i]);
    }
    cudaArray_t a_planck = nullptr;
    qplanck pl_h;
    pl_h.tex = tex_f1(planck_h.data(), 4096, 1, &a_planck);
    qplanck* pl_d = up(&pl_h, 1);

    qbase base_h; base_h.pidx = 0xffffffffffffffffull;
    qbase* base_d = up(&base_h, 1);

    qcerenkov ck_h; memset(&ck_h, 0, sizeof(ck_h));
    ck_h.base = base_d; ck_h.bnd = bnd_d;
    qcerenkov* ck_d = up(&ck_h, 1);

    XORWOW* states = nullptr;
    cudaMalloc(&states, sizeof(XORWOW) * (N > 0 ? N : 1));
    if (N > 0) ref_curand_init_k<<<(unsigned)((N + 127) / 128), 128>>>(seed, (int)N, states);
    qrng<XORWOW> rng_h;
    rng_h.seed = seed; rng_h.offset = 0; rng_h.skipahead_event_offset = skip; rng_h.uploaded_states = states;
    qrng<XORWOW>* rng_d = up(&rng_h, 1);

    sevent ev_h; memset(&ev_h, 0, sizeof(ev_h));
    ev_h.max_bounce = max_bounce;
    ev_h.max_seq = 1;
    ev_h.index = event_index;
    ev_h.num_seed = (size_t)N;
    ev_h.num_photon = (size_t)N;
    ev_h.num_genstep = (size_t)G;
    ev_h.genstep = up((const quad6*)gs, (size_t)G);
    ev_h.seed = up(seed_h.data(), (size_t)N);
    cudaMalloc(&ev_h.photon, sizeof(sphoton) * (N > 0 ? N : 1));
    // input photons: generate_photon copies evt->photon[photon_id] (qudarap/qsim.h:2557), as QEvt
    // uploads them before the launch (qudarap/QEvt.cc:540-560)
    cudaMemset(ev_h.photon, 0, sizeof(sphoton) * (N > 0 ? N : 1));
    if (input_photon && num_input > 0 && N > 0)
        cudaMemcpy(ev_h.photon, input_photon, sizeof(sphoton) * (size_t)(num_input < N ? num_input : N), cudaMemcpyHostToDevice);
    cudaMalloc(&ev_h.seq, sizeof(sseq) * (N > 0 ? N : 1));
    cudaMemset(ev_h.seq, 0, sizeof(sseq) * (N > 0 ? N : 1));
    const size_t nrec = record_out && N > 0 ? (size_t)N * (size_t)max_record : 0;
    if (nrec) {
        ev_h.max_record = max_record;
        ev_h.max_prd = max_record;
        cudaMalloc(&ev_h.record, sizeof(sphoton) * nrec);
        cudaMalloc(&ev_h.prd, sizeof(quad2) * nrec);
        cudaMemset(ev_h.record, 0, sizeof(sphoton) * nrec);
        cudaMemset(ev_h.prd, 0, sizeof(quad2) * nrec);
    }
    sevent* ev_d = up(&ev_h, 1);

    qsim sim_h; memset(&sim_h, 0, sizeof(sim_h));
    sim_h.base = base_d; sim_h.evt = ev_d; sim_h.rng = rng_d; sim_h.bnd = bnd_d;
    sim_h.cerenkov = ck_d; sim_h.scint = sc_d; sim_h.planck = pl_d;
    qsim* sim_d = up(&sim_h, 1);

    if (N > 0) ref_simulate_k<<<(unsigned)((N + 127) / 128), 128>>>(sim_d, ev_d, S, tmin, tmin0, eps0mask, max_time);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && N > 0) {
        cudaMemcpy(photon_out, ev_h.photon, sizeof(sphoton) * N, cudaMemcpyDeviceToHost);
        cudaMemcpy(seq_out, ev_h.seq, sizeof(sseq) * N, cudaMemcpyDeviceToHost);
        if (nrec) {
            cudaMemcpy(record_out, ev_h.record, sizeof(sphoton) * nrec, cudaMemcpyDeviceToHost);
            cudaMemcpy(prd_out, ev_h.prd, sizeof(quad2) * nrec, cudaMemcpyDeviceToHost);
        }
    }
    if (nrec) { cudaFree(ev_h.record); cudaFree(ev_h.prd); }
    cudaDestroyTextureObject(t_bnd); cudaDestroyTextureObject(t_icdf); cudaDestroyTextureObject(pl_h.tex);
    cudaFreeArray(a_bnd); cudaFreeArray(a_icdf); cudaFreeArray(a_planck); cudaFree(pl_d);
    cudaFree((void*)S.node); if (S.plan) cudaFree((void*)S.plan); cudaFree((void*)S.itra); cudaFree((void*)S.inst_inv); cudaFree((void*)S.pair_inst);
    cudaFree((void*)S.pair_node); cudaFree((void*)S.pair_gpbd); cudaFree((void*)S.pair_iiid);
    cudaFree(meta_d); cudaFree(bnd_h.optical); cudaFree(bnd_d); cudaFree(sc_d); cudaFree(base_d); cudaFree(ck_d);
    cudaFree(states); cudaFree(rng_d); cudaFree(ev_h.genstep); cudaFree(ev_h.seed); cudaFree(ev_h.photon);
    cudaFree(ev_h.seq); cudaFree(ev_d); cudaFree(sim_d);
    return e == cudaSuccess ? 0 : -2;
}

extern "C" int ref_scan_run(const float* node, int nn, const float* itra, int nt, const float* plan, int npl, int root, float tmin,
                            const float* rays, long long n, float* out)
{
    const CSGNode* dn = up((const CSGNode*)node, (size_t)nn);
    const qat4* dt = up((const qat4*)itra, (size_t)nt);
    const float4* dp = up((const float4*)plan, (size_t)npl);
    float* dr = up(rays, (size_t)(6 * n));
    float4* dout = nullptr;
    cudaMalloc(&dout, sizeof(float4) * (n > 0 ? n : 1));
    if (n > 0) ref_scan_k<<<(unsigned)((n + 127) / 128), 128>>>(dn + root, dp, dt, tmin, dr, n, dout);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && n > 0) cudaMemcpy(out, dout, sizeof(float4) * n, cudaMemcpyDeviceToHost);
    cudaFree((void*)dn); cudaFree((void*)dt); cudaFree((void*)dp); cudaFree(dr); cudaFree(dout);
    return e == cudaSuccess ? 0 : -2;
}
