// ref_csg_scan.cc : TEST INFRASTRUCTURE ONLY — the reference's CSG intersector run on the CPU.
//
// Compiled by oracle/Makefile (target `ref`) with g++ against the unmodified reference headers
// where they lie in the reference checkout (CSG/csg_intersect_{tree,node,leaf*}.h,
// sysrap/{scuda,squad,sqat4}.h, CSG/CSGNode.h); the output is oracle/_ref/libref_csg.so.
// This mirrors the reference's own non-OptiX scan harness CSGParams::intersect
// (CSG/CSGParams.h:72-95) over SoA rays, with std::thread over the host cores.
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>
#include "scuda.h"
#include "squad.h"
#include "sqat4.h"
#include "CSGNode.h"
#include "csg_intersect_leaf.h"
#include "csg_intersect_node.h"
#include "csg_intersect_tree.h"

extern "C" int ref_csg_scan(const float* node, const float* itra, const float* plan, int root, float tmin, const float* rays,
                            long long n, float* out, int nthread)
{
    const CSGNode* nd = reinterpret_cast<const CSGNode*>(node) + root;
    const qat4* it = reinterpret_cast<const qat4*>(itra);
    const float4* pl = reinterpret_cast<const float4*>(plan);
    if (nthread < 1) nthread = 1;
    auto work = [&](long long a, long long b) {
        for (long long i = a; i < b; i++) {
            float3 o = make_float3(rays[i], rays[n + i], rays[2 * n + i]);
            float3 d = make_float3(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]);
            float4 is = make_float4(0.f, 0.f, 0.f, 0.f);
            bool v = intersect_prim(is, nd, pl, it, tmin, o, d, false);
            out[4 * i + 0] = v ? is.x : 0.f;
            out[4 * i + 1] = v ? is.y : 0.f;
            out[4 * i + 2] = v ? is.z : 0.f;
            out[4 * i + 3] = v ? is.w : 0.f;
        }
    };
    std::vector<std::thread> th;
    long long chunk = (n + nthread - 1) / nthread;
    for (int t = 0; t < nthread; t++) {
        long long a = t * chunk, b = a + chunk < n ? a + chunk : n;
        if (a < b) th.emplace_back(work, a, b);
    }
    for (auto& t : th) t.join();
    return 0;
}

// The slab, infinite-cylinder and disc leaves are compiled by the reference only under
// CSG_EXTRA (CSG/csg_intersect_leaf.h:100-108,224-232), where the plane leaf beside them does
// not compile; their own headers are included here and called directly, one leaf per scan.
#include "csg_intersect_leaf_slab.h"
#include "csg_intersect_leaf_infcylinder.h"
#include "csg_intersect_leaf_disc.h"

extern "C" int ref_leaf_extra_scan(int typecode, const float* q0q1, float tmin, const float* rays, long long n, float* out)
{
    quad q0, q1;
    std::memcpy(&q0, q0q1, 16);
    std::memcpy(&q1, q0q1 + 4, 16);
    for (long long i = 0; i < n; i++) {
        float3 o = make_float3(rays[i], rays[n + i], rays[2 * n + i]);
        float3 d = make_float3(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]);
        float4 is = make_float4(0.f, 0.f, 0.f, 0.f);
        bool v = false;
        switch (typecode) {
            case CSG_SLAB: intersect_leaf_slab(v, is, q0, q1, tmin, o, d); break;
            case CSG_INFCYLINDER: intersect_leaf_infcylinder(v, is, q0, q1, tmin, o, d); break;
            case CSG_DISC: intersect_leaf_disc(v, is, q0, q1, tmin, o, d); break;
            default: return -1;
        }
        out[4 * i + 0] = v ? is.x : 0.f;
        out[4 * i + 1] = v ? is.y : 0.f;
        out[4 * i + 2] = v ? is.z : 0.f;
        out[4 * i + 3] = v ? is.w : 0.f;
    }
    return 0;
}
