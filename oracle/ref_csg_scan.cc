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

extern "C" int ref_csg_scan(const float* node, const float* itra, int root, float tmin, const float* rays,
                            long long n, float* out, int nthread)
{
    const CSGNode* nd = reinterpret_cast<const CSGNode*>(node) + root;
    const qat4* it = reinterpret_cast<const qat4*>(itra);
    if (nthread < 1) nthread = 1;
    auto work = [&](long long a, long long b) {
        for (long long i = a; i < b; i++) {
            float3 o = make_float3(rays[i], rays[n + i], rays[2 * n + i]);
            float3 d = make_float3(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]);
            float4 is = make_float4(0.f, 0.f, 0.f, 0.f);
            bool v = intersect_prim(is, nd, nullptr, it, tmin, o, d, false);
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
