// phx_bvh.h : host-side 4-wide BVH builder interface (see phx_bvh.cc)
#pragma once
#include <vector>
#include "phx_pod.h"

struct PhxLeafInput {
    float bbox[6];      // prim box in the instance (object) frame : mn.xyz, mx.xyz
    float xform[16];    // instance transform, row-vector convention (rows q0..q3), object -> world
    float sphere[4];    // world-space bounding sphere of the leaf: centre xyz, radius
    double wbox[6];     // a world box from the prim's CSG tree (lo xyz, hi xyz), when has_wbox
    int has_wbox;       //   the leaf's box is the overlap of this and the prim box's corner box
    phx_leaf leaf;
};

struct PhxBvh4Result {
    std::vector<phx_bvh4_node> nodes;
    std::vector<phx_leaf> leaves;   // reordered to match the leaf ranges in nodes
    std::vector<phx_leaf> globals;  // leaves tested by every ray before the traversal (input order)
    std::vector<float> leaf_sphere, global_sphere;   // 4 floats per leaf, same orders
    float cull[4] = { 0.f, 0.f, 0.f, 0.f };   // empty ball of the BVH leaves: centre xyz, radius^2 (0: none)
    int leaf_count = 0;
    int max_depth = 0;
};

// Leaves whose box surface area is at least global_frac of the scene box's (at most max_global of
// them, the largest) are kept out of the hierarchy: every ray would enter their boxes anyway, so
// they are tested first, coherently across a warp, and their hit shortens the traversal.
int phx_build_bvh4(const std::vector<PhxLeafInput>& in, PhxBvh4Result& out, double global_frac = 0.25, int max_global = 16);
