// phx_bvh.h : host-side 4-wide BVH builder interface (see phx_bvh.cc)
#pragma once
#include <vector>
#include "phx_pod.h"

struct PhxLeafInput {
    float bbox[6];      // prim box in the instance (object) frame : mn.xyz, mx.xyz
    float xform[16];    // instance transform, row-vector convention (rows q0..q3), object -> world
    phx_leaf leaf;
};

struct PhxBvh4Result {
    std::vector<phx_bvh4_node> nodes;
    std::vector<phx_leaf> leaves;   // reordered to match the leaf ranges in nodes
    int leaf_count = 0;
    int max_depth = 0;
};

int phx_build_bvh4(const std::vector<PhxLeafInput>& in, PhxBvh4Result& out);
