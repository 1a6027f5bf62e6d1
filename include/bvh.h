// bvh.h -- linear BVH over a triangle soup.
//
// Drop-in for the reference header include/bvh.h:1-26.  BvhNode keeps the
// reference's 40-byte layout; the node array is in breadth-first order with
// the root at index 0, leaves have triCount > 0 and left = right = -1,
// internal nodes have triCount = 0 and firstTri = -1.
#pragma once

#include <cstdint>
#include <vector>

#include "scene.h"

struct BvhNode
{
    float bbMin[3];
    float bbMax[3];
    int left;      // -1 for a leaf
    int right;     // -1 for a leaf
    int firstTri;  // leaf: first triangle after BuildBVH's reorder; internal: -1
    int triCount;  // 0 = internal, > 0 = leaf
};
static_assert(sizeof(BvhNode) == 40, "BvhNode must stay 40 bytes (reference ABI)");

struct Bvh
{
    std::vector<BvhNode> nodes;
    int rootIdx = 0;
};

// Builds the BVH on the GPU (Morton codes, radix sort, radix-tree split,
// bottom-up refit) and reorders scene.triangles in place so each leaf covers
// a contiguous range.  The node array is bit-identical to the reference's
// CPU build (src/bvh.cpp:164-211); see lumina.h for the C entry point.
void BuildBVH(Scene& scene, Bvh& out);
