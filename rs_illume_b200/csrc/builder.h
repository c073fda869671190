// Host-side acceleration-structure construction.
#pragma once
#include <stdint.h>
#include <string>
#include <vector>

#include "layout.h"

namespace ilm {

struct Box {
    float mn[3], mx[3];
};
Box empty_box();                  // Bounds3::default (min = MAX, max = -MAX)

struct BuildPrim {
    uint32_t prim;                // primitive id
    Box bounds;
    float centroid[3];
};

// SAH binary build with 12 buckets and BVHAccel's leaf rule (bvh.rs:95-247,
// with the centroid-bound, bucket-index and argmin repairs), flattened
// depth-first as flatten_bvh_tree (bvh.rs:504-537).  On return `prims` is in
// leaf order (the order of BVHAccel's ordered_prims) and leaf offsets index it.
// Subtrees are built on up to `threads` host threads; the result does not
// depend on the thread count.
void sah_build(std::vector<BuildPrim>& prims, int max_prims_in_node, int threads,
               std::vector<BinNode>& nodes);

// Collapses the binary tree into W-wide compressed nodes (W = 4 or 8).
// `prims` is the leaf-ordered list from sah_build (for per-primitive boxes).
// Outputs the node array (raw bytes, node 0 = root) and, for each primitive
// record slot of the wide layout, the index into `prims` it holds.
void collapse_wide(const std::vector<BinNode>& bin, const std::vector<BuildPrim>& prims, int width,
                   std::vector<uint8_t>& node_bytes, uint32_t* n_nodes,
                   std::vector<uint32_t>& record_order);

// Triangle bound as Triangle::world_bound (shapes/triangle.rs:126-132).
Box triangle_bound(const float* p0, const float* p1, const float* p2);
// Centroid as Bounds3::centroid (geometry/bounds3.rs:238-242).
void box_centroid(const Box& b, float c[3]);
// (p2-p0)x(p1-p0) evaluated as Vector3::cross (f64, rounded) has zero
// squared length (shapes/triangle.rs:281-289).
bool triangle_degenerate(const float* p0, const float* p1, const float* p2);
// Sphere::new derived values and world bound (shapes/sphere.rs:50-75;
// geometry/bounds3.rs:320-356).
struct SphereInput {
    float o2w[16], w2o[16];
    float radius, z_min, z_max, phi_max_deg;
    int32_t reverse;
    int32_t kind = 0;              // kQuadric*
    float height = 0.0f, inner_radius = 0.0f;
    float p1[3] = {0, 0, 0}, p2[3] = {0, 0, 0};
};
// False when a hyperboloid's implicit coefficients do not come out finite.
bool make_sphere(const SphereInput& in, SphereRec* out);
SphereRec make_sphere(const SphereInput& in);
// Curve::new for one segment (shapes/curve.rs:30-91): the segment's control
// points blossomed from the curve's for [u_min, u_max], the ribbon normals'
// angle; type 0 flat, 1 cylinder, 2 ribbon.
struct CurveInput {
    float o2w[16], w2o[16];
    float cp[12];
    float width[2];
    float n[6];
    float u_min, u_max;
    int32_t type;
    int32_t reverse;
};
SphereRec make_curve(const CurveInput& in);
// World bound of a quadric or curve record (geometry/bounds3.rs:320-356 on
// the object box; a curve's box is its segment's control points padded by
// half the larger end width, curve.rs:255-268).
Box sphere_bound(const SphereRec& s);

// One shape list entry: a triangle mesh (world-space vertices) or a sphere set.
struct MeshView {
    bool is_spheres;
    const float* xyz;
    const uint32_t* idx;
    const SphereRec* spheres;
    uint32_t n_prims;
};

// Everything the device needs for one acceleration structure, built on the
// host: the SAH binary tree, the layout for `width`, and primitive records in
// traversal order.
struct HostLayout {
    int width = 8;                      // 2, 4, 8, or kLayoutKdTree
    uint32_t n_prims = 0;
    std::vector<BinNode> bin_nodes;
    std::vector<uint32_t> prim_order;   // BVHAccel ordered_prims as primitive ids
    std::vector<uint8_t> node_bytes;
    uint32_t n_nodes = 0;
    std::vector<PrimRec> records;
    std::vector<SphereRec> spheres;
    float bound[6];
    std::vector<uint32_t> kd_index;     // kd-tree: leaf primitive runs (records in id order)
    int kd_max_depth = 0;               // kd-tree: the depth limit used
};

// KdTreeAccel::new parameters (accelerators/kdtreeaccel.rs:25-32).
struct KdParams {
    int isect_cost = 80;
    int traversal_cost = 1;
    float empty_bonus = 0.5f;
    uint32_t max_prims = 1;
    int max_depth = -1;                 // <= 0: round(8 + 1.3 log2(N))
};

// KdTreeAccel::build_tree (kdtreeaccel.rs:90-244) over the primitives' world
// bounds: SAH over the sorted bound edges of one axis at a time (the largest
// extent first, then the others when no edge lies strictly inside the node),
// leaves below max_prims primitives, at max_depth, after three bad refines,
// or when the best split costs over four times the leaf with fewer than 16
// primitives.  Nodes come out depth first (below child next, as the
// reference allocates them); subtrees near the root are built on up to
// `threads` host threads into separate arrays and spliced in that order, so
// the result does not depend on the thread count.  Edges at equal position
// and type are ordered by primitive id.
void kd_build(const std::vector<Box>& bounds, const Box& root, const KdParams& p, int threads,
              std::vector<KdNode>& nodes, std::vector<uint32_t>& index);
// The default depth limit round(8 + 1.3 log2(n)) (kdtreeaccel.rs:34-36).
int kd_default_depth(uint64_t n);

// KdTreeAccel::new followed by the device layout: kd nodes in node_bytes,
// leaf runs in kd_index, one primitive record per primitive id.
std::string build_kd_layout(const std::vector<MeshView>& meshes, const KdParams& p, int threads, HostLayout& out);

// Loop subdivision (shapes/loop_subdiv.rs, pbrt-v3's LoopSubdivide): `levels`
// refinements of the triangle mesh (p: 3 floats per vertex, idx: 3 per face),
// vertices moved to the limit surface, limit normals (unnormalised) per vertex.
// Throws std::runtime_error on an invalid or non-manifold mesh.
void loop_subdivide(const std::vector<float>& p, const std::vector<uint32_t>& idx, int levels,
                    std::vector<float>& p_out, std::vector<uint32_t>& idx_out, std::vector<float>& n_out);

// BVHAccel::new (bvh.rs:32-93) followed by the device layout.  Returns an
// empty string on success or a description of the failure.
std::string build_layout(const std::vector<MeshView>& meshes, int width, int max_prims_in_node, int threads,
                         HostLayout& out);

}  // namespace ilm
