// Device data layouts shared by the host builder and the CUDA kernels.
#pragma once
#include <stdint.h>

namespace ilm {

// Binary node, byte-compatible with LinearBVHNode (accelerators/bvh.rs:665-673)
// at its intended 32-byte size: bounds, offset (leaf: first primitive record;
// interior: second child), n_prims (0 = interior), split axis.
struct BinNode {
    float bmin[3], bmax[3];
    int32_t offset;
    uint16_t n_prims;
    uint8_t axis;
    uint8_t pad;
};
static_assert(sizeof(BinNode) == 32, "BinNode must be 32 bytes");

// Primitive record, 48 bytes = 3 x 16-byte loads, stored in traversal order.
// Triangle: three world-space vertices.  Sphere: index into the sphere table.
struct PrimRec {
    float p0[3]; uint32_t prim;    // original primitive id
    float p1[3]; uint32_t flags;   // kPrimDegenerate | kPrimSphere
    float p2[3]; uint32_t aux;     // sphere index
};
static_assert(sizeof(PrimRec) == 48, "PrimRec must be 48 bytes");
enum : uint32_t {
    // (p2-p0)x(p1-p0) has zero squared length: Triangle::intersect rejects it
    // (shapes/triangle.rs:281-289); Triangle::intersect_p does not.
    kPrimDegenerate = 1u,
    kPrimSphere = 2u,
};

// Sphere record (shapes/sphere.rs:15-75) with Sphere::new's derived values.
// A sphere or another quadric (kind).  radius and z_min / z_max bound the
// object box for every kind; a disk keeps its height in z_min (= z_max) and
// its inner radius in theta_min, a cone its height in z_max (z_min = 0), a
// hyperboloid its largest radius in radius and p1, p2, ah, ch in aux.
// A curve segment (kQuadricCurve) keeps its control points, widths, u range
// and ribbon normals in aux and its type in theta_min (shapes.cuh).
enum : int32_t {
    kQuadricSphere = 0, kQuadricDisk = 1, kQuadricCylinder = 2, kQuadricCone = 3,
    kQuadricParaboloid = 4, kQuadricHyperboloid = 5, kQuadricCurve = 6
};
struct SphereRec {
    float o2w[16];
    float w2o[16];
    float radius, z_min, z_max, theta_min, theta_max, phi_max;
    int32_t reverse;
    int32_t kind;
    float aux[24];
};
static_assert(sizeof(SphereRec) == 256, "SphereRec must be 256 bytes");

// Compressed wide node.  Child boxes are quantised to 8 bits per plane on a
// per-node grid: plane = fma(2^23 + q, 2^(e-127), origin), where origin is the
// grid start biased by -2^23 * 2^(e-127) (so the kernel forms 2^23 + q with
// one byte permute and subtracts nothing), with q rounded outward at build
// time so every dequantised box contains its child's exact box.
//   word 0: origin x, y, z (float), packed = ex | ey<<8 | ez<<16 | imask<<24
//   word 1: child_base, prim_base, meta[W] ...
//   then qlo_x[W], qlo_y[W], qlo_z[W], qhi_x[W], qhi_y[W], qhi_z[W] (bytes)
// meta byte per child: 0 = empty slot.  Interior (imask bit set): low 5 bits
// = offset from child_base (interior children are contiguous).  Leaf: bits
// 5..7 = primitive count (1..4), low 5 bits = offset from prim_base.
template <int W> struct WideNode;

template <> struct WideNode<8> {           // 80 bytes
    float origin[3];
    uint32_t packed;
    uint32_t child_base, prim_base;
    uint8_t meta[8];
    uint8_t qlo[3][8];
    uint8_t qhi[3][8];
};
static_assert(sizeof(WideNode<8>) == 80, "WideNode<8> must be 80 bytes");

template <> struct WideNode<4> {           // 64 bytes
    float origin[3];
    uint32_t packed;
    uint32_t child_base, prim_base;
    uint8_t meta[4];
    uint8_t qlo_x[4];
    uint8_t qlo_y[4], qlo_z[4], qhi_x[4], qhi_y[4];
    uint8_t qhi_z[4];
    uint32_t pad[3];
};
static_assert(sizeof(WideNode<4>) == 64, "WideNode<4> must be 64 bytes");

// kd-tree node, the 8-byte KdAccelNode (accelerators/kdtreeaccel.rs:470-545):
//   word : interior -> split position (float bits); leaf of one primitive ->
//          its id; leaf of several -> first slot of its run in the index list
//   flags: low 2 bits = split axis (0..2) or 3 for a leaf; the upper 30 bits =
//          the above child's node index (interior) or the primitive count (leaf)
// The below child of an interior node is the next node.
struct KdNode {
    uint32_t word;
    uint32_t flags;
};
static_assert(sizeof(KdNode) == 8, "KdNode must be 8 bytes");
constexpr uint32_t kKdLeaf = 3u;
// Layout code of a kd-tree accel (the BVH layouts are their widths 2, 4, 8).
constexpr int kLayoutKdTree = 1;
// Deepest kd-tree accepted: the traversal keeps at most one deferred node per
// level on its 64-entry stack.
constexpr int kKdMaxDepth = 64;

// Stack / entry encoding used by the wide traversal kernels.
constexpr uint32_t kLeafFlag = 0x80000000u;
constexpr uint32_t kMaxLeafPrims = 4;     // per wide-node child slot
constexpr uint32_t kMaxPrimsPerNode = 32; // 5-bit leaf offsets

// Per-ray status written in place of a primitive id when traversal had to give
// up (stack overflow or iteration cap); the context's error word is set too.
constexpr uint32_t kHitTraversalError = 0xFFFFFFFEu;

// Device error word bits.
enum : uint32_t { kErrStackOverflow = 1u, kErrIterationCap = 2u };

}  // namespace ilm
