// Host-side SAH build and wide-node collapse.  Compiled with
// -ffp-contract=off so every float expression rounds as in the reference
// (Rust never fuses multiply-add); the binary tree therefore matches
// BVHAccel's node for node.
#include "builder.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <thread>

namespace ilm {

namespace {

inline float fmin_rs(float a, float b) { return a < b ? a : b; }   // Point3::min (point3.rs:70-79)
inline float fmax_rs(float a, float b) { return a > b ? a : b; }   // Point3::max (point3.rs:83-92)

inline void box_union(Box& a, const Box& b) {
    for (int k = 0; k < 3; ++k) {
        a.mn[k] = fmin_rs(a.mn[k], b.mn[k]);
        a.mx[k] = fmax_rs(a.mx[k], b.mx[k]);
    }
}
inline void box_union_pt(Box& a, const float* p) {
    for (int k = 0; k < 3; ++k) {
        a.mn[k] = fmin_rs(a.mn[k], p[k]);
        a.mx[k] = fmax_rs(a.mx[k], p[k]);
    }
}
// Bounding3::surface_area (bounds3.rs:59-62)
inline float surface_area(const Box& b) {
    float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
    return 2.0f * (dx * dy + dx * dz + dy * dz);
}
// Bounding3::maximum_extent (bounds3.rs:53-56)
inline int maximum_extent(const Box& b) {
    float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
    if (dx > dy && dx > dz) return 0;
    if (dy > dz) return 1;
    return 2;
}
// Bounds3::offset along one axis (bounds3.rs:178-193)
inline float offset_axis(const Box& b, const float* p, int a) {
    float o = p[a] - b.mn[a];
    if (b.mx[a] > b.mn[a]) o /= b.mx[a] - b.mn[a];
    return o;
}
// SAH bucket with the cast applied after the multiply (pbrt-v3 semantics;
// bvh.rs:176 casts first, which only ever yields bucket 0 or 12).
inline int bucket_of(const Box& cb, const float* c, int a) {
    int b = (int)(12.0f * offset_axis(cb, c, a));
    return b == 12 ? 11 : b;
}

struct TreeNode {
    Box bounds;
    int32_t child[2];
    uint32_t start, count;   // leaf range in the (partitioned) primitive array
    uint8_t axis;
};

class SahBuilder {
public:
    SahBuilder(std::vector<BuildPrim>& p, int max_prims, int threads)
        : p_(p), max_prims_(max_prims), nodes_(2 * p.size() + 1) {
        spawn_depth_ = 0;
        while ((1 << spawn_depth_) < threads && spawn_depth_ < 6) ++spawn_depth_;
    }
    int32_t run() { return build(0, (uint32_t)p_.size(), 0); }
    const std::vector<TreeNode>& nodes() const { return nodes_; }

private:
    int32_t alloc() {
        uint32_t i = next_.fetch_add(1);
        if (i >= nodes_.size()) throw std::runtime_error("SAH builder node pool exhausted");
        return (int32_t)i;
    }
    int32_t leaf(uint32_t start, uint32_t end, const Box& b) {
        int32_t i = alloc();
        TreeNode& n = nodes_[i];
        n.bounds = b;
        n.child[0] = n.child[1] = -1;
        n.start = start;
        n.count = end - start;
        n.axis = 0;
        return i;
    }
    // recursive_build (bvh.rs:95-247), SAH split method.
    int32_t build(uint32_t start, uint32_t end, int depth) {
        Box bounds = empty_box();
        for (uint32_t i = start; i < end; ++i) box_union(bounds, p_[i].bounds);
        uint32_t n = end - start;
        if (n == 1) return leaf(start, end, bounds);
        // centroid bounds: union of centroids (bvh.rs:125-128 unions primitive
        // bounds into an immutable binding; the pbrt intent is centroids)
        Box cb = empty_box();
        for (uint32_t i = start; i < end; ++i) box_union_pt(cb, p_[i].centroid);
        int dim = maximum_extent(cb);
        uint32_t mid = (start + end) / 2;
        if (cb.mx[dim] == cb.mn[dim]) return leaf(start, end, bounds);   // bvh.rs:133-141
        if (n <= 2) {
            // equal-count split of two: the reference's partial_sort pass swaps
            // the pair iff c[1] < c[0] (slice_extension.rs:45-72)
            if (p_[start + 1].centroid[dim] < p_[start].centroid[dim]) std::swap(p_[start], p_[start + 1]);
        } else {
            uint32_t count[12] = {0};
            Box bb[12];
            for (int b = 0; b < 12; ++b) bb[b] = empty_box();
            for (uint32_t i = start; i < end; ++i) {
                int b = bucket_of(cb, p_[i].centroid, dim);
                count[b] += 1;
                box_union(bb[b], p_[i].bounds);
            }
            float cost[11];
            for (int i = 0; i < 11; ++i) {
                Box b0 = empty_box(), b1 = empty_box();
                uint32_t c0 = 0, c1 = 0;
                for (int j = 0; j <= i; ++j) { box_union(b0, bb[j]); c0 += count[j]; }
                for (int j = i + 1; j < 12; ++j) { box_union(b1, bb[j]); c1 += count[j]; }
                cost[i] = 1.0f + ((float)c0 * surface_area(b0) + (float)c1 * surface_area(b1)) /
                                     surface_area(bounds);
            }
            float min_cost = cost[0];
            int split = 0;
            for (int i = 1; i < 11; ++i)
                if (cost[i] < min_cost) { min_cost = cost[i]; split = i; }   // first minimum wins
            float leaf_cost = (float)n;
            if (n > (uint32_t)max_prims_ || min_cost < leaf_cost) {
                // SliceExtension::partition (slice_extension.rs:20-43): find the
                // first element failing the predicate, then swap later passing
                // elements down to it.
                uint32_t first = end;
                for (uint32_t i = start; i < end; ++i)
                    if (bucket_of(cb, p_[i].centroid, dim) > split) { first = i; break; }
                if (first != end)
                    for (uint32_t i = first; i < end; ++i)
                        if (bucket_of(cb, p_[i].centroid, dim) <= split) std::swap(p_[i], p_[first++]);
                mid = first;
            } else {
                return leaf(start, end, bounds);
            }
        }
        int32_t self = alloc();
        int32_t c0, c1;
        if (depth < spawn_depth_ && n > 4096) {
            std::thread t([&] { c0 = build(start, mid, depth + 1); });
            c1 = build(mid, end, depth + 1);
            t.join();
        } else {
            c0 = build(start, mid, depth + 1);
            c1 = build(mid, end, depth + 1);
        }
        // init_interior (bvh.rs:707-719)
        TreeNode& nd = nodes_[self];
        nd.bounds = nodes_[c0].bounds;
        box_union(nd.bounds, nodes_[c1].bounds);
        nd.child[0] = c0;
        nd.child[1] = c1;
        nd.start = 0;
        nd.count = 0;
        nd.axis = (uint8_t)dim;
        return self;
    }

    std::vector<BuildPrim>& p_;
    int max_prims_;
    int spawn_depth_;
    std::vector<TreeNode> nodes_;
    std::atomic<uint32_t> next_{0};
};

// flatten_bvh_tree (bvh.rs:504-537)
uint32_t flatten(const std::vector<TreeNode>& t, int32_t node, std::vector<BinNode>& out) {
    uint32_t my = (uint32_t)out.size();
    out.emplace_back();
    const TreeNode& n = t[node];
    BinNode b;
    std::memset(&b, 0, sizeof b);
    for (int k = 0; k < 3; ++k) { b.bmin[k] = n.bounds.mn[k]; b.bmax[k] = n.bounds.mx[k]; }
    if (n.child[0] < 0) {
        if (n.count >= 65536) throw std::runtime_error("leaf with >= 65536 primitives");
        b.offset = (int32_t)n.start;
        b.n_prims = (uint16_t)n.count;
        out[my] = b;
    } else {
        flatten(t, n.child[0], out);
        b.offset = (int32_t)flatten(t, n.child[1], out);
        b.axis = n.axis;
        out[my] = b;
    }
    return my;
}

}  // namespace

Box empty_box() {
    Box b;
    for (int k = 0; k < 3; ++k) {
        b.mn[k] = std::numeric_limits<float>::max();
        b.mx[k] = -std::numeric_limits<float>::max();
    }
    return b;
}

Box triangle_bound(const float* p0, const float* p1, const float* p2) {
    Box b;
    for (int k = 0; k < 3; ++k) {     // Bounds3f::new(p0, p1) then union p2
        b.mn[k] = fmin_rs(p0[k], p1[k]);
        b.mx[k] = fmax_rs(p0[k], p1[k]);
    }
    box_union_pt(b, p2);
    return b;
}

void box_centroid(const Box& b, float c[3]) {
    for (int k = 0; k < 3; ++k) c[k] = b.mn[k] * 0.5f + b.mx[k] * 0.5f;
}

bool triangle_degenerate(const float* p0, const float* p1, const float* p2) {
    float a[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    float b[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    double ax = a[0], ay = a[1], az = a[2], bx = b[0], by = b[1], bz = b[2];
    float nx = (float)((ay * bz) - (az * by));
    float ny = (float)((az * bx) - (ax * bz));
    float nz = (float)((ax * by) - (ay * bx));
    return nx * nx + ny * ny + nz * nz == 0.0f;
}

SphereRec make_sphere(const SphereInput& in) {
    SphereRec s;
    make_sphere(in, &s);
    return s;
}

bool make_sphere(const SphereInput& in, SphereRec* out) {
    SphereRec& s = *out;
    std::memset(&s, 0, sizeof s);
    std::memcpy(s.o2w, in.o2w, sizeof s.o2w);
    std::memcpy(s.w2o, in.w2o, sizeof s.w2o);
    auto clamp = [](float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); };
    float mn = std::fmin(in.z_min, in.z_max), mx = std::fmax(in.z_min, in.z_max);
    const float kPi = 3.14159265358979323846f;
    s.radius = in.radius;
    s.phi_max = (kPi / 180.0f) * clamp(in.phi_max_deg, 0.0f, 360.0f);
    s.reverse = in.reverse;
    s.kind = in.kind;
    switch (in.kind) {
        case kQuadricDisk:   // Disk::new (disk.rs:27-47)
            s.z_min = s.z_max = in.height;
            s.theta_min = in.inner_radius;
            break;
        case kQuadricCylinder:   // Cylinder::new (cylinder.rs:26-46), z range ordered and phi in radians as pbrt
            s.z_min = mn;
            s.z_max = mx;
            break;
        case kQuadricCone:   // Cone::new (cone.rs:26-41)
            s.z_min = 0.0f;
            s.z_max = in.height;
            break;
        case kQuadricParaboloid:   // Paraboloid::new (paraboloid.rs:26-47), z range ordered as pbrt
            s.z_min = mn;
            s.z_max = mx;
            break;
        case kQuadricHyperboloid: {   // Hyperboloid::new (hyperboloid.rs:31-77)
            float p1[3] = {in.p1[0], in.p1[1], in.p1[2]}, p2[3] = {in.p2[0], in.p2[1], in.p2[2]};
            float r1 = std::sqrt(p1[0] * p1[0] + p1[1] * p1[1]);
            float r2 = std::sqrt(p2[0] * p2[0] + p2[1] * p2[1]);
            s.radius = r1 > r2 ? r1 : r2;
            s.z_min = std::fmin(p1[2], p2[2]);
            s.z_max = std::fmax(p1[2], p2[2]);
            // the implicit coefficients need p2.z != 0: swap when it is 0
            // (hyperboloid.rs:42-47 swaps on the opposite test; pbrt's rule)
            if (p2[2] == 0.0f) for (int k = 0; k < 3; ++k) std::swap(p1[k], p2[k]);
            float pp[3] = {p1[0], p1[1], p1[2]};
            float ah = INFINITY, ch = INFINITY;
            // step pp away from p1 until both coefficients are finite numbers
            // (the reference's loop tests infinities only; pbrt's also NaN)
            for (int it = 0; it < 64 && !(std::isfinite(ah) && std::isfinite(ch)); ++it) {
                for (int k = 0; k < 3; ++k) pp[k] = pp[k] + 2.0f * (p2[k] - p1[k]);
                float xy1 = pp[0] * pp[0] + pp[1] * pp[1];
                float xy2 = p2[0] * p2[0] + p2[1] * p2[1];
                ah = (1.0f / xy1 - (pp[2] * pp[2]) / (xy1 * p2[2] * p2[2])) /
                     (1.0f - (xy2 * pp[2] * pp[2]) / (xy1 * p2[2] * p2[2]));
                ch = (ah * xy2 - 1.0f) / (p2[2] * p2[2]);
            }
            for (int k = 0; k < 3; ++k) { s.aux[k] = p1[k]; s.aux[3 + k] = p2[k]; }
            s.aux[6] = ah;
            s.aux[7] = ch;
            return std::isfinite(ah) && std::isfinite(ch) && s.z_min < s.z_max;
        }
        default:   // Sphere::new (sphere.rs:50-75)
            s.z_min = clamp(mn, -in.radius, in.radius);
            s.z_max = clamp(mx, -in.radius, in.radius);
            s.theta_min = std::acos(clamp(mn / in.radius, -1.0f, 1.0f));
            s.theta_max = std::acos(clamp(mx / in.radius, -1.0f, 1.0f));
    }
    return true;
}

namespace {
// lerp(t, a, b) = a (1 - t) + b t (core/pbrt.rs:41-47)
inline float lerpf(float t, float a, float b) { return a * (1.0f - t) + b * t; }
// blossom_bezier (curve.rs:406-412)
void blossom(const float* p, float u0, float u1, float u2, float* out) {
    float a[3][3], b[2][3];
    for (int k = 0; k < 3; ++k) {
        for (int i = 0; i < 3; ++i) a[i][k] = lerpf(u0, p[3 * i + k], p[3 * (i + 1) + k]);
        for (int i = 0; i < 2; ++i) b[i][k] = lerpf(u1, a[i][k], a[i + 1][k]);
        out[k] = b[0][k] * (1.0f - u2) + b[1][k] * u2;
    }
}
}  // namespace

SphereRec make_curve(const CurveInput& in) {
    SphereRec s;
    std::memset(&s, 0, sizeof s);
    std::memcpy(s.o2w, in.o2w, sizeof s.o2w);
    std::memcpy(s.w2o, in.w2o, sizeof s.w2o);
    s.kind = kQuadricCurve;
    s.theta_min = (float)in.type;
    s.reverse = in.reverse;
    blossom(in.cp, in.u_min, in.u_min, in.u_min, &s.aux[0]);
    blossom(in.cp, in.u_min, in.u_min, in.u_max, &s.aux[3]);
    blossom(in.cp, in.u_min, in.u_max, in.u_max, &s.aux[6]);
    blossom(in.cp, in.u_max, in.u_max, in.u_max, &s.aux[9]);
    s.aux[12] = in.width[0];
    s.aux[13] = in.width[1];
    s.aux[14] = in.u_min;
    s.aux[15] = in.u_max;
    if (in.type == 2) {   // CurveCommon::new with normals (curve.rs:39-52)
        float n[6];
        for (int e = 0; e < 2; ++e) {
            const float* v = in.n + 3 * e;
            float inv = 1.0f / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            for (int k = 0; k < 3; ++k) n[3 * e + k] = v[k] * inv;
        }
        float dot = n[0] * n[3] + n[1] * n[4] + n[2] * n[5];
        float angle = std::acos(dot < 0.0f ? 0.0f : (dot > 1.0f ? 1.0f : dot));
        std::memcpy(&s.aux[16], n, sizeof n);
        s.aux[22] = angle;
        s.aux[23] = 1.0f / std::sin(angle);
    }
    return s;
}

Box sphere_bound(const SphereRec& s) {
    float omn[3] = {-s.radius, -s.radius, s.z_min}, omx[3] = {s.radius, s.radius, s.z_max};
    if (s.kind == kQuadricCurve) {
        const float* c = s.aux;
        for (int k = 0; k < 3; ++k) {
            omn[k] = std::fmin(std::fmin(c[k], c[3 + k]), std::fmin(c[6 + k], c[9 + k]));
            omx[k] = std::fmax(std::fmax(c[k], c[3 + k]), std::fmax(c[6 + k], c[9 + k]));
        }
        float w = std::fmax(lerpf(s.aux[14], s.aux[12], s.aux[13]), lerpf(s.aux[15], s.aux[12], s.aux[13])) * 0.5f;
        for (int k = 0; k < 3; ++k) { omn[k] -= w; omx[k] += w; }
    }
    float bmin[3] = {s.o2w[3], s.o2w[7], s.o2w[11]}, bmax[3] = {s.o2w[3], s.o2w[7], s.o2w[11]};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float a = s.o2w[4 * i + j] * omn[j];
            float b = s.o2w[4 * i + j] * omx[j];
            if (a < b) { bmin[i] += a; bmax[i] += b; } else { bmin[i] += b; bmax[i] += a; }
        }
    Box r;
    for (int k = 0; k < 3; ++k) { r.mn[k] = bmin[k]; r.mx[k] = bmax[k]; }
    return r;
}

void sah_build(std::vector<BuildPrim>& prims, int max_prims_in_node, int threads,
               std::vector<BinNode>& nodes) {
    nodes.clear();
    if (prims.empty()) return;
    SahBuilder b(prims, max_prims_in_node, threads < 1 ? 1 : threads);
    int32_t root = b.run();
    nodes.reserve(2 * prims.size());
    flatten(b.nodes(), root, nodes);
}

// ------------------------------------------------------------------ collapse
namespace {

struct Entry {
    bool interior;      // binary interior node
    uint32_t bin;       // binary node index (interior)
    uint32_t start, count;
    Box box;
};

struct Collapser {
    const std::vector<BinNode>& bin;
    const std::vector<BuildPrim>& prims;
    int W;

    Entry from_bin(uint32_t i) const {
        const BinNode& n = bin[i];
        Entry e;
        e.interior = n.n_prims == 0;
        e.bin = i;
        e.start = e.interior ? 0 : (uint32_t)n.offset;
        e.count = e.interior ? 0 : n.n_prims;
        for (int k = 0; k < 3; ++k) { e.box.mn[k] = n.bmin[k]; e.box.mx[k] = n.bmax[k]; }
        return e;
    }
    Entry range(uint32_t start, uint32_t count) const {
        Entry e;
        e.interior = false;
        e.bin = 0;
        e.start = start;
        e.count = count;
        e.box = empty_box();
        for (uint32_t i = start; i < start + count; ++i) box_union(e.box, prims[i].bounds);
        return e;
    }
    static bool expandable(const Entry& e) { return e.interior || e.count > kMaxLeafPrims; }
    void split(const Entry& e, Entry out[2]) const {
        if (e.interior) {
            out[0] = from_bin(e.bin + 1);
            out[1] = from_bin((uint32_t)bin[e.bin].offset);
        } else {
            uint32_t h = e.count / 2;
            out[0] = range(e.start, h);
            out[1] = range(e.start + h, e.count - h);
        }
    }
    std::vector<Entry> children_of(const Entry& e) const {
        std::vector<Entry> c;
        if (!expandable(e)) { c.push_back(e); return c; }
        Entry s[2];
        split(e, s);
        c.push_back(s[0]);
        c.push_back(s[1]);
        while ((int)c.size() < W) {
            int best = -1;
            float best_sa = -1.0f;
            for (size_t i = 0; i < c.size(); ++i)
                if (expandable(c[i])) {
                    float sa = surface_area(c[i].box);
                    if (sa > best_sa) { best_sa = sa; best = (int)i; }
                }
            if (best < 0) break;
            split(c[best], s);
            c[best] = s[0];
            c.insert(c.begin() + best + 1, s[1]);
        }
        return c;
    }
};

// Dequantised plane q of an axis with scale s and biased origin b, exactly as
// the kernel computes it: fmaf(2^23 + q, s, b).  2^23 + q is the float whose
// low mantissa byte is q, which the kernel forms with one byte permute.
float dequant(int q, float s, float b) { return std::fma((float)(8388608 + q), s, b); }

// Biased origin for grid start `mn`: the largest float b with
// 2^23 * s + b <= mn, so that dequant(0) <= mn.
float biased_origin(float mn, float s) {
    double d = (double)mn - std::ldexp((double)s, 23);
    float b = (float)d;
    if ((double)b > d) b = std::nextafter(b, -INFINITY);
    return b;
}

// Every child plane of one axis rounded outward on the grid (scale s, biased
// origin b), checked with the kernel's arithmetic; false when 255 steps do not
// reach a plane.
bool quantize_axis(float b, float s, const std::vector<Entry>& ch, int axis, uint8_t* qlo, uint8_t* qhi) {
    const double base = (double)dequant(0, s, b);
    for (size_t c = 0; c < ch.size(); ++c) {
        float lo = ch[c].box.mn[axis], hi = ch[c].box.mx[axis];
        double fl = std::floor(((double)lo - base) / (double)s);
        double fh = std::ceil(((double)hi - base) / (double)s);
        int ql = (int)std::max(0.0, std::min(255.0, fl));
        int qh = (int)std::max(0.0, std::min(256.0, fh));
        while (ql > 0 && dequant(ql, s, b) > lo) --ql;
        while (qh <= 255 && dequant(qh, s, b) < hi) ++qh;
        if (qh > 255 || dequant(ql, s, b) > lo) return false;
        qlo[c] = (uint8_t)ql;
        qhi[c] = (uint8_t)qh;
    }
    return true;
}

}  // namespace

void collapse_wide(const std::vector<BinNode>& bin, const std::vector<BuildPrim>& prims, int width,
                   std::vector<uint8_t>& node_bytes, uint32_t* n_nodes,
                   std::vector<uint32_t>& record_order) {
    if (width != 4 && width != 8) throw std::runtime_error("wide collapse supports width 4 or 8");
    node_bytes.clear();
    record_order.clear();
    *n_nodes = 0;
    if (bin.empty()) return;
    const size_t nb = width == 8 ? sizeof(WideNode<8>) : sizeof(WideNode<4>);
    Collapser col{bin, prims, width};
    std::vector<Entry> queue;
    queue.push_back(col.from_bin(0));
    std::vector<uint8_t> bytes(nb, 0);
    for (size_t qi = 0; qi < queue.size(); ++qi) {
        Entry e = queue[qi];
        std::vector<Entry> ch = col.children_of(e);
        // node bounds = union of children
        Box nbx = empty_box();
        for (auto& c : ch) box_union(nbx, c.box);
        uint8_t meta[8] = {0}, qlo[3][8] = {{0}}, qhi[3][8] = {{0}}, ex[3];
        uint32_t imask = 0;
        uint32_t child_base = (uint32_t)queue.size();
        uint32_t prim_base = (uint32_t)record_order.size();
        uint32_t n_int = 0, prim_off = 0;
        for (size_t c = 0; c < ch.size(); ++c) {
            if (Collapser::expandable(ch[c])) {
                meta[c] = (uint8_t)((1u << 5) | n_int);
                imask |= 1u << c;
                queue.push_back(ch[c]);
                ++n_int;
            } else {
                meta[c] = (uint8_t)((ch[c].count << 5) | prim_off);
                for (uint32_t k = 0; k < ch[c].count; ++k) record_order.push_back(ch[c].start + k);
                prim_off += ch[c].count;
            }
        }
        if (prim_off > kMaxPrimsPerNode) throw std::runtime_error("wide node holds too many primitives");
        float origin[3];
        for (int a = 0; a < 3; ++a) {
            // 254 steps over the extent leave one for the biased origin's
            // rounding below the node's lower plane
            double ext = (double)nbx.mx[a] - (double)nbx.mn[a];
            int e2 = -126;
            if (ext > 0.0) e2 = std::max(-126, (int)std::ceil(std::log2(ext / 254.0)));
            // a step far below the plane's float spacing only spends passes
            float mag = std::max(std::fabs(nbx.mn[a]), std::fabs(nbx.mx[a]));
            if (mag > 0.0f) e2 = std::max(e2, std::ilogb(mag) - 23 - 8);
            for (;;) {
                float sc = std::ldexp(1.0f, e2);
                origin[a] = biased_origin(nbx.mn[a], sc);
                if (std::isfinite(origin[a]) && quantize_axis(origin[a], sc, ch, a, qlo[a], qhi[a])) break;
                if (++e2 > 104) throw std::runtime_error("cannot quantise node bounds");
            }
            ex[a] = (uint8_t)(e2 + 127);
        }
        uint32_t packed = (uint32_t)ex[0] | ((uint32_t)ex[1] << 8) | ((uint32_t)ex[2] << 16) | (imask << 24);
        size_t base = qi * nb;
        node_bytes.resize((qi + 1) * nb);
        if (width == 8) {
            WideNode<8> w;
            std::memset(&w, 0, sizeof w);
            std::memcpy(w.origin, origin, sizeof origin);
            w.packed = packed;
            w.child_base = child_base;
            w.prim_base = prim_base;
            std::memcpy(w.meta, meta, 8);
            std::memcpy(w.qlo, qlo, sizeof qlo);
            std::memcpy(w.qhi, qhi, sizeof qhi);
            std::memcpy(&node_bytes[base], &w, sizeof w);
        } else {
            WideNode<4> w;
            std::memset(&w, 0, sizeof w);
            std::memcpy(w.origin, origin, sizeof origin);
            w.packed = packed;
            w.child_base = child_base;
            w.prim_base = prim_base;
            std::memcpy(w.meta, meta, 4);
            std::memcpy(w.qlo_x, qlo[0], 4);
            std::memcpy(w.qlo_y, qlo[1], 4);
            std::memcpy(w.qlo_z, qlo[2], 4);
            std::memcpy(w.qhi_x, qhi[0], 4);
            std::memcpy(w.qhi_y, qhi[1], 4);
            std::memcpy(w.qhi_z, qhi[2], 4);
            std::memcpy(&node_bytes[base], &w, sizeof w);
        }
    }
    *n_nodes = (uint32_t)queue.size();
}

std::string build_layout(const std::vector<MeshView>& meshes, int width, int max_prims_in_node, int threads,
                         HostLayout& out) {
    if (width != 2 && width != 4 && width != 8) return "width must be 2, 4 or 8";
    if (max_prims_in_node < 1 || max_prims_in_node > 255) return "max_prims_in_node must be in [1, 255]";
    out = HostLayout();
    out.width = width;
    uint64_t total = 0;
    for (const MeshView& m : meshes) total += m.n_prims;
    if (total >= (1ull << 28)) return "more than 2^28 primitives";
    // Primitive info in list order (bvh.rs:49-53).
    struct Src { uint32_t mesh, local, sphere_slot; };
    std::vector<BuildPrim> prims;
    std::vector<Src> src;
    prims.reserve(total);
    src.reserve(total);
    uint32_t pid = 0;
    for (uint32_t k = 0; k < meshes.size(); ++k) {
        const MeshView& m = meshes[k];
        for (uint32_t i = 0; i < m.n_prims; ++i, ++pid) {
            BuildPrim bp;
            bp.prim = pid;
            if (m.is_spheres) {
                bp.bounds = sphere_bound(m.spheres[i]);
                src.push_back({k, i, (uint32_t)out.spheres.size()});
                out.spheres.push_back(m.spheres[i]);
            } else {
                const uint32_t* ix = &m.idx[3ull * i];
                bp.bounds = triangle_bound(m.xyz + 3ull * ix[0], m.xyz + 3ull * ix[1], m.xyz + 3ull * ix[2]);
                src.push_back({k, i, 0});
            }
            box_centroid(bp.bounds, bp.centroid);
            prims.push_back(bp);
        }
    }
    out.n_prims = (uint32_t)total;
    try {
        sah_build(prims, max_prims_in_node, threads, out.bin_nodes);
    } catch (const std::exception& e) {
        return e.what();
    }
    out.prim_order.resize(prims.size());
    for (size_t i = 0; i < prims.size(); ++i) out.prim_order[i] = prims[i].prim;
    if (!out.bin_nodes.empty()) {
        for (int k = 0; k < 3; ++k) { out.bound[k] = out.bin_nodes[0].bmin[k]; out.bound[3 + k] = out.bin_nodes[0].bmax[k]; }
    } else {
        Box e = empty_box();
        for (int k = 0; k < 3; ++k) { out.bound[k] = e.mn[k]; out.bound[3 + k] = e.mx[k]; }
    }
    std::vector<uint32_t> record_order;   // indices into the leaf-ordered `prims`
    if (width == 2) {
        out.n_nodes = (uint32_t)out.bin_nodes.size();
        out.node_bytes.resize(out.bin_nodes.size() * sizeof(BinNode));
        if (!out.bin_nodes.empty()) std::memcpy(out.node_bytes.data(), out.bin_nodes.data(), out.node_bytes.size());
        record_order.resize(prims.size());
        for (size_t i = 0; i < prims.size(); ++i) record_order[i] = (uint32_t)i;
    } else {
        try {
            collapse_wide(out.bin_nodes, prims, width, out.node_bytes, &out.n_nodes, record_order);
        } catch (const std::exception& e) {
            return e.what();
        }
    }
    out.records.resize(record_order.size());
    for (size_t r = 0; r < record_order.size(); ++r) {
        const BuildPrim& bp = prims[record_order[r]];
        const Src& s = src[bp.prim];
        const MeshView& m = meshes[s.mesh];
        PrimRec& pr = out.records[r];
        std::memset(&pr, 0, sizeof pr);
        pr.prim = bp.prim;
        if (m.is_spheres) {
            pr.flags = kPrimSphere;
            pr.aux = s.sphere_slot;
        } else {
            const uint32_t* ix = &m.idx[3ull * s.local];
            std::memcpy(pr.p0, m.xyz + 3ull * ix[0], 12);
            std::memcpy(pr.p1, m.xyz + 3ull * ix[1], 12);
            std::memcpy(pr.p2, m.xyz + 3ull * ix[2], 12);
            pr.flags = triangle_degenerate(pr.p0, pr.p1, pr.p2) ? kPrimDegenerate : 0u;
        }
    }
    return std::string();
}

}  // namespace ilm
