// Host-side kd-tree build (KdTreeAccel, accelerators/kdtreeaccel.rs:25-244).
// Compiled with -ffp-contract=off: the split costs round as the reference's
// f32 expressions do, so the node array is the reference's node for node.
//
// Repairs against the reference (which does not compile as written):
//  * the split axis is rebound on each retry (`let axis` is immutable in
//    kdtreeaccel.rs:130 although 189 assigns it; pbrt-v3's retrySplit intent);
//  * edges of one axis are sorted by (position, start before end) as
//    kdtreeaccel.rs:142-148, then by primitive id, so the order of equal
//    edges -- which decides the children of primitives that touch the split
//    plane -- is fixed instead of left to an unstable sort.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <thread>

#include "builder.h"

namespace ilm {

namespace {

struct Edge {
    float t;
    uint32_t prim;
    uint32_t end;      // 0 = EdgeType::Start, 1 = EdgeType::End
};

inline bool edge_less(const Edge& a, const Edge& b) {
    if (a.t != b.t) return a.t < b.t;
    if (a.end != b.end) return a.end < b.end;
    return a.prim < b.prim;
}

// Bounding3::surface_area / maximum_extent (geometry/bounds3.rs:53-62).
inline float box_area(const Box& b) {
    float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
    return 2.0f * (dx * dy + dx * dz + dy * dz);
}
inline int box_max_extent(const Box& b) {
    float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
    if (dx > dy && dx > dz) return 0;
    if (dy > dz) return 1;
    return 2;
}

// One subtree's output with node and index numbering local to it.
struct KdPart {
    std::vector<KdNode> nodes;
    std::vector<uint32_t> index;
};

// Appends `src` (numbered from 0) to `dst`, moving its above-child links and
// leaf runs past what `dst` already holds.
void splice(KdPart& dst, const KdPart& src) {
    const uint64_t nb = dst.nodes.size(), ib = dst.index.size();
    if (nb + src.nodes.size() >= (1ull << 30)) throw std::runtime_error("kd-tree above 2^30 nodes");
    for (KdNode n : src.nodes) {
        if ((n.flags & 3u) == kKdLeaf) {
            if ((n.flags >> 2) > 1) n.word += (uint32_t)ib;
        } else {
            n.flags = (n.flags & 3u) | ((uint32_t)((n.flags >> 2) + nb) << 2);
        }
        dst.nodes.push_back(n);
    }
    dst.index.insert(dst.index.end(), src.index.begin(), src.index.end());
}

class KdBuilder {
public:
    KdBuilder(const std::vector<Box>& bounds, const KdParams& p, int threads) : b_(bounds), p_(p) {
        while ((1 << spawn_levels_) < threads && spawn_levels_ < 6) ++spawn_levels_;
    }

    // build_tree (kdtreeaccel.rs:90-244) for the node about to be appended.
    void build(const Box& nb, const std::vector<uint32_t>& prims, int depth, int bad_refines, int level,
               KdPart& out) {
        const size_t node = out.nodes.size();
        if (node >= (1u << 30)) throw std::runtime_error("kd-tree above 2^30 nodes");
        out.nodes.push_back(KdNode{0u, 0u});
        const size_t n = prims.size();
        if (n <= p_.max_prims || depth == 0) {
            leaf(prims, node, out);
            return;
        }
        // Split choice (kdtreeaccel.rs:120-195).
        int best_axis = -1;
        size_t best_offset = 0;
        float best_cost = INFINITY;
        const float old_cost = (float)((uint64_t)p_.isect_cost * n);
        const float total_sa = box_area(nb);
        const float inv_total_sa = 1.0f / total_sa;
        const float d[3] = {nb.mx[0] - nb.mn[0], nb.mx[1] - nb.mn[1], nb.mx[2] - nb.mn[2]};
        std::vector<Edge>& edges = scratch();
        int axis = box_max_extent(nb);
        for (int retries = 0;;) {
            edges.resize(2 * n);
            for (size_t i = 0; i < n; ++i) {
                const Box& pb = b_[prims[i]];
                edges[2 * i] = Edge{pb.mn[axis], prims[i], 0u};
                edges[2 * i + 1] = Edge{pb.mx[axis], prims[i], 1u};
            }
            std::sort(edges.begin(), edges.end(), edge_less);
            const int o0 = (axis + 1) % 3, o1 = (axis + 2) % 3;
            size_t n_below = 0, n_above = n;
            for (size_t i = 0; i < 2 * n; ++i) {
                if (edges[i].end) --n_above;
                const float et = edges[i].t;
                if (et > nb.mn[axis] && et < nb.mx[axis]) {
                    float below_sa = 2.0f * (d[o0] * d[o1] + (et - nb.mn[axis]) * (d[o0] + d[o1]));
                    float above_sa = 2.0f * (d[o0] * d[o1] + (nb.mx[axis] - et) * (d[o0] + d[o1]));
                    float p_below = below_sa * inv_total_sa;
                    float p_above = above_sa * inv_total_sa;
                    float eb = (n_above == 0 || n_below == 0) ? p_.empty_bonus : 0.0f;
                    float cost = (float)p_.traversal_cost +
                                 (float)p_.isect_cost * (1.0f - eb) *
                                     (p_below * (float)n_below + p_above * (float)n_above);
                    if (cost < best_cost) {
                        best_cost = cost;
                        best_axis = axis;
                        best_offset = i;
                    }
                }
                if (!edges[i].end) ++n_below;
            }
            if (best_axis == -1 && retries < 2) {
                ++retries;
                axis = (axis + 1) % 3;
                continue;
            }
            break;
        }
        if (best_cost > old_cost) ++bad_refines;
        if ((best_cost > 4.0f * old_cost && n < 16) || best_axis == -1 || bad_refines == 3) {
            leaf(prims, node, out);
            return;
        }
        // The last sort was along best_axis: a retry happens only when the
        // axis before it found no candidate edge.  Classify (kdtreeaccel.rs:206-219).
        std::vector<uint32_t> prims0, prims1;
        for (size_t i = 0; i < best_offset; ++i)
            if (!edges[i].end) prims0.push_back(edges[i].prim);
        for (size_t i = best_offset + 1; i < 2 * n; ++i)
            if (edges[i].end) prims1.push_back(edges[i].prim);
        const float t_split = edges[best_offset].t;
        Box b0 = nb, b1 = nb;
        b0.mx[best_axis] = t_split;
        b1.mn[best_axis] = t_split;
        if (level < spawn_levels_ && prims0.size() + prims1.size() > 4096) {
            KdPart below, above;
            std::exception_ptr err;
            std::thread th([&] {
                try {
                    build(b1, prims1, depth - 1, bad_refines, level + 1, above);
                } catch (...) {
                    err = std::current_exception();
                }
            });
            try {
                build(b0, prims0, depth - 1, bad_refines, level + 1, below);
            } catch (...) {
                th.join();
                throw;
            }
            th.join();
            if (err) std::rethrow_exception(err);
            // the below subtree lands at node + 1, the above child right after it
            out.nodes.reserve(out.nodes.size() + below.nodes.size() + above.nodes.size());
            const uint64_t base = out.nodes.size();
            splice(out, below);
            interior(out, node, best_axis, (uint32_t)(base + below.nodes.size()), t_split);
            splice(out, above);
        } else {
            build(b0, prims0, depth - 1, bad_refines, level + 1, out);
            const size_t above_child = out.nodes.size();
            interior(out, node, best_axis, (uint32_t)above_child, t_split);
            build(b1, prims1, depth - 1, bad_refines, level + 1, out);
        }
    }

private:
    static std::vector<Edge>& scratch() {
        thread_local std::vector<Edge> e;
        return e;
    }
    // KdAccelNode::init_leaf (kdtreeaccel.rs:476-490)
    static void leaf(const std::vector<uint32_t>& prims, size_t node, KdPart& out) {
        KdNode& k = out.nodes[node];
        const size_t n = prims.size();
        k.flags = kKdLeaf | ((uint32_t)n << 2);
        if (n == 0) {
            k.word = 0u;
        } else if (n == 1) {
            k.word = prims[0];
        } else {
            k.word = (uint32_t)out.index.size();
            out.index.insert(out.index.end(), prims.begin(), prims.end());
        }
    }
    // KdAccelNode::init_interior (kdtreeaccel.rs:492-496)
    static void interior(KdPart& out, size_t node, int axis, uint32_t above, float split) {
        KdNode& k = out.nodes[node];
        std::memcpy(&k.word, &split, 4);
        k.flags = (uint32_t)axis | (above << 2);
    }

    const std::vector<Box>& b_;
    KdParams p_;
    int spawn_levels_ = 0;
};

}  // namespace

int kd_default_depth(uint64_t n) {
    if (n == 0) return 0;
    return (int)std::lround(8.0 + 1.3 * std::log2((double)n));
}

void kd_build(const std::vector<Box>& bounds, const Box& root, const KdParams& p, int threads,
              std::vector<KdNode>& nodes, std::vector<uint32_t>& index) {
    nodes.clear();
    index.clear();
    if (bounds.empty()) return;
    std::vector<uint32_t> all(bounds.size());
    for (size_t i = 0; i < all.size(); ++i) all[i] = (uint32_t)i;
    const int depth = p.max_depth > 0 ? p.max_depth : kd_default_depth(bounds.size());
    KdPart out;
    KdBuilder(bounds, p, threads).build(root, all, depth, 0, 0, out);
    nodes.swap(out.nodes);
    index.swap(out.index);
}

std::string build_kd_layout(const std::vector<MeshView>& meshes, const KdParams& p, int threads, HostLayout& out) {
    if (p.isect_cost < 0 || p.traversal_cost < 0) return "costs must be non-negative";
    if (!(p.empty_bonus >= 0.0f && p.empty_bonus <= 1.0f)) return "empty_bonus must be in [0, 1]";
    out = HostLayout();
    out.width = kLayoutKdTree;
    uint64_t total = 0;
    for (const MeshView& m : meshes) total += m.n_prims;
    if (total >= (1ull << 28)) return "more than 2^28 primitives";
    const int depth = p.max_depth > 0 ? p.max_depth : kd_default_depth(total);
    if (depth > kKdMaxDepth) return "max_depth above 64";
    out.kd_max_depth = depth;
    out.n_prims = (uint32_t)total;
    // World bounds and records in primitive-id order (kdtreeaccel.rs:38-46).
    std::vector<Box> bounds;
    bounds.reserve(total);
    out.records.resize(total);
    Box root = empty_box();
    uint32_t pid = 0;
    for (const MeshView& m : meshes) {
        for (uint32_t i = 0; i < m.n_prims; ++i, ++pid) {
            PrimRec& pr = out.records[pid];
            std::memset(&pr, 0, sizeof pr);
            pr.prim = pid;
            Box b;
            if (m.is_spheres) {
                b = sphere_bound(m.spheres[i]);
                pr.flags = kPrimSphere;
                pr.aux = (uint32_t)out.spheres.size();
                out.spheres.push_back(m.spheres[i]);
            } else {
                const uint32_t* ix = &m.idx[3ull * i];
                std::memcpy(pr.p0, m.xyz + 3ull * ix[0], 12);
                std::memcpy(pr.p1, m.xyz + 3ull * ix[1], 12);
                std::memcpy(pr.p2, m.xyz + 3ull * ix[2], 12);
                pr.flags = triangle_degenerate(pr.p0, pr.p1, pr.p2) ? kPrimDegenerate : 0u;
                b = triangle_bound(pr.p0, pr.p1, pr.p2);
            }
            for (int k = 0; k < 3; ++k) {
                root.mn[k] = root.mn[k] < b.mn[k] ? root.mn[k] : b.mn[k];
                root.mx[k] = root.mx[k] > b.mx[k] ? root.mx[k] : b.mx[k];
            }
            bounds.push_back(b);
        }
    }
    for (int k = 0; k < 3; ++k) { out.bound[k] = root.mn[k]; out.bound[3 + k] = root.mx[k]; }
    std::vector<KdNode> nodes;
    KdParams q = p;
    q.max_depth = depth;
    try {
        kd_build(bounds, root, q, threads, nodes, out.kd_index);
    } catch (const std::exception& e) {
        return e.what();
    }
    out.n_nodes = (uint32_t)nodes.size();
    out.node_bytes.resize(nodes.size() * sizeof(KdNode));
    if (!nodes.empty()) std::memcpy(out.node_bytes.data(), nodes.data(), out.node_bytes.size());
    out.prim_order.resize(total);
    for (uint32_t i = 0; i < total; ++i) out.prim_order[i] = i;
    return std::string();
}

}  // namespace ilm
