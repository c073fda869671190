// Wide-BVH traversal state shared by the single-scene and batched kernels.
//
// Nodes are the compressed layout of layout.h: 8-bit child planes on a
// per-node power-of-two grid, dequantised with one fma each and rounded
// outward at build time, so every test below is at least as permissive as
// Bounds3::intersect_p on the exact child box (geometry/bounds3.rs:284-318).
// Hit children are sorted by entry distance (sorting network on keys that
// pack the distance's bits with the slot) and pushed far-to-near.
#pragma once
#include "trace_common.cuh"

namespace ilm {

template <int W> struct WideWords;
template <> struct WideWords<8> { static constexpr int kWords = 5; };
template <> struct WideWords<4> { static constexpr int kWords = 4; };

// Byte i of a W-byte array split over 32-bit words lo (bytes 0-3) and hi (4-7).
__device__ __forceinline__ uint32_t byte_of(uint32_t lo, uint32_t hi, int i) {
    return __byte_perm(i < 4 ? lo : hi, 0u, (uint32_t)(i & 3) | 0x4440u);
}

// The float 2^23 + byte, formed by one byte permute that writes the byte into
// the low mantissa bits of 2^23 (no integer-to-float conversion: those issue
// on the narrow XU pipe, which 48 conversions per node saturate).  Nodes
// store their origin biased by -2^23 * scale, so fma(2^23 + q, scale, origin)
// is the dequantised plane with no subtraction of the bias.
__device__ __forceinline__ float byte_float(uint32_t lo, uint32_t hi, int i) {
    return __uint_as_float(__byte_perm(i < 4 ? lo : hi, 0x4B000000u, (uint32_t)(i & 3) | 0x7650u));
}

// Decoded node, with near/far planes already swapped for the ray octant.
template <int W>
struct WideView {
    float ox, oy, oz, sx, sy, sz;
    uint32_t imask, child_base, prim_base;
    uint32_t meta[2];
    uint32_t nq[3][2], fq[3][2];   // near / far quantised planes per axis
};

template <int W>
__device__ __forceinline__ WideView<W> load_wide(const uint4* __restrict__ nodes, uint32_t idx, bool negx,
                                                 bool negy, bool negz) {
    WideView<W> v;
    const uint4* p = nodes + (size_t)idx * WideWords<W>::kWords;
    uint4 w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2), w3 = __ldg(p + 3);
    v.ox = __uint_as_float(w0.x); v.oy = __uint_as_float(w0.y); v.oz = __uint_as_float(w0.z);
    v.sx = __uint_as_float((w0.w & 0xFFu) << 23);
    v.sy = __uint_as_float(((w0.w >> 8) & 0xFFu) << 23);
    v.sz = __uint_as_float(((w0.w >> 16) & 0xFFu) << 23);
    v.imask = w0.w >> 24;
    v.child_base = w1.x;
    v.prim_base = w1.y;
    uint32_t lo[3][2], hi[3][2];
    if (W == 8) {
        uint4 w4 = __ldg(p + 4);
        v.meta[0] = w1.z; v.meta[1] = w1.w;
        lo[0][0] = w2.x; lo[0][1] = w2.y; lo[1][0] = w2.z; lo[1][1] = w2.w;
        lo[2][0] = w3.x; lo[2][1] = w3.y; hi[0][0] = w3.z; hi[0][1] = w3.w;
        hi[1][0] = w4.x; hi[1][1] = w4.y; hi[2][0] = w4.z; hi[2][1] = w4.w;
    } else {
        v.meta[0] = w1.z; v.meta[1] = 0;
        lo[0][0] = w1.w; lo[1][0] = w2.x; lo[2][0] = w2.y; hi[0][0] = w2.z; hi[1][0] = w2.w;
        hi[2][0] = w3.x;
        lo[0][1] = lo[1][1] = lo[2][1] = hi[0][1] = hi[1][1] = hi[2][1] = 0;
    }
    bool neg[3] = {negx, negy, negz};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            v.nq[a][h] = neg[a] ? hi[a][h] : lo[a][h];
            v.fq[a][h] = neg[a] ? lo[a][h] : hi[a][h];
        }
    return v;
}

// Slab test of child i (Bounds3::intersect_p semantics on the dequantised
// box; fmaxf/fminf skip a NaN slab, which can only widen the accepted set).
template <int W>
__device__ __forceinline__ bool child_hit(const WideView<W>& v, int i, const RayIn& r, float ix, float iy,
                                          float iz, float tmax, float& tn_out) {
    uint32_t m = byte_of(v.meta[0], v.meta[1], i);
    float nx = fmaf(byte_float(v.nq[0][0], v.nq[0][1], i), v.sx, v.ox);
    float fx = fmaf(byte_float(v.fq[0][0], v.fq[0][1], i), v.sx, v.ox);
    float ny = fmaf(byte_float(v.nq[1][0], v.nq[1][1], i), v.sy, v.oy);
    float fy = fmaf(byte_float(v.fq[1][0], v.fq[1][1], i), v.sy, v.oy);
    float nz = fmaf(byte_float(v.nq[2][0], v.nq[2][1], i), v.sz, v.oz);
    float fz = fmaf(byte_float(v.fq[2][0], v.fq[2][1], i), v.sz, v.oz);
    float tnx = __fmul_rn(__fsub_rn(nx, r.ox), ix), tfx = __fmul_rn(__fsub_rn(fx, r.ox), ix);
    float tny = __fmul_rn(__fsub_rn(ny, r.oy), iy), tfy = __fmul_rn(__fsub_rn(fy, r.oy), iy);
    float tnz = __fmul_rn(__fsub_rn(nz, r.oz), iz), tfz = __fmul_rn(__fsub_rn(fz, r.oz), iz);
    float tn = fmaxf(fmaxf(tnx, tny), tnz);
    float tf = __fmul_rn(fminf(fminf(tfx, tfy), tfz), kBoxRobust);
    tn_out = tn;
    return m != 0u && tn <= tf && tn < tmax && tf > 0.0f;
}

template <int W>
__device__ __forceinline__ uint32_t child_entry(const WideView<W>& v, uint32_t slot) {
    uint32_t m = byte_of(v.meta[0], v.meta[1], (int)slot);
    if ((v.imask >> slot) & 1u) return v.child_base + (m & 31u);
    return kLeafFlag | ((v.prim_base + (m & 31u)) << 3) | ((m >> 5) - 1u);
}

__device__ __forceinline__ void cswap(uint32_t& a, uint32_t& b) {
    uint32_t lo = min(a, b), hi = max(a, b);
    a = lo; b = hi;
}

template <int W>
__device__ __forceinline__ void sort_keys(uint32_t* k) {
    if (W == 8) {
        // Batcher odd-even merge sort, 19 comparators
        cswap(k[0], k[1]); cswap(k[2], k[3]); cswap(k[4], k[5]); cswap(k[6], k[7]);
        cswap(k[0], k[2]); cswap(k[1], k[3]); cswap(k[4], k[6]); cswap(k[5], k[7]);
        cswap(k[1], k[2]); cswap(k[5], k[6]);
        cswap(k[0], k[4]); cswap(k[1], k[5]); cswap(k[2], k[6]); cswap(k[3], k[7]);
        cswap(k[2], k[4]); cswap(k[3], k[5]);
        cswap(k[1], k[2]); cswap(k[3], k[4]); cswap(k[5], k[6]);
    } else {
        cswap(k[0], k[1]); cswap(k[2], k[3]);
        cswap(k[0], k[2]); cswap(k[1], k[3]);
        cswap(k[1], k[2]);
    }
}

// A subtree handed to another lane that the donor's own pop would have culled
// (no node or leaf entry has all bits set: that would be a leaf of 8 records
// at 2^28 - 1; kd-tree node indices stay below 2^30).
constexpr uint32_t kNoEntry = 0xFFFFFFFFu;

// Per-lane traversal state of one ray over 4- or 8-wide nodes: hit children
// sorted by entry distance and pushed far-to-near, one stack entry (node or
// leaf, with its entry distance) per child.
//
// The stack is a local array of the launching kernel (Entry stk[kDepth]),
// handed to the constructor, never a member: a struct that holds a
// dynamically indexed array is kept whole in local memory, and every scalar
// of the traversal state (ray, current node, best hit) would be loaded from
// and stored to local memory at each step beside it.
template <int W, int kStack, bool kAny, bool kAnalytic = true>
struct WideTracerSorted {
    using Entry = uint2;
    static constexpr int kDepth = kStack;
    RayIn ray;
    float ix, iy, iz;
    bool negx, negy, negz, tr_ready, occluded;
    TriRay tr;
    float best_t, bu, bv;
    uint32_t best, status, cur, iter;
    int sp;
    uint2* stack;

    __device__ __forceinline__ explicit WideTracerSorted(uint2* s) : stack(s) {}

    __device__ __forceinline__ void init(const RayIn& r) {
        ray = r;
        best_t = r.tmax; bu = 0.0f; bv = 0.0f;
        best = ILM_MISS;
        occluded = false;
        status = 0;
        ix = __frcp_rn(r.dx); iy = __frcp_rn(r.dy); iz = __frcp_rn(r.dz);   // == 1/d exactly
        negx = ix < 0.0f; negy = iy < 0.0f; negz = iz < 0.0f;
        tr_ready = false;
        cur = 0; iter = 0; sp = 0;
    }

    // The root box test BVHAccel performs first (the root node's bounds are
    // the world bound).
    __device__ __forceinline__ bool enters(const float* b) const {
        return box_intersect_p(b[0], b[1], b[2], b[3], b[4], b[5], ray, ix, iy, iz, negx, negy, negz, ray.tmax);
    }

    // Starts on subtree `node` of a ray another lane is tracing, with that
    // lane's reciprocal directions and `bound` (its best distance so far) as
    // the limit; the hit found, if any, is this lane's own.
    __device__ __forceinline__ void adopt(const RayIn& r, float rx, float ry, float rz, float bound, uint32_t node) {
        ray = r;
        ix = rx; iy = ry; iz = rz;
        negx = ix < 0.0f; negy = iy < 0.0f; negz = iz < 0.0f;
        best_t = bound; bu = 0.0f; bv = 0.0f;
        best = ILM_MISS;
        occluded = false;
        status = 0;
        tr_ready = false;
        cur = node; iter = 0; sp = 0;
    }

    // Split tail: stages the top stack entry for another lane (4 uint4: the
    // entry, tmax, best distance, owner lane; the ray with its reciprocal
    // directions), and adopts such a staging; take() is false for an entry
    // the donor's pop would have culled.
    __device__ __forceinline__ void give(uint4* s, uint32_t owner) {
        const uint2 e = pop_one();
        const bool live = kAny || __uint_as_float(e.y) < best_t;
        s[0] = make_uint4(live ? e.x : kNoEntry, __float_as_uint(ray.tmax), __float_as_uint(best_t), owner);
        s[1] = make_uint4(__float_as_uint(ray.ox), __float_as_uint(ray.oy), __float_as_uint(ray.oz),
                          __float_as_uint(ix));
        s[2] = make_uint4(__float_as_uint(ray.dx), __float_as_uint(ray.dy), __float_as_uint(ray.dz),
                          __float_as_uint(iy));
        s[3].x = __float_as_uint(iz);
    }
    __device__ __forceinline__ bool take(const uint4* s, uint32_t& owner) {
        const uint4 h = s[0];
        if (h.x == kNoEntry) return false;
        const uint4 r0 = s[1], r1 = s[2];
        adopt(RayIn{__uint_as_float(r0.x), __uint_as_float(r0.y), __uint_as_float(r0.z), __uint_as_float(r1.x),
                    __uint_as_float(r1.y), __uint_as_float(r1.z), __uint_as_float(h.y)},
              __uint_as_float(r0.w), __uint_as_float(r1.w), __uint_as_float(s[3].x), __uint_as_float(h.z), h.x);
        owner = h.w;
        return true;
    }

    __device__ __forceinline__ void push(uint2 e) { stack[sp++] = e; }
    __device__ __forceinline__ uint2 pop_one() { return stack[--sp]; }

    // Next stacked entry still nearer than the current hit; false when none.
    __device__ __forceinline__ bool pop() {
        while (sp > 0) {
            uint2 e = pop_one();
            if (kAny || __uint_as_float(e.y) < best_t) { cur = e.x; return true; }
        }
        return false;
    }

    // Interior node `cur`: true when the traversal continues into a child.
    __device__ __forceinline__ bool node(const uint4* __restrict__ nodes) {
        WideView<W> nv = load_wide<W>(nodes, cur, negx, negy, negz);
        float lim = kAny ? ray.tmax : best_t;
        if (kAny) {
            uint32_t first = 0xFFFFFFFFu;
#pragma unroll
            for (int c = 0; c < W; ++c) {
                float tn;
                if (child_hit<W>(nv, c, ray, ix, iy, iz, lim, tn)) {
                    uint32_t e = child_entry<W>(nv, (uint32_t)c);
                    if (first == 0xFFFFFFFFu) first = e;
                    else if (sp < kStack) push(make_uint2(e, 0u));
                    else status = kErrStackOverflow;
                }
            }
            if (first != 0xFFFFFFFFu && !status) { cur = first; return true; }
            return false;
        }
        uint32_t keys[W];
        int nhit = 0;
#pragma unroll
        for (int c = 0; c < W; ++c) {
            float tn;
            bool h = child_hit<W>(nv, c, ray, ix, iy, iz, lim, tn);
            keys[c] = h ? ((__float_as_uint(fmaxf(tn, 0.0f)) & ~7u) | (uint32_t)c) : 0xFFFFFFFFu;
            nhit += h ? 1 : 0;
        }
        if (nhit == 0) return false;
        sort_keys<W>(keys);
        if (sp + nhit - 1 > kStack) { status = kErrStackOverflow; return false; }
#pragma unroll
        for (int j = W - 1; j >= 1; --j)
            if (j < nhit) push(make_uint2(child_entry<W>(nv, keys[j] & 7u), keys[j] & ~7u));
        cur = child_entry<W>(nv, keys[0] & 7u);
        return true;
    }

    __device__ __forceinline__ void leaf(const PrimRec* __restrict__ prims, const SphereRec* __restrict__ spheres) {
        uint32_t start = (cur & ~kLeafFlag) >> 3, cnt = (cur & 7u) + 1u;
        for (uint32_t k = 0; k < cnt; ++k) {
            float t, u, v;
            uint32_t pid;
            if (kAny) {
                if (prim_test<false, kAnalytic>(prims, spheres, start + k, tr, tr_ready, ray, ray.tmax, t, u, v,
                                                pid)) {
                    occluded = true;
                    return;
                }
            } else if (prim_test<true, kAnalytic>(prims, spheres, start + k, tr, tr_ready, ray, best_t, t, u, v,
                                                  pid) &&
                       (t < best_t || (t == best_t && pid < best))) {
                best_t = t; best = pid; bu = u; bv = v;
            }
        }
    }

    // Advances by one node or one leaf; true when the ray is finished.
    __device__ __forceinline__ bool step(const TraceArgs& a) {
        if (++iter > a.max_iter) { status = kErrIterationCap; return true; }
        if (cur & kLeafFlag) {
            leaf(a.prims, a.spheres);
            if (kAny && occluded) return true;
        } else if (node(static_cast<const uint4*>(a.nodes))) {
            return false;
        } else if (status) {
            return true;
        }
        return !pop();
    }

    __device__ __forceinline__ void write(uint64_t i, const TraceArgs& a) const {
        if (status) atomicOr(a.err, status);
        if (kAny) {
            a.occ[i] = status ? kHitTraversalError : (occluded ? 1u : 0u);
        } else {
            if (status) store_hit(a.hits, i, kHitTraversalError, ray.tmax, 0.0f, 0.0f);
            else store_hit(a.hits, i, best, best == ILM_MISS ? ray.tmax : best_t, bu, bv);
        }
    }
};


// Per-lane traversal state of one ray over the binary layout (the reference's
// 32-byte LinearBVHNode, accelerators/bvh.rs:665-673): the ordered traversal of
// BVHAccel::intersect / intersect_p (bvh.rs:563-662, the far child pushed on
// both branches), one node visit per step, exactly as k_trace_bin runs it, so
// the records (and which rays reach a limit) are the same.  The stack has the
// reference's 64 entries (bvh.rs:573) whatever the caller's depth; like
// WideTracerSorted's, it is the launching kernel's array.
template <bool kAny, bool kAnalytic = true>
struct BinTracer {
    using Entry = uint32_t;
    static constexpr int kDepth = 64;
    RayIn ray;
    float ix, iy, iz;
    bool negx, negy, negz, tr_ready, occluded;
    TriRay tr;
    float best_t, bu, bv;
    uint32_t best, status, cur, iter;
    int sp;
    uint32_t* stack;

    __device__ __forceinline__ explicit BinTracer(uint32_t* s) : stack(s) {}

    __device__ __forceinline__ void init(const RayIn& r) {
        ray = r;
        best_t = r.tmax; bu = 0.0f; bv = 0.0f;
        best = ILM_MISS;
        occluded = false;
        status = 0;
        ix = __frcp_rn(r.dx); iy = __frcp_rn(r.dy); iz = __frcp_rn(r.dz);   // == 1/d exactly
        negx = ix < 0.0f; negy = iy < 0.0f; negz = iz < 0.0f;
        tr_ready = false;
        cur = 0; iter = 0; sp = 0;
    }

    __device__ __forceinline__ bool enters(const float* b) const {
        return box_intersect_p(b[0], b[1], b[2], b[3], b[4], b[5], ray, ix, iy, iz, negx, negy, negz, ray.tmax);
    }

    // Visits node `cur`; true when the ray is finished.
    __device__ __forceinline__ bool step(const TraceArgs& a) {
        if (++iter > a.max_iter) { status = kErrIterationCap; return true; }
        const float4* np = reinterpret_cast<const float4*>(static_cast<const BinNode*>(a.nodes) + cur);
        const float4 n0 = __ldg(np), n1 = __ldg(np + 1);
        // n0 = (minx, miny, minz, maxx), n1 = (maxy, maxz, offset, n_prims | axis << 16)
        if (box_intersect_p(n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, ray, ix, iy, iz, negx, negy, negz,
                            kAny ? ray.tmax : best_t)) {
            const uint32_t meta = __float_as_uint(n1.w);
            const uint32_t nprims = meta & 0xFFFFu;
            const uint32_t off = __float_as_uint(n1.z);
            if (nprims == 0) {
                if (sp == 64) { status = kErrStackOverflow; return true; }
                const uint32_t axis = (meta >> 16) & 0xFFu;
                const bool neg = axis == 0 ? negx : (axis == 1 ? negy : negz);
                if (neg) { stack[sp++] = cur + 1; cur = off; }
                else { stack[sp++] = off; cur = cur + 1; }
                return false;
            }
            for (uint32_t k = 0; k < nprims; ++k) {
                float t, u, v;
                uint32_t pid;
                if (kAny) {
                    if (prim_test<false, kAnalytic>(a.prims, a.spheres, off + k, tr, tr_ready, ray, ray.tmax, t, u,
                                                    v, pid)) {
                        occluded = true;
                        return true;
                    }
                } else if (prim_test<true, kAnalytic>(a.prims, a.spheres, off + k, tr, tr_ready, ray, best_t, t, u,
                                                      v, pid) &&
                           (t < best_t || (t == best_t && pid < best))) {
                    best_t = t; best = pid; bu = u; bv = v;
                }
            }
        }
        if (sp == 0) return true;
        cur = stack[--sp];
        return false;
    }

    __device__ __forceinline__ void write(uint64_t i, const TraceArgs& a) const {
        if (status) atomicOr(a.err, status);
        if (kAny) {
            a.occ[i] = status ? kHitTraversalError : (occluded ? 1u : 0u);
        } else {
            if (status) store_hit(a.hits, i, kHitTraversalError, ray.tmax, 0.0f, 0.0f);
            else store_hit(a.hits, i, best, best == ILM_MISS ? ray.tmax : best_t, bu, bv);
        }
    }
};

// The tracer of a width: sorted children for 4- and 8-wide nodes, the
// reference's ordered traversal for binary nodes.
template <int W, int kStack, bool kAny, bool kAnalytic>
struct TracerOf { using type = WideTracerSorted<W, kStack, kAny, kAnalytic>; };
template <int kStack, bool kAny, bool kAnalytic>
struct TracerOf<2, kStack, kAny, kAnalytic> { using type = BinTracer<kAny, kAnalytic>; };
template <int W, int kStack, bool kAny, bool kAnalytic = true>
using WideTracer = typename TracerOf<W, kStack, kAny, kAnalytic>::type;

// Split tail of the pooled persistent schedule (k_trace_wide_persistent).
// Once the work counter has run out, a warp's last rays finish with its idle
// lanes helping them; without help the launch lasts as long as its longest
// rays, which make ten times the median number of node visits.  A ray's lane
// (its owner) keeps traversing; each pass, every idle lane takes the top stack
// entry of a lane that has one (owner or helper) and traverses that subtree
// with a copy of the ray, bounded by the donor's best distance so far.  A
// helper that finishes hands its best hit to the owner, which keeps the
// smaller (t, primitive id), the tie rule of every traversal here: the nearest
// hit is the nearest whichever lane tests it, and culling only skips subtrees
// that cannot hold a nearer hit, so the records are the lone traversal's --
// except that of two hits at exactly the same t the split keeps the smaller
// primitive id where the lone traversal may keep the first it found.  Any-hit
// owners stop at the first occlusion any of their lanes finds, and their
// helpers stop with them.  An owner writes its record once its own traversal
// and all its helpers are done.  Nothing waits on another warp; every lane's
// traversal is bounded by the iteration cap.
//
// Lane roles, packed with the owner lane (bits 2-6) and an owner's count of
// helpers (bits 8-13) in one word.
enum : uint32_t { kFree = 0, kOwner = 1, kWaiting = 2, kHelper = 3 };
__device__ __forceinline__ uint32_t role_of(uint32_t st) { return st & 3u; }
__device__ __forceinline__ uint32_t owner_of(uint32_t st) { return (st >> 2) & 31u; }

// Words of the per-warp shared area of the pooled schedule: the pool of
// entering rays' offsets, each lane's ray id, and 16 staging slots of 16
// words for handed-over subtrees (a tracer's give / take).
constexpr int kPoolWords = 64;
constexpr int kIdWords = 64;
constexpr int kSplitSlots = 16;
constexpr int kWarpWords = kPoolWords + kIdWords + kSplitSlots * 16;

// Idle lanes take stacked subtrees: the j-th lane holding an entry stages its
// top entry in slot j (the tracer's give: the entry with its range, the ray,
// the donor's best distance and owner), and the j-th idle lane adopts slot j
// (take).  Helpers first lower their bound to their owner's best distance when
// that is nearer.
template <class Tracer, bool kAny>
__device__ __forceinline__ void share_subtrees(Tracer& T, uint32_t& st, bool owner_occluded, uint32_t* warp_words) {
    const unsigned lane = threadIdx.x & 31u;
    if (!kAny) {
        const float ob = __shfl_sync(0xFFFFFFFFu, T.best_t, owner_of(st));
        if (role_of(st) == kHelper && ob < T.best_t) { T.best_t = ob; T.best = ILM_MISS; }
    }
    const uint32_t role = role_of(st);
    const unsigned idle = __ballot_sync(0xFFFFFFFFu, role == kFree);
    const unsigned don = __ballot_sync(0xFFFFFFFFu, (role == kOwner || role == kHelper) && T.sp > 0 &&
                                                        !T.status && !(kAny && owner_occluded));
    const unsigned pairs = min(__popc(idle), __popc(don));
    if (pairs == 0u) return;
    const unsigned below = (1u << lane) - 1u;
    const unsigned irank = __popc(idle & below), drank = __popc(don & below);
    uint4* stage = reinterpret_cast<uint4*>(warp_words + kPoolWords + kIdWords);
    if (((don >> lane) & 1u) && drank < pairs) T.give(stage + 4 * drank, owner_of(st));
    __syncwarp();
    bool take = false;
    uint32_t o = 0;
    if (role == kFree && irank < pairs) {
        take = T.take(stage + 4 * irank, o);
        if (take) st = kHelper | (o << 2);
    }
    __syncwarp();
    unsigned fresh = __ballot_sync(0xFFFFFFFFu, take);
    while (fresh != 0u) {
        const int k = __ffs(fresh) - 1;
        fresh &= fresh - 1u;
        if (lane == __shfl_sync(0xFFFFFFFFu, o, k)) st += 1u << 8;
    }
}

// Helpers that finished this pass report to their owners, one at a time.
template <class Tracer, bool kAny>
__device__ __forceinline__ void merge_helpers(Tracer& T, uint32_t& st, unsigned fin) {
    const unsigned lane = threadIdx.x & 31u;
    while (fin != 0u) {
        const int k = __ffs(fin) - 1;
        fin &= fin - 1u;
        const unsigned o = __shfl_sync(0xFFFFFFFFu, owner_of(st), k);
        const float t = __shfl_sync(0xFFFFFFFFu, T.best_t, k);
        const uint32_t p = __shfl_sync(0xFFFFFFFFu, T.best, k);
        const float u = __shfl_sync(0xFFFFFFFFu, T.bu, k);
        const float v = __shfl_sync(0xFFFFFFFFu, T.bv, k);
        const uint32_t es = __shfl_sync(0xFFFFFFFFu, T.status, k);
        const int oc = __shfl_sync(0xFFFFFFFFu, (int)T.occluded, k);
        if (lane == o) {
            T.status |= es;
            if (kAny) {
                T.occluded = T.occluded || oc;
            } else if (p != ILM_MISS && (t < T.best_t || (t == T.best_t && p < T.best))) {
                T.best_t = t; T.best = p; T.bu = u; T.bv = v;
            }
            st -= 1u << 8;
        }
    }
}

// Warp-level ray claiming of the persistent schedules: kChunk rays per
// atomicAdd on a device counter.
constexpr uint32_t kChunk = 64;

}  // namespace ilm
