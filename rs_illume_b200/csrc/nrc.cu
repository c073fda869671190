// Neural radiance cache: input encoding, a 5 x 64 ReLU MLP on the BF16
// tensor cores (tcgen05.mma, FP32 accumulators in TMEM), relative-L2 loss
// and Adam.
// No counterpart in the reference (a learned component added on top of the
// path tracer); the method follows published neural radiance caching:
//   inputs: position (12-frequency sin/cos per axis, 72), outgoing direction
//   and normal (one-blob, 32 bins on each of theta/pi and phi/2pi, 128),
//   albedo (3) = 203, padded to 208;
//   layers 208->64, 4 x (64->64), 64->16 (first 3 outputs = RGB radiance),
//   ReLU between, no biases;
//   loss = mean over samples and channels of (p - y)^2 / (sg(p)^2 + 0.01).
//
// Kernels
//   k_mlp_fwd_tc<train>  forward pass: per 128-row tile a warpgroup encodes its
//                  rows straight into layer 0's A operand in shared memory,
//                  one thread issues the MMAs, each layer's accumulator comes
//                  back through tcgen05.ld as the next layer's A; training
//                  also stores the encoding and the bf16 activations
//   k_mlp_bwd_tc   loss gradient, then back through the layers the same way
//                  (transposed weights), storing dOut
//   k_wgrad_tc     dW_l = dOut_l^T * in_l for all six layers on tcgen05
//                  (M = outputs, N = inputs, K = batch rows, both operands
//                  MN-major as the rows are stored, staged by 16-byte
//                  cp.async into two buffers); split-K over the rows, one FP32
//                  partial per CTA, no atomics
//   k_reduce_adam  sums the CTA partials, Adam on the FP32 master weights,
//                  bf16 weight packs and the inference moving average
//   k_nrc_encode   the encoding alone (for inspection)
// Row counts may live in device memory (NrcCount), so the path tracer enqueues
// inference and training without reading its queue sizes on the host.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "context.h"
#include "illume_gpu.h"
#include "nrc.h"
#include "pcg32.h"

namespace ilm {
namespace nrc {

constexpr int kIn = 208, kInReal = 203, kHid = 64, kOut = 16, kLayers = 6;
__host__ __device__ constexpr int in_dim(int l) { return l == 0 ? kIn : kHid; }
__host__ __device__ constexpr int out_dim(int l) { return l == 5 ? kOut : kHid; }
// FP32 parameter offsets, row-major [out][in]
__host__ __device__ constexpr int param_off(int l) {
    return l == 0 ? 0 : kHid * kIn + (l - 1) * kHid * kHid;
}
constexpr int kParams = kHid * kIn + 4 * kHid * kHid + kOut * kHid;   // 30720
// bf16 inference pack in the tensor cores' canonical K-major layout without
// swizzle: layer l's [out][in] matrix as 8x8 core matrices of 128 contiguous
// bytes, core matrix (o/8, i/8) at (o/8 * in/8 + i/8) * 64 elements from the
// layer's start (param_off(l)), row o%8 at 8 elements, column i%8.
__host__ __device__ constexpr int tc_index(int l, int o, int i) {
    return param_off(l) + ((o >> 3) * (in_dim(l) >> 3) + (i >> 3)) * 64 + (o & 7) * 8 + (i & 7);
}
// Transposed bf16 pack for the backward pass, the same canonical layout:
// layer l >= 1 as W_l^T ([in][out], N = in, K = out), core matrix (i/8, o/8)
// at (i/8 * out/8 + o/8) * 64 elements from tcb_off(l).
__host__ __device__ constexpr int tcb_off(int l) { return (l - 1) * kHid * kHid; }   // l = 1..5
__host__ __device__ constexpr int tcb_index(int l, int o, int i) {
    return tcb_off(l) + ((i >> 3) * (out_dim(l) >> 3) + (o >> 3)) * 64 + (i & 7) * 8 + (o & 7);
}
constexpr int kTcbElems = 4 * kHid * kHid + kHid * kOut;   // 17408
constexpr float kLossEps = 0.01f;
constexpr int kMaxPartials = 148;   // CTAs of k_wgrad_tc (one FP32 partial gradient each)

struct Enc {   // position normalisation: q = (p - origin) * scale
    float x0, y0, z0, sx, sy, sz;
};

struct AdamArgs {
    float lr, b1, b2, eps;
    float ema_a;   // moving-average decay (0 = off)
    float wd;      // decoupled weight decay (AdamW; 0 = none)
};

// Optimiser counters in device memory, so that a captured training step
// replays with the right bias corrections.
struct StepState {
    int step;        // Adam steps taken
    int ema_steps;   // Adam steps since the inference weights restarted
};

__device__ __forceinline__ uint32_t rows_of(const NrcCount& c) {
    uint32_t n = c.cap;
    if (c.dev) {
        unsigned long long d = *c.dev;
        n = d < (unsigned long long)c.cap ? (uint32_t)d : c.cap;
    }
    if (c.batches > 1) n = n > c.batch ? (n - c.batch + c.batches - 1) / c.batches : 0u;
    return n;
}

// 16-byte global -> shared copy; zero-filled when !ok.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool ok) {
    uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    int sz = ok ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(sz));
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ uint32_t pack(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float lo_of(uint32_t p) { return __uint_as_float(p << 16); }
__device__ __forceinline__ float hi_of(uint32_t p) { return __uint_as_float(p & 0xFFFF0000u); }

// Copies n bf16 (a multiple of 8) from global to shared memory with 16-byte loads.
__device__ __forceinline__ void stage(__nv_bfloat16* dst, const __nv_bfloat16* src, int n) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (int i = threadIdx.x; i < n / 8; i += blockDim.x) d[i] = s[i];
}

// ---------------------------------------------------------------- encoding
// What the encoder needs of one input row.
struct RowIn {
    float q[3];     // normalised position
    float u[4];     // theta/pi, phi/2pi of the direction, then of the normal
    float alb[3];
    float ps[3], pc[3];   // encoding state: the last octave's (sin, cos) per axis
};

__device__ __forceinline__ RowIn load_row(const float* __restrict__ raw, uint32_t r, const Enc& e) {
    const float* p = raw + 12 * (size_t)r;
    RowIn v;
    v.q[0] = (p[0] - e.x0) * e.sx;
    v.q[1] = (p[1] - e.y0) * e.sy;
    v.q[2] = (p[2] - e.z0) * e.sz;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        float x = p[3 + 3 * k], y = p[4 + 3 * k], z = p[5 + 3 * k];
        v.u[2 * k] = acosf(fminf(fmaxf(z, -1.0f), 1.0f)) * (1.0f / 3.14159265358979f);
        v.u[2 * k + 1] = atan2f(y, x) * (0.5f / 3.14159265358979f) + 0.5f;
    }
    v.alb[0] = p[9];
    v.alb[1] = p[10];
    v.alb[2] = p[11];
    return v;
}

// The eight features 8 KC .. 8 KC + 7 of a row as four bf16 pairs (pair t =
// features 8 KC + 2t, 8 KC + 2t + 1).  The layout:
//   [0, 72)    axis f / 24, octave k = (f % 24) / 2: (sin, cos)(2^k pi q)
//   [72, 200)  one-blob of u[(f - 72) / 32], bin j = (f - 72) % 32:
//              exp(-((u - (j + 1/2)/32) * 32)^2 / 2)
//   200..202   albedo, then zeros
// Groups are evaluated in order (KC = 0, 1, ... 25), and two recurrences cut
// the special-function work:
//   * octaves: one sincospi per axis at octave 0, then the double angle,
//     sin 2x = 2 sin x cos x, cos 2x = (cos x - sin x)(cos x + sin x); the
//     error doubles per octave, about 2^11 float ulps at octave 11, far below
//     a bf16 ulp; the last octave of a group is kept in the row state;
//   * one-blob bins: two exps per group of 8 bins, g_j = exp(-d_j^2 / 2) and
//     the ratio r_j = g_{j+1} / g_j = exp(d_j - 1/2) (d_{j+1} = d_j - 1), then
//     g_{j+1} = g_j r_j and r_{j+1} = r_j / e; relative error grows by a few
//     ulps per step.
template <int KC>
__device__ __forceinline__ uint4 feature_group(RowIn& v) {
    constexpr int F = 8 * KC;
    uint4 q;
    if constexpr (F < 72) {
        constexpr int a = F / 24, o0 = (F % 24) >> 1;
        float s, c;
        if constexpr (o0 == 0) {
            sincospif(v.q[a], &s, &c);
        } else {
            s = 2.0f * v.ps[a] * v.pc[a];
            c = (v.pc[a] - v.ps[a]) * (v.pc[a] + v.ps[a]);
        }
        uint32_t w[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            w[t] = pack(s, c);
            if (t < 3) {
                const float s2 = 2.0f * s * c, c2 = (c - s) * (c + s);
                s = s2;
                c = c2;
            }
        }
        v.ps[a] = s;
        v.pc[a] = c;
        q = make_uint4(w[0], w[1], w[2], w[3]);
    } else if constexpr (F < 200) {
        constexpr int ui = (F - 72) >> 5, j0 = (F - 72) & 31;
        constexpr float kInvE = 0.36787944117144233f;   // e^-1
        const float d = (v.u[ui] - (j0 + 0.5f) * (1.0f / 32.0f)) * 32.0f;
        float g = __expf(-0.5f * d * d), r = __expf(d - 0.5f);
        float gv[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            gv[k] = g;
            g *= r;
            r *= kInvE;
        }
        q = make_uint4(pack(gv[0], gv[1]), pack(gv[2], gv[3]), pack(gv[4], gv[5]), pack(gv[6], gv[7]));
    } else {
        q = make_uint4(pack(v.alb[0], v.alb[1]), pack(v.alb[2], 0.0f), 0u, 0u);
    }
    return q;
}

// Whole-row encoder (104 words) for k_nrc_encode.
template <int B>
__device__ __forceinline__ void encode_row(RowIn& v, uint32_t* out) {
    const uint4 q = feature_group<B>(v);
    out[4 * B] = q.x;
    out[4 * B + 1] = q.y;
    out[4 * B + 2] = q.z;
    out[4 * B + 3] = q.w;
    if constexpr (B + 1 < kIn / 8) encode_row<B + 1>(v, out);
}

__global__ void k_nrc_encode(const float* __restrict__ raw, uint32_t n, Enc ec, __nv_bfloat16* __restrict__ enc) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    RowIn v = load_row(raw, i, ec);
    encode_row<0>(v, reinterpret_cast<uint32_t*>(enc + (size_t)i * kIn));
}

// ---------------------------------------------------------------- forward on tcgen05
// k_mlp_fwd_tc: the forward pass on the 5th-generation tensor cores.
// A CTA of 1, 2 or 4 warpgroups (blockDim / 128; few per CTA for small
// batches, so that the tiles spread over the SMs); each warpgroup owns 128-row tiles (thread t
// = row t), its own A operand buffer in shared memory, 64 TMEM columns of
// FP32 accumulator (rows = TMEM lanes) and an mbarrier.  Per tile:
//   layer 0 in two K halves (features 0-111, 112-207): the threads evaluate
//     their row's encoding into A, one thread issues tcgen05.mma
//     (M 128, N 64, K 16, bf16 x bf16 -> f32) and commits to the mbarrier;
//   layers 1-4: tcgen05.ld of the accumulator, ReLU, bf16 into A, MMA;
//   layer 5: N = 16, the first 3 columns are the output.
// Training also stores each row's encoding ([n][208] bf16) and its five
// ReLU'd activations (layer l at acts + l * ld * 64, [n][64] bf16), the bf16
// values that go into the next layer's A operand.
// The weights (61,440 bytes, all layers) are staged once per CTA.  Operands
// use the canonical K-major layout without swizzle: 8x8 core matrices of 128
// contiguous bytes; LBO = 128 bytes (next core matrix along K), SBO = the
// stride between 8-row groups.  Every mbarrier wait is bounded; a timeout
// sets kErrMlpTimeout in *err and the warpgroup stops.
constexpr int kTcGroups = 4;                                   // warpgroups per CTA, at most
constexpr int kTcHalfCols = 14;                                // core-matrix columns of an A buffer (112 features)
constexpr int kTcABytes = 128 / 8 * kTcHalfCols * 128;         // 28,672
constexpr int kTcWBytes = kParams * 2;                         // 61,440
constexpr int kTcSmem = kTcWBytes + kTcGroups * kTcABytes;     // 176,128 at 4 warpgroups
constexpr uint32_t kErrMlpTimeout = 4u;
constexpr uint32_t kTcWaitCap = 1u << 22;   // try_wait polls before a wait gives up
constexpr uint32_t kTcDrainCap = 1u << 26;  // further polls for a batch whose wait gave up

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start, LBO, SBO (bytes), version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor, kind::f16: D f32, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void group_sync(int g) {
    asm volatile("bar.sync %0, 128;" ::"r"(g + 1) : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// Row t's 8 features F..F+7 (F = 8 * KC) into core-matrix column c of an A
// buffer, and into the row's stored encoding when genc is set.
template <int KC>
__device__ __forceinline__ void put_features(uint8_t* a, int c, int row, RowIn& v, uint4* genc) {
    const uint4 q = feature_group<KC>(v);
    *reinterpret_cast<uint4*>(a + ((row >> 3) * kTcHalfCols + c) * 128 + (row & 7) * 16) = q;
    if (genc) genc[KC] = q;
}
template <int KC, int KEND>
__device__ __forceinline__ void encode_cols(uint8_t* a, int c0, int row, RowIn& v, uint4* genc) {
    put_features<KC>(a, KC - c0, row, v, genc);
    if constexpr (KC + 1 < KEND) encode_cols<KC + 1, KEND>(a, c0, row, v, genc);
}

// One warpgroup's MMA batch: layer with `ksteps` K-steps of 16, A from
// `a_base` (SBO a_sbo), B = layer weights from `w_base` (SBO w_sbo) starting at
// K-step k0; then commit and (thread 0) wait.  Returns false on a timeout.
__device__ __forceinline__ bool mma_batch(int g, int t, uint32_t tmem_d, uint32_t a_base, uint32_t a_sbo,
                                          uint32_t w_base, uint32_t w_sbo, int k0, int ksteps, int n_out,
                                          bool accumulate, uint32_t mbar, uint32_t& phase, volatile int* fail) {
    fence_proxy_async();   // the A tile written by this warpgroup, visible to the tensor core
    tc_fence_before();     // the accumulator reads above, ordered before the MMAs below
    group_sync(g);
    if (t == 0) {
        tc_fence_after();
        const uint32_t idesc = idesc_bf16(128, n_out);
        for (int k = 0; k < ksteps; ++k) {
            uint64_t da = umma_desc(a_base + (uint32_t)k * 256u, 128u, a_sbo);
            uint64_t db = umma_desc(w_base + (uint32_t)(k0 + k) * 256u, 128u, w_sbo);
            umma(tmem_d, da, db, idesc, (accumulate || k > 0) ? 1u : 0u);
        }
        umma_commit(mbar);
        uint32_t it = 0;
        while (!mbar_try_wait(mbar, phase) && ++it < kTcWaitCap) {}
        if (it >= kTcWaitCap) *fail = 1;
    }
    phase ^= 1u;
    group_sync(g);
    tc_fence_after();
    return *fail == 0;
}

// Accumulator row t (64 columns) -> ReLU -> bf16 A operand (K = 64, SBO 1024),
// and into the row's stored activation ([64] bf16) when gact is set.
__device__ __forceinline__ void acc_to_a(uint32_t tmem_row, uint8_t* a, int row, uint4* gact) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float v[16];
        tmem_ld16(tmem_row + 16 * q, v);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            uint4 w;
            w.x = pack(fmaxf(v[8 * h], 0.0f), fmaxf(v[8 * h + 1], 0.0f));
            w.y = pack(fmaxf(v[8 * h + 2], 0.0f), fmaxf(v[8 * h + 3], 0.0f));
            w.z = pack(fmaxf(v[8 * h + 4], 0.0f), fmaxf(v[8 * h + 5], 0.0f));
            w.w = pack(fmaxf(v[8 * h + 6], 0.0f), fmaxf(v[8 * h + 7], 0.0f));
            *reinterpret_cast<uint4*>(a + ((row >> 3) * 8 + 2 * q + h) * 128 + (row & 7) * 16) = w;
            if (gact) gact[2 * q + h] = w;
        }
    }
}

// TMEM, barriers and failure flags of a tcgen05 MLP kernel: allocation of
// 64 columns per warpgroup (64, 128 or 256: powers of two) by warp 0 and the
// fences that publish them.
__device__ __forceinline__ void tc_setup(uint64_t* mbar, int* fail, uint32_t* tmem_base) {
    const uint32_t groups = blockDim.x >> 7;
    if (threadIdx.x < groups) {
        mbar_init(smem_u32(&mbar[threadIdx.x]));
        fail[threadIdx.x] = 0;
    }
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_base)),
                     "r"(64u * groups));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

// Reports a timed-out wait and frees the TMEM.  Every warpgroup has stopped
// issuing by then: its last batch was committed and waited for, or its wait
// gave up.  A warpgroup whose wait gave up first drains that batch: its issuing
// thread waits again, up to kTcDrainCap more polls, on the same mbarrier phase
// (the parity before mma_batch's flip, phase ^ 1), so tcgen05.dealloc does not
// free columns an MMA may still write.  If the drain runs out too, the columns
// are freed all the same -- a CTA that kept them would leave the tcgen05.alloc
// of later CTAs on its SM waiting -- and the error word marks the launch's
// results as invalid.  The CTA barrier below follows every warpgroup's exit.
__device__ __forceinline__ void tc_teardown(const int* fail, uint32_t tmem_base, uint32_t* err, uint32_t mbar,
                                            uint32_t phase) {
    const int g = threadIdx.x >> 7;
    if ((threadIdx.x & 127) == 0 && fail[g]) {
        uint32_t it = 0;
        while (!mbar_try_wait(mbar, phase ^ 1u) && ++it < kTcDrainCap) {}
        atomicOr(err, kErrMlpTimeout);
    }
    tc_fence_before();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(64u * (blockDim.x >> 7)));
    }
}

template <bool kTrain>
__global__ void __launch_bounds__(128 * kTcGroups, 1) k_mlp_fwd_tc(const float* __restrict__ raw, NrcCount cnt,
                                                                   Enc ec, const __nv_bfloat16* __restrict__ wtc,
                                                                   float* __restrict__ out, uint32_t* err,
                                                                   uint32_t ld, __nv_bfloat16* __restrict__ acts,
                                                                   __nv_bfloat16* __restrict__ enc) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ __align__(8) uint64_t mbar[kTcGroups];
    __shared__ int fail[kTcGroups];
    __shared__ uint32_t tmem_base;
    const int warp = threadIdx.x >> 5, g = warp >> 2, t = threadIdx.x & 127;
    // stage the weights; barriers; TMEM (64 columns per warpgroup)
    {
        const uint4* src = reinterpret_cast<const uint4*>(wtc);
        uint4* dst = reinterpret_cast<uint4*>(tc_smem);
        for (int k = threadIdx.x; k < kTcWBytes / 16; k += blockDim.x) dst[k] = src[k];
    }
    tc_setup(mbar, fail, &tmem_base);
    const uint32_t n = rows_of(cnt);
    const uint32_t tmem_d = tmem_base + 64u * g;                          // this warpgroup's columns
    const uint32_t tmem_row = tmem_d + ((uint32_t)(32 * (warp & 3)) << 16);   // this warp's lanes
    uint8_t* a = tc_smem + kTcWBytes + g * kTcABytes;
    const uint32_t a_base = smem_u32(a), w_base = smem_u32(tc_smem);
    const uint32_t mb = smem_u32(&mbar[g]);
    uint32_t phase = 0;
    const uint32_t tiles = (n + 127) / 128;
    const uint32_t groups = blockDim.x >> 7;
    for (uint32_t tile = blockIdx.x * groups + g; tile < tiles; tile += gridDim.x * groups) {
        const uint32_t row = tile * 128 + t;
        const bool keep = kTrain && row < n;
        RowIn v = {};
        if (row < n) v = load_row(raw, row, ec);
        uint4* genc = keep ? reinterpret_cast<uint4*>(enc + (size_t)row * kIn) : nullptr;
        // layer 0, features 0-111 (K-steps 0-6)
        encode_cols<0, kTcHalfCols>(a, 0, t, v, genc);
        if (!mma_batch(g, t, tmem_d, a_base, kTcHalfCols * 128, w_base + 2 * param_off(0), 26 * 128, 0, 7, 64,
                       false, mb, phase, &fail[g]))
            break;
        // features 112-207 (K-steps 7-12), accumulated
        encode_cols<kTcHalfCols, 26>(a, kTcHalfCols, t, v, genc);
        if (!mma_batch(g, t, tmem_d, a_base, kTcHalfCols * 128, w_base + 2 * param_off(0), 26 * 128, 7, 6, 64,
                       true, mb, phase, &fail[g]))
            break;
        bool ok = true;
        for (int l = 1; l <= 5 && ok; ++l) {
            acc_to_a(tmem_row, a, t,
                     keep ? reinterpret_cast<uint4*>(acts + (size_t)(l - 1) * ld * kHid + (size_t)row * kHid) : nullptr);
            ok = mma_batch(g, t, tmem_d, a_base, 8 * 128, w_base + 2 * param_off(l), 8 * 128, 0, 4, l == 5 ? 16 : 64,
                           false, mb, phase, &fail[g]);
        }
        if (!ok) break;
        float o[16];
        tmem_ld16(tmem_row, o);
        if (row < n) {
            out[3 * (size_t)row] = o[0];
            out[3 * (size_t)row + 1] = o[1];
            out[3 * (size_t)row + 2] = o[2];
        }
    }
    tc_teardown(fail, tmem_base, err, mb, phase);
}

// ---------------------------------------------------------------- inference on tcgen05, two tiles per warpgroup
// k_mlp_infer_tc: the inference forward with two 128-row tiles in flight per
// warpgroup.  Each tile (slot) has its own A buffer (128 rows x 64 features,
// 16 KB), its own 64 TMEM columns and its own mbarrier; the warpgroup
// alternates between its slots, so while one slot's MMAs run the threads
// produce the other slot's next A operand (encoding or accumulator -> ReLU ->
// bf16).  Layer 0 is issued in four parts of K = 64, 64, 64 and 16 features
// (features 0-63, 64-127, 128-191, 192-207), so an A buffer holds 64
// features; a tile takes nine MMA batches (four layer-0 parts, five layers).
// With 4 warpgroups per CTA, 8 tiles are in flight per SM (192,512 bytes of
// shared memory, all 512 TMEM columns).  Waits are bounded; a warpgroup
// whose wait gives up drains both slots' last commits before the TMEM is
// freed.
constexpr int kInfABytes = 128 / 8 * 8 * 128;                        // 16,384
constexpr int kInfSmem = kTcWBytes + kTcGroups * 2 * kInfABytes;      // 192,512

// The features of layer-0 part p (groups 8p .. 8p + 7, at most 25) into
// columns 0.. of an A buffer (8 core-matrix columns, SBO 1024).
template <int KC, int KEND>
__device__ __forceinline__ void encode_part(uint8_t* a, int c0, int row, RowIn& v) {
    const uint4 q = feature_group<KC>(v);
    *reinterpret_cast<uint4*>(a + ((row >> 3) * 8 + (KC - c0)) * 128 + (row & 7) * 16) = q;
    if constexpr (KC + 1 < KEND) encode_part<KC + 1, KEND>(a, c0, row, v);
}

// Issues one batch (no wait): fences, group barrier, one thread issues and
// commits to the slot's mbarrier.
__device__ __forceinline__ void inf_issue(int g, int t, uint32_t tmem_d, uint32_t a_base, uint32_t a_sbo,
                                          uint32_t w_base, uint32_t w_sbo, int k0, int ksteps, int n_out,
                                          bool accumulate, uint32_t mbar) {
    fence_proxy_async();
    tc_fence_before();
    group_sync(g);
    if (t == 0) {
        tc_fence_after();
        const uint32_t idesc = idesc_bf16(128, n_out);
        for (int k = 0; k < ksteps; ++k) {
            const uint64_t da = umma_desc(a_base + (uint32_t)k * 256u, 128u, a_sbo);
            const uint64_t db = umma_desc(w_base + (uint32_t)(k0 + k) * 256u, 128u, w_sbo);
            umma(tmem_d, da, db, idesc, (accumulate || k > 0) ? 1u : 0u);
        }
        umma_commit(mbar);
    }
}

// Waits for the slot's last batch (issuing thread, bounded); false on a timeout.
__device__ __forceinline__ bool inf_wait(int g, int t, uint32_t mbar, uint32_t& phase, volatile int* fail) {
    if (t == 0) {
        uint32_t it = 0;
        while (!mbar_try_wait(mbar, phase) && ++it < kTcWaitCap) {}
        if (it >= kTcWaitCap) *fail = 1;
    }
    phase ^= 1u;
    group_sync(g);
    tc_fence_after();
    return *fail == 0;
}

// Batch k (0-8) of the slot's tile: its A operand, then the issue.
__device__ __forceinline__ void inf_step(int k, int g, int t, uint8_t* a, uint32_t a_base, uint32_t w_base,
                                         uint32_t tmem_d, uint32_t tmem_row, RowIn& v, uint32_t mbar) {
    if (k < 4) {
        switch (k) {
            case 0: encode_part<0, 8>(a, 0, t, v); break;
            case 1: encode_part<8, 16>(a, 8, t, v); break;
            case 2: encode_part<16, 24>(a, 16, t, v); break;
            default: encode_part<24, 26>(a, 24, t, v); break;
        }
        inf_issue(g, t, tmem_d, a_base, 8 * 128, w_base + 2 * param_off(0), 26 * 128, 4 * k, k < 3 ? 4 : 1, 64,
                  k > 0, mbar);
    } else {
        const int l = k - 3;
        acc_to_a(tmem_row, a, t, nullptr);
        inf_issue(g, t, tmem_d, a_base, 8 * 128, w_base + 2 * param_off(l), 8 * 128, 0, 4, l == 5 ? 16 : 64, false,
                  mbar);
    }
}

__global__ void __launch_bounds__(128 * kTcGroups, 1) k_mlp_infer_tc(const float* __restrict__ raw, NrcCount cnt,
                                                                     Enc ec, const __nv_bfloat16* __restrict__ wtc,
                                                                     float* __restrict__ out, uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ __align__(8) uint64_t mbar[2 * kTcGroups];
    __shared__ int fail[kTcGroups];
    __shared__ uint32_t tmem_base;
    const int warp = threadIdx.x >> 5, g = warp >> 2, t = threadIdx.x & 127;
    const uint32_t groups = blockDim.x >> 7;
    {
        const uint4* src = reinterpret_cast<const uint4*>(wtc);
        uint4* dst = reinterpret_cast<uint4*>(tc_smem);
        for (int k = threadIdx.x; k < kTcWBytes / 16; k += blockDim.x) dst[k] = src[k];
    }
    if (threadIdx.x < 2 * groups) mbar_init(smem_u32(&mbar[threadIdx.x]));
    if (threadIdx.x < groups) fail[threadIdx.x] = 0;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(128u * groups));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t n = rows_of(cnt);
    const uint32_t w_base = smem_u32(tc_smem);
    // per slot: A buffer, TMEM columns (and this warp's lanes), mbarrier
    auto a_of = [&](int sl) { return tc_smem + kTcWBytes + (2 * g + sl) * kInfABytes; };
    auto tmem_of = [&](int sl) { return tmem_base + 64u * (2u * g + sl); };
    auto lanes_of = [&](int sl) { return tmem_of(sl) + ((uint32_t)(32 * (warp & 3)) << 16); };
    auto mb_of = [&](int sl) { return smem_u32(&mbar[2 * g + sl]); };
    uint32_t phase[2] = {0u, 0u};
    // a committed batch not yet waited for, and its phase parity
    bool pending[2] = {false, false};
    uint32_t pend_par[2] = {0u, 0u};
    const uint32_t tiles = (n + 127) / 128, pairs = (tiles + 1) / 2;
    bool ok = true;
    for (uint32_t pr = blockIdx.x * groups + g; pr < pairs && ok; pr += gridDim.x * groups) {
        RowIn v[2];
#pragma unroll
        for (int sl = 0; sl < 2; ++sl) {
            const uint32_t row = (2 * pr + sl) * 128 + t;
            v[sl] = RowIn{};
            if (row < n) v[sl] = load_row(raw, row, ec);
        }
        for (int k = 0; k < 9 && ok; ++k) {
#pragma unroll
            for (int sl = 0; sl < 2; ++sl) {
                if (k > 0) {
                    ok = inf_wait(g, t, mb_of(sl), phase[sl], &fail[g]);
                    if (!ok) break;
                    pending[sl] = false;
                }
                pend_par[sl] = phase[sl];
                uint8_t* buf = a_of(sl);
                inf_step(k, g, t, buf, smem_u32(buf), w_base, tmem_of(sl), lanes_of(sl), v[sl], mb_of(sl));
                pending[sl] = true;
            }
        }
        if (!ok) break;
#pragma unroll
        for (int sl = 0; sl < 2; ++sl) {
            ok = ok && inf_wait(g, t, mb_of(sl), phase[sl], &fail[g]);
            if (!ok) break;
            pending[sl] = false;
            float o[16];
            tmem_ld16(lanes_of(sl), o);
            const uint32_t row = (2 * pr + sl) * 128 + t;
            if (row < n) {
                out[3 * (size_t)row] = o[0];
                out[3 * (size_t)row + 1] = o[1];
                out[3 * (size_t)row + 2] = o[2];
            }
        }
    }
    // a wait that gave up: drain both slots' outstanding commits, then
    // report; see tc_teardown
    if (t == 0 && fail[g]) {
#pragma unroll
        for (int sl = 0; sl < 2; ++sl) {
            if (!pending[sl]) continue;
            uint32_t it = 0;
            while (!mbar_try_wait(mb_of(sl), pend_par[sl]) && ++it < kTcDrainCap) {}
        }
        atomicOr(err, kErrMlpTimeout);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(128u * groups));
    }
}

// ---------------------------------------------------------------- backward on tcgen05
// k_mlp_bwd_tc: loss gradient (mean over the n rows and 3 channels), then
// dOut of every layer back to the input (layer l at douts + l * ld * 64:
// layers 0-4 [n][64], layer 5 [n][16]); accumulates the loss sum.  The tile
// scheme of k_mlp_fwd_tc: thread t of a warpgroup owns row t, writes its
// dOut_l into the A operand (K-major, no swizzle) and one thread issues
// dAct_{l-1} = dOut_l * W_l with B = W_l^T from the transposed pack (N = 64
// inputs, K = the layer's outputs: 16 for layer 5, else 64).  dOut_l is
// dAct_l where layer l's stored activation is positive (ReLU), else 0.
constexpr int kTcbWBytes = kTcbElems * 2;                       // 34,816
constexpr int kTcbABytes = 128 / 8 * 8 * 128;                  // 16,384 (K = 64)
constexpr int kTcbSmem = kTcbWBytes + kTcGroups * kTcbABytes;   // 100,352 at 4 warpgroups

__global__ void __launch_bounds__(128 * kTcGroups, 1) k_mlp_bwd_tc(const float* __restrict__ pred,
                                                                   const float* __restrict__ target, NrcCount cnt,
                                                                   uint32_t ld, const __nv_bfloat16* __restrict__ acts,
                                                                   const __nv_bfloat16* __restrict__ wtcb,
                                                                   __nv_bfloat16* __restrict__ douts,
                                                                   float* __restrict__ loss_sum, uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ __align__(8) uint64_t mbar[kTcGroups];
    __shared__ int fail[kTcGroups];
    __shared__ uint32_t tmem_base;
    const int warp = threadIdx.x >> 5, g = warp >> 2, t = threadIdx.x & 127;
    {
        const uint4* src = reinterpret_cast<const uint4*>(wtcb);
        uint4* dst = reinterpret_cast<uint4*>(tc_smem);
        for (int k = threadIdx.x; k < kTcbWBytes / 16; k += blockDim.x) dst[k] = src[k];
    }
    tc_setup(mbar, fail, &tmem_base);
    const uint32_t n = rows_of(cnt);
    const float scale = n > 0 ? 1.0f / (3.0f * (float)n) : 0.0f;
    const uint32_t tmem_d = tmem_base + 64u * g;
    const uint32_t tmem_row = tmem_d + ((uint32_t)(32 * (warp & 3)) << 16);
    uint8_t* a = tc_smem + kTcbWBytes + g * kTcbABytes;
    const uint32_t a_base = smem_u32(a), w_base = smem_u32(tc_smem);
    const uint32_t mb = smem_u32(&mbar[g]);
    uint32_t phase = 0;
    float loss = 0.0f;
    const uint32_t tiles = (n + 127) / 128;
    const uint32_t groups = blockDim.x >> 7;
    for (uint32_t tile = blockIdx.x * groups + g; tile < tiles; tile += gridDim.x * groups) {
        const uint32_t row = tile * 128 + t;
        const bool ok = row < n;
        // dL/dpred of the row's 3 channels -> dOut5 (K = 16: two core-matrix columns)
        float d[3] = {0.0f, 0.0f, 0.0f};
        if (ok) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float p = pred[3 * (size_t)row + c], y = target[3 * (size_t)row + c];
                const float den = p * p + kLossEps, e = p - y;
                loss += e * e / den;
                d[c] = 2.0f * e / den * scale;
            }
        }
        const uint4 q0 = make_uint4(pack(d[0], d[1]), pack(d[2], 0.0f), 0u, 0u), q1 = make_uint4(0u, 0u, 0u, 0u);
        if (ok) {
            uint4* g5 = reinterpret_cast<uint4*>(douts + (size_t)5 * ld * kHid + (size_t)row * kOut);
            g5[0] = q0;
            g5[1] = q1;
        }
        *reinterpret_cast<uint4*>(a + ((t >> 3) * 2) * 128 + (t & 7) * 16) = q0;
        *reinterpret_cast<uint4*>(a + ((t >> 3) * 2 + 1) * 128 + (t & 7) * 16) = q1;
        // dAct4 = dOut5 * W5
        if (!mma_batch(g, t, tmem_d, a_base, 2 * 128, w_base + 2 * tcb_off(5), 2 * 128, 0, 1, 64, false, mb, phase,
                       &fail[g]))
            break;
        bool go = true;
        for (int l = 4; l >= 0 && go; --l) {
            const uint4* gact = reinterpret_cast<const uint4*>(acts + (size_t)l * ld * kHid + (size_t)row * kHid);
            uint4* gd = reinterpret_cast<uint4*>(douts + (size_t)l * ld * kHid + (size_t)row * kHid);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float v[16];
                tmem_ld16(tmem_row + 16 * q, v);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint4 m = ok ? gact[2 * q + h] : make_uint4(0u, 0u, 0u, 0u);
                    const uint32_t mw[4] = {m.x, m.y, m.z, m.w};
                    uint32_t w[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const float lo = lo_of(mw[k]) > 0.0f ? v[8 * h + 2 * k] : 0.0f;
                        const float hi = hi_of(mw[k]) > 0.0f ? v[8 * h + 2 * k + 1] : 0.0f;
                        w[k] = pack(lo, hi);
                    }
                    const uint4 wv = make_uint4(w[0], w[1], w[2], w[3]);
                    if (ok) gd[2 * q + h] = wv;
                    *reinterpret_cast<uint4*>(a + ((t >> 3) * 8 + 2 * q + h) * 128 + (t & 7) * 16) = wv;
                }
            }
            if (l == 0) break;
            // dAct_{l-1} = dOut_l * W_l
            go = mma_batch(g, t, tmem_d, a_base, 8 * 128, w_base + 2 * tcb_off(l), 8 * 128, 0, 4, 64, false, mb,
                           phase, &fail[g]);
        }
        if (!go) break;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
    if ((threadIdx.x & 31) == 0 && loss != 0.0f) atomicAdd(loss_sum, loss);
    tc_teardown(fail, tmem_base, err, mb, phase);
}

// ---------------------------------------------------------------- weight gradient on tcgen05
// k_wgrad_tc: dW_l[o][i] = sum over rows r of dOut_l[r][o] * in_l[r][i], split
// over the batch rows and the six layers: CTA (c, l) takes layer l's rows
// [c * R, (c + 1) * R) and writes layer l's slice of partial c (k_reduce_adam
// sums the partials).  One warpgroup per CTA; D = A * B with M = o, N = i
// (208 or 64), K = rows, FP32 D in TMEM (256 or 64 columns).
// Both operands are MN-major without swizzle, which is how the rows are stored
// (features contiguous): a core matrix is 8 consecutive rows (K) x 8 features
// (MN), 16 contiguous bytes per row, so staging is one 16-byte cp.async per
// (row, 8 features), no transpose.
//   A (dOut_l^T): core matrix (o/8, r/8) at (r/8) * LBO_A + (o/8) * 128,
//                 LBO_A = O * 16 (an 8-row group of all O outputs), SBO = 128;
//   B (in_l):     core matrix (i/8, r/8) at (r/8) * LBO_B + (i/8) * 128,
//                 LBO_B = I * 16, SBO = 128.
// The MMA has M = 128 and the layer O = 64 or 16 real rows: the descriptor's
// MN groups past O/8 read the bytes that follow (the next 8-row groups, and up
// to kWgPad bytes past the tile, reserved), and the D rows they give are never
// read.  Rows are staged kWgRows at a time into two buffers: one buffer's MMAs
// run while the other fills.  Waits are bounded as in the forward kernel.
constexpr int kWgRows = 64;                                   // rows per staging step (4 MMAs of K = 16)
constexpr int kWgPad = 2048;                                  // bytes past an A tile its descriptor reads
constexpr int kWgABytes = kWgRows / 8 * kHid * 16 + kWgPad;   // 10,240
constexpr int kWgBBytes = kWgRows / 8 * kIn * 16;             // 26,624
constexpr int kWgBuf = kWgABytes + kWgBBytes;                 // 36,864
constexpr int kWgSmem = 2 * kWgBuf;                           // 73,728
constexpr int kWgMinRows = 256;                               // rows per CTA, at least

__device__ __forceinline__ uint32_t idesc_bf16_mn(int m, int n) {
    return idesc_bf16(m, n) | (1u << 15) | (1u << 16);        // A and B MN-major
}

// Layer l's operand tiles for rows r0 .. r0 + kWgRows - 1 (zeros past n).
__device__ __forceinline__ void wg_stage(uint8_t* buf, int l, uint32_t r0, uint32_t n, uint32_t ld,
                                         const __nv_bfloat16* __restrict__ enc, const __nv_bfloat16* __restrict__ acts,
                                         const __nv_bfloat16* __restrict__ douts) {
    const int O = out_dim(l), I = in_dim(l);
    const __nv_bfloat16* dsrc = douts + (size_t)l * ld * kHid;
    const __nv_bfloat16* isrc = l == 0 ? enc : acts + (size_t)(l - 1) * ld * kHid;
    const int oc = O / 8, ic = I / 8;
    uint8_t* a = buf;
    uint8_t* b = buf + kWgABytes;
    for (int e = threadIdx.x; e < kWgRows * (oc + ic); e += blockDim.x) {
        const int r = e / (oc + ic), c = e - r * (oc + ic);
        const uint32_t row = r0 + (uint32_t)r;
        const bool ok = row < n;
        const size_t src_row = ok ? row : 0;
        if (c < oc)
            cp_async16(a + (r >> 3) * (O * 16) + c * 128 + (r & 7) * 16, dsrc + src_row * O + c * 8, ok);
        else
            cp_async16(b + (r >> 3) * (I * 16) + (c - oc) * 128 + (r & 7) * 16, isrc + src_row * I + (c - oc) * 8, ok);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// Bounded wait of the issuing thread on an mbarrier phase; false on a timeout.
__device__ __forceinline__ bool wg_wait(uint32_t mbar, uint32_t parity) {
    uint32_t it = 0;
    while (!mbar_try_wait(mbar, parity) && ++it < kTcWaitCap) {}
    return it < kTcWaitCap;
}

// Also advances the step counters (read by k_reduce_adam, which follows).
__global__ void __launch_bounds__(128, 1) k_wgrad_tc(NrcCount cnt, uint32_t ld, uint32_t rows_per_cta,
                                                     const __nv_bfloat16* __restrict__ enc,
                                                     const __nv_bfloat16* __restrict__ acts,
                                                     const __nv_bfloat16* __restrict__ douts,
                                                     float* __restrict__ partial, StepState* st, int do_step,
                                                     uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t wg_smem[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ int fail[1];
    __shared__ uint32_t tmem_base;
    const uint32_t n = rows_of(cnt);
    if (do_step && n > 0 && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {   // an empty batch takes no step
        st->step += 1;
        st->ema_steps += 1;
    }
    const int t = threadIdx.x, warp = t >> 5;
    const int l = blockIdx.y;                        // this CTA's layer
    const uint32_t cols = l == 0 ? 256u : 64u;       // TMEM columns: N = 208 or 64, a power of two
    if (t < 2) mbar_init(smem_u32(&mbar[t]));
    if (t == 0) fail[0] = 0;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_d = tmem_base;
    const uint32_t row0 = blockIdx.x * rows_per_cta;
    const int steps = (int)(rows_per_cta / kWgRows);
    float* part = partial + (size_t)blockIdx.x * kParams;
    bool ok = true;
    // the issuing thread's last commit (barrier and phase parity): a later
    // commit covers every earlier MMA, so a drain waits on this one
    uint32_t last_bar = 0, last_parity = 0;
    wg_stage(wg_smem, l, row0, n, ld, enc, acts, douts);
    for (int s = 0; s < steps && ok; ++s) {
        const int b = s & 1;
        uint8_t* buf = wg_smem + b * kWgBuf;
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        fence_proxy_async();        // this thread's copies, visible to the tensor core
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
            const int O = out_dim(l), I = in_dim(l);
            const uint32_t a0 = smem_u32(buf), b0 = smem_u32(buf + kWgABytes);
            const uint32_t idesc = idesc_bf16_mn(128, I);
#pragma unroll 1
            for (int ks = 0; ks < kWgRows / 16; ++ks) {
                const uint64_t da = umma_desc(a0 + (uint32_t)(ks * 2 * O * 16), (uint32_t)(O * 16), 128u);
                const uint64_t db = umma_desc(b0 + (uint32_t)(ks * 2 * I * 16), (uint32_t)(I * 16), 128u);
                umma(tmem_d, da, db, idesc, (s > 0 || ks > 0) ? 1u : 0u);
            }
            umma_commit(smem_u32(&mbar[b]));
            last_bar = smem_u32(&mbar[b]);
            last_parity = (uint32_t)(s >> 1) & 1u;
        }
        // refill the other buffer with step s + 1 once step s - 1's MMAs (its
        // last reader) are done
        if (s + 1 < steps) {
            if (s >= 1) {
                if (t == 0 && !wg_wait(smem_u32(&mbar[b ^ 1]), ((s - 1) >> 1) & 1)) fail[0] = 1;
                __syncthreads();
                if (fail[0]) { ok = false; break; }
            }
            wg_stage(wg_smem + (b ^ 1) * kWgBuf, l, row0 + (uint32_t)((s + 1) * kWgRows), n, ld, enc, acts, douts);
        }
        if (s == steps - 1) {
            // layer l complete: D rows o < O to this CTA's partial
            if (t == 0 && !wg_wait(smem_u32(&mbar[b]), (s >> 1) & 1)) fail[0] = 1;
            __syncthreads();
            if (fail[0]) { ok = false; break; }
            tc_fence_after();
            const int O = out_dim(l), I = in_dim(l);
            if (warp * 32 < O) {
                float* dst = part + param_off(l) + (size_t)(warp * 32 + (t & 31)) * I;
                const bool real = warp * 32 + (t & 31) < O;
                for (int c0 = 0; c0 < I; c0 += 16) {
                    float v[16];
                    tmem_ld16(tmem_d + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
                    if (real) {
                        float4* d4 = reinterpret_cast<float4*>(dst + c0);
                        d4[0] = make_float4(v[0], v[1], v[2], v[3]);
                        d4[1] = make_float4(v[4], v[5], v[6], v[7]);
                        d4[2] = make_float4(v[8], v[9], v[10], v[11]);
                        d4[3] = make_float4(v[12], v[13], v[14], v[15]);
                    }
                }
            }
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    // a wait that gave up: drain the last commit before the TMEM is freed
    // (as tc_teardown does), then report
    if (t == 0 && fail[0]) {
        uint32_t it = 0;
        while (!mbar_try_wait(last_bar, last_parity) && ++it < kTcDrainCap) {}
        atomicOr(err, kErrMlpTimeout);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(cols));
    }
}

// ---------------------------------------------------------------- optimiser
__device__ __forceinline__ void param_coords(int p, int& l, int& o, int& i) {
    l = 0;
    while (l < 5 && p >= param_off(l + 1)) ++l;
    int local = p - param_off(l), in = in_dim(l);
    o = local / in;
    i = local - o * in;
}

// grad = sum of the CTA partials; with do_step, Adam on the FP32 master
// weights (bias corrections 1 - beta^step; rows 3..15 of the output layer and
// the padded inputs stay zero), the bf16 training packs (forward and
// transposed, both in the tensor cores' canonical layout), and the inference
// pack: with ema_a > 0, ema = ema_a * ema + (1 - ema_a) * w (ema
// starts at 0) and the pack holds ema / (1 - ema_a^ema_steps), else w.
__global__ void k_reduce_adam(const float* __restrict__ partial, int n_part, NrcCount cnt, float* __restrict__ grad,
                              float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, AdamArgs ar,
                              const StepState* __restrict__ st, int do_step, __nv_bfloat16* __restrict__ wtc,
                              __nv_bfloat16* __restrict__ wtcb, float* __restrict__ ema,
                              __nv_bfloat16* __restrict__ winf) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float gsum = 0.0f;
    for (int k = 0; k < n_part; ++k) gsum += partial[(size_t)k * kParams + p];
    grad[p] = gsum;
    if (!do_step || rows_of(cnt) == 0) return;
    const float step = (float)st->step;
    const float c1 = 1.0f - powf(ar.b1, step), c2 = 1.0f - powf(ar.b2, step);
    int l, o, i;
    param_coords(p, l, o, i);
    float x = w[p];
    bool frozen = (l == 5 && o >= 3) || (l == 0 && i >= kInReal);
    if (!frozen) {
        float mm = ar.b1 * m[p] + (1.0f - ar.b1) * gsum;
        float vv = ar.b2 * v[p] + (1.0f - ar.b2) * gsum * gsum;
        m[p] = mm;
        v[p] = vv;
        x -= ar.lr * ((mm / c1) / (sqrtf(vv / c2) + ar.eps) + ar.wd * x);
        w[p] = x;
    }
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    wtc[tc_index(l, o, i)] = h;
    if (l >= 1) wtcb[tcb_index(l, o, i)] = h;
    float xi = x;
    if (ar.ema_a > 0.0f) {
        float e = ar.ema_a * ema[p] + (1.0f - ar.ema_a) * x;
        ema[p] = e;
        xi = e / (1.0f - powf(ar.ema_a, (float)st->ema_steps));
    }
    winf[tc_index(l, o, i)] = __float2bfloat16_rn(xi);
}

// Packs the master weights (after creation or replacement) and restarts the
// moving average: the inference pack holds w.
__global__ void k_pack(const float* __restrict__ w, __nv_bfloat16* __restrict__ wtc,
                       __nv_bfloat16* __restrict__ wtcb, float* __restrict__ ema, __nv_bfloat16* __restrict__ winf,
                       StepState* st) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) st->ema_steps = 0;
    if (p >= kParams) return;
    int l, o, i;
    param_coords(p, l, o, i);
    __nv_bfloat16 h = __float2bfloat16_rn(w[p]);
    wtc[tc_index(l, o, i)] = h;
    winf[tc_index(l, o, i)] = h;
    if (l >= 1) wtcb[tcb_index(l, o, i)] = h;
    ema[p] = 0.0f;
}

}  // namespace nrc
}  // namespace ilm

using namespace ilm;
using namespace ilm::nrc;

struct ilm_nrc {
    ilm_nrc_config cfg;
    DeviceBuffer state;                          // StepState
    DeviceBuffer w, m, v, grad, wtc, wtcb;       // params and their training packs
    DeviceBuffer ema, winf;                      // moving average and its inference pack
    DeviceBuffer partial;                        // k_wgrad_tc partial sums
    DeviceBuffer err;                            // device error word (kErrMlpTimeout)
    DeviceBuffer raw, enc, out, target, acts, douts, loss;
    cudaStream_t stream = nullptr;
    ~ilm_nrc() {
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// Launch shape of a tcgen05 MLP kernel for n rows: one 128-row tile per
// warpgroup in flight, 4 warpgroups per CTA when the tiles fill the SMs that
// way, else 2 or 1 so that they spread over more SMs (up to 2 CTAs per SM:
// TMEM and shared memory allow it); each CTA stages the weights once and
// strides over tiles.
struct TcLaunch {
    unsigned grid, threads;
    size_t smem;
};
TcLaunch tc_launch(uint32_t n, int w_bytes, int a_bytes) {
    const uint32_t tiles = (n + 127) / 128;
    const uint32_t groups = tiles >= 4u * 148u ? 4u : (tiles >= 2u * 148u ? 2u : 1u);
    uint32_t grid = (tiles + groups - 1) / groups;
    const uint32_t cap = groups == 4 ? 148u : 296u;
    grid = grid < 1 ? 1 : (grid > cap ? cap : grid);
    return {grid, 128u * groups, (size_t)w_bytes + groups * (size_t)a_bytes};
}

Enc enc_params(const ilm_nrc* h) {
    const float* b = h->cfg.bound;
    return Enc{b[0], b[1], b[2], 1.0f / fmaxf(b[3] - b[0], 1e-12f), 1.0f / fmaxf(b[4] - b[1], 1e-12f),
               1.0f / fmaxf(b[5] - b[2], 1e-12f)};
}

cudaError_t pack(ilm_nrc* h, cudaStream_t s) {
    k_pack<<<(kParams + 255) / 256, 256, 0, s>>>(
        static_cast<const float*>(h->w.ptr), static_cast<__nv_bfloat16*>(h->wtc.ptr),
        static_cast<__nv_bfloat16*>(h->wtcb.ptr), static_cast<float*>(h->ema.ptr),
        static_cast<__nv_bfloat16*>(h->winf.ptr), static_cast<StepState*>(h->state.ptr));
    return cudaGetLastError();
}

// Rows per batch that a count can give (the batch's share of the cap).
uint32_t batch_cap(const NrcCount& c) { return c.batches > 1 ? (c.cap + c.batches - 1) / c.batches : c.cap; }

cudaError_t reserve_train(ilm_nrc* h, uint32_t rows) {
    cudaError_t e;
    if ((e = h->enc.reserve((size_t)rows * kIn * 2)) != cudaSuccess) return e;
    if ((e = h->out.reserve((size_t)rows * 3 * 4)) != cudaSuccess) return e;
    if ((e = h->acts.reserve((size_t)rows * 5 * kHid * 2)) != cudaSuccess) return e;
    return h->douts.reserve((size_t)rows * 6 * kHid * 2);
}

// Training runs on the current weights and stores the encoding and the
// activations (layer stride = the batch's row cap); inference runs on the
// moving-average pack.
cudaError_t forward(ilm_nrc* h, const float* raw, NrcCount cnt, bool train, float* out, cudaStream_t s) {
    const uint32_t rows = batch_cap(cnt);
    uint32_t* err = static_cast<uint32_t*>(h->err.ptr);
    const TcLaunch L = tc_launch(rows, kTcWBytes, kTcABytes);
    if (train)
        k_mlp_fwd_tc<true><<<L.grid, L.threads, L.smem, s>>>(
            raw, cnt, enc_params(h), static_cast<const __nv_bfloat16*>(h->wtc.ptr), out, err, rows,
            static_cast<__nv_bfloat16*>(h->acts.ptr), static_cast<__nv_bfloat16*>(h->enc.ptr));
    else {
        // inference: two tiles per warpgroup, 4 warpgroups per CTA, one CTA per SM
        const uint32_t pairs = (rows + 255) / 256;   // two 128-row tiles per pair
        const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(148, (pairs + kTcGroups - 1) / kTcGroups));
        k_mlp_infer_tc<<<grid, 128 * kTcGroups, kInfSmem, s>>>(
            raw, cnt, enc_params(h), static_cast<const __nv_bfloat16*>(h->winf.ptr), out, err);
    }
    return cudaGetLastError();
}

// Loss gradient into h->grad (and the loss sum into h->loss, zeroed first);
// with do_step, one Adam step.
cudaError_t train_rows(ilm_nrc* h, const float* raw, const float* target, NrcCount cnt, int do_step,
                       cudaStream_t s) {
    cudaError_t e;
    const uint32_t cap = batch_cap(cnt);   // layer stride of acts / douts
    if ((e = reserve_train(h, cap)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(h->loss.ptr, 0, 4, s)) != cudaSuccess) return e;
    float* pred = static_cast<float*>(h->out.ptr);
    if ((e = forward(h, raw, cnt, true, pred, s)) != cudaSuccess) return e;
    const __nv_bfloat16* acts = static_cast<const __nv_bfloat16*>(h->acts.ptr);
    __nv_bfloat16* douts = static_cast<__nv_bfloat16*>(h->douts.ptr);
    const TcLaunch L = tc_launch(cap, kTcbWBytes, kTcbABytes);
    k_mlp_bwd_tc<<<L.grid, L.threads, L.smem, s>>>(
        pred, target, cnt, cap, acts, static_cast<const __nv_bfloat16*>(h->wtcb.ptr), douts,
        static_cast<float*>(h->loss.ptr), static_cast<uint32_t*>(h->err.ptr));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // split-K over the rows: kWgMinRows or more per CTA (a multiple of
    // kWgRows), at most kMaxPartials CTAs
    uint32_t per_cta = (cap + kMaxPartials - 1) / kMaxPartials;
    per_cta = std::max<uint32_t>(kWgMinRows, (per_cta + kWgRows - 1) / kWgRows * kWgRows);
    const int n_part = (int)std::max<uint32_t>(1, (cap + per_cta - 1) / per_cta);
    StepState* st = static_cast<StepState*>(h->state.ptr);
    k_wgrad_tc<<<dim3(n_part, kLayers), 128, kWgSmem, s>>>(cnt, cap, per_cta, static_cast<const __nv_bfloat16*>(h->enc.ptr), acts,
                                            douts, static_cast<float*>(h->partial.ptr), st, do_step,
                                            static_cast<uint32_t*>(h->err.ptr));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    AdamArgs ar{h->cfg.lr, h->cfg.beta1, h->cfg.beta2, h->cfg.eps,
                h->cfg.ema > 0.0f && h->cfg.ema < 1.0f ? h->cfg.ema : 0.0f, h->cfg.weight_decay};
    k_reduce_adam<<<(kParams + 255) / 256, 256, 0, s>>>(
        static_cast<const float*>(h->partial.ptr), n_part, cnt, static_cast<float*>(h->grad.ptr),
        static_cast<float*>(h->w.ptr), static_cast<float*>(h->m.ptr), static_cast<float*>(h->v.ptr), ar, st, do_step,
        static_cast<__nv_bfloat16*>(h->wtc.ptr), static_cast<__nv_bfloat16*>(h->wtcb.ptr),
        static_cast<float*>(h->ema.ptr), static_cast<__nv_bfloat16*>(h->winf.ptr));
    return cudaGetLastError();
}

// Device copy of host-or-device input into dst (grown as needed).
cudaError_t take(DeviceBuffer& dst, const float* src, size_t bytes, cudaStream_t s) {
    cudaError_t e = dst.reserve(bytes);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(dst.ptr, src, bytes, cudaMemcpyDefault, s);
}

}  // namespace

namespace ilm {

cudaError_t nrc_infer_async(ilm_nrc* h, const float* raw, NrcCount n, float* out, cudaStream_t s) {
    return forward(h, raw, n, false, out, s);
}

cudaError_t nrc_train_async(ilm_nrc* h, const float* raw, const float* target, NrcCount n, cudaStream_t s) {
    return train_rows(h, raw, target, n, 1, s);
}

cudaError_t nrc_reserve(ilm_nrc* h, uint32_t rows) { return reserve_train(h, rows); }

uint32_t* nrc_error_word(ilm_nrc* h) { return static_cast<uint32_t*>(h->err.ptr); }

}  // namespace ilm

extern "C" {

int32_t ilm_nrc_create(ilm_context* ctx, const ilm_nrc_config* cfg, ilm_nrc** out) {
    if (!ctx || !cfg || !out) return ILM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!(cfg->weight_decay >= 0.0f) || !std::isfinite(cfg->weight_decay) || !(cfg->weight_decay * cfg->lr < 1.0f)) {
        set_error(ctx, "ilm_nrc_create: weight_decay must be finite, >= 0 and below 1 / lr");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    auto h = std::make_unique<ilm_nrc>();
    h->cfg = *cfg;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    for (DeviceBuffer* b : {&h->w, &h->m, &h->v, &h->grad, &h->ema})
        if ((e = b->reserve(kParams * 4)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->partial.reserve((size_t)kMaxPartials * kParams * 4)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->wtc.reserve(kParams * 2)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->winf.reserve(kParams * 2)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->wtcb.reserve(kTcbElems * 2)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->loss.reserve(4)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->err.reserve(4)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    cudaMemset(h->err.ptr, 0, 4);
    if ((e = h->state.reserve(sizeof(StepState))) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    cudaMemset(h->state.ptr, 0, sizeof(StepState));
    // He-uniform initialisation from PCG32; padded inputs and output rows 3..15 zero
    std::vector<float> w(kParams, 0.0f);
    Pcg32 rng(cfg->seed);
    for (int l = 0; l < kLayers; ++l) {
        int in = in_dim(l), fan = l == 0 ? kInReal : in;
        float s = std::sqrt(6.0f / (float)fan);
        for (int o = 0; o < out_dim(l); ++o)
            for (int i = 0; i < in; ++i) {
                float u = rng.uniform_float();
                bool zero = (l == 0 && i >= kInReal) || (l == 5 && o >= 3);
                w[param_off(l) + o * in + i] = zero ? 0.0f : (2.0f * u - 1.0f) * s;
            }
    }
    cudaMemcpy(h->w.ptr, w.data(), kParams * 4, cudaMemcpyHostToDevice);
    cudaMemset(h->m.ptr, 0, kParams * 4);
    cudaMemset(h->v.ptr, 0, kParams * 4);
    cudaMemset(h->wtc.ptr, 0, kParams * 2);
    cudaMemset(h->winf.ptr, 0, kParams * 2);
    cudaMemset(h->wtcb.ptr, 0, kTcbElems * 2);
    cudaFuncSetAttribute(k_mlp_fwd_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    cudaFuncSetAttribute(k_mlp_fwd_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    cudaFuncSetAttribute(k_mlp_bwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcbSmem);
    cudaFuncSetAttribute(k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgSmem);
    cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kInfSmem);
    if ((e = pack(h.get(), h->stream)) != cudaSuccess) return cuda_fail(ctx, e, "nrc pack");
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    *out = h.release();
    return ILM_OK;
}

int32_t ilm_nrc_destroy(ilm_context* ctx, ilm_nrc* h) {
    if (!ctx || !h) return ILM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(h->stream);
    delete h;
    return ILM_OK;
}

int32_t ilm_nrc_params(ilm_context* ctx, ilm_nrc* h, float* get, const float* set) {
    if (!ctx || !h) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    cudaStreamSynchronize(h->stream);
    cudaError_t e;
    if (set) {
        if ((e = cudaMemcpy(h->w.ptr, set, kParams * 4, cudaMemcpyDefault)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
        if ((e = pack(h, h->stream)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
        cudaStreamSynchronize(h->stream);
    }
    if (get && (e = cudaMemcpy(get, h->w.ptr, kParams * 4, cudaMemcpyDefault)) != cudaSuccess)
        return cuda_fail(ctx, e, "nrc");
    return ILM_OK;
}

int32_t ilm_nrc_infer(ilm_context* ctx, ilm_nrc* h, const float* inputs, uint64_t n, float* out, void* stream) {
    if (!ctx || !h || (n && (!inputs || !out))) return ILM_ERR_INVALID_ARGUMENT;
    if (n == 0) return ILM_OK;
    if (n > (1ull << 28)) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    cudaError_t e;
    bool dev_in = classify(inputs) == PtrKind::kDevice, dev_out = classify(out) == PtrKind::kDevice;
    const float* raw = inputs;
    if (!dev_in) {
        if ((e = take(h->raw, inputs, n * 12 * 4, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
        raw = static_cast<const float*>(h->raw.ptr);
    }
    float* dst = out;
    if (!dev_out) {
        if ((e = h->out.reserve(n * 12)) != cudaSuccess) return cuda_fail(ctx, e, "nrc buffers");
        dst = static_cast<float*>(h->out.ptr);
    }
    if ((e = forward(h, raw, NrcCount{nullptr, (uint32_t)n, 1, 0}, false, dst, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "nrc forward");
    if (!dev_out) {
        cudaMemcpyAsync(out, dst, n * 12, cudaMemcpyDeviceToHost, s);
        uint32_t flags = 0;
        cudaMemcpyAsync(&flags, h->err.ptr, 4, cudaMemcpyDeviceToHost, s);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
        if (flags) {
            set_error(ctx, "ilm_nrc_infer: a tensor-core wait ran out of time");
            return ILM_ERR_TIMEOUT;
        }
    }
    return ILM_OK;
}

static int32_t train_impl(ilm_context* ctx, ilm_nrc* h, const float* inputs, const float* targets, uint64_t n,
                          float* loss, float* grad_out, int step, void* stream) {
    if (!ctx || !h || !inputs || !targets || n == 0 || n > (1ull << 24)) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    cudaError_t e;
    const float* raw = inputs;
    if (classify(inputs) != PtrKind::kDevice) {
        if ((e = take(h->raw, inputs, n * 12 * 4, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
        raw = static_cast<const float*>(h->raw.ptr);
    }
    const float* tg = targets;
    if (classify(targets) != PtrKind::kDevice) {
        if ((e = take(h->target, targets, n * 3 * 4, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
        tg = static_cast<const float*>(h->target.ptr);
    }
    if ((e = train_rows(h, raw, tg, NrcCount{nullptr, (uint32_t)n, 1, 0}, step, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "nrc training");
    if (grad_out) cudaMemcpyAsync(grad_out, h->grad.ptr, kParams * 4, cudaMemcpyDefault, s);
    if (loss) {
        float ls = 0.0f;
        cudaMemcpyAsync(&ls, h->loss.ptr, 4, cudaMemcpyDeviceToHost, s);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
        *loss = ls / (3.0f * (float)n);
    } else if (grad_out) {
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    }
    return ILM_OK;
}

int32_t ilm_nrc_train_step(ilm_context* ctx, ilm_nrc* h, const float* inputs, const float* targets, uint64_t n,
                           float* loss, void* stream) {
    return train_impl(ctx, h, inputs, targets, n, loss, nullptr, 1, stream);
}

int32_t ilm_nrc_gradients(ilm_context* ctx, ilm_nrc* h, const float* inputs, const float* targets, uint64_t n,
                          float* grad_out, float* loss) {
    return train_impl(ctx, h, inputs, targets, n, loss, grad_out, 0, nullptr);
}

int32_t ilm_nrc_encode(ilm_context* ctx, ilm_nrc* h, const float* inputs, uint64_t n, void* enc_out) {
    if (!ctx || !h || !inputs || !enc_out || n == 0 || n > (1ull << 28)) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    cudaError_t e;
    if ((e = take(h->raw, inputs, n * 12 * 4, h->stream)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->enc.reserve(n * kIn * 2)) != cudaSuccess) return cuda_fail(ctx, e, "nrc buffers");
    k_nrc_encode<<<(unsigned)((n + 127) / 128), 128, 0, h->stream>>>(static_cast<const float*>(h->raw.ptr),
                                                                     (uint32_t)n, enc_params(h),
                                                                     static_cast<__nv_bfloat16*>(h->enc.ptr));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "nrc encode");
    cudaMemcpyAsync(enc_out, h->enc.ptr, n * kIn * 2, cudaMemcpyDefault, h->stream);
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    return ILM_OK;
}

}  // extern "C"
