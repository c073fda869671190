// Neural radiance cache: input encoding, a 5 x 64 ReLU MLP on BF16 tensor
// cores (mma.sync m16n8k16, FP32 accumulation), relative-L2 loss and Adam.
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
//   k_nrc_encode   raw (p, wo, n, albedo) -> 208 bf16
//   k_mlp_fwd      one warp per 16 rows: every layer's output fragments are
//                  turned into the next layer's A fragments in registers;
//                  weights in shared memory (rows padded to avoid bank
//                  conflicts); training stores the bf16 activations
//   k_mlp_bwd      loss gradient, then back through the layers the same way
//                  (transposed weights in shared memory), storing dOut
//   k_mlp_wgrad    dW = dOut^T * in, reduced over the batch: each CTA stages a
//                  64-row chunk transposed in shared memory, warps own output
//                  tiles, partial sums are added to the FP32 gradient
//   k_adam         Adam on FP32 master weights; writes the bf16 weight packs
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "context.h"
#include "illume_gpu.h"
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
// bf16 packs: forward W_l rows padded to in+8; backward W_l^T (l >= 1) rows
// padded to out+8
__host__ __device__ constexpr int fwd_stride(int l) { return in_dim(l) + 8; }
__host__ __device__ constexpr int fwd_off(int l) {
    return l == 0 ? 0 : kHid * (kIn + 8) + (l - 1) * kHid * (kHid + 8);
}
constexpr int kFwdElems = kHid * (kIn + 8) + 4 * kHid * (kHid + 8) + kOut * (kHid + 8);   // 33408
__host__ __device__ constexpr int bwd_stride(int l) { return out_dim(l) + 8; }
__host__ __device__ constexpr int bwd_off(int l) { return (l - 1) * kHid * (kHid + 8); }   // l = 1..5
constexpr int kBwdElems = 4 * kHid * (kHid + 8) + kHid * (kOut + 8);                        // 19968
constexpr float kLossEps = 0.01f;

__device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
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

// C fragments of 8 n-tiles (64 columns) -> ReLU'd bf16 A fragments of 4 k-steps.
__device__ __forceinline__ void to_a_frags(const float (&c)[8][4], uint32_t (&a)[4][4], bool relu) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float v[8];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            v[q] = c[2 * j][q];
            v[4 + q] = c[2 * j + 1][q];
        }
        if (relu)
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = fmaxf(v[q], 0.0f);
        a[j][0] = pack(v[0], v[1]);
        a[j][1] = pack(v[2], v[3]);
        a[j][2] = pack(v[4], v[5]);
        a[j][3] = pack(v[6], v[7]);
    }
}

// Stores / loads 4 k-steps of A fragments as a [rows][64] bf16 tile (row
// stride 32 words).
__device__ __forceinline__ void store_frags(uint32_t* base, uint32_t row0, uint32_t nrows, const uint32_t (&a)[4][4]) {
    const unsigned lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u;
    uint32_t r0 = row0 + g, r1 = row0 + g + 8;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (r0 < nrows) { base[r0 * 32 + 8 * j + t] = a[j][0]; base[r0 * 32 + 8 * j + 4 + t] = a[j][2]; }
        if (r1 < nrows) { base[r1 * 32 + 8 * j + t] = a[j][1]; base[r1 * 32 + 8 * j + 4 + t] = a[j][3]; }
    }
}

// Multiplies A fragments (16 x 64, four k-steps) by a 64-wide weight block in
// shared memory: out[nt] += A * B where B[k][n] = w[n * stride + k].
template <int NT>
__device__ __forceinline__ void gemm64(float (&acc)[NT][4], const uint32_t (&a)[4][4], const __nv_bfloat16* w,
                                       int stride) {
    const unsigned lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[nt][q] = 0.0f;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const __nv_bfloat16* p = w + (nt * 8 + g) * stride + ks * 16 + 2 * t;
            uint32_t b0 = *reinterpret_cast<const uint32_t*>(p);
            uint32_t b1 = *reinterpret_cast<const uint32_t*>(p + 8);
            mma(acc[nt], a[ks], b0, b1);
        }
}

__global__ void k_nrc_encode(const float* __restrict__ raw, uint32_t n, float bx0, float by0, float bz0, float sx,
                             float sy, float sz, __nv_bfloat16* __restrict__ enc) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = raw + 12 * (size_t)i;
    uint32_t* out = reinterpret_cast<uint32_t*>(enc + (size_t)i * kIn);
    float q[3] = {(r[0] - bx0) * sx, (r[1] - by0) * sy, (r[2] - bz0) * sz};
    int w = 0;
    // 72: for each axis, 12 octaves of (sin, cos)(2^k pi q)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float f = q[a];
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            float s, c;
            sincospif(f, &s, &c);
            out[w++] = pack(s, c);
            f *= 2.0f;
        }
    }
    // 128: one-blob of (theta/pi, phi/2pi) for wo then n, 32 bins, sigma 1/32
#pragma unroll
    for (int v = 0; v < 2; ++v) {
        float x = r[3 + 3 * v], y = r[4 + 3 * v], z = r[5 + 3 * v];
        float th = acosf(fminf(fmaxf(z, -1.0f), 1.0f)) * (1.0f / 3.14159265358979f);
        float ph = atan2f(y, x) * (0.5f / 3.14159265358979f) + 0.5f;
        float u[2] = {th, ph};
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int j = 0; j < 32; j += 2) {
                float d0 = (u[h] - (j + 0.5f) * (1.0f / 32.0f)) * 32.0f;
                float d1 = (u[h] - (j + 1.5f) * (1.0f / 32.0f)) * 32.0f;
                out[w++] = pack(__expf(-0.5f * d0 * d0), __expf(-0.5f * d1 * d1));
            }
    }
    // albedo (3) and 5 zeros of padding
    out[w++] = pack(r[9], r[10]);
    out[w++] = pack(r[11], 0.0f);
    out[w++] = 0u;
    out[w++] = 0u;
}

// Forward pass; kTrain stores the five hidden activations (bf16 [n][64]).
template <bool kTrain>
__global__ void __launch_bounds__(128) k_mlp_fwd(const __nv_bfloat16* __restrict__ enc, uint32_t n,
                                                 const __nv_bfloat16* __restrict__ wfwd, float* __restrict__ out,
                                                 __nv_bfloat16* __restrict__ acts) {
    extern __shared__ __align__(16) __nv_bfloat16 sw[];
    stage(sw, wfwd, kFwdElems);
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u, warp = threadIdx.x >> 5;
    const uint32_t* enc32 = reinterpret_cast<const uint32_t*>(enc);
    for (uint32_t tile = blockIdx.x * 4 + warp; tile * 16 < n; tile += gridDim.x * 4) {
        const uint32_t row0 = tile * 16, r0 = row0 + g, r1 = row0 + g + 8;
        float acc[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[nt][q] = 0.0f;
        // layer 0: K = 208 (13 k-steps), A straight from the encoded inputs
#pragma unroll 1
        for (int ks = 0; ks < 13; ++ks) {
            uint32_t a[4];
            a[0] = r0 < n ? enc32[(size_t)r0 * 104 + 8 * ks + t] : 0u;
            a[1] = r1 < n ? enc32[(size_t)r1 * 104 + 8 * ks + t] : 0u;
            a[2] = r0 < n ? enc32[(size_t)r0 * 104 + 8 * ks + 4 + t] : 0u;
            a[3] = r1 < n ? enc32[(size_t)r1 * 104 + 8 * ks + 4 + t] : 0u;
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const __nv_bfloat16* p = sw + fwd_off(0) + (nt * 8 + g) * fwd_stride(0) + ks * 16 + 2 * t;
                mma(acc[nt], a, *reinterpret_cast<const uint32_t*>(p), *reinterpret_cast<const uint32_t*>(p + 8));
            }
        }
        uint32_t af[4][4];
        to_a_frags(acc, af, true);
        if (kTrain) store_frags(reinterpret_cast<uint32_t*>(acts), row0, n, af);
#pragma unroll 1
        for (int l = 1; l <= 4; ++l) {
            gemm64<8>(acc, af, sw + fwd_off(l), fwd_stride(l));
            to_a_frags(acc, af, true);
            if (kTrain) store_frags(reinterpret_cast<uint32_t*>(acts + (size_t)l * n * kHid), row0, n, af);
        }
        float o[2][4];
        gemm64<2>(o, af, sw + fwd_off(5), fwd_stride(5));
        // columns 0..2 of n-tile 0: lanes t = 0 (cols 0, 1) and t = 1 (col 2)
        if (t == 0) {
            if (r0 < n) { out[3 * (size_t)r0] = o[0][0]; out[3 * (size_t)r0 + 1] = o[0][1]; }
            if (r1 < n) { out[3 * (size_t)r1] = o[0][2]; out[3 * (size_t)r1 + 1] = o[0][3]; }
        } else if (t == 1) {
            if (r0 < n) out[3 * (size_t)r0 + 2] = o[0][0];
            if (r1 < n) out[3 * (size_t)r1 + 2] = o[0][2];
        }
    }
}

// Backward pass: loss gradient and dOut of every layer (bf16: layers 0-4
// [n][64], layer 5 [n][16]); accumulates the loss sum.
__global__ void __launch_bounds__(128) k_mlp_bwd(const float* __restrict__ pred, const float* __restrict__ target,
                                                 uint32_t n, float scale, const __nv_bfloat16* __restrict__ acts,
                                                 const __nv_bfloat16* __restrict__ wbwd,
                                                 __nv_bfloat16* __restrict__ douts, float* __restrict__ loss_sum) {
    extern __shared__ __align__(16) __nv_bfloat16 sw[];
    stage(sw, wbwd, kBwdElems);
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u, warp = threadIdx.x >> 5;
    float loss = 0.0f;
    for (uint32_t tile = blockIdx.x * 4 + warp; tile * 16 < n; tile += gridDim.x * 4) {
        const uint32_t row0 = tile * 16, r0 = row0 + g, r1 = row0 + g + 8;
        // dL/dpred for this lane's output columns 2t, 2t+1 (only 0..2 exist)
        float d[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            uint32_t r = h ? r1 : r0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                uint32_t c = 2 * t + q;
                if (r < n && c < 3) {
                    float p = pred[3 * (size_t)r + c], y = target[3 * (size_t)r + c];
                    float den = p * p + kLossEps;
                    float e = p - y;
                    loss += e * e / den;
                    d[h][q] = 2.0f * e / den * scale;
                }
            }
        }
        uint32_t a5[4] = {pack(d[0][0], d[0][1]), pack(d[1][0], d[1][1]), 0u, 0u};
        // store dOut5 ([n][16], 8 words per row)
        uint32_t* d5 = reinterpret_cast<uint32_t*>(douts + (size_t)5 * n * kHid);
        if (r0 < n) { d5[r0 * 8 + t] = a5[0]; d5[r0 * 8 + 4 + t] = 0u; }
        if (r1 < n) { d5[r1 * 8 + t] = a5[1]; d5[r1 * 8 + 4 + t] = 0u; }
        // dAct4 = dOut5 * W5 (K = 16): B[k][n] = W5[k][n] = W5^T[n][k]
        float acc[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[nt][q] = 0.0f;
            const __nv_bfloat16* p = sw + bwd_off(5) + (nt * 8 + g) * bwd_stride(5) + 2 * t;
            mma(acc[nt], a5, *reinterpret_cast<const uint32_t*>(p), *reinterpret_cast<const uint32_t*>(p + 8));
        }
#pragma unroll 1
        for (int l = 4; l >= 0; --l) {
            // ReLU mask from the stored activation of layer l
            const uint32_t* act = reinterpret_cast<const uint32_t*>(acts + (size_t)l * n * kHid);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                uint32_t m0 = r0 < n ? act[r0 * 32 + 4 * nt + t] : 0u;
                uint32_t m1 = r1 < n ? act[r1 * 32 + 4 * nt + t] : 0u;
                acc[nt][0] = lo_of(m0) > 0.0f ? acc[nt][0] : 0.0f;
                acc[nt][1] = hi_of(m0) > 0.0f ? acc[nt][1] : 0.0f;
                acc[nt][2] = lo_of(m1) > 0.0f ? acc[nt][2] : 0.0f;
                acc[nt][3] = hi_of(m1) > 0.0f ? acc[nt][3] : 0.0f;
            }
            uint32_t af[4][4];
            to_a_frags(acc, af, false);
            store_frags(reinterpret_cast<uint32_t*>(douts + (size_t)l * n * kHid), row0, n, af);
            if (l == 0) break;
            // dAct_{l-1} = dOut_l * W_l: B[k][n] = W_l[k][n] = W_l^T[n][k]
            gemm64<8>(acc, af, sw + bwd_off(l), bwd_stride(l));
        }
    }
    // warp-reduce the loss, one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
    if (lane == 0) atomicAdd(loss_sum, loss);
}

// dW_l[o][i] = sum_r dOut_l[r][o] * in_l[r][i], reduced over the batch.
// OUT in {16, 64}, IN in {64, 208}; 8 warps; 64-row chunks.
template <int OUT, int IN>
__global__ void __launch_bounds__(256) k_mlp_wgrad(const __nv_bfloat16* __restrict__ dout, int dout_cols,
                                                   const __nv_bfloat16* __restrict__ in, uint32_t n,
                                                   float* __restrict__ grad) {
    constexpr int kRows = 64, kStride = kRows + 8;
    constexpr int kMT = OUT / 16, kNT = IN / 8, kTiles = kMT * kNT, kPerWarp = (kTiles + 7) / 8;
    __shared__ __align__(16) __nv_bfloat16 sd[OUT * kStride];   // dOut^T chunk
    __shared__ __align__(16) __nv_bfloat16 sa[IN * kStride];    // in^T chunk
    const unsigned lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u, warp = threadIdx.x >> 5;
    float acc[kPerWarp][4];
#pragma unroll
    for (int k = 0; k < kPerWarp; ++k)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[k][q] = 0.0f;
    const uint32_t chunks = (n + kRows - 1) / kRows;
    for (uint32_t ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
        const uint32_t base = ch * kRows;
        __syncthreads();
        // stage transposed: element (r, c) -> s[c * kStride + r]
        for (int e = threadIdx.x; e < kRows * OUT; e += blockDim.x) {
            int r = e / OUT, c = e % OUT;
            sd[c * kStride + r] = base + r < n ? dout[(size_t)(base + r) * dout_cols + c] : __float2bfloat16(0.0f);
        }
        for (int e = threadIdx.x; e < kRows * IN; e += blockDim.x) {
            int r = e / IN, c = e % IN;
            sa[c * kStride + r] = base + r < n ? in[(size_t)(base + r) * IN + c] : __float2bfloat16(0.0f);
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < kRows / 16; ++ks)
#pragma unroll
            for (int k = 0; k < kPerWarp; ++k) {
                int tile = warp + 8 * k;
                if (tile < kTiles) {
                    int mt = tile / kNT, nt = tile % kNT;
                    const __nv_bfloat16* pa = sd + (mt * 16 + g) * kStride + ks * 16 + 2 * t;
                    uint32_t a[4] = {*reinterpret_cast<const uint32_t*>(pa),
                                     *reinterpret_cast<const uint32_t*>(pa + 8 * kStride),
                                     *reinterpret_cast<const uint32_t*>(pa + 8),
                                     *reinterpret_cast<const uint32_t*>(pa + 8 * kStride + 8)};
                    const __nv_bfloat16* pb = sa + (nt * 8 + g) * kStride + ks * 16 + 2 * t;
                    mma(acc[k], a, *reinterpret_cast<const uint32_t*>(pb), *reinterpret_cast<const uint32_t*>(pb + 8));
                }
            }
    }
#pragma unroll
    for (int k = 0; k < kPerWarp; ++k) {
        int tile = warp + 8 * k;
        if (tile < kTiles) {
            int mt = tile / kNT, nt = tile % kNT;
            int o0 = mt * 16 + g, i0 = nt * 8 + 2 * t;
            atomicAdd(&grad[o0 * IN + i0], acc[k][0]);
            atomicAdd(&grad[o0 * IN + i0 + 1], acc[k][1]);
            atomicAdd(&grad[(o0 + 8) * IN + i0], acc[k][2]);
            atomicAdd(&grad[(o0 + 8) * IN + i0 + 1], acc[k][3]);
        }
    }
}

// Adam on the FP32 master weights (rows 3..15 of the output layer stay zero),
// then the bf16 forward and transposed packs.  With ema_a > 0 a step also
// updates ema = ema_a * ema + (1 - ema_a) * w (ema starts at 0) and the
// inference pack holds ema / ce (ce = 1 - ema_a^steps, the zero-start
// correction); without a step the inference pack holds w and ema restarts.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                       int do_step, __nv_bfloat16* __restrict__ wfwd, __nv_bfloat16* __restrict__ wbwd,
                       float* __restrict__ ema, float ema_a, float ce, __nv_bfloat16* __restrict__ winf) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    int l = 0;
    while (l < 5 && p >= param_off(l + 1)) ++l;
    int local = p - param_off(l), in = in_dim(l), o = local / in, i = local % in;
    float x = w[p];
    bool frozen = (l == 5 && o >= 3) || (l == 0 && i >= kInReal);
    if (do_step && !frozen) {
        float gr = grad[p];
        float mm = b1 * m[p] + (1.0f - b1) * gr;
        float vv = b2 * v[p] + (1.0f - b2) * gr * gr;
        m[p] = mm;
        v[p] = vv;
        x -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
        w[p] = x;
    }
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    wfwd[fwd_off(l) + o * fwd_stride(l) + i] = h;
    if (l >= 1) wbwd[bwd_off(l) + i * bwd_stride(l) + o] = h;
    float xi = x;
    if (ema_a > 0.0f) {
        if (do_step) {
            float e = ema_a * ema[p] + (1.0f - ema_a) * x;
            ema[p] = e;
            xi = e / ce;
        } else {
            ema[p] = 0.0f;
        }
    }
    winf[fwd_off(l) + o * fwd_stride(l) + i] = __float2bfloat16_rn(xi);
}

}  // namespace nrc
}  // namespace ilm

using namespace ilm;
using namespace ilm::nrc;

struct ilm_nrc {
    ilm_nrc_config cfg;
    int step = 0;
    int ema_steps = 0;                           // Adam steps since the inference weights restarted
    DeviceBuffer w, m, v, grad, wfwd, wbwd;      // params and packs
    DeviceBuffer ema, winf;                      // moving average and its inference pack
    DeviceBuffer raw, enc, out, target, acts, douts, loss;
    uint32_t cap = 0;
    cudaStream_t stream = nullptr;
    ~ilm_nrc() {
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

cudaError_t ensure_capacity(ilm_nrc* h, uint32_t n) {
    if (n <= h->cap) return cudaSuccess;
    uint32_t c = 1024;
    while (c < n) c <<= 1;
    cudaError_t e;
    if ((e = h->raw.reserve((size_t)c * 12 * 4)) != cudaSuccess) return e;
    if ((e = h->enc.reserve((size_t)c * kIn * 2)) != cudaSuccess) return e;
    if ((e = h->out.reserve((size_t)c * 3 * 4)) != cudaSuccess) return e;
    if ((e = h->target.reserve((size_t)c * 3 * 4)) != cudaSuccess) return e;
    if ((e = h->acts.reserve((size_t)c * 5 * kHid * 2)) != cudaSuccess) return e;
    if ((e = h->douts.reserve((size_t)c * 6 * kHid * 2)) != cudaSuccess) return e;
    h->cap = c;
    return cudaSuccess;
}

// Re-packs the bf16 weights (and optionally takes an Adam step).
cudaError_t adam(ilm_nrc* h, int do_step, cudaStream_t s) {
    if (do_step) h->step += 1;
    h->ema_steps = do_step ? h->ema_steps + 1 : 0;
    float c1 = 1.0f - std::pow(h->cfg.beta1, (float)(h->step > 0 ? h->step : 1));
    float c2 = 1.0f - std::pow(h->cfg.beta2, (float)(h->step > 0 ? h->step : 1));
    float ea = h->cfg.ema > 0.0f && h->cfg.ema < 1.0f ? h->cfg.ema : 0.0f;
    float ce = ea > 0.0f ? 1.0f - (float)std::pow((double)ea, (double)(h->ema_steps > 0 ? h->ema_steps : 1)) : 1.0f;
    k_adam<<<(kParams + 255) / 256, 256, 0, s>>>(
        static_cast<float*>(h->w.ptr), static_cast<const float*>(h->grad.ptr), static_cast<float*>(h->m.ptr),
        static_cast<float*>(h->v.ptr), h->cfg.lr, h->cfg.beta1, h->cfg.beta2, h->cfg.eps, c1, c2, do_step,
        static_cast<__nv_bfloat16*>(h->wfwd.ptr), static_cast<__nv_bfloat16*>(h->wbwd.ptr),
        static_cast<float*>(h->ema.ptr), ea, ce, static_cast<__nv_bfloat16*>(h->winf.ptr));
    return cudaGetLastError();
}

int blocks_for(uint32_t n, int rows_per_block) {
    int b = (int)((n + rows_per_block - 1) / rows_per_block);
    return b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b);
}

cudaError_t encode(ilm_nrc* h, const float* raw_dev, uint32_t n, cudaStream_t s) {
    const float* b = h->cfg.bound;
    float sx = 1.0f / fmaxf(b[3] - b[0], 1e-12f), sy = 1.0f / fmaxf(b[4] - b[1], 1e-12f),
          sz = 1.0f / fmaxf(b[5] - b[2], 1e-12f);
    k_nrc_encode<<<(n + 127) / 128, 128, 0, s>>>(raw_dev, n, b[0], b[1], b[2], sx, sy, sz,
                                                 static_cast<__nv_bfloat16*>(h->enc.ptr));
    return cudaGetLastError();
}

cudaError_t forward(ilm_nrc* h, uint32_t n, bool train, float* out_dev, cudaStream_t s) {
    size_t smem = (size_t)kFwdElems * 2;
    if (train)
        k_mlp_fwd<true><<<blocks_for(n, 64), 128, smem, s>>>(static_cast<const __nv_bfloat16*>(h->enc.ptr), n,
                                                             static_cast<const __nv_bfloat16*>(h->wfwd.ptr), out_dev,
                                                             static_cast<__nv_bfloat16*>(h->acts.ptr));
    else   // inference reads the moving-average pack
        k_mlp_fwd<false><<<blocks_for(n, 64), 128, smem, s>>>(static_cast<const __nv_bfloat16*>(h->enc.ptr), n,
                                                              static_cast<const __nv_bfloat16*>(h->winf.ptr), out_dev,
                                                              nullptr);
    return cudaGetLastError();
}

// Loss gradient into h->grad (zeroed first) and the loss sum into h->loss.
cudaError_t gradients(ilm_nrc* h, uint32_t n, cudaStream_t s) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(h->grad.ptr, 0, kParams * 4, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(h->loss.ptr, 0, 4, s)) != cudaSuccess) return e;
    if ((e = forward(h, n, true, static_cast<float*>(h->out.ptr), s)) != cudaSuccess) return e;
    const __nv_bfloat16* acts = static_cast<const __nv_bfloat16*>(h->acts.ptr);
    __nv_bfloat16* douts = static_cast<__nv_bfloat16*>(h->douts.ptr);
    k_mlp_bwd<<<blocks_for(n, 64), 128, (size_t)kBwdElems * 2, s>>>(
        static_cast<const float*>(h->out.ptr), static_cast<const float*>(h->target.ptr), n, 1.0f / (3.0f * n),
        acts, static_cast<const __nv_bfloat16*>(h->wbwd.ptr), douts, static_cast<float*>(h->loss.ptr));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    float* gr = static_cast<float*>(h->grad.ptr);
    const __nv_bfloat16* enc = static_cast<const __nv_bfloat16*>(h->enc.ptr);
    int wb = blocks_for(n, 64 * 4);
    k_mlp_wgrad<64, 208><<<wb, 256, 0, s>>>(douts, kHid, enc, n, gr + param_off(0));
    for (int l = 1; l <= 4; ++l)
        k_mlp_wgrad<64, 64><<<wb, 256, 0, s>>>(douts + (size_t)l * n * kHid, kHid, acts + (size_t)(l - 1) * n * kHid,
                                               n, gr + param_off(l));
    k_mlp_wgrad<16, 64><<<wb, 256, 0, s>>>(douts + (size_t)5 * n * kHid, kOut, acts + (size_t)4 * n * kHid, n,
                                           gr + param_off(5));
    return cudaGetLastError();
}

// Device copy of host-or-device input into h's buffer.
cudaError_t take(DeviceBuffer& dst, const float* src, size_t bytes, cudaStream_t s) {
    if (!src) return cudaSuccess;
    return cudaMemcpyAsync(dst.ptr, src, bytes, cudaMemcpyDefault, s);
}

}  // namespace

extern "C" {

int32_t ilm_nrc_create(ilm_context* ctx, const ilm_nrc_config* cfg, ilm_nrc** out) {
    if (!ctx || !cfg || !out) return ILM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    auto h = std::make_unique<ilm_nrc>();
    h->cfg = *cfg;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    for (DeviceBuffer* b : {&h->w, &h->m, &h->v, &h->grad, &h->ema})
        if ((e = b->reserve(kParams * 4)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->wfwd.reserve(kFwdElems * 2)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->winf.reserve(kFwdElems * 2)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->wbwd.reserve(kBwdElems * 2)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = h->loss.reserve(4)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
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
    cudaMemset(h->wfwd.ptr, 0, kFwdElems * 2);
    cudaMemset(h->winf.ptr, 0, kFwdElems * 2);
    cudaMemset(h->wbwd.ptr, 0, kBwdElems * 2);
    cudaMemset(h->ema.ptr, 0, kParams * 4);
    cudaFuncSetAttribute(k_mlp_fwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdElems * 2);
    cudaFuncSetAttribute(k_mlp_fwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdElems * 2);
    if ((e = adam(h.get(), 0, h->stream)) != cudaSuccess) return cuda_fail(ctx, e, "nrc pack");
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
        if ((e = adam(h, 0, h->stream)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
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
    if ((e = ensure_capacity(h, (uint32_t)n)) != cudaSuccess) return cuda_fail(ctx, e, "nrc buffers");
    bool dev_in = classify(inputs) == PtrKind::kDevice, dev_out = classify(out) == PtrKind::kDevice;
    const float* raw = inputs;
    if (!dev_in) {
        if ((e = take(h->raw, inputs, n * 12 * 4, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
        raw = static_cast<const float*>(h->raw.ptr);
    }
    if ((e = encode(h, raw, (uint32_t)n, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc encode");
    float* dst = dev_out ? out : static_cast<float*>(h->out.ptr);
    if ((e = forward(h, (uint32_t)n, false, dst, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc forward");
    if (!dev_out) {
        cudaMemcpyAsync(out, dst, n * 12, cudaMemcpyDeviceToHost, s);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    }
    return ILM_OK;
}

static int32_t train_impl(ilm_context* ctx, ilm_nrc* h, const float* inputs, const float* targets, uint64_t n,
                          float* loss, float* grad_out, int step, void* stream) {
    if (!ctx || !h || !inputs || !targets || n == 0 || n > (1ull << 24)) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    cudaError_t e;
    if ((e = ensure_capacity(h, (uint32_t)n)) != cudaSuccess) return cuda_fail(ctx, e, "nrc buffers");
    const float* raw = inputs;
    if (classify(inputs) != PtrKind::kDevice) {
        if ((e = take(h->raw, inputs, n * 12 * 4, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
        raw = static_cast<const float*>(h->raw.ptr);
    }
    if ((e = take(h->target, targets, n * 3 * 4, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = encode(h, raw, (uint32_t)n, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc encode");
    if ((e = gradients(h, (uint32_t)n, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc gradients");
    if (step && (e = adam(h, 1, s)) != cudaSuccess) return cuda_fail(ctx, e, "nrc adam");
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
    if (!ctx || !h || !inputs || !enc_out || n == 0) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    cudaError_t e;
    if ((e = ensure_capacity(h, (uint32_t)n)) != cudaSuccess) return cuda_fail(ctx, e, "nrc buffers");
    if ((e = take(h->raw, inputs, n * 12 * 4, h->stream)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    if ((e = encode(h, static_cast<const float*>(h->raw.ptr), (uint32_t)n, h->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "nrc encode");
    cudaMemcpyAsync(enc_out, h->enc.ptr, n * kIn * 2, cudaMemcpyDefault, h->stream);
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_fail(ctx, e, "nrc");
    return ILM_OK;
}

}  // extern "C"
