// surrogate.cu - kernels of the BF16 convolutional field surrogate
// (include/dsmc_surrogate.h).
//
// The 3x3 convolutions are implicit GEMMs on the tensor cores with
// mma.sync.m16n8k16 (bf16 in, fp32 accumulate); tiles move global -> shared
// with cp.async and shared -> registers with ldmatrix, in a 3-stage pipeline.
//   forward  C[pixel][cout]       = sum_(tap, cin) X[pixel + tap][cin] W[cout][tap][cin]
//   dgrad    the forward with the weights rotated by 180 degrees and the
//            channel roles swapped (stride 1, padding 1: the transpose of a
//            3x3 convolution is a 3x3 convolution)
//   wgrad    C[cout][(tap, cin)]  = sum_pixel dY[pixel][cout] X[pixel + tap][cin]
//            (split over pixels, FP32 atomics into dW)
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/dsmc_surrogate.h"

namespace {

constexpr int OK = 0, ERR_ARG = 2, ERR_CUDA = 50;

using bf16 = __nv_bfloat16;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte asynchronous copy; zero fill when !valid (src must still be a
// mapped address: the callers pass the tensor's base then).
__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void ldsm_x4(uint32_t r[4], const void *p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t r[4], const void *p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x2(uint32_t r[2], const void *p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t r[2], const void *p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2])
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, "
                 "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Eight bf16 (16 bytes) as floats.
struct V8 {
    float v[8];
};
__device__ __forceinline__ V8 ld8(const bf16 *p)
{
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
    V8 r;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 f = __bfloat1622float2(h[i]);
        r.v[2 * i] = f.x;
        r.v[2 * i + 1] = f.y;
    }
    return r;
}
__device__ __forceinline__ void st8(bf16 *p, const V8 &r)
{
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i)
        h[i] = __floats2bfloat162_rn(r.v[2 * i], r.v[2 * i + 1]);
    *reinterpret_cast<uint4 *>(p) = u;
}

// ---------------------------------------------------------------------------
// Forward (and dgrad): CTA tile 128 pixels x 64 output channels, k-tiles of
// 32 input channels of one tap; 8 warps as 4 (pixels) x 2 (channels), each
// 32 x 32.  Shared rows are padded to 40 elements (80 bytes) so ldmatrix's
// eight 16-byte rows fall on distinct banks.
// ---------------------------------------------------------------------------
constexpr int FBM = 128, FBN = 64, FBK = 32, FST = 3, FLD = FBK + 8;

__global__ void __launch_bounds__(256)
    k_conv_fwd(const bf16 *__restrict__ x, const bf16 *__restrict__ w,
               const float *__restrict__ bias, const bf16 *__restrict__ res, bf16 *__restrict__ y,
               float *__restrict__ y32, int N, int H, int W, int Cin, int Cout, int relu)
{
    __shared__ __align__(128) bf16 sA[FST][FBM][FLD];
    __shared__ __align__(128) bf16 sB[FST][FBN][FLD];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int M = N * H * W;
    const int m0 = blockIdx.x * FBM, n0 = blockIdx.y * FBN;
    const int cblocks = Cin / FBK;
    const int KT = 9 * cblocks;

    // The two A rows this thread copies, and its B row.
    int an[2], ah[2], aw[2];
    bool am[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int m = m0 + (tid >> 2) + 64 * i;
        am[i] = m < M;
        const int mm = am[i] ? m : 0;
        an[i] = mm / (H * W);
        ah[i] = (mm / W) % H;
        aw[i] = mm % W;
    }
    const int chunk = (tid & 3) * 8;
    const int bco = n0 + (tid >> 2);

    auto load = [&](int kt, int st) {
        const int tap = kt / cblocks, cb = (kt % cblocks) * FBK;
        const int kh = tap / 3, kw = tap % 3;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int hh = ah[i] + kh - 1, ww = aw[i] + kw - 1;
            const bool ok = am[i] && hh >= 0 && hh < H && ww >= 0 && ww < W;
            const bf16 *src =
                ok ? x + ((static_cast<int64_t>(an[i]) * H + hh) * W + ww) * Cin + cb + chunk : x;
            cp_async16(&sA[st][(tid >> 2) + 64 * i][chunk], src, ok);
        }
        const bool okb = bco < Cout;
        const bf16 *srcb = okb ? w + (static_cast<int64_t>(bco) * 9 + tap) * Cin + cb + chunk : w;
        cp_async16(&sB[st][tid >> 2][chunk], srcb, okb);
    };

    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int k = 0; k < 4; ++k)
                acc[i][j][k] = 0.0f;

#pragma unroll
    for (int s = 0; s < FST - 1; ++s) {
        if (s < KT)
            load(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<FST - 2>();
        __syncthreads();
        if (kt + FST - 1 < KT)
            load(kt + FST - 1, (kt + FST - 1) % FST);
        cp_async_commit();
        const int st = kt % FST;
#pragma unroll
        for (int kk = 0; kk < FBK; kk += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
                ldsm_x4(a[mi], &sA[st][wm * 32 + mi * 16 + (lane & 15)][kk + (lane >> 4) * 8]);
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
                ldsm_x2(b[ni], &sB[st][wn * 32 + ni * 8 + (lane & 7)][kk + ((lane >> 3) & 1) * 8]);
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                    mma_bf16(acc[mi][ni], a[mi], b[ni]);
        }
    }
    cp_async_wait<0>();

    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int m = m0 + wm * 32 + mi * 16 + g + half * 8;
            if (m >= M)
                continue;
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) {
                const int co = n0 + wn * 32 + ni * 8 + 2 * t;
                if (co >= Cout)
                    continue;
                float v0 = acc[mi][ni][2 * half] + (bias ? bias[co] : 0.0f);
                float v1 = acc[mi][ni][2 * half + 1] + (bias ? bias[co + 1] : 0.0f);
                if (relu) {
                    v0 = fmaxf(v0, 0.0f);
                    v1 = fmaxf(v1, 0.0f);
                }
                const int64_t o = static_cast<int64_t>(m) * Cout + co;
                if (res) {
                    const __nv_bfloat162 r = *reinterpret_cast<const __nv_bfloat162 *>(res + o);
                    v0 += __bfloat162float(r.x);
                    v1 += __bfloat162float(r.y);
                }
                if (y)
                    *reinterpret_cast<__nv_bfloat162 *>(y + o) = __floats2bfloat162_rn(v0, v1);
                if (y32)
                    *reinterpret_cast<float2 *>(y32 + o) = make_float2(v0, v1);
            }
        }
}

// w_rot[ci][tap][co] = w[co][8 - tap][ci]: the weights of the dgrad conv.
__global__ void k_rotate(const bf16 *__restrict__ w, bf16 *__restrict__ w_rot, int Cin, int Cout)
{
    const int64_t total = static_cast<int64_t>(Cout) * 9 * Cin;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int ci = static_cast<int>(i % Cin);
        const int tap = static_cast<int>((i / Cin) % 9);
        const int co = static_cast<int>(i / (9 * static_cast<int64_t>(Cin)));
        w_rot[(static_cast<int64_t>(ci) * 9 + (8 - tap)) * Cout + co] = w[i];
    }
}

// ---------------------------------------------------------------------------
// wgrad: CTA tile 64 output channels x 32 input channels of one tap, k-tiles
// of 32 pixels; the pixels of the problem are split over gridDim.z.  Shared
// tiles are stored pixel-major as they sit in memory and read transposed
// with ldmatrix.trans.  8 warps as 4 (cout) x 2 (cin), each 16 x 16.
// ---------------------------------------------------------------------------
constexpr int WBM = 64, WBN = 32, WBK = 32, WST = 3, WLDA = WBM + 8, WLDB = WBN + 8;

__global__ void __launch_bounds__(256)
    k_conv_wgrad(const bf16 *__restrict__ dy, const bf16 *__restrict__ x, float *__restrict__ dw,
                 int N, int H, int W, int Cin, int Cout, int per_split)
{
    __shared__ __align__(128) bf16 sA[WST][WBK][WLDA];
    __shared__ __align__(128) bf16 sB[WST][WBK][WLDB];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int M = N * H * W;
    const int co0 = blockIdx.x * WBM;
    const int cblocks = Cin / WBN;
    const int tap = blockIdx.y / cblocks, ci0 = (blockIdx.y % cblocks) * WBN;
    const int kh = tap / 3, kw = tap % 3;
    const int p_begin = blockIdx.z * per_split;
    const int p_end = min(M, p_begin + per_split);
    const int KT = (p_end - p_begin + WBK - 1) / WBK;

    auto load = [&](int kt, int st) {
        const int pbase = p_begin + kt * WBK;
        {   // A: 32 pixels x 64 channels of dY, 8 chunks per pixel
            const int r = tid >> 3, c = (tid & 7) * 8;
            const int p = pbase + r;
            const bool ok = p < p_end && co0 + c < Cout;
            const bf16 *src = ok ? dy + static_cast<int64_t>(p) * Cout + co0 + c : dy;
            cp_async16(&sA[st][r][c], src, ok);
        }
        if (tid < 128) { // B: 32 pixels x 32 channels of X shifted by the tap
            const int r = tid >> 2, c = (tid & 3) * 8;
            const int p = pbase + r;
            bool ok = p < p_end;
            const bf16 *src = x;
            if (ok) {
                const int n = p / (H * W), hh = (p / W) % H + kh - 1, ww = p % W + kw - 1;
                ok = hh >= 0 && hh < H && ww >= 0 && ww < W;
                if (ok)
                    src = x + ((static_cast<int64_t>(n) * H + hh) * W + ww) * Cin + ci0 + c;
            }
            cp_async16(&sB[st][r][c], src, ok);
        }
    };

    float acc[2][4];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int k = 0; k < 4; ++k)
            acc[j][k] = 0.0f;

#pragma unroll
    for (int s = 0; s < WST - 1; ++s) {
        if (s < KT)
            load(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<WST - 2>();
        __syncthreads();
        if (kt + WST - 1 < KT)
            load(kt + WST - 1, (kt + WST - 1) % WST);
        cp_async_commit();
        const int st = kt % WST;
#pragma unroll
        for (int kk = 0; kk < WBK; kk += 16) {
            uint32_t a[4], b[2][2];
            ldsm_x4_t(a, &sA[st][kk + (lane & 7) + ((lane >> 4) << 3)]
                             [wm * 16 + ((lane >> 3) & 1) * 8]);
#pragma unroll
            for (int ni = 0; ni < 2; ++ni)
                ldsm_x2_t(b[ni], &sB[st][kk + (lane & 7) + (((lane >> 3) & 1) << 3)]
                                    [wn * 16 + ni * 8]);
#pragma unroll
            for (int ni = 0; ni < 2; ++ni)
                mma_bf16(acc[ni], a, b[ni]);
        }
    }
    cp_async_wait<0>();

    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int co = co0 + wm * 16 + g + half * 8;
        if (co >= Cout)
            continue;
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) {
            const int ci = ci0 + wn * 16 + ni * 8 + 2 * t;
            float *o = dw + (static_cast<int64_t>(co) * 9 + tap) * Cin + ci;
            atomicAdd(o, acc[ni][2 * half]);
            atomicAdd(o + 1, acc[ni][2 * half + 1]);
        }
    }
}

// db[c] += sum over pixels of dy[pixel][c]: each thread sums one 8-channel
// group over a strided set of pixels, the CTA reduces in shared memory and
// adds with one atomic per channel.
__global__ void k_bias_grad(const bf16 *__restrict__ dy, float *__restrict__ db, int M, int C)
{
    const int c8 = C / 8;                 // channel groups (4..16)
    const int lanes = blockDim.x / c8;    // pixel lanes of the CTA
    const int g = threadIdx.x % c8, lp = threadIdx.x / c8;
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (lp < lanes)
        for (int p = blockIdx.x * lanes + lp; p < M; p += gridDim.x * lanes) {
            const V8 v = ld8(dy + static_cast<int64_t>(p) * C + 8 * g);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                s[k] += v.v[k];
        }
    __shared__ float part[256][9];
#pragma unroll
    for (int k = 0; k < 8; ++k)
        part[threadIdx.x][k] = s[k];
    __syncthreads();
    if (threadIdx.x < C) {
        const int gg = threadIdx.x / 8, k = threadIdx.x % 8;
        float t = 0.0f;
        for (int l = 0; l < lanes; ++l)
            t += part[l * c8 + gg][k];
        atomicAdd(db + threadIdx.x, t);
    }
}

// ---------------------------------------------------------------------------
// Elementwise kernels.  Channel counts are multiples of 32, so every kernel
// moves 8 bf16 (16 bytes) per thread and step, never across a pixel.
// ---------------------------------------------------------------------------
// Grid-stride over n8 = count / 8 vectors.
#define FOR_V8(n8)                                                                         \
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < (n8); \
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)

__global__ void k_relu_bwd(bf16 *dy, const bf16 *y, int64_t n8)
{
    FOR_V8(n8)
    {
        V8 g = ld8(dy + 8 * i);
        const V8 a = ld8(y + 8 * i);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            g.v[k] = a.v[k] > 0.0f ? g.v[k] : 0.0f;
        st8(dy + 8 * i, g);
    }
}

__global__ void k_add(bf16 *a, const bf16 *b, int64_t n8)
{
    FOR_V8(n8)
    {
        V8 x = ld8(a + 8 * i);
        const V8 y = ld8(b + 8 * i);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            x.v[k] += y.v[k];
        st8(a + 8 * i, x);
    }
}

// Output vector i of (n, h/2, w/2, c): c8 = c / 8 vectors per pixel.
__global__ void k_pool_fwd(const bf16 *x, bf16 *y, int N, int H, int W, int C)
{
    const int c8 = C / 8, Ho = H / 2, Wo = W / 2;
    const int64_t n8 = static_cast<int64_t>(N) * Ho * Wo * c8;
    FOR_V8(n8)
    {
        const int cv = static_cast<int>(i % c8);
        const int64_t pix = i / c8;
        const int wo = static_cast<int>(pix % Wo), ho = static_cast<int>((pix / Wo) % Ho);
        const int64_t n = pix / (static_cast<int64_t>(Wo) * Ho);
        const bf16 *b = x + ((n * H + 2 * ho) * W + 2 * wo) * C + 8 * cv;
        const int64_t row = static_cast<int64_t>(W) * C;
        const V8 a = ld8(b), bb = ld8(b + C), cc = ld8(b + row), dd = ld8(b + row + C);
        V8 r;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            r.v[k] = 0.25f * (a.v[k] + bb.v[k] + cc.v[k] + dd.v[k]);
        st8(y + 8 * i, r);
    }
}

// Input-gradient vector i of (n, h, w, c).
__global__ void k_pool_bwd(const bf16 *dy, bf16 *dx, int N, int H, int W, int C)
{
    const int c8 = C / 8;
    const int64_t n8 = static_cast<int64_t>(N) * H * W * c8;
    FOR_V8(n8)
    {
        const int cv = static_cast<int>(i % c8);
        const int64_t pix = i / c8;
        const int w = static_cast<int>(pix % W), h = static_cast<int>((pix / W) % H);
        const int64_t n = pix / (static_cast<int64_t>(W) * H);
        V8 g = ld8(dy + ((n * (H / 2) + h / 2) * (W / 2) + w / 2) * C + 8 * cv);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            g.v[k] *= 0.25f;
        st8(dx + 8 * i, g);
    }
}

// (n, h, w, c) -> (n, 2h, 2w, c), nearest: output vector i.
__global__ void k_up_fwd(const bf16 *x, bf16 *y, int N, int H, int W, int C)
{
    const int c8 = C / 8;
    const int64_t n8 = static_cast<int64_t>(N) * 4 * H * W * c8;
    FOR_V8(n8)
    {
        const int cv = static_cast<int>(i % c8);
        const int64_t pix = i / c8;
        const int w2 = static_cast<int>(pix % (2 * W)), h2 = static_cast<int>((pix / (2 * W)) % (2 * H));
        const int64_t n = pix / (4 * static_cast<int64_t>(W) * H);
        *reinterpret_cast<uint4 *>(y + 8 * i) = *reinterpret_cast<const uint4 *>(
            x + ((n * H + h2 / 2) * W + w2 / 2) * C + 8 * cv);
    }
}

// Input-gradient vector i of (n, h, w, c) from dy of (n, 2h, 2w, c).
__global__ void k_up_bwd(const bf16 *dy, bf16 *dx, int N, int H, int W, int C)
{
    const int c8 = C / 8;
    const int64_t n8 = static_cast<int64_t>(N) * H * W * c8;
    FOR_V8(n8)
    {
        const int cv = static_cast<int>(i % c8);
        const int64_t pix = i / c8;
        const int w = static_cast<int>(pix % W), h = static_cast<int>((pix / W) % H);
        const int64_t n = pix / (static_cast<int64_t>(W) * H);
        const bf16 *b = dy + ((n * 2 * H + 2 * h) * (2 * W) + 2 * w) * C + 8 * cv;
        const int64_t row = 2 * static_cast<int64_t>(W) * C;
        const V8 a = ld8(b), bb = ld8(b + C), cc = ld8(b + row), dd = ld8(b + row + C);
        V8 r;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            r.v[k] = a.v[k] + bb.v[k] + cc.v[k] + dd.v[k];
        st8(dx + 8 * i, r);
    }
}

__global__ void k_mask_sum(const float *mask, int64_t n, float *sum)
{
    float s = 0.0f;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        s += mask[i];
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(sum, s);
}

__global__ void k_mse(const float *out, const float *tgt, const float *mask, const float *msum,
                      bf16 *dy, float *loss, int64_t pixels, int C, int K)
{
    const float scale = 1.0f / (static_cast<float>(K) * fmaxf(*msum, 1.0f));
    float l = 0.0f;
    for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < pixels;
         p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float mk = mask[p];
        for (int c = 0; c < C; ++c) {
            float g = 0.0f;
            if (c < K && mk != 0.0f) {
                const float d = out[p * C + c] - tgt[p * K + c];
                l += d * d * scale;
                g = 2.0f * d * scale;
            }
            dy[p * C + c] = __float2bfloat16(g);
        }
    }
    for (int o = 16; o > 0; o >>= 1)
        l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(loss, l);
}

__global__ void k_adam(float *w, bf16 *wb, const float *g, float *m, float *v, int64_t n, float lr,
                       float b1, float b2, float eps, float c1, float c2)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb)
            wb[i] = __float2bfloat16(wi);
    }
}

__global__ void k_to_bf16(const float *x, bf16 *y, int64_t n)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

int grid_for(int64_t n) { return static_cast<int>(n / 256 + 1 < 4096 ? n / 256 + 1 : 4096); }

int status() { return cudaGetLastError() == cudaSuccess ? OK : ERR_CUDA; }

bool conv_shape_ok(int n, int h, int w, int cin, int cout)
{
    return n > 0 && h > 0 && w > 0 && cin > 0 && cout > 0 && cin % 32 == 0 && cout % 32 == 0 &&
           static_cast<int64_t>(n) * h * w < (int64_t(1) << 31) / 128;
}

} // namespace

extern "C" {

int dsmc_sg_conv_fwd(const uint16_t *x, const uint16_t *w, const float *bias, const uint16_t *res,
                     uint16_t *y, float *y32, int n, int h, int w_, int cin, int cout, int relu,
                     void *stream)
{
    if (!x || !w || (!y && !y32) || !conv_shape_ok(n, h, w_, cin, cout))
        return ERR_ARG;
    const int M = n * h * w_;
    dim3 grid((M + FBM - 1) / FBM, (cout + FBN - 1) / FBN);
    k_conv_fwd<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const bf16 *>(x), reinterpret_cast<const bf16 *>(w), bias,
        reinterpret_cast<const bf16 *>(res), reinterpret_cast<bf16 *>(y), y32, n, h, w_, cin,
        cout, relu);
    return status();
}

int dsmc_sg_conv_dgrad(const uint16_t *dy, const uint16_t *w, uint16_t *w_rot, uint16_t *dx,
                       int n, int h, int w_, int cin, int cout, void *stream)
{
    if (!dy || !w || !w_rot || !dx || !conv_shape_ok(n, h, w_, cin, cout))
        return ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_rotate<<<grid_for(int64_t(9) * cin * cout), 256, 0, s>>>(
        reinterpret_cast<const bf16 *>(w), reinterpret_cast<bf16 *>(w_rot), cin, cout);
    return dsmc_sg_conv_fwd(dy, w_rot, nullptr, nullptr, dx, nullptr, n, h, w_, cout, cin, 0,
                            stream);
}

int dsmc_sg_conv_wgrad(const uint16_t *dy, const uint16_t *x, float *dw, float *db, int n, int h,
                       int w_, int cin, int cout, void *stream)
{
    if (!dy || !x || !dw || !conv_shape_ok(n, h, w_, cin, cout) || (db && cout > 256))
        return ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int M = n * h * w_;
    const int tiles = ((cout + WBM - 1) / WBM) * 9 * (cin / WBN);
    // Enough pixel splits for ~4 CTAs per SM of a 148-SM part, at least
    // 512 pixels each.
    int splits = (4 * 148 + tiles - 1) / tiles;
    splits = splits < 1 ? 1 : splits;
    int per = (M + splits - 1) / splits;
    per = per < 512 ? 512 : ((per + WBK - 1) / WBK) * WBK;
    splits = (M + per - 1) / per;
    dim3 grid((cout + WBM - 1) / WBM, 9 * (cin / WBN), splits);
    k_conv_wgrad<<<grid, 256, 0, s>>>(reinterpret_cast<const bf16 *>(dy),
                                      reinterpret_cast<const bf16 *>(x), dw, n, h, w_, cin, cout,
                                      per);
    if (db) {
        k_bias_grad<<<512, 256, 0, s>>>(reinterpret_cast<const bf16 *>(dy), db, M, cout);
    }
    return status();
}

int dsmc_sg_relu_bwd(uint16_t *dy, const uint16_t *y, int64_t count, void *stream)
{
    if (!dy || !y || count < 0)
        return ERR_ARG;
    if (count % 8)
        return ERR_ARG;
    k_relu_bwd<<<grid_for(count / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<bf16 *>(dy), reinterpret_cast<const bf16 *>(y), count / 8);
    return status();
}

int dsmc_sg_pool_fwd(const uint16_t *x, uint16_t *y, int n, int h, int w_, int c, void *stream)
{
    if (!x || !y || n <= 0 || h <= 0 || w_ <= 0 || c <= 0 || h % 2 || w_ % 2 || c % 8)
        return ERR_ARG;
    k_pool_fwd<<<grid_for(int64_t(n) * h * w_ * c / 32), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const bf16 *>(x), reinterpret_cast<bf16 *>(y), n, h, w_, c);
    return status();
}

int dsmc_sg_pool_bwd(const uint16_t *dy, uint16_t *dx, int n, int h, int w_, int c, void *stream)
{
    if (!dy || !dx || n <= 0 || h <= 0 || w_ <= 0 || c <= 0 || h % 2 || w_ % 2 || c % 8)
        return ERR_ARG;
    k_pool_bwd<<<grid_for(int64_t(n) * h * w_ * c / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const bf16 *>(dy), reinterpret_cast<bf16 *>(dx), n, h, w_, c);
    return status();
}

int dsmc_sg_up_fwd(const uint16_t *x, uint16_t *y, int n, int h, int w_, int c, void *stream)
{
    if (!x || !y || n <= 0 || h <= 0 || w_ <= 0 || c <= 0 || c % 8)
        return ERR_ARG;
    k_up_fwd<<<grid_for(int64_t(n) * 4 * h * w_ * c / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const bf16 *>(x), reinterpret_cast<bf16 *>(y), n, h, w_, c);
    return status();
}

int dsmc_sg_up_bwd(const uint16_t *dy, uint16_t *dx, int n, int h, int w_, int c, void *stream)
{
    if (!dy || !dx || n <= 0 || h <= 0 || w_ <= 0 || c <= 0 || c % 8)
        return ERR_ARG;
    k_up_bwd<<<grid_for(int64_t(n) * h * w_ * c / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const bf16 *>(dy), reinterpret_cast<bf16 *>(dx), n, h, w_, c);
    return status();
}

int dsmc_sg_add(uint16_t *a, const uint16_t *b, int64_t count, void *stream)
{
    if (!a || !b || count < 0)
        return ERR_ARG;
    if (count % 8)
        return ERR_ARG;
    k_add<<<grid_for(count / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<bf16 *>(a), reinterpret_cast<const bf16 *>(b), count / 8);
    return status();
}

int dsmc_sg_mse(const float *out, const float *target, const float *mask, uint16_t *dy,
                float *loss, int64_t pixels, int c, int k, void *stream)
{
    if (!out || !target || !mask || !dy || !loss || pixels <= 0 || k <= 0 || k > c)
        return ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // loss[0] = loss, loss[1] = sum of the mask (scratch).
    if (cudaMemsetAsync(loss, 0, 2 * sizeof(float), s) != cudaSuccess)
        return ERR_CUDA;
    k_mask_sum<<<grid_for(pixels), 256, 0, s>>>(mask, pixels, loss + 1);
    k_mse<<<grid_for(pixels), 256, 0, s>>>(out, target, mask, loss + 1,
                                           reinterpret_cast<bf16 *>(dy), loss, pixels, c, k);
    return status();
}

int dsmc_sg_adam(float *w, uint16_t *w_bf16, const float *g, float *m, float *v, int64_t count,
                 float lr, float beta1, float beta2, float eps, int t, void *stream)
{
    if (!w || !g || !m || !v || count < 0 || t < 1)
        return ERR_ARG;
    const float c1 = 1.0f - powf(beta1, static_cast<float>(t));
    const float c2 = 1.0f - powf(beta2, static_cast<float>(t));
    k_adam<<<grid_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w, reinterpret_cast<bf16 *>(w_bf16), g, m, v, count, lr, beta1, beta2, eps, c1, c2);
    return status();
}

int dsmc_sg_to_bf16(const float *x, uint16_t *y, int64_t count, void *stream)
{
    if (!x || !y || count < 0)
        return ERR_ARG;
    k_to_bf16<<<grid_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        x, reinterpret_cast<bf16 *>(y), count);
    return status();
}

} // extern "C"
