// surrogate.cu - kernels of the BF16 convolutional field surrogate
// (include/dsmc_surrogate.h).
//
// The 3x3 convolutions are implicit GEMMs on the tensor cores.  Forward and
// dgrad run on the 5th-generation tensor cores (tcgen05.mma, operands in
// shared memory, FP32 accumulator in tensor memory, read back with
// tcgen05.ld); the weight gradient uses mma.sync.m16n8k16 with tiles moved
// global -> shared by cp.async and shared -> registers by ldmatrix.
//   forward  C[pixel][cout]       = sum_(tap, cin) X[pixel + tap][cin] W[cout][tap][cin]
//   dgrad    the forward with the weights rotated by 180 degrees and the
//            channel roles swapped (stride 1, padding 1: the transpose of a
//            3x3 convolution is a 3x3 convolution)
//   wgrad    C[cout][(tap, cin)]  = sum_pixel dY[pixel][cout] X[pixel + tap][cin]
//            (split over pixels, FP32 atomics into dW)
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/dsmc_surrogate.h"

namespace {

constexpr int OK = 0, ERR_ARG = 2, ERR_CUDA = 50, ERR_TIMEOUT = 60;

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

__device__ __forceinline__ void ldsm_x4_t(uint32_t r[4], const void *p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
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
// Forward (and dgrad) on the 5th-generation tensor cores.
//
// Persistent CTAs over tiles of TBM = 128 pixels x BN output channels,
// warp-specialised: warps 0-3 gather the operands, one thread of warp 4
// issues the MMAs into one of two tensor-memory accumulators (warp 4 also
// allocates them), and warps 5-8 run the epilogue of the previous tile from
// the other accumulator (warp w reads tensor-memory lanes 32 (w % 4) ..,
// thread lane l of it accumulator row 32 (w % 4) + l).  The reduction index is k = tap * Cin + ci, cut into
// chunks of TBK = 64; a chunk is gathered with cp.async (the implicit
// im2col: 8 consecutive k of a pixel are 16 contiguous bytes of x, zeros
// outside the image or beyond the 9 taps) into one of 2-3 stages.  Each
// gatherer waits for its own copies, fences them to the async proxy and
// arrives on the stage's `full` barrier; the MMA thread waits on it, issues
// the chunk's four tcgen05.mma (M 128, N BN, K 16) and commits them to the
// stage's `empty` barrier, which the gatherers wait on before the refill.
//
// Shared operands are K-major with the 128-byte swizzle: a row's 64 k (128
// bytes) fill one 128-byte line, 8-row groups are 1024-byte atoms, and the
// 16-byte piece j of row r sits at piece j ^ (r % 8) of its line:
//   (r / 8) * 1024 + (r % 8) * 128 + ((j ^ (r % 8)) * 16).
// A warp's copies then cover whole global lines (8 lanes per row) and whole
// shared lines (no bank conflict).  Descriptor: stride-byte offset 1024 (the
// next 8 rows), leading-byte offset unused (16), layout SWIZZLE_128B; the
// j-th K-16 step starts 32 j bytes into the atom.
// ---------------------------------------------------------------------------
constexpr int TBM = 128, TBK = 64;
// Stages per CTA and CTAs per SM (bounded by the 512 tensor-memory columns,
// 2 BN a CTA): measured on B200, deeper stages lose to more CTAs.
template <int BN> __host__ __device__ constexpr int tc_stages() { return BN == 64 ? 2 : 3; }
template <int BN> constexpr int tc_ctas_per_sm() { return BN == 128 ? 2 : (BN == 64 ? 4 : 3); }
constexpr int TC_THREADS = TBM + 32 + TBM; // gatherers, MMA warp, epilogue
// AMODE 3 (Cin 32, tiles of 16 pixels x 8 rows): per tile one halo box per
// tap column (dw), 10 rows x 16 pixels x 32 channels, read once for that
// column's three taps (dh), whose A operands are the box's rows dh .. dh + 7
// (1024 bytes apart: whole 64-byte-swizzle atoms); the weights of all 9
// taps stay in shared memory for the CTA's life.  Per tile 30 KB cross
// from L2 instead of 80 KB of tap boxes plus the weights.
constexpr int H3W = 16, H3H = 8;
constexpr uint32_t A3_BYTES = (H3H + 2) * H3W * 64;
constexpr uint32_t TC_SPIN_LIMIT = 1u << 22;

__device__ int g_tc_error; // a bounded wait of a tensor-core kernel gave up

__device__ __forceinline__ void tc_mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void tc_mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool tc_mbar_wait(uint64_t *bar, uint32_t parity)
{
    for (uint32_t spins = 0; spins < TC_SPIN_LIMIT; ++spins) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(smem_u32(bar)), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}
// The next arrival on `bar` also expects `bytes` from bulk tensor copies.
__device__ __forceinline__ void tc_mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// TMA tile loads (no multicast) completing on an mbarrier of this CTA.
// Coordinates are elements, innermost first; boxes outside the tensor read
// zeros.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, int c3, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
                 "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
                 : "memory");
}
// Shared-memory matrix descriptor: K-major, 64-byte swizzle (rows of 32
// bf16, 8-row atoms of 512 bytes), version 1.
__device__ __forceinline__ uint64_t umma_desc_sw64(uint32_t saddr)
{
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (1ull << 16) |
           (static_cast<uint64_t>(512 >> 4) << 32) | (1ull << 46) | (4ull << 61);
}
// Shared-memory matrix descriptor: K-major, 128-byte swizzle, version 1.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr)
{
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (1ull << 16) | // LBO (unused)
           (static_cast<uint64_t>(1024 >> 4) << 32) |                     // SBO: 8 rows
           (1ull << 46) |                                                 // version
           (2ull << 61);                                                  // SWIZZLE_128B
}
// Byte offset of 16-byte piece j of row r in a swizzled operand.
__device__ __forceinline__ uint32_t sw128_off(int r, int j)
{
    return static_cast<uint32_t>((r >> 3) * 1024 + (r & 7) * 128 + ((j ^ (r & 7)) << 4));
}
// Instruction descriptor: bf16 A and B (K-major), FP32 accumulator, M x N.
template <int BN> __host__ __device__ constexpr uint32_t umma_idesc()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(BN >> 3) << 17) |
           (static_cast<uint32_t>(TBM >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                 : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t r[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Stages plus 1 KB to align the first to a swizzle atom.
template <int BN> constexpr int tc_smem() { return tc_stages<BN>() * (TBM + BN) * TBK * 2 + 1024; }
// CTAs per SM of AMODE 3 (measured: for 64 channels what its shared memory
// lets reside, 3 instead of the tap-tile form's 4; 4 for 32 channels, which
// would fit, measured slower than 3).
template <int BN> constexpr int tc_ctas_per_sm3() { return BN == 128 ? 2 : 3; }
template <int BN> constexpr int tc_smem3()
{
    return tc_stages<BN>() * static_cast<int>(A3_BYTES) + 9 * BN * 64 + 1024;
}

// The forward epilogue of 16 channels co .. co + 15 at element offset o
// (pixel * Cout + co): bias and ReLU on the accumulators v, then the residual
// (added to y, or as the skip sum ysum = bf16(y) + res, y kept for the
// ReLU's gradient) and the bf16 / FP32 stores.
__device__ __forceinline__ void fwd_store16(float v[16], int64_t o, int co,
                                            const float *__restrict__ bias, int relu,
                                            const bf16 *__restrict__ res, bf16 *__restrict__ y,
                                            bf16 *__restrict__ ysum, float *__restrict__ y32)
{
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        v[e] += bias ? bias[co + e] : 0.0f;
        if (relu)
            v[e] = fmaxf(v[e], 0.0f);
    }
    if (ysum) {
#pragma unroll
        for (int h8 = 0; h8 < 2; ++h8) {
            const V8 rr = ld8(res + o + 8 * h8);
            V8 out;
#pragma unroll
            for (int e = 0; e < 8; ++e)
                out.v[e] = static_cast<float>(__float2bfloat16(v[8 * h8 + e])) + rr.v[e];
            st8(ysum + o + 8 * h8, out);
        }
    } else if (res) {
#pragma unroll
        for (int h8 = 0; h8 < 2; ++h8) {
            const V8 rr = ld8(res + o + 8 * h8);
#pragma unroll
            for (int e = 0; e < 8; ++e)
                v[8 * h8 + e] += rr.v[e];
        }
    }
    if (y) {
#pragma unroll
        for (int h8 = 0; h8 < 2; ++h8) {
            V8 out;
#pragma unroll
            for (int e = 0; e < 8; ++e)
                out.v[e] = v[8 * h8 + e];
            st8(y + o + 8 * h8, out);
        }
    }
    if (y32) {
#pragma unroll
        for (int e4 = 0; e4 < 4; ++e4)
            *reinterpret_cast<float4 *>(y32 + o + 4 * e4) =
                make_float4(v[4 * e4], v[4 * e4 + 1], v[4 * e4 + 2], v[4 * e4 + 3]);
    }
}

// AMODE selects how the stages are filled: 0, the cp.async im2col gather
// (any shape); 1 and 2, TMA tile loads by one thread, for shapes whose
// 128-pixel tile is a BW x BH rectangle of one image: the input through a
// 4-D map [N][H][W][Cin] whose box is read at the tap's offset (zeros
// outside the image are the padding), the weights through a 2-D map
// [Cout][9 Cin].  AMODE 1 (Cin a multiple of 64): one box of 64 channels per
// chunk, 128-byte swizzle, as the gather lays it out.  AMODE 2 (Cin 32): a
// chunk is two taps, two boxes of 32 channels in 64-byte-swizzled K-major
// tiles of 8 KB each (a tenth tap reads a box wholly outside the image).
// AMODE 3: the halo boxes described at A3_BYTES (Cin 32, Cout = BN, W a
// multiple of 16, H of 8), the weights through a 2-D map [Cout][9 Cin] in
// boxes of 32 k (one tap) x BN rows, 64-byte swizzle.
template <int BN, int AMODE>
__global__ void __launch_bounds__(TC_THREADS)
    k_conv_fwd_tc(const bf16 *__restrict__ x, const bf16 *__restrict__ w,
                  const float *__restrict__ bias, const bf16 *__restrict__ res,
                  bf16 *__restrict__ y, bf16 *__restrict__ ysum, float *__restrict__ y32, int N,
                  int H, int W, int Cin,
                  int Cout, int relu, const __grid_constant__ CUtensorMap tmx,
                  const __grid_constant__ CUtensorMap tmw, int BW, int BH)
{
    static_assert(BN == 32 || BN == 64 || BN == 128, "tensor-memory columns: a power of 2");
    static_assert(AMODE >= 0 && AMODE <= 3,
                  "gather, TMA 128-byte, TMA 64-byte tap tiles, TMA halo boxes");
    constexpr int TST = tc_stages<BN>();
    constexpr uint32_t A_BYTES = TBM * TBK * 2, B_BYTES = BN * TBK * 2;
    constexpr uint32_t STAGE = AMODE == 3 ? A3_BYTES : A_BYTES + B_BYTES;
    extern __shared__ __align__(1024) unsigned char tc_smem_dyn[];
    __shared__ uint64_t bar_full[TST], bar_empty[TST];
    __shared__ uint64_t bar_acc_full[2], bar_acc_empty[2];
    __shared__ uint64_t bar_done;
    __shared__ uint64_t bar_w; // AMODE 3: the resident weights have landed
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int M = N * H * W;
    const int K = 9 * Cin;
    const int KT = AMODE == 3 ? 3 : (K + TBK - 1) / TBK; // AMODE 3: one chunk per tap column
    const int ntiles_n = Cout / BN;
    const int ntiles = AMODE == 3 ? N * (H / H3H) * (W / H3W)
                                  : ((M + TBM - 1) / TBM) * ntiles_n;
    // AMODE 3: image and top-left pixel of tile t (row-major over 16 x 8 tiles).
    auto tile3 = [&](int t, int &img, int &th, int &tw) {
        const int tx = W / H3W, per = tx * (H / H3H);
        img = t / per;
        const int r = t % per;
        th = (r / tx) * H3H;
        tw = (r % tx) * H3W;
    };

    if (warp == 4) { // two accumulators: the epilogue of a tile overlaps the next
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&s_tmem)), "r"(2 * BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < TST; ++i) {
            tc_mbar_init(&bar_full[i], AMODE ? 1 : TBM); // the TMA thread or every gatherer
            tc_mbar_init(&bar_empty[i], 1);  // one tcgen05.commit
        }
        for (int i = 0; i < 2; ++i) {
            tc_mbar_init(&bar_acc_full[i], 1);    // one tcgen05.commit
            tc_mbar_init(&bar_acc_empty[i], TBM); // every epilogue thread arrives
        }
        tc_mbar_init(&bar_done, 1);
        tc_mbar_init(&bar_w, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    bool ok = true;
    // The swizzle acts on address bits: stages start on 1024-byte boundaries.
    unsigned char *tc_smem_raw =
        tc_smem_dyn + ((1024u - (smem_u32(tc_smem_dyn) & 1023u)) & 1023u);
    unsigned char *const w3_smem = tc_smem_raw + TST * A3_BYTES; // AMODE 3 weights

    if (AMODE == 3 && warp < 4) {
        if (tid == 0) { // TMA producer: the weights once, then per tile a box per tap column
            tc_mbar_expect_tx(&bar_w, 9u * BN * 64u);
            for (int tap = 0; tap < 9; ++tap)
                tma_load_2d(w3_smem + tap * BN * 64, &tmw, 32 * tap, 0, &bar_w);
            int g = 0;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                int img, th, tw;
                tile3(t, img, th, tw);
                for (int d = 0; d < 3; ++d, ++g) { // tap column dw = d - 1
                    const int st = g % TST;
                    if (g >= TST)
                        ok = tc_mbar_wait(&bar_empty[st],
                                          static_cast<uint32_t>(((g - TST) / TST) & 1));
                    if (!ok)
                        break;
                    tc_mbar_expect_tx(&bar_full[st], A3_BYTES);
                    // Rows th - 1 .. th + 8, pixels tw + d - 1 ..: zeros outside
                    // the image are the padding.
                    tma_load_4d(tc_smem_raw + st * A3_BYTES, &tmx, 0, tw + d - 1, th - 1, img,
                                &bar_full[st]);
                }
            }
        }
    } else if (AMODE && warp < 4) {
        if (tid == 0) { // TMA producer: chunks in the order the MMA thread takes them
            int g = 0;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const int m0 = (t / ntiles_n) * TBM, n0 = (t % ntiles_n) * BN;
                const int img = m0 / (H * W), rem = m0 % (H * W);
                const int h0 = rem / W, w0 = rem % W;
                for (int kc = 0; kc < KT; ++kc, ++g) {
                    const int st = g % TST;
                    if (g >= TST)
                        ok = tc_mbar_wait(&bar_empty[st],
                                          static_cast<uint32_t>(((g - TST) / TST) & 1));
                    if (!ok)
                        break;
                    unsigned char *sa = tc_smem_raw + st * STAGE;
                    tc_mbar_expect_tx(&bar_full[st], STAGE);
                    if (AMODE == 1) {
                        const int k = kc * TBK, tap = k / Cin;
                        tma_load_4d(sa, &tmx, k % Cin, w0 + tap % 3 - 1, h0 + tap / 3 - 1, img,
                                    &bar_full[st]);
                    } else {
#pragma unroll
                        for (int half = 0; half < 2; ++half) {
                            const int tap = 2 * kc + half;
                            const int hh = tap < 9 ? h0 + tap / 3 - 1 : -BH - 1;
                            tma_load_4d(sa + half * (A_BYTES / 2), &tmx, 0, w0 + tap % 3 - 1, hh,
                                        img, &bar_full[st]);
                        }
                    }
                    tma_load_2d(sa + A_BYTES, &tmw, kc * TBK, n0, &bar_full[st]);
                }
            }
        }
    } else if (warp < 4) {
        // Gatherer: piece j = tid % 8 of rows tid / 8 + 16 i of A (i < 8)
        // and of B (i < BN / 16).  Chunks are counted across the CTA's tiles
        // (g), so the stage ring runs on from one tile to the next.
        const int j = tid & 7, r0 = tid >> 3;
        int g = 0;
        auto publish = [&](int gc) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_mbar_arrive(&bar_full[gc % TST]);
        };
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const int m0 = (t / ntiles_n) * TBM, n0 = (t % ntiles_n) * BN;
            int ah[TBM / 16], aw[TBM / 16];
            bool am[TBM / 16];
#pragma unroll
            for (int i = 0; i < TBM / 16; ++i) {
                const int m = m0 + r0 + 16 * i;
                am[i] = m < M;
                const int mm = am[i] ? m : 0;
                ah[i] = (mm / W) % H;
                aw[i] = mm % W;
            }
            // Element offset of row r0 in x; row r0 + 16 i is 16 i Cin on.
            const int64_t arow = static_cast<int64_t>(m0 + r0) * Cin;
            for (int kc = 0; kc < KT; ++kc, ++g) {
                const int st = g % TST;
                if (g >= TST && ok)
                    ok = tc_mbar_wait(&bar_empty[st],
                                      static_cast<uint32_t>(((g - TST) / TST) & 1));
                if (ok) {
                    unsigned char *sa = tc_smem_raw + st * STAGE;
                    unsigned char *sb = sa + A_BYTES;
                    const int k = kc * TBK + 8 * j;
                    const bool kin = k < K;
                    const int tap = kin ? k / Cin : 0, ci = k % Cin;
                    const int dh = tap / 3 - 1, dw = tap % 3 - 1;
                    // The tap's pixel is dh W + dw pixels from the row's own.
                    const int64_t koff = arow + static_cast<int64_t>(dh * W + dw) * Cin + ci;
                    const int64_t rstep = 16 * static_cast<int64_t>(Cin);
#pragma unroll
                    for (int i = 0; i < TBM / 16; ++i) {
                        const int hh = ah[i] + dh, ww = aw[i] + dw;
                        const bool v = am[i] && kin && hh >= 0 && hh < H && ww >= 0 && ww < W;
                        const bf16 *src = v ? x + (koff + i * rstep) : x;
                        cp_async16(sa + sw128_off(r0 + 16 * i, j), src, v);
                    }
#pragma unroll
                    for (int i = 0; i < BN / 16; ++i) {
                        const int row = r0 + 16 * i;
                        const int co = n0 + row;
                        const bool v = co < Cout && kin;
                        // w[co][tap][ci] is w[co][k]: k runs over taps and channels.
                        const bf16 *src = v ? w + static_cast<int64_t>(co) * K + k : w;
                        cp_async16(sb + sw128_off(row, j), src, v);
                    }
                }
                cp_async_commit();
                // Keep TST - 1 chunks in flight; a chunk's barrier gets this
                // thread's arrival once its copies have landed.
                if (g >= TST - 1) {
                    cp_async_wait<TST - 1>();
                    publish(g - (TST - 1));
                }
            }
        }
        cp_async_wait<0>();
        for (int gc = g - (TST - 1) < 0 ? 0 : g - (TST - 1); gc < g; ++gc)
            publish(gc);
    } else if (warp == 4) {
        if (lane == 0) { // MMA issuer
            int g = 0, i = 0;
            if (AMODE == 3)
                ok = tc_mbar_wait(&bar_w, 0);
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++i) {
                const int b = i & 1;
                if (i >= 2)
                    ok = tc_mbar_wait(&bar_acc_empty[b],
                                      static_cast<uint32_t>(((i >> 1) - 1) & 1));
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                for (int kc = 0; kc < KT && ok; ++kc, ++g) {
                    const int st = g % TST;
                    ok = tc_mbar_wait(&bar_full[st], static_cast<uint32_t>((g / TST) & 1));
                    if (!ok)
                        break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = smem_u32(tc_smem_raw + st * STAGE), sb = sa + A_BYTES;
                    if constexpr (AMODE == 3) {
                        // Chunk kc is tap column dw = kc - 1; tap (dh, dw) reads
                        // box rows dh + 1 .. dh + 8, 1024 bytes per row of 16
                        // pixels, and weight box 3 (dh + 1) + kc.
                        const uint32_t sw = smem_u32(w3_smem);
#pragma unroll
                        for (int r = 0; r < 3; ++r)
#pragma unroll
                            for (int kk = 0; kk < 2; ++kk)
                                umma_bf16(tmem + static_cast<uint32_t>(b * BN),
                                          umma_desc_sw64(sa + 1024u * r + 32 * kk),
                                          umma_desc_sw64(sw + (3 * r + kc) * BN * 64 + 32 * kk),
                                          umma_idesc<BN>(), (kc > 0 || r > 0 || kk > 0) ? 1u : 0u);
                    } else {
#pragma unroll
                        for (int kk = 0; kk < TBK / 16; ++kk) {
                            // AMODE 2: k 0-31 in the first 64-byte-swizzled
                            // tile, 32-63 in the second.
                            const uint64_t da =
                                AMODE == 2 ? umma_desc_sw64(sa + (kk >> 1) * (A_BYTES / 2) +
                                                            32 * (kk & 1))
                                           : umma_desc_sw128(sa + 32 * kk);
                            umma_bf16(tmem + static_cast<uint32_t>(b * BN), da,
                                      umma_desc_sw128(sb + 32 * kk), umma_idesc<BN>(),
                                      (kc > 0 || kk > 0) ? 1u : 0u);
                        }
                    }
                    umma_commit(&bar_empty[st]);
                }
                umma_commit(&bar_acc_full[b]);
            }
            umma_commit(&bar_done); // arrives once every MMA issued above is complete
        }
    } else {
        // Epilogue: warps 5-8; warp w reads tensor-memory lanes 32 (w % 4) ..
        const int q = warp & 3;
        const int row = 32 * q + lane;
        int i = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
            const int b = i & 1;
            if (ok)
                ok = tc_mbar_wait(&bar_acc_full[b], static_cast<uint32_t>((i >> 1) & 1));
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int m, n0;
            if (AMODE == 3) { // accumulator row = pixel (th + row / 16, tw + row % 16)
                int img, th, tw;
                tile3(t, img, th, tw);
                m = (img * H + th + row / H3W) * W + tw + row % H3W;
                n0 = 0;
            } else {
                m = (t / ntiles_n) * TBM + row;
                n0 = (t % ntiles_n) * BN;
            }
            const bool am = m < M;
            // Rolled: each load waits for its tensor-memory read anyway, and
            // unrolled copies of the store paths spill.
#pragma unroll 1
            for (int c = 0; c < BN; c += 16) {
                uint32_t r[16];
                tmem_ld16(tmem + (static_cast<uint32_t>(32 * q) << 16) +
                              static_cast<uint32_t>(b * BN + c),
                          r);
                const int co = n0 + c;
                if (!ok || !am || co >= Cout)
                    continue;
                float v[16];
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    v[e] = __uint_as_float(r[e]);
                fwd_store16(v, static_cast<int64_t>(m) * Cout + co, co, bias, relu, res, y, ysum,
                            y32);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            tc_mbar_arrive(&bar_acc_empty[b]); // this buffer may be reused
        }
    }
    // Every MMA is complete before the tensor memory is released.
    const bool done = tc_mbar_wait(&bar_done, 0);
    if (!__syncthreads_and(ok && done) && tid == 0)
        atomicExch(&g_tc_error, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 4)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(2 * BN)
                     : "memory");
}

// ---------------------------------------------------------------------------
// Weight gradient on the 5th-generation tensor cores (Cin 32, 64 or 128;
// Cout up to 256).  A CTA takes a group of TAPS = 128 / Cin taps and a range
// of pixels and accumulates
//   D[(tap, ci)][co] = sum_p X[p + off(tap)][ci] dY[p][co]
// in tensor memory (M 128 = taps x Cin, N = Cout rounded up to NB; K =
// 64-pixel chunks), then adds D to dW with FP32 atomics, coalesced over the
// input channels of a warp.  Both operands are MN-major (the pixel is the
// reduction index; channels are contiguous in memory), 128-byte swizzled:
// element (row m, pixel k) at
//   (m / 64) * 1024 + (k / 8) * SBO + (k % 8) * 128 + (((m % 64) / 8) ^ (k % 8)) * 16,
// SBO being the bytes of one 8-pixel group of all the rows; the descriptor's
// leading-byte offset is the 1024 between 64-row atoms, and the j-th K-16
// step starts 2 j groups in.  Rows of a tap past the ninth and columns past
// Cout are zero-filled.  Gatherers, MMA thread and barriers as in the
// forward kernel; 3 stages, 1-3 CTAs per SM by NB.
// ---------------------------------------------------------------------------
constexpr int WG_PIX = 64, WG_ST = 3;
constexpr int WG_THREADS = 128 + 32;

// MN-major descriptor with the given leading (between MN atoms) and stride
// (between 8-deep K groups) byte offsets; layout 2 = 128-byte swizzle (64-wide
// atoms), 4 = 64-byte swizzle (32-wide atoms).
__device__ __forceinline__ uint64_t umma_desc_mn(uint32_t saddr, uint32_t lbo, uint32_t sbo,
                                                 uint32_t layout)
{
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) |
           (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) |
           (static_cast<uint64_t>(layout) << 61);
}
__device__ __forceinline__ uint64_t umma_desc_sw128_mn(uint32_t saddr, uint32_t sbo)
{
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(1024 >> 4) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}
// bf16 x bf16 -> FP32, both operands MN-major, M 128 x N.
template <int N> __host__ __device__ constexpr uint32_t umma_idesc_mn()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
           (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(128 >> 4) << 24);
}
__device__ __forceinline__ uint32_t sw128_mn_off(int m, int k, uint32_t sbo)
{
    return static_cast<uint32_t>((m >> 6) * 1024) + static_cast<uint32_t>(k >> 3) * sbo +
           static_cast<uint32_t>((k & 7) * 128 + ((((m & 63) >> 3) ^ (k & 7)) << 4));
}
template <int NB> __host__ __device__ constexpr int wg_stage() { return 128 * WG_PIX * 2 + NB * WG_PIX * 2; }
template <int NB> constexpr int wg_smem() { return WG_ST * wg_stage<NB>() + 1024; }
template <int NB> constexpr int wg_ctas_per_sm() { return NB <= 64 ? 3 : (NB == 128 ? 2 : 1); }

// TMA: the stages are filled by one thread with tile loads for shapes whose
// 64-pixel chunks are BW x BH rectangles of one image: per tap a box of
// CB = min(Cin, 64) channels x 64 pixels from a 4-D map of X (zeros outside
// the image; a tap past the ninth reads a box wholly outside), and NB / 64
// boxes of 64 channels x 64 pixels from a 2-D map of dY [pixels][Cout]
// (zeros past Cout).  A box is rows of pixels as they sit in memory, which
// is the MN-major swizzled tile: atoms along M a box apart (LBO), 8-pixel
// groups one atom row apart (SBO); 64-byte swizzle for Cin 32.  NB 32 (Cout
// 32, TMA only): one dY box of 32 channels, 64-byte swizzle, N = 32.
template <int CI, int NB, bool TMA>
__global__ void __launch_bounds__(WG_THREADS)
    k_conv_wgrad_tc(const bf16 *__restrict__ dy, const bf16 *__restrict__ x,
                    float *__restrict__ dw, int N, int H, int W, int Cout, int per,
                    const __grid_constant__ CUtensorMap tmx,
                    const __grid_constant__ CUtensorMap tmy, int BW, int BH)
{
    static_assert(CI == 32 || CI == 64 || CI == 128, "taps x Cin fill the 128 rows");
    static_assert(NB == 32 || NB == 64 || NB == 128 || NB == 256,
                  "one 32-channel or whole 64-channel swizzle atoms");
    static_assert(NB != 32 || TMA, "32 output channels: TMA boxes only");
    constexpr int TAPS = 128 / CI;
    constexpr uint32_t A_BYTES = 128 * WG_PIX * 2;
    constexpr uint32_t STAGE = wg_stage<NB>();
    constexpr uint32_t SBO_A = 2 * 1024, SBO_B = (NB / 64) * 1024;
    extern __shared__ __align__(1024) unsigned char wg_smem_dyn[];
    __shared__ uint64_t bar_full[WG_ST], bar_empty[WG_ST];
    __shared__ uint64_t bar_done;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int M = N * H * W;
    const int tap0 = blockIdx.y * TAPS;
    const int p_begin = blockIdx.x * per;
    const int p_end = min(M, p_begin + per);
    const int KT = p_end > p_begin ? (p_end - p_begin + WG_PIX - 1) / WG_PIX : 0;

    if (warp == 4) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&s_tmem)), "r"(NB)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < WG_ST; ++i) {
            tc_mbar_init(&bar_full[i], TMA ? 1 : 128);
            tc_mbar_init(&bar_empty[i], 1);
        }
        tc_mbar_init(&bar_done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    bool ok = true;
    unsigned char *sm = wg_smem_dyn + ((1024u - (smem_u32(wg_smem_dyn) & 1023u)) & 1023u);

    constexpr int CB = CI < 64 ? CI : 64;                  // channels of an X box
    constexpr int YC = NB < 64 ? NB : 64;                  // channels of a dY box
    constexpr uint32_t XBOX = CB * WG_PIX * 2, YBOX = YC * WG_PIX * 2;
    if (TMA && warp < 4) {
        if (tid == 0) {
            for (int kc = 0; kc < KT; ++kc) {
                const int st = kc % WG_ST;
                if (kc >= WG_ST)
                    ok = tc_mbar_wait(&bar_empty[st],
                                      static_cast<uint32_t>(((kc - WG_ST) / WG_ST) & 1));
                if (!ok)
                    break;
                unsigned char *sa = sm + st * STAGE;
                const int p0 = p_begin + kc * WG_PIX;
                const int img = p0 / (H * W), rem = p0 % (H * W);
                const int h0 = rem / W, w0 = rem % W;
                tc_mbar_expect_tx(&bar_full[st], STAGE);
#pragma unroll
                for (int b = 0; b < 128 / CB; ++b) {
                    // Box b: tap tap0 + b (Cin <= 64) or channels 64 b of tap0.
                    const int tap = CI <= 64 ? tap0 + b : tap0;
                    const int hh = tap < 9 ? h0 + tap / 3 - 1 : -BH - 1;
                    tma_load_4d(sa + b * XBOX, &tmx, CI <= 64 ? 0 : 64 * b, w0 + tap % 3 - 1, hh,
                                img, &bar_full[st]);
                }
#pragma unroll
                for (int b = 0; b < NB / YC; ++b)
                    tma_load_2d(sa + A_BYTES + b * YBOX, &tmy, YC * b, p0, &bar_full[st]);
            }
        }
    } else if (warp < 4) {
        // The 16 pieces of 8 rows a thread gathers: row 8 j = (tap tl, input
        // channels ci8 .. ci8 + 7), the same for every chunk.
        const int j = tid & 15;
        const int tap = tap0 + (8 * j) / CI, ci8 = (8 * j) % CI;
        const bool tap_ok = tap < 9;
        const int dh = tap / 3 - 1, dwx = tap % 3 - 1;
        // Element offsets of the thread's first X and dY pieces in chunk 0;
        // piece i is 8 i pixels on, a chunk 64 pixels.
        const int64_t xoff0 =
            (static_cast<int64_t>(p_begin) + (tid >> 4) + static_cast<int64_t>(dh) * W + dwx) * CI +
            ci8;
        constexpr int BJ = NB / 8; // 16-byte pieces of a dY row
        const int jb = tid % BJ;
        const bool col_ok = 8 * jb < Cout;
        const int64_t yoff0 = static_cast<int64_t>(p_begin + tid / BJ) * Cout + 8 * jb;
        const int64_t ystep = static_cast<int64_t>(128 / BJ) * Cout;
        // Row and column of the thread's 8 pixels (tid / 16 + 8 i of each
        // chunk), stepped by 64 pixels a chunk instead of divided out.
        int hh[8], ww[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int p = p_begin + (tid >> 4) + 8 * i;
            hh[i] = (p / W) % H;
            ww[i] = p % W;
        }
        auto publish = [&](int kc) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_mbar_arrive(&bar_full[kc % WG_ST]);
        };
        for (int kc = 0; kc < KT; ++kc) {
            const int st = kc % WG_ST;
            if (kc >= WG_ST && ok)
                ok = tc_mbar_wait(&bar_empty[st], static_cast<uint32_t>(((kc - WG_ST) / WG_ST) & 1));
            if (ok) {
                unsigned char *sa = sm + st * STAGE;
                const int p0 = p_begin + kc * WG_PIX;
                const int64_t xoff = xoff0 + static_cast<int64_t>(kc) * WG_PIX * CI;
                const int64_t yoff = yoff0 + static_cast<int64_t>(kc) * WG_PIX * Cout;
                // X at the taps: 64 pixels x 16 pieces of 8 rows.
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int pp = (tid >> 4) + 8 * i;
                    const int h2 = hh[i] + dh, w2 = ww[i] + dwx;
                    const bool v =
                        tap_ok && p0 + pp < p_end && h2 >= 0 && h2 < H && w2 >= 0 && w2 < W;
                    const bf16 *src = v ? x + (xoff + 8 * i * CI) : x;
                    cp_async16(sa + sw128_mn_off(8 * j, pp, SBO_A), src, v);
                }
                // dY: 64 pixels x NB / 8 pieces of 8 output channels.
#pragma unroll
                for (int i = 0; i < BJ * WG_PIX / 128; ++i) {
                    const int pp = tid / BJ + (128 / BJ) * i;
                    const bool v = col_ok && p0 + pp < p_end;
                    const bf16 *src = v ? dy + (yoff + i * ystep) : dy;
                    cp_async16(sa + A_BYTES + sw128_mn_off(8 * jb, pp, SBO_B), src, v);
                }
            }
            cp_async_commit();
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                ww[i] += WG_PIX;
                while (ww[i] >= W) {
                    ww[i] -= W;
                    hh[i] = hh[i] + 1 == H ? 0 : hh[i] + 1;
                }
            }
            if (kc >= WG_ST - 1) {
                cp_async_wait<WG_ST - 1>();
                publish(kc - (WG_ST - 1));
            }
        }
        cp_async_wait<0>();
        for (int kc = KT - (WG_ST - 1) < 0 ? 0 : KT - (WG_ST - 1); kc < KT; ++kc)
            publish(kc);
    } else if (tid == 128) {
        for (int kc = 0; kc < KT && ok; ++kc) {
            const int st = kc % WG_ST;
            ok = tc_mbar_wait(&bar_full[st], static_cast<uint32_t>((kc / WG_ST) & 1));
            if (!ok)
                break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_u32(sm + st * STAGE);
#pragma unroll
            for (int kk = 0; kk < WG_PIX / 16; ++kk) {
                // TMA boxes: 8-pixel groups of CB (X) or YC (dY) channels.
                const uint64_t da =
                    TMA ? umma_desc_mn(sa + kk * 2 * (CB * 16), XBOX, CB * 16, CB == 64 ? 2 : 4)
                        : umma_desc_sw128_mn(sa + kk * 2 * SBO_A, SBO_A);
                const uint64_t db =
                    TMA ? umma_desc_mn(sa + A_BYTES + kk * 2 * (YC * 16), YBOX, YC * 16,
                                       YC == 64 ? 2 : 4)
                        : umma_desc_sw128_mn(sa + A_BYTES + kk * 2 * SBO_B, SBO_B);
                umma_bf16(tmem, da, db, umma_idesc_mn<NB>(), (kc > 0 || kk > 0) ? 1u : 0u);
            }
            umma_commit(&bar_empty[st]);
        }
        umma_commit(&bar_done);
    }
    const bool done = tc_mbar_wait(&bar_done, 0);
    const bool ok_all = __syncthreads_and(ok && done);
    if (!ok_all && tid == 0)
        atomicExch(&g_tc_error, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok_all && warp < 4 && KT > 0) {
        // Tensor-memory lane = row = (tap, input channel); columns = Cout.
        const int tap = tap0 + tid / CI, ci = tid % CI;
        const bool row_ok = tap < 9;
        float *d = dw + static_cast<int64_t>(tap) * CI + ci;
#pragma unroll 1
        for (int c = 0; c < NB && c < Cout; c += 16) {
            uint32_t r[16];
            tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c),
                      r);
            if (!row_ok)
                continue;
#pragma unroll
            for (int e = 0; e < 16; ++e)
                if (c + e < Cout)
                    atomicAdd(d + static_cast<int64_t>(c + e) * 9 * CI, __uint_as_float(r[e]));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 4)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NB)
                     : "memory");
}

// ---------------------------------------------------------------------------
// wgrad for Cin 32 on images of 16-pixel columns and 8-pixel rows, Cout = NB
// (32 or 64).  Per 16 x 8-pixel tile: one halo box of X, 10 rows (th - 1 ..
// th + 8) x 16 pixels x 32 channels (the forward's AMODE 3 box), and three
// boxes of dY, 8 rows x 16 pixels x NB channels, at columns tw + 1, tw,
// tw - 1.  One MMA per image row of the tile: M = 128 rows (four 32-row
// atoms, taps dh = -1, 0, 1 and a fourth whose rows are discarded) x N = 3
// NB (taps dw = -1, 0, 1) x K = 16 pixels, both operands MN-major.  The A
// atom of dh is the X box shifted by dh + 1 image rows (1024 bytes, whole
// 64-byte-swizzle atoms: leading offset 1024, stride 512 between 8-pixel
// groups; the fourth atom reads a row past the box, inside the slot); the B
// atom of dw is the dY box shifted by -dw columns (leading offset one box).
// So pixel p pairs X[p + (dh, 0)] with dY[p - (0, dw)]: over a row of tiles
// each q = p - (0, dw) meets X[q + (dh, dw)] once; the column a shift
// leaves out meets only padding, the one it brings in reads dY's zero fill.
// Per tile 34 KB (NB 32) cross from L2 and 8 MMAs of N = 96 issue, against
// 120 KB and 24 MMAs of N = 32 for the tap-box form's three tap groups; 3/4
// of the MMA rows are useful in both.  Tap (dh, dw) accumulates into tensor-
// memory lanes 32 (dh + 1) + ci, columns (dw + 1) NB + co, over all the
// CTA's tiles; one CTA per SM over a contiguous range of tiles; producer
// thread 0, MMA thread 32, epilogue warps 0-2 (the lanes of useful atoms).
// ---------------------------------------------------------------------------
constexpr uint32_t WH_XSLOT = (H3H + 3) * H3W * 64; // a box and the fourth atom's extra row
template <int NB> __host__ __device__ constexpr int wh_stages() { return NB == 32 ? 6 : 3; }
template <int NB> __host__ __device__ constexpr uint32_t wh_ybytes() { return H3W * H3H * NB * 2; }
template <int NB> __host__ __device__ constexpr uint32_t wh_stage()
{
    return WH_XSLOT + 3 * wh_ybytes<NB>();
}
template <int NB> constexpr int wh_smem()
{
    return wh_stages<NB>() * static_cast<int>(wh_stage<NB>()) + 1024;
}

template <int NB>
__global__ void __launch_bounds__(128, 1)
    k_conv_wgrad_halo(float *__restrict__ dw, int N, int H, int W, int per,
                      const __grid_constant__ CUtensorMap tmx,
                      const __grid_constant__ CUtensorMap tmy)
{
    static_assert(NB == 32 || NB == 64, "one dY box of 32 or 64 channels");
    constexpr int WH_ST = wh_stages<NB>();
    constexpr uint32_t STAGE = wh_stage<NB>(), YBYTES = wh_ybytes<NB>();
    constexpr uint32_t TCOLS = NB == 32 ? 128 : 256; // 3 NB accumulator columns
    static_assert(STAGE % 1024 == 0 && WH_XSLOT % 1024 == 0, "swizzle atoms stay aligned");
    extern __shared__ __align__(1024) unsigned char wh_smem_dyn[];
    __shared__ uint64_t bar_full[WH_ST], bar_empty[WH_ST];
    __shared__ uint64_t bar_done;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tx = W / H3W, tpi = tx * (H / H3H);
    const int ntiles = N * tpi;
    const int t_begin = blockIdx.x * per;
    const int KT = max(0, min(ntiles, t_begin + per) - t_begin);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&s_tmem)), "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 32) {
        for (int i = 0; i < WH_ST; ++i) {
            tc_mbar_init(&bar_full[i], 1);
            tc_mbar_init(&bar_empty[i], 1);
        }
        tc_mbar_init(&bar_done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    bool ok = true;
    unsigned char *sm = wh_smem_dyn + ((1024u - (smem_u32(wh_smem_dyn) & 1023u)) & 1023u);

    if (tid == 0) {
        for (int kc = 0; kc < KT; ++kc) {
            const int st = kc % WH_ST;
            if (kc >= WH_ST)
                ok = tc_mbar_wait(&bar_empty[st], static_cast<uint32_t>(((kc - WH_ST) / WH_ST) & 1));
            if (!ok)
                break;
            const int t = t_begin + kc, img = t / tpi, r = t % tpi;
            const int th = (r / tx) * H3H, tw = (r % tx) * H3W;
            unsigned char *sa = sm + st * STAGE;
            tc_mbar_expect_tx(&bar_full[st], A3_BYTES + 3 * YBYTES);
            tma_load_4d(sa, &tmx, 0, tw, th - 1, img, &bar_full[st]);
#pragma unroll
            for (int d = 0; d < 3; ++d) // tap dw = d - 1: dY shifted by -dw columns
                tma_load_4d(sa + WH_XSLOT + d * YBYTES, &tmy, 0, tw + 1 - d, th, img,
                            &bar_full[st]);
        }
    } else if (tid == 32) {
        for (int kc = 0; kc < KT && ok; ++kc) {
            const int st = kc % WH_ST;
            ok = tc_mbar_wait(&bar_full[st], static_cast<uint32_t>((kc / WH_ST) & 1));
            if (!ok)
                break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_u32(sm + st * STAGE), sy = sa + WH_XSLOT;
#pragma unroll
            for (int kk = 0; kk < H3H; ++kk) {
                // K step kk: image row kk of the tile (two 8-pixel groups).
                const uint64_t da = umma_desc_mn(sa + kk * 1024, 1024, 512, 4);
                const uint64_t db =
                    umma_desc_mn(sy + kk * 2 * (NB * 16), YBYTES, NB * 16, NB == 64 ? 2 : 4);
                umma_bf16(tmem, da, db, umma_idesc_mn<3 * NB>(), (kc > 0 || kk > 0) ? 1u : 0u);
            }
            umma_commit(&bar_empty[st]);
        }
        umma_commit(&bar_done);
    }
    const bool done = tc_mbar_wait(&bar_done, 0);
    const bool ok_all = __syncthreads_and(ok && done);
    if (!ok_all && tid == 0)
        atomicExch(&g_tc_error, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok_all && warp < 3 && KT > 0) {
        // Lane 32 a + ci, column d NB + co: dW[co][3 a + d][ci].
#pragma unroll 1
        for (int d = 0; d < 3; ++d) {
            float *dst = dw + (warp * 3 + d) * 32 + (tid & 31);
#pragma unroll 1
            for (int c = 0; c < NB; c += 16) {
                uint32_t r[16];
                tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) +
                              static_cast<uint32_t>(d * NB + c),
                          r);
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    atomicAdd(dst + static_cast<int64_t>(c + e) * 9 * 32, __uint_as_float(r[e]));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS)
                     : "memory");
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

// The rotation of several layers' weights in one launch: layer blockIdx.y
// starts at element off[l] of both w and w_rot.
constexpr int ROT_MAX_LAYERS = 32;
struct RotTable {
    int64_t off[ROT_MAX_LAYERS];
    int cin[ROT_MAX_LAYERS], cout[ROT_MAX_LAYERS];
};

__global__ void k_rotate_layers(const bf16 *__restrict__ w, bf16 *__restrict__ w_rot,
                                const RotTable t)
{
    const int l = blockIdx.y;
    const int Cin = t.cin[l], Cout = t.cout[l];
    const bf16 *src = w + t.off[l];
    bf16 *dst = w_rot + t.off[l];
    const int64_t total = static_cast<int64_t>(Cout) * 9 * Cin;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int ci = static_cast<int>(i % Cin);
        const int tap = static_cast<int>((i / Cin) % 9);
        const int co = static_cast<int>(i / (9 * static_cast<int64_t>(Cin)));
        dst[(static_cast<int64_t>(ci) * 9 + (8 - tap)) * Cout + co] = src[i];
    }
}

// ---------------------------------------------------------------------------
// wgrad for the shapes the tensor-core kernel does not take (Cin other than
// 32, 64, 128, or Cout > 256): CTA tile 64 output channels x 32 input
// channels of one tap, k-tiles
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

// One pass over a layer's output gradient dy [M][C] for the backward step:
// skip (when given) receives dy as it comes (skip_acc 0: a copy, the skip
// source's first gradient; 1: added), then dy = y > 0 ? dy : 0 (when y is
// given: the ReLU), then db[c] += the sum over pixels of the result.  Lanes
// and reduction as in k_bias_grad.
__global__ void k_relu_bias_bwd(bf16 *__restrict__ dy, const bf16 *__restrict__ y,
                                bf16 *__restrict__ skip, int skip_acc, float *__restrict__ db,
                                int M, int C)
{
    const int c8 = C / 8;
    const int lanes = blockDim.x / c8;
    const int g = threadIdx.x % c8, lp = threadIdx.x / c8;
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (lp < lanes)
        for (int p = blockIdx.x * lanes + lp; p < M; p += gridDim.x * lanes) {
            const int64_t o = static_cast<int64_t>(p) * C + 8 * g;
            V8 v = ld8(dy + o);
            if (skip) {
                if (skip_acc) {
                    V8 k = ld8(skip + o);
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        k.v[e] += v.v[e];
                    st8(skip + o, k);
                } else {
                    st8(skip + o, v);
                }
            }
            if (y) {
                const V8 a = ld8(y + o);
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    v.v[e] = a.v[e] > 0.0f ? v.v[e] : 0.0f;
                st8(dy + o, v);
            }
#pragma unroll
            for (int e = 0; e < 8; ++e)
                s[e] += v.v[e];
        }
    __shared__ float part[256][9];
#pragma unroll
    for (int e = 0; e < 8; ++e)
        part[threadIdx.x][e] = s[e];
    __syncthreads();
    if (threadIdx.x < C) {
        const int gg = threadIdx.x / 8, e = threadIdx.x % 8;
        float t = 0.0f;
        for (int l = 0; l < lanes; ++l)
            t += part[l * c8 + gg][e];
        atomicAdd(db + threadIdx.x, t);
    }
}

// Sum of v over the CTA (blockDim.x a multiple of 32, at most 1024), valid
// in thread 0.
__device__ __forceinline__ float block_sum(float v)
{
    __shared__ float ws[32];
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0)
        ws[threadIdx.x >> 5] = v;
    __syncthreads();
    float t = 0.0f;
    if (threadIdx.x == 0)
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w)
            t += ws[w];
    return t;
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

// Input-gradient vector i of (n, h, w, c); acc: added to dx.
__global__ void k_pool_bwd(const bf16 *dy, bf16 *dx, int N, int H, int W, int C, int acc)
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
        if (acc) {
            const V8 d = ld8(dx + 8 * i);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                g.v[k] = d.v[k] + static_cast<float>(__float2bfloat16(g.v[k]));
        }
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

// Input-gradient vector i of (n, h, w, c) from dy of (n, 2h, 2w, c); acc:
// added to dx.
__global__ void k_up_bwd(const bf16 *dy, bf16 *dx, int N, int H, int W, int C, int acc)
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
        if (acc) {
            const V8 d = ld8(dx + 8 * i);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                r.v[k] = d.v[k] + static_cast<float>(__float2bfloat16(r.v[k]));
        }
        st8(dx + 8 * i, r);
    }
}

// One atomic per CTA.
__global__ void k_mask_sum(const float *mask, int64_t n, float *sum)
{
    float s = 0.0f;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        s += mask[i];
    s = block_sum(s);
    if (threadIdx.x == 0)
        atomicAdd(sum, s);
}

// Masked MSE over the first K of C channels and its gradient: one thread per
// (pixel, 8-channel group), a 16-byte store of the gradient; groups past K
// store zeros and read nothing.  One atomic per CTA for the loss.
__global__ void k_mse(const float *out, const float *tgt, const float *mask, const float *msum,
                      bf16 *dy, float *loss, int64_t pixels, int C, int K)
{
    const float scale = 1.0f / (static_cast<float>(K) * fmaxf(*msum, 1.0f));
    const int c8 = C / 8;
    float l = 0.0f;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
         i < pixels * c8; i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t p = i / c8;
        const int c0 = 8 * static_cast<int>(i % c8);
        V8 r;
#pragma unroll
        for (int e = 0; e < 8; ++e)
            r.v[e] = 0.0f;
        if (c0 < K && mask[p] != 0.0f) {
#pragma unroll
            for (int e = 0; e < 8; ++e)
                if (c0 + e < K) {
                    const float d = out[p * C + c0 + e] - tgt[p * K + c0 + e];
                    l += d * d * scale;
                    r.v[e] = 2.0f * d * scale;
                }
        }
        st8(dy + p * C + c0, r);
    }
    l = block_sum(l);
    if (threadIdx.x == 0)
        atomicAdd(loss, l);
}

// hp, when given, holds {lr, c1, c2} in device memory (a captured step
// whose learning rate and bias corrections change from replay to replay).
__global__ void k_adam(float *w, bf16 *wb, const float *g, float *m, float *v, int64_t n, float lr,
                       float b1, float b2, float eps, float c1, float c2, const float *hp)
{
    if (hp) {
        lr = hp[0];
        c1 = hp[1];
        c2 = hp[2];
    }
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

// cuTensorMapEncodeTiled from the driver, found once through the runtime.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// The TMA maps of one convolution: the input [N][H][W][Cin] read in boxes of
// cb channels x bw x bh pixels, the weights [Cout][9 Cin] in boxes of 64 k x
// bn rows.  False when the shape or the pointers do not suit them.
bool conv_tma_maps(const bf16 *x, const bf16 *w, int n, int h, int w_, int cin, int cout, int bn,
                   int cb, int bw, int bh, CUtensorMap *mx, CUtensorMap *mw)
{
    auto enc = tensor_map_encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(x) & 15u) || (reinterpret_cast<uintptr_t>(w) & 15u))
        return false;
    const cuuint64_t xd[4] = {cuuint64_t(cin), cuuint64_t(w_), cuuint64_t(h), cuuint64_t(n)};
    const cuuint64_t xs[3] = {cuuint64_t(cin) * 2, cuuint64_t(w_) * cin * 2,
                              cuuint64_t(h) * w_ * cin * 2};
    const cuuint32_t xb[4] = {cuuint32_t(cb), cuuint32_t(bw), cuuint32_t(bh), 1};
    const cuuint32_t one[4] = {1, 1, 1, 1};
    if (enc(mx, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(x), xd, xs, xb, one,
            CU_TENSOR_MAP_INTERLEAVE_NONE,
            cb == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    const cuuint64_t wd[2] = {cuuint64_t(9) * cin, cuuint64_t(cout)};
    const cuuint64_t ws[1] = {cuuint64_t(9) * cin * 2};
    const cuuint32_t wb[2] = {cuuint32_t(TBK), cuuint32_t(bn)};
    return enc(mw, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(w), wd, ws, wb, one,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The TMA maps of AMODE 3: the input [N][H][W][32] in halo boxes of 32
// channels x 16 pixels x 10 rows, the weights [Cout][9 x 32] in boxes of one
// tap (32 k) x bn rows, both with the 64-byte swizzle.
// The halo boxes of a [N][H][W][32] input: 32 channels x 16 pixels x 10 rows.
bool halo_x_map(const bf16 *x, int n, int h, int w_, CUtensorMap *mx)
{
    auto enc = tensor_map_encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(x) & 15u))
        return false;
    const cuuint64_t xd[4] = {32, cuuint64_t(w_), cuuint64_t(h), cuuint64_t(n)};
    const cuuint64_t xs[3] = {64, cuuint64_t(w_) * 64, cuuint64_t(h) * w_ * 64};
    const cuuint32_t xb[4] = {32, H3W, H3H + 2, 1};
    const cuuint32_t one[4] = {1, 1, 1, 1};
    return enc(mx, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(x), xd, xs, xb, one,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool conv_tma_maps3(const bf16 *x, const bf16 *w, int n, int h, int w_, int cout, int bn,
                    CUtensorMap *mx, CUtensorMap *mw)
{
    auto enc = tensor_map_encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(w) & 15u) || !halo_x_map(x, n, h, w_, mx))
        return false;
    const cuuint32_t one[4] = {1, 1, 1, 1};
    const cuuint64_t wd[2] = {9 * 32, cuuint64_t(cout)};
    const cuuint64_t ws[1] = {9 * 32 * 2};
    const cuuint32_t wb[2] = {32, cuuint32_t(bn)};
    return enc(mw, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(w), wd, ws, wb, one,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, int AMODE>
int conv_fwd_tc_mode(const bf16 *x, const bf16 *w, const float *bias, const bf16 *res, bf16 *y,
                     bf16 *ysum, float *y32, int n, int h, int w_, int cin, int cout, int relu,
                     const CUtensorMap &mx, const CUtensorMap &mw, int bw, int bh, cudaStream_t s)
{
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    constexpr int smem = AMODE == 3 ? tc_smem3<BN>() : tc_smem<BN>();
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_conv_fwd_tc<BN, AMODE>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    });
    if (attr != cudaSuccess)
        return ERR_CUDA;
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return ERR_CUDA;
    }
    // Persistent: tc_ctas_per_sm CTAs per SM, each taking tiles
    // blockIdx.x + i * gridDim.x.
    const int M = n * h * w_;
    const int64_t tiles = AMODE == 3 ? int64_t(n) * (h / H3H) * (w_ / H3W)
                                     : static_cast<int64_t>((M + TBM - 1) / TBM) * (cout / BN);
    const int per_sm = AMODE == 3 ? tc_ctas_per_sm3<BN>() : tc_ctas_per_sm<BN>();
    const int grid = static_cast<int>(tiles < int64_t(sms) * per_sm ? tiles : int64_t(sms) * per_sm);
    k_conv_fwd_tc<BN, AMODE><<<grid, TC_THREADS, smem, s>>>(
        x, w, bias, res, y, ysum, y32, n, h, w_, cin, cout, relu, mx, mw, bw, bh);
    return status();
}

// Halo boxes (AMODE 3) for Cin 32 with one channel tile on 16 x 8-pixel
// tiles; else TMA tiles when every 128-pixel tile is a rectangle of one
// image (W a divisor or a multiple of 128, H W a multiple of 128) and Cin is
// 32 or a multiple of 64; the cp.async gather otherwise.
template <int BN>
int conv_fwd_tc(const bf16 *x, const bf16 *w, const float *bias, const bf16 *res, bf16 *y,
                bf16 *ysum, float *y32, int n, int h, int w_, int cin, int cout, int relu,
                cudaStream_t s)
{
    CUtensorMap mx, mw;
#ifndef DSMC_CONV_HALO
#define DSMC_CONV_HALO 1
#endif

    if (DSMC_CONV_HALO && cin == 32 && cout == BN && w_ % H3W == 0 && h % H3H == 0 &&
        conv_tma_maps3(x, w, n, h, w_, cout, BN, &mx, &mw))
        return conv_fwd_tc_mode<BN, 3>(x, w, bias, res, y, ysum, y32, n, h, w_, cin, cout, relu, mx,
                                       mw, H3W, H3H, s);
    const bool rect = (w_ % TBM == 0 || TBM % w_ == 0) && (int64_t(h) * w_) % TBM == 0;
    const int bw = w_ < TBM ? w_ : TBM, bh = TBM / bw;
    if (rect && cin % 64 == 0 &&
        conv_tma_maps(x, w, n, h, w_, cin, cout, BN, 64, bw, bh, &mx, &mw))
        return conv_fwd_tc_mode<BN, 1>(x, w, bias, res, y, ysum, y32, n, h, w_, cin, cout, relu, mx,
                                       mw, bw, bh, s);
    if (rect && cin == 32 && conv_tma_maps(x, w, n, h, w_, cin, cout, BN, 32, bw, bh, &mx, &mw))
        return conv_fwd_tc_mode<BN, 2>(x, w, bias, res, y, ysum, y32, n, h, w_, cin, cout, relu, mx,
                                       mw, bw, bh, s);
    memset(&mx, 0, sizeof(mx));
    memset(&mw, 0, sizeof(mw));
    return conv_fwd_tc_mode<BN, 0>(x, w, bias, res, y, ysum, y32, n, h, w_, cin, cout, relu, mx, mw,
                                   0, 0, s);
}
// Weight gradient on the tensor cores: groups of 128 / Cin taps x splits of
// the pixels.
// The TMA maps of the weight gradient: X [N][H][W][Cin] in boxes of cb
// channels x bw x bh pixels (128- or 64-byte swizzle), dY [pixels][Cout] in
// boxes of 64 channels x 64 pixels.  False when they do not suit.
bool wgrad_tma_maps(const bf16 *dy, const bf16 *x, int n, int h, int w_, int cin, int cout,
                    int cb, int bw, int bh, CUtensorMap *mx, CUtensorMap *my, int yc = 64)
{
    auto enc = tensor_map_encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(x) & 15u) || (reinterpret_cast<uintptr_t>(dy) & 15u))
        return false;
    const cuuint32_t one[4] = {1, 1, 1, 1};
    const cuuint64_t xd[4] = {cuuint64_t(cin), cuuint64_t(w_), cuuint64_t(h), cuuint64_t(n)};
    const cuuint64_t xs[3] = {cuuint64_t(cin) * 2, cuuint64_t(w_) * cin * 2,
                              cuuint64_t(h) * w_ * cin * 2};
    const cuuint32_t xb[4] = {cuuint32_t(cb), cuuint32_t(bw), cuuint32_t(bh), 1};
    if (enc(mx, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(x), xd, xs, xb, one,
            CU_TENSOR_MAP_INTERLEAVE_NONE,
            cb == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    const cuuint64_t yd[2] = {cuuint64_t(cout), cuuint64_t(n) * h * w_};
    const cuuint64_t ys[1] = {cuuint64_t(cout) * 2};
    const cuuint32_t yb[2] = {cuuint32_t(yc), cuuint32_t(WG_PIX)};
    return enc(my, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(dy), yd, ys, yb, one,
               CU_TENSOR_MAP_INTERLEAVE_NONE,
               yc == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// NB 32 (Cout 32: N 32 instead of a zero-filled 64, half the MMA work) has
// no gather form: it returns WG_NOT_TAKEN when the chunks are no rectangles.
constexpr int WG_NOT_TAKEN = -1;

template <int CI, int NB>
int wgrad_tc(const bf16 *dy, const bf16 *x, float *dw, int n, int h, int w_, int cout,
             cudaStream_t s)
{
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        if constexpr (NB != 32)
            attr = cudaFuncSetAttribute(k_conv_wgrad_tc<CI, NB, false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        wg_smem<NB>());
        if (attr == cudaSuccess)
            attr = cudaFuncSetAttribute(k_conv_wgrad_tc<CI, NB, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        wg_smem<NB>());
    });
    if (attr != cudaSuccess)
        return ERR_CUDA;
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return ERR_CUDA;
    }
    constexpr int groups = (9 + 128 / CI - 1) / (128 / CI);
    const int M = n * h * w_;
    const int chunks = (M + WG_PIX - 1) / WG_PIX;
    // One wave: whole splits per tap group that fit the resident CTAs.
    int splits = sms * wg_ctas_per_sm<NB>() / groups;
    splits = splits < 1 ? 1 : (splits < chunks ? splits : chunks);
    const int per = ((chunks + splits - 1) / splits) * WG_PIX;
    splits = (M + per - 1) / per;
    // TMA when every 64-pixel chunk is a rectangle of one image.
    CUtensorMap mx, my;
    const bool rect = (w_ % WG_PIX == 0 || WG_PIX % w_ == 0) && (int64_t(h) * w_) % WG_PIX == 0;
    const int bw = w_ < WG_PIX ? w_ : WG_PIX, bh = WG_PIX / bw;
    if (rect && wgrad_tma_maps(dy, x, n, h, w_, CI, cout, CI < 64 ? CI : 64, bw, bh, &mx, &my,
                               NB < 64 ? NB : 64)) {
        k_conv_wgrad_tc<CI, NB, true><<<dim3(splits, groups), WG_THREADS, wg_smem<NB>(), s>>>(
            dy, x, dw, n, h, w_, cout, per, mx, my, bw, bh);
    } else if constexpr (NB == 32) {
        return WG_NOT_TAKEN;
    } else {
        memset(&mx, 0, sizeof(mx));
        memset(&my, 0, sizeof(my));
        k_conv_wgrad_tc<CI, NB, false><<<dim3(splits, groups), WG_THREADS, wg_smem<NB>(), s>>>(
            dy, x, dw, n, h, w_, cout, per, mx, my, 0, 0);
    }
    return status();
}

// The halo-box weight gradient (Cin 32, Cout = NB, 16 x 8-pixel tiles); false
// when the maps do not suit.
template <int NB>
bool wgrad_halo(const bf16 *dy, const bf16 *x, float *dw, int n, int h, int w_, cudaStream_t s,
                int *st)
{
    auto enc = tensor_map_encoder();
    CUtensorMap mx, my;
    if (!enc || (reinterpret_cast<uintptr_t>(dy) & 15u) || !halo_x_map(x, n, h, w_, &mx))
        return false;
    const cuuint64_t yd[4] = {NB, cuuint64_t(w_), cuuint64_t(h), cuuint64_t(n)};
    const cuuint64_t ys[3] = {NB * 2, cuuint64_t(w_) * NB * 2, cuuint64_t(h) * w_ * NB * 2};
    const cuuint32_t yb[4] = {NB, H3W, H3H, 1};
    const cuuint32_t one[4] = {1, 1, 1, 1};
    if (enc(&my, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(dy), yd, ys, yb, one,
            CU_TENSOR_MAP_INTERLEAVE_NONE,
            NB == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_conv_wgrad_halo<NB>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, wh_smem<NB>());
    });
    static int sms = 0;
    if (attr == cudaSuccess && sms == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            sms = 0;
    }
    if (attr != cudaSuccess || sms == 0) {
        *st = ERR_CUDA;
        return true;
    }
    // One CTA per SM, each a contiguous range of tiles.
    const int ntiles = n * (h / H3H) * (w_ / H3W);
    const int per = (ntiles + sms - 1) / sms;
    const int splits = (ntiles + per - 1) / per;
    k_conv_wgrad_halo<NB><<<splits, 128, wh_smem<NB>(), s>>>(dw, n, h, w_, per, mx, my);
    *st = status();
    return true;
}

template <int CI>
int wgrad_tc_n(const bf16 *dy, const bf16 *x, float *dw, int n, int h, int w_, int cout,
               cudaStream_t s)
{
#ifndef DSMC_WGRAD_HALO
#define DSMC_WGRAD_HALO 1
#endif
    if (DSMC_WGRAD_HALO && CI == 32 && h % H3H == 0 && w_ % H3W == 0) {
        int st = OK;
        if (cout == 32 && wgrad_halo<32>(dy, x, dw, n, h, w_, s, &st))
            return st;
        if (cout == 64 && wgrad_halo<64>(dy, x, dw, n, h, w_, s, &st))
            return st;
    }
    if (cout == 32) {
        const int st = wgrad_tc<CI, 32>(dy, x, dw, n, h, w_, cout, s);
        if (st != WG_NOT_TAKEN)
            return st;
    }
    if (cout <= 64)
        return wgrad_tc<CI, 64>(dy, x, dw, n, h, w_, cout, s);
    if (cout <= 128)
        return wgrad_tc<CI, 128>(dy, x, dw, n, h, w_, cout, s);
    return wgrad_tc<CI, 256>(dy, x, dw, n, h, w_, cout, s);
}

int conv_fwd_launch(const bf16 *x, const bf16 *w, const float *bias, const bf16 *res, bf16 *y,
                    bf16 *ysum, float *y32, int n, int h, int w_, int cin, int cout, int relu,
                    cudaStream_t s)
{
    // The widest channel tile that divides Cout and still gives every SM a
    // tile; for small images (16x16 x 32 is 64 pixel tiles) 64 channels.
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return ERR_CUDA;
    }
    const int64_t mt = (int64_t(n) * h * w_ + TBM - 1) / TBM;
    if (cout % 128 == 0 && mt * (cout / 128) >= sms)
        return conv_fwd_tc<128>(x, w, bias, res, y, ysum, y32, n, h, w_, cin, cout, relu, s);
    if (cout % 64 == 0)
        return conv_fwd_tc<64>(x, w, bias, res, y, ysum, y32, n, h, w_, cin, cout, relu, s);
    return conv_fwd_tc<32>(x, w, bias, res, y, ysum, y32, n, h, w_, cin, cout, relu, s);
}

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
    return conv_fwd_launch(reinterpret_cast<const bf16 *>(x), reinterpret_cast<const bf16 *>(w),
                           bias, reinterpret_cast<const bf16 *>(res), reinterpret_cast<bf16 *>(y),
                           nullptr, y32, n, h, w_, cin, cout, relu,
                           static_cast<cudaStream_t>(stream));
}

int dsmc_sg_conv_fwd_skip(const uint16_t *x, const uint16_t *w, const float *bias,
                          const uint16_t *skip, uint16_t *y, uint16_t *ysum, int n, int h, int w_,
                          int cin, int cout, int relu, void *stream)
{
    if (!x || !w || !skip || !y || !ysum || !conv_shape_ok(n, h, w_, cin, cout))
        return ERR_ARG;
    return conv_fwd_launch(reinterpret_cast<const bf16 *>(x), reinterpret_cast<const bf16 *>(w),
                           bias, reinterpret_cast<const bf16 *>(skip),
                           reinterpret_cast<bf16 *>(y), reinterpret_cast<bf16 *>(ysum), nullptr,
                           n, h, w_, cin, cout, relu, static_cast<cudaStream_t>(stream));
}

int dsmc_sg_check(void *stream)
{
    if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess)
        return ERR_CUDA;
    int flag = 0;
    if (cudaMemcpyFromSymbol(&flag, g_tc_error, sizeof(int)) != cudaSuccess)
        return ERR_CUDA;
    if (flag) {
        const int zero = 0;
        if (cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int)) != cudaSuccess)
            return ERR_CUDA;
        return ERR_TIMEOUT;
    }
    return OK;
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

int dsmc_sg_rotate_layers(const uint16_t *w, uint16_t *w_rot, const int64_t *offsets,
                          const int *cin, const int *cout, int layers, void *stream)
{
    if (!w || !w_rot || !offsets || !cin || !cout || layers < 0 || layers > ROT_MAX_LAYERS)
        return ERR_ARG;
    RotTable t;
    int64_t most = 0;
    for (int l = 0; l < layers; ++l) {
        if (offsets[l] < 0 || offsets[l] % 8 || cin[l] <= 0 || cout[l] <= 0)
            return ERR_ARG;
        t.off[l] = offsets[l];
        t.cin[l] = cin[l];
        t.cout[l] = cout[l];
        const int64_t k = int64_t(9) * cin[l] * cout[l];
        most = k > most ? k : most;
    }
    if (layers == 0)
        return OK;
    const int bx = static_cast<int>(most / 256 + 1 < 256 ? most / 256 + 1 : 256);
    k_rotate_layers<<<dim3(bx, layers), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const bf16 *>(w), reinterpret_cast<bf16 *>(w_rot), t);
    return status();
}

int dsmc_sg_conv_wgrad(const uint16_t *dy, const uint16_t *x, float *dw, float *db, int n, int h,
                       int w_, int cin, int cout, void *stream)
{
    if (!dy || !x || !dw || !conv_shape_ok(n, h, w_, cin, cout) || (db && cout > 256))
        return ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int M = n * h * w_;
    if ((cin == 32 || cin == 64 || cin == 128) && cout <= 256) {
        const bf16 *dyb = reinterpret_cast<const bf16 *>(dy);
        const bf16 *xb = reinterpret_cast<const bf16 *>(x);
        const int st = cin == 128  ? wgrad_tc_n<128>(dyb, xb, dw, n, h, w_, cout, s)
                       : cin == 64 ? wgrad_tc_n<64>(dyb, xb, dw, n, h, w_, cout, s)
                                   : wgrad_tc_n<32>(dyb, xb, dw, n, h, w_, cout, s);
        if (st != OK)
            return st;
        if (db)
            k_bias_grad<<<512, 256, 0, s>>>(reinterpret_cast<const bf16 *>(dy), db, M, cout);
        return status();
    }
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

int dsmc_sg_pool_bwd_acc(const uint16_t *dy, uint16_t *dx, int n, int h, int w_, int c,
                         int accumulate, void *stream)
{
    if (!dy || !dx || n <= 0 || h <= 0 || w_ <= 0 || c <= 0 || h % 2 || w_ % 2 || c % 8)
        return ERR_ARG;
    k_pool_bwd<<<grid_for(int64_t(n) * h * w_ * c / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const bf16 *>(dy), reinterpret_cast<bf16 *>(dx), n, h, w_, c,
        accumulate ? 1 : 0);
    return status();
}

int dsmc_sg_pool_bwd(const uint16_t *dy, uint16_t *dx, int n, int h, int w_, int c, void *stream)
{
    return dsmc_sg_pool_bwd_acc(dy, dx, n, h, w_, c, 0, stream);
}

int dsmc_sg_up_fwd(const uint16_t *x, uint16_t *y, int n, int h, int w_, int c, void *stream)
{
    if (!x || !y || n <= 0 || h <= 0 || w_ <= 0 || c <= 0 || c % 8)
        return ERR_ARG;
    k_up_fwd<<<grid_for(int64_t(n) * 4 * h * w_ * c / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const bf16 *>(x), reinterpret_cast<bf16 *>(y), n, h, w_, c);
    return status();
}

int dsmc_sg_up_bwd_acc(const uint16_t *dy, uint16_t *dx, int n, int h, int w_, int c,
                       int accumulate, void *stream)
{
    if (!dy || !dx || n <= 0 || h <= 0 || w_ <= 0 || c <= 0 || c % 8)
        return ERR_ARG;
    k_up_bwd<<<grid_for(int64_t(n) * h * w_ * c / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const bf16 *>(dy), reinterpret_cast<bf16 *>(dx), n, h, w_, c,
        accumulate ? 1 : 0);
    return status();
}

int dsmc_sg_up_bwd(const uint16_t *dy, uint16_t *dx, int n, int h, int w_, int c, void *stream)
{
    return dsmc_sg_up_bwd_acc(dy, dx, n, h, w_, c, 0, stream);
}

int dsmc_sg_relu_bias_bwd(uint16_t *dy, const uint16_t *y, uint16_t *skip, int skip_accumulate,
                          float *db, int64_t pixels, int c, void *stream)
{
    if (!dy || !db || pixels < 0 || pixels > INT32_MAX || c < 8 || c > 256 || c % 8)
        return ERR_ARG;
    k_relu_bias_bwd<<<592, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<bf16 *>(dy), reinterpret_cast<const bf16 *>(y),
        reinterpret_cast<bf16 *>(skip), skip_accumulate ? 1 : 0, db, static_cast<int>(pixels), c);
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
    if (!out || !target || !mask || !dy || !loss || pixels <= 0 || k <= 0 || k > c || c % 8)
        return ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // loss[0] = loss, loss[1] = sum of the mask (scratch).
    if (cudaMemsetAsync(loss, 0, 2 * sizeof(float), s) != cudaSuccess)
        return ERR_CUDA;
    k_mask_sum<<<592, 256, 0, s>>>(mask, pixels, loss + 1);
    k_mse<<<grid_for(pixels * (c / 8) / 4), 256, 0, s>>>(
        out, target, mask, loss + 1, reinterpret_cast<bf16 *>(dy), loss, pixels, c, k);
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
        w, reinterpret_cast<bf16 *>(w_bf16), g, m, v, count, lr, beta1, beta2, eps, c1, c2,
        nullptr);
    return status();
}

int dsmc_sg_adam_dev(float *w, uint16_t *w_bf16, const float *g, float *m, float *v,
                     int64_t count, const float *step, float beta1, float beta2, float eps,
                     void *stream)
{
    if (!w || !g || !m || !v || !step || count < 0)
        return ERR_ARG;
    k_adam<<<grid_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w, reinterpret_cast<bf16 *>(w_bf16), g, m, v, count, 0.0f, beta1, beta2, eps, 1.0f, 1.0f,
        step);
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
