/*
 * The proposal network of the prior-net form: 3x3 convolutions over NHWC
 * BF16 activations on the tcgen05 tensor cores (FP32 accumulation in TMEM),
 * with fused epilogues, plus weight packing.  No counterpart in the
 * reference: the network proposes a plane per coarse pixel, and its
 * proposals enter PatchMatch only as extra candidates scored by the
 * unchanged NCC cost.
 *
 * Implicit GEMM without an im2col copy.  A CTA computes 128 consecutive
 * output pixels of one image row (M = 128) for all output channels (N =
 * COUT).  Its input halo, 3 rows x 130 pixels, sits in shared memory as
 * channel groups of 8: slab cg holds [row][pixel][8 channels], 16 bytes per
 * pixel, so 8 consecutive pixels of one channel group are one 128-byte core
 * matrix.  The A operand of tap (dy, dx) is then the same halo with its start
 * address moved by (dy * 130 + dx) * 16 bytes: SBO = 128 B (next 8 pixels),
 * LBO = one slab (next 8 channels).  Weights sit as [tap][cin group][cout
 * group][8 x 8] core matrices (SBO 128 B along N, LBO one cout-group row
 * along K).  9 taps x CIN/16 MMAs of 128 x COUT x 16 accumulate in TMEM;
 * four warps read the 128 x COUT accumulator back (one TMEM lane quarter
 * each) and apply the epilogue.
 *
 * The halo comes in by TMA (one 3-D tiled load per channel group, box 8 x
 * 130 x 3, out-of-image rows and columns filled with zeros by the unit:
 * the convolution's zero padding) or, for checking, by thread loads.
 */
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "hpm_b200.h"
#include "hpm_tc.cuh"

namespace hpm {

/* set by a convolution whose wait ran out (see kWaitCycles) */
__device__ int g_net_error;

namespace {

constexpr int kTileM = 128;
constexpr int kHaloW = kTileM + 2;
constexpr int kHaloBytes = 3 * kHaloW * 16; /* one channel group: 6240 B */
constexpr int kSlab = 6272;                 /* slab stride, a multiple of 128 B */
constexpr long long kWaitCycles = 4000000000LL; /* ~2 s at 2 GHz */

/* Shared memory of one CTA.  The A region is large enough that every
 * address an MMA may read stays inside it even under the other reading of
 * the two stride fields (the M stride taken as the slab): a mistaken
 * descriptor gives wrong numbers, never an out-of-bounds access. */
template <int CIN, int COUT>
struct ConvSmem {
    static constexpr int CG = CIN / 8, OG = COUT / 8;
    static constexpr int kAStartMax = (CG - 2 > 0 ? CG - 2 : 0) * kSlab + (2 * kHaloW + 2) * 16;
    static constexpr int kAReach = kAStartMax + 15 * kSlab + 2 * 128 + 128;
    static constexpr int kA = ((kAReach > CG * kSlab ? kAReach : CG * kSlab) + 1023) / 1024 * 1024;
    static constexpr int kB = 9 * CIN * COUT * 2;
    static constexpr int kBReach = ((8 * CG + CG - 2 > 0 ? 8 * CG + CG - 2 : 0) * OG) * 128 + OG * OG * 128 + 256;
    static constexpr int kBRegion = ((kBReach > kB ? kBReach : kB) + 1023) / 1024 * 1024;
    static constexpr int kBytes = kA + kBRegion + 64;
};

enum { kEpiReluBf16 = 0, kEpiBiasF32 = 1, kEpiDreluBf16 = 2 };

template <int COUT>
__device__ __forceinline__ void load_acc(uint32_t taddr, uint32_t *r)
{
    if constexpr (COUT == 32)
        tc::tmem_ld32(taddr, r);
    else
        tc::tmem_ld16(taddr, r);
}

template <int CIN, int COUT, int EPI, bool TMA>
__global__ void __launch_bounds__(128, 1)
    k_conv3x3(const __grid_constant__ CUtensorMap tmap, const __nv_bfloat16 *__restrict__ x, int h, int w,
              const uint4 *__restrict__ wpk, const float *__restrict__ bias, const __nv_bfloat16 *__restrict__ aux,
              void *__restrict__ y, int *__restrict__ err)
{
    using L = ConvSmem<CIN, COUT>;
    constexpr int CG = L::CG, OG = L::OG;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sA = smem;
    uint8_t *sB = smem + L::kA;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sB + L::kBRegion); /* [0] loads, [1] MMAs */
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_x = (w + kTileM - 1) / kTileM;
    const int ty = blockIdx.x / tiles_x, x0 = (blockIdx.x % tiles_x) * kTileM;

    if ((tc::smem_u32(smem) & 1023u) != 0) { /* TMA and the descriptors assume 1 KB alignment */
        if (tid == 0) atomicExch(err, 2);
        return;
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, 32);
    if (tid == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if constexpr (TMA) {
        if (tid == 0) {
            tc::mbar_expect_tx(&bar[0], CG * kHaloBytes);
            for (int cg = 0; cg < CG; ++cg) tc::tma_load_3d(sA + cg * kSlab, &tmap, &bar[0], cg * 8, x0 - 1, ty - 1);
        }
    } else {
        for (int i = tid; i < CG * 3 * kHaloW; i += 128) {
            const int cg = i / (3 * kHaloW), r = (i / kHaloW) % 3, p = i % kHaloW;
            const int gy = ty + r - 1, gx = x0 + p - 1;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy >= 0 && gy < h && gx >= 0 && gx < w)
                v = *reinterpret_cast<const uint4 *>(x + ((size_t)gy * w + gx) * CIN + cg * 8);
            *reinterpret_cast<uint4 *>(sA + cg * kSlab + (r * kHaloW + p) * 16) = v;
        }
    }
    for (int i = tid; i < L::kB / 16; i += 128) reinterpret_cast<uint4 *>(sB)[i] = wpk[i];
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;
    if constexpr (TMA) ok = tc::mbar_wait(&bar[0], 0, kWaitCycles);
    if (tid == 0 && ok) {
        const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
        constexpr uint32_t idesc = tc::idesc_bf16(128, COUT, 0, 0);
        int k = 0;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const int dy = t / 3, dx = t % 3;
#pragma unroll
            for (int ks = 0; ks < CIN / 16; ++ks, ++k) {
                const uint64_t ad = tc::smem_desc(a0 + 2 * ks * kSlab + (dy * kHaloW + dx) * 16, kSlab, 128);
                const uint64_t bd = tc::smem_desc(b0 + (t * CG + 2 * ks) * OG * 128, OG * 128, 128);
                tc::mma_bf16(tmem, ad, bd, idesc, k > 0);
            }
        }
        tc::mma_commit(&bar[1]);
    }
    const bool loaded = __syncthreads_and(ok) != 0;
    ok = loaded && tc::mbar_wait(&bar[1], 0, kWaitCycles);
    ok = __syncthreads_and(ok) != 0;
    tc::fence_after_sync();
    if (ok) {
        uint32_t r[COUT];
        load_acc<COUT>(tmem + ((uint32_t)(warp * 32) << 16), r);
        tc::tmem_wait_ld();
        const int m = warp * 32 + lane, gx = x0 + m;
        if (gx < w) {
            const size_t o = ((size_t)ty * w + gx) * COUT;
            if constexpr (EPI == kEpiBiasF32) {
                float *yo = static_cast<float *>(y) + o;
#pragma unroll
                for (int n = 0; n < COUT; n += 4)
                    *reinterpret_cast<float4 *>(yo + n) =
                        make_float4(__uint_as_float(r[n]) + bias[n], __uint_as_float(r[n + 1]) + bias[n + 1],
                                    __uint_as_float(r[n + 2]) + bias[n + 2], __uint_as_float(r[n + 3]) + bias[n + 3]);
            } else {
                __nv_bfloat16 *yo = static_cast<__nv_bfloat16 *>(y) + o;
                __align__(16) __nv_bfloat162 v[COUT / 2];
                if constexpr (EPI == kEpiReluBf16) {
#pragma unroll
                    for (int n = 0; n < COUT; n += 2)
                        v[n / 2] = __floats2bfloat162_rn(fmaxf(__uint_as_float(r[n]) + bias[n], 0.0f),
                                                         fmaxf(__uint_as_float(r[n + 1]) + bias[n + 1], 0.0f));
                } else {
                    const __nv_bfloat16 *ax = aux + o;
#pragma unroll
                    for (int n = 0; n < COUT; n += 2) {
                        const float g0 = __bfloat162float(ax[n]) > 0.0f ? __uint_as_float(r[n]) : 0.0f;
                        const float g1 = __bfloat162float(ax[n + 1]) > 0.0f ? __uint_as_float(r[n + 1]) : 0.0f;
                        v[n / 2] = __floats2bfloat162_rn(g0, g1);
                    }
                }
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q)
                    reinterpret_cast<uint4 *>(yo)[q] = reinterpret_cast<const uint4 *>(v)[q];
            }
        }
    } else {
        if (tid == 0) atomicExch(err, 1);
        /* give copies and MMAs still in flight a second bounded wait before
         * the shared memory and the TMEM columns are released */
        if constexpr (TMA) tc::mbar_wait(&bar[0], 0, kWaitCycles);
        if (loaded) tc::mbar_wait(&bar[1], 0, kWaitCycles);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 32);
}

/* Weight gradient dW[cout][cin][tap] += sum over pixels p of
 * dY[p][cout] * X[p + shift(tap)][cin], on the tensor cores with the pixels
 * as the K dimension.  Both operands are MN-major (8 channels contiguous per
 * pixel, as NHWC stores them):
 *   A = (tap slot, cin) x pixels: TG = 128 / CIN taps per M = 128 group
 *       (4 for 32 channels, 8 for 16), 9 taps in NG groups, unused slots
 *       zero; core matrix (m group, 8 pixels) at m * 128 + kgroup * 2048.
 *   B = cout x pixels: core matrix (n group, 8 pixels) at n * 128 +
 *       kgroup * OG * 128.
 * A persistent CTA walks its 128-pixel row tiles and accumulates NG
 * accumulators of 128 x COUT in TMEM across all of them, then adds them to
 * dW (FP32, OIHW) with atomics. */
template <int CIN, int COUT>
struct WgradSmem {
    static constexpr int CG = CIN / 8, OG = COUT / 8, TG = 128 / CIN, NG = (9 + TG - 1) / TG;
    static constexpr int kAGroup = 16 * 16 * 128; /* 16 pixel groups x 16 m groups */
    static constexpr int kA = NG * kAGroup;
    static constexpr int kB = 16 * OG * 128 + 1024; /* + reach of the other stride reading */
    /* under the other reading of the two strides the last A group reaches
     * 7 * 4096 + 15 * 2048 + 255 bytes past its start: one group of slack */
    static constexpr int kBytes = kA + kB + kAGroup + 64;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128, 1)
    k_conv_wgrad(const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ dy, int h, int w,
                 float *__restrict__ dw, int *__restrict__ err)
{
    using L = WgradSmem<CIN, COUT>;
    constexpr int CG = L::CG, OG = L::OG, TG = L::TG, NG = L::NG;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sA = smem;
    uint8_t *sB = smem + L::kA;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sB + L::kB + L::kAGroup);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    static_assert(L::kBytes <= 227 * 1024, "shared memory of one CTA");
    if ((tc::smem_u32(smem) & 1023u) != 0) {
        if (tid == 0) atomicExch(err, 2);
        return;
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, 128);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    const int tiles_x = (w + kTileM - 1) / kTileM, tiles = h * tiles_x;
    bool ok = true;
    uint32_t phase = 0;
    int issued = 0;
    for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const int ty = tile / tiles_x, x0 = (tile % tiles_x) * kTileM;
        /* B: dY of the tile's 128 pixels */
        for (int i = tid; i < kTileM * OG; i += 128) {
            const int p = i / OG, og = i % OG, gx = x0 + p;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gx < w) v = *reinterpret_cast<const uint4 *>(dy + ((size_t)ty * w + gx) * COUT + og * 8);
            *reinterpret_cast<uint4 *>(sB + (p >> 3) * (OG * 128) + og * 128 + (p & 7) * 16) = v;
        }
        /* A: the input at each tap's shift, zero outside the image */
        for (int i = tid; i < NG * TG * CG * kTileM; i += 128) {
            const int p = i % kTileM, rest = i / kTileM;
            const int cg = rest % CG, slot = rest / CG; /* slot = g * TG + tl */
            const int g = slot / TG, tl = slot % TG, t = slot;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (t < 9) {
                const int gy = ty + t / 3 - 1, gx = x0 + p + t % 3 - 1;
                if (x0 + p < w && gy >= 0 && gy < h && gx >= 0 && gx < w)
                    v = *reinterpret_cast<const uint4 *>(x + ((size_t)gy * w + gx) * CIN + cg * 8);
            }
            *reinterpret_cast<uint4 *>(sA + g * L::kAGroup + (p >> 3) * 2048 + (tl * CG + cg) * 128 + (p & 7) * 16) = v;
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
            const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
            constexpr uint32_t idesc = tc::idesc_bf16(128, COUT, 1, 1);
#pragma unroll
            for (int g = 0; g < NG; ++g)
#pragma unroll
                for (int ks = 0; ks < kTileM / 16; ++ks) {
                    const uint64_t ad = tc::smem_desc(a0 + g * L::kAGroup + ks * 2 * 2048, 2048, 128);
                    const uint64_t bd = tc::smem_desc(b0 + ks * 2 * OG * 128, OG * 128, 128);
                    tc::mma_bf16(tmem + g * COUT, ad, bd, idesc, (issued > 0 || ks > 0) ? 1u : 0u);
                }
            tc::mma_commit(bar);
        }
        issued = 1;
        /* the next tile overwrites the operands: wait for these MMAs */
        ok = tc::mbar_wait(bar, phase, kWaitCycles);
        phase ^= 1;
        ok = __syncthreads_and(ok) != 0;
    }
    tc::fence_after_sync();
    if (ok && issued) {
        /* row m of group g: tap g * TG + m / CIN, input channel m % CIN */
        const int m = warp * 32 + lane, tl = m / CIN, ci = m % CIN;
#pragma unroll
        for (int g = 0; g < NG; ++g) {
            uint32_t r[COUT];
            load_acc<COUT>(tmem + g * COUT + ((uint32_t)(warp * 32) << 16), r);
            tc::tmem_wait_ld();
            const int t = g * TG + tl;
            if (t < 9)
#pragma unroll
                for (int n = 0; n < COUT; ++n) atomicAdd(&dw[((size_t)n * CIN + ci) * 9 + t], __uint_as_float(r[n]));
        }
    } else if (!ok) {
        if (tid == 0) atomicExch(err, 1);
        tc::mbar_wait(bar, phase ^ 1, kWaitCycles);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

/* Bias gradient db[c] += sum over pixels of dY[p][c] (dY FP32 or BF16). */
template <typename T, int C>
__global__ void k_bias_grad(const T *__restrict__ dy, long long n, float *__restrict__ db)
{
    float acc[C];
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = 0.0f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] += (float)dy[p * C + c];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        float v = acc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&db[c], v);
    }
}

/* Weights [cout][cin][3][3] FP32 (PyTorch's OIHW) into the shared-memory
 * image of k_conv3x3: [tap][cin/8][cout/8][8 cout][8 cin] BF16.  mode 1
 * packs the weights of the data-gradient convolution instead: the kernel
 * flipped and cin/cout exchanged (output channels = the layer's inputs). */
__global__ void k_pack_weights(const float *__restrict__ wt, int cout, int cin, int mode,
                               __nv_bfloat16 *__restrict__ out)
{
    const int oc = mode ? cin : cout, ic = mode ? cout : cin; /* of the packed convolution */
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 9 * oc * ic) return;
    const int k8 = i & 7, n8 = (i >> 3) & 7;
    const int rest = i >> 6;
    const int og = rest % (oc / 8), cg = (rest / (oc / 8)) % (ic / 8), t = rest / ((oc / 8) * (ic / 8));
    const int n = og * 8 + n8, k = cg * 8 + k8; /* packed conv: output n, input k */
    float v;
    if (!mode)
        v = wt[((size_t)n * cin + k) * 9 + t];
    else
        v = wt[((size_t)k * cin + n) * 9 + (8 - t)];
    out[i] = __float2bfloat16_rn(v);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

/* 3-D map over NHWC BF16 activations: (channel, x, y), box 8 x 130 x 3. */
bool make_halo_map(CUtensorMap *m, const void *x, int h, int w, int c)
{
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h};
    const cuuint64_t strides[2] = {(cuuint64_t)c * 2, (cuuint64_t)w * c * 2};
    const cuuint32_t box[3] = {8, (cuuint32_t)kHaloW, 3};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void *>(x), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int CIN, int COUT, int EPI, bool TMA>
cudaError_t launch_conv(const CUtensorMap &m, const void *x, int h, int w, const void *wpk, const float *bias,
                        const void *aux, void *y, int *err, cudaStream_t s)
{
    using L = ConvSmem<CIN, COUT>;
    static_assert(L::kBytes <= 227 * 1024, "shared memory of one CTA");
    auto kern = k_conv3x3<CIN, COUT, EPI, TMA>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kBytes);
    if (e != cudaSuccess) return e;
    const int tiles = h * ((w + kTileM - 1) / kTileM);
    kern<<<tiles, 128, L::kBytes, s>>>(m, static_cast<const __nv_bfloat16 *>(x), h, w, static_cast<const uint4 *>(wpk),
                                      bias, static_cast<const __nv_bfloat16 *>(aux), y, err);
    return cudaGetLastError();
}

template <int CIN, int COUT, bool TMA>
cudaError_t launch_conv_epi(int epi, const CUtensorMap &m, const void *x, int h, int w, const void *wpk,
                            const float *bias, const void *aux, void *y, int *err, cudaStream_t s)
{
    switch (epi) {
    case kEpiReluBf16: return launch_conv<CIN, COUT, kEpiReluBf16, TMA>(m, x, h, w, wpk, bias, aux, y, err, s);
    case kEpiBiasF32: return launch_conv<CIN, COUT, kEpiBiasF32, TMA>(m, x, h, w, wpk, bias, aux, y, err, s);
    default: return launch_conv<CIN, COUT, kEpiDreluBf16, TMA>(m, x, h, w, wpk, bias, aux, y, err, s);
    }
}

template <bool TMA>
cudaError_t launch_conv_any(int cin, int cout, int epi, const CUtensorMap &m, const void *x, int h, int w,
                            const void *wpk, const float *bias, const void *aux, void *y, int *err, cudaStream_t s)
{
    if (cin == 16 && cout == 32) return launch_conv_epi<16, 32, TMA>(epi, m, x, h, w, wpk, bias, aux, y, err, s);
    if (cin == 32 && cout == 32) return launch_conv_epi<32, 32, TMA>(epi, m, x, h, w, wpk, bias, aux, y, err, s);
    if (cin == 32 && cout == 16) return launch_conv_epi<32, 16, TMA>(epi, m, x, h, w, wpk, bias, aux, y, err, s);
    if (cin == 16 && cout == 16) return launch_conv_epi<16, 16, TMA>(epi, m, x, h, w, wpk, bias, aux, y, err, s);
    return cudaErrorInvalidValue;
}

}  // namespace

/* Internal launcher for the flow: FP32-free NHWC BF16 convolution. */
cudaError_t net_conv3x3(const void *x, int h, int w, int cin, const void *wpk, const float *bias, int cout, int epi,
                        const void *aux, void *y, int *err, bool use_tma, cudaStream_t s)
{
    CUtensorMap m;
    memset(&m, 0, sizeof(m));
    if (use_tma && !make_halo_map(&m, x, h, w, cin)) return cudaErrorNotSupported;
    return use_tma ? launch_conv_any<true>(cin, cout, epi, m, x, h, w, wpk, bias, aux, y, err, s)
                   : launch_conv_any<false>(cin, cout, epi, m, x, h, w, wpk, bias, aux, y, err, s);
}

cudaError_t net_pack_weights(const float *wt, int cout, int cin, int mode, void *out, cudaStream_t s)
{
    const int n = 9 * cout * cin;
    k_pack_weights<<<(n + 255) / 256, 256, 0, s>>>(wt, cout, cin, mode, static_cast<__nv_bfloat16 *>(out));
    return cudaGetLastError();
}

cudaError_t net_conv_wgrad(const void *x, const void *dy, int h, int w, int cin, int cout, float *dw, int *err,
                           int ctas, cudaStream_t s)
{
    auto run = [&](auto kern, int bytes) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
        const int tiles = h * ((w + kTileM - 1) / kTileM);
        kern<<<tiles < ctas ? tiles : ctas, 128, bytes, s>>>(static_cast<const __nv_bfloat16 *>(x),
                                                             static_cast<const __nv_bfloat16 *>(dy), h, w, dw, err);
        return cudaGetLastError();
    };
    if (cin == 16 && cout == 32) return run(k_conv_wgrad<16, 32>, WgradSmem<16, 32>::kBytes);
    if (cin == 32 && cout == 32) return run(k_conv_wgrad<32, 32>, WgradSmem<32, 32>::kBytes);
    if (cin == 32 && cout == 16) return run(k_conv_wgrad<32, 16>, WgradSmem<32, 16>::kBytes);
    if (cin == 16 && cout == 16) return run(k_conv_wgrad<16, 16>, WgradSmem<16, 16>::kBytes);
    return cudaErrorInvalidValue;
}

cudaError_t net_bias_grad(const void *dy, int is_f32, long long n, int c, float *db, cudaStream_t s)
{
    const int blocks = 296;
    if (is_f32 && c == 16) k_bias_grad<float, 16><<<blocks, 256, 0, s>>>(static_cast<const float *>(dy), n, db);
    else if (is_f32 && c == 32) k_bias_grad<float, 32><<<blocks, 256, 0, s>>>(static_cast<const float *>(dy), n, db);
    else if (!is_f32 && c == 16)
        k_bias_grad<__nv_bfloat16, 16><<<blocks, 256, 0, s>>>(static_cast<const __nv_bfloat16 *>(dy), n, db);
    else if (!is_f32 && c == 32)
        k_bias_grad<__nv_bfloat16, 32><<<blocks, 256, 0, s>>>(static_cast<const __nv_bfloat16 *>(dy), n, db);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace hpm

namespace {
bool supported(int cin, int cout) { return (cin == 16 || cin == 32) && (cout == 16 || cout == 32); }
}  // namespace

extern "C" int hpm_net_pack_weights(const float *weights, int cout, int cin, int mode, void *packed, void *stream)
{
    if (!weights || !packed || (mode != 0 && mode != 1)) return HPM_ERR_ARG;
    if (!(mode ? supported(cout, cin) : supported(cin, cout))) return HPM_ERR_ARG;
    return hpm::net_pack_weights(weights, cout, cin, mode, packed, static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? HPM_OK
               : HPM_ERR_CUDA;
}

extern "C" int hpm_net_conv3x3(const void *x, int h, int w, int cin, const void *packed, const float *bias, int cout,
                               int epilogue, const void *aux, void *y, int use_tma, int *err, void *stream)
{
    if (!x || !packed || !y || h < 1 || w < 1 || !supported(cin, cout) || epilogue < 0 || epilogue > 2)
        return HPM_ERR_ARG;
    if (epilogue != 2 && !bias) return HPM_ERR_ARG;
    if (epilogue == 2 && !aux) return HPM_ERR_ARG;
    int *e = err;
    if (!e && cudaGetSymbolAddress(reinterpret_cast<void **>(&e), hpm::g_net_error) != cudaSuccess) return HPM_ERR_CUDA;
    const cudaError_t r =
        hpm::net_conv3x3(x, h, w, cin, packed, bias, cout, epilogue, aux, y, e, use_tma != 0, static_cast<cudaStream_t>(stream));
    return r == cudaSuccess ? HPM_OK : (r == cudaErrorNotSupported ? HPM_ERR_STATE : HPM_ERR_CUDA);
}

extern "C" int hpm_net_conv_wgrad(const void *x, const void *dy, int h, int w, int cin, int cout, float *dw,
                                  float *db, int *err, void *stream)
{
    if (!x || !dy || !dw || h < 1 || w < 1 || !supported(cin, cout)) return HPM_ERR_ARG;
    int *e = err;
    if (!e && cudaGetSymbolAddress(reinterpret_cast<void **>(&e), hpm::g_net_error) != cudaSuccess) return HPM_ERR_CUDA;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (hpm::net_conv_wgrad(x, dy, h, w, cin, cout, dw, e, sms, s) != cudaSuccess) return HPM_ERR_CUDA;
    if (db && hpm::net_bias_grad(dy, 0, (long long)h * w, cout, db, s) != cudaSuccess) return HPM_ERR_CUDA;
    return HPM_OK;
}
