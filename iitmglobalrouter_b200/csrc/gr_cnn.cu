// gr_cnn.cu -- the congestion lookahead network: a stack of 3x3 convolutions
// over the per-layer demand / capacity grid, BF16 tensor-core GEMMs with FP32
// accumulation, trained and run entirely by the kernels in this file.
//
// A layer maps Cin channels of an H x W grid to Cout channels:
//   forward   col[m][k] = X[ci][y+dy][x+dx]          (im2col, k = ci*9 + (dy+1)*3 + dx+1, m = y*W + x)
//             Z[m][n]   = sum_k col[m][k] * Wt[k][n] (GEMM, mma.sync m16n8k16 bf16 -> f32)
//             Y[n][m]   = act(Z[m][n] + b[n])         (ReLU on every layer but the last)
//   backward  dZ = dY * act'(Z)                     (ReLU mask from the layer's output)
//             dW[n][k]  = sum_m col[m][k] dZ[n][m],   db[n] = sum_m dZ[n][m]
//                         (one tensor-core GEMM over the positions with the patches
//                          gathered on the fly and a row of ones for the bias)
//             dX[ci]    = sum over co, taps of dZ[co] shifted * W[co][ci] flipped
//                         (a 3x3 convolution of dZ with the weights transposed and
//                          rotated by 180 degrees: the forward convolution kernel)
// The loss is the mean squared error of the last layer against the target;
// parameters are FP32 masters updated by Adam, cast to BF16 for the GEMMs.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/iitmgr_b200.h"

namespace {

#define CN_CK(call)                                                                                \
    do {                                                                                           \
        cudaError_t _e = (call);                                                                   \
        if (_e != cudaSuccess) {                                                                   \
            fprintf(stderr, "iitmgr_b200: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(_e), \
                    __FILE__, __LINE__);                                                           \
            return GR_ERR_CUDA;                                                                    \
        }                                                                                          \
    } while (0)

constexpr int kMaxLayers = 8;

int round_up(int v, int m) { return (v + m - 1) / m * m; }

// ------------------------------------------------------------------ GEMM
// C[m][n] (f32) = or += sum over k in this block's range of A(m,k) * B(k,n),
// A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn] (bf16), C(m,n) at
// C[m*scm + n*scn]. Block tile 64 x 32, four warps of 16 rows each, k steps
// of 16 staged in shared memory; out-of-range elements read as zero.
// blockIdx.z splits the k range (atomic = 1 adds into C with atomics).
constexpr int kBM = 64, kBN = 32, kBK = 16;

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const __nv_bfloat16 *__restrict__ A,
                                              long long sam, long long sak, const __nv_bfloat16 *__restrict__ B,
                                              long long sbk, long long sbn, float *__restrict__ C, long long scm,
                                              long long scn, int kchunk, int atomic) {
    __shared__ __nv_bfloat16 As[kBM][kBK + 2];
    __shared__ __nv_bfloat16 Bs[kBK][kBN + 2];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
    const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[j][q] = 0.0f;
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);
    for (int k0 = kb; k0 < ke; k0 += kBK) {
        for (int i = tid; i < kBM * kBK; i += 128) {
            const int r = i / kBK, c = i % kBK, m = m0 + r, k = k0 + c;
            As[r][c] = (m < M && k < ke) ? A[(long long)m * sam + (long long)k * sak] : zero;
        }
        for (int i = tid; i < kBK * kBN; i += 128) {
            const int r = i / kBN, c = i % kBN, k = k0 + r, n = n0 + c;
            Bs[r][c] = (k < ke && n < N) ? B[(long long)k * sbk + (long long)n * sbn] : zero;
        }
        __syncthreads();
        const int r0 = warp * 16;
        uint32_t a[4];
        a[0] = pack2(As[r0 + g][2 * t], As[r0 + g][2 * t + 1]);
        a[1] = pack2(As[r0 + g + 8][2 * t], As[r0 + g + 8][2 * t + 1]);
        a[2] = pack2(As[r0 + g][2 * t + 8], As[r0 + g][2 * t + 9]);
        a[3] = pack2(As[r0 + g + 8][2 * t + 8], As[r0 + g + 8][2 * t + 9]);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int nn = j * 8 + g;
            const uint32_t b0 = pack2(Bs[2 * t][nn], Bs[2 * t + 1][nn]);
            const uint32_t b1 = pack2(Bs[2 * t + 8][nn], Bs[2 * t + 9][nn]);
            asm volatile(
                "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};\n"
                : "+f"(acc[j][0]), "+f"(acc[j][1]), "+f"(acc[j][2]), "+f"(acc[j][3])
                : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int m = m0 + warp * 16 + g + (q >= 2 ? 8 : 0), n = n0 + j * 8 + 2 * t + (q & 1);
            if (m < M && n < N) {
                float *p = C + (long long)m * scm + (long long)n * scn;
                if (atomic) atomicAdd(p, acc[j][q]);
                else *p = acc[j][q];
            }
        }
}

// ------------------------------------------------------------------ tcgen05 helpers
// (used by the forward / input-gradient convolution k_conv_strip and the
// weight-gradient kernel k_wgrad_tc below)
constexpr int kConvThreads = 256, kConvRows = 128, kConvTmemCols = 32;
constexpr int kConvSmemMax = 200 * 1024;
constexpr long long kConvWaitLimit = 1ll << 24;  // mbarrier polls before the kernel reports a stall

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start, leading (k chunk) and stride (row
// group) byte offsets in 16-byte units, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t umma_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kConvWaitLimit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

// ------------------------------------------------------------------ forward convolution on tcgen05
// A 3 x 3 convolution as an implicit GEMM with no patch matrix. A CTA computes a strip of 128
// positions of one grid row (x0 .. x0 + 127 of row y) x Nt output channels.
// Its input halo -- rows y - 1 .. y + 1, columns x0 - 1 .. x0 + 128, every
// channel rounded up to a multiple of 16 -- is stored as bf16 in planes of 8
// channels: plane c, halo row r, column q at ((c * 3 + r) * 130 + q) * 16
// bytes, the 8 channels of a cell as one 16-byte row. In that layout the
// 128 x 16 A operand of tap (dy, dx) and channel pair (2s, 2s + 1) is a
// canonical no-swizzle K-major matrix as it lies: 8-row core matrices of
// consecutive columns (stride 128 B), the second 8 channels one plane on
// (LBO = 3 * 130 * 16 B), starting at plane 2s, row dy, column dx. So one
// thread issues 9 taps x (channels / 16) MMAs straight from the halo into
// one FP32 accumulator (128 lanes x Nt columns of tensor memory); the
// weights of tap t are an Nt x channels matrix W[n][ci * 9 + t] in the same
// layout. The epilogue reads the accumulator with tcgen05.ld (warp w: lanes
// 32 (w % 4) .., columns 16 (w / 4) ..), adds the bias, applies ReLU and
// writes Y[n][y][x] (32 consecutive positions per warp) and, when training,
// the pre-activation Z[m][n].
constexpr int kStripX = 128, kStripCols = kStripX + 2;

__host__ __device__ constexpr int strip_cpad(int cin) { return (cin + 15) / 16 * 16; }
__host__ __device__ constexpr int strip_smem_bytes(int Nt, int cin) {
    return 1024 + strip_cpad(cin) / 8 * 3 * kStripCols * 16 + 9 * Nt * strip_cpad(cin) * 2 + 64;
}

// The shared-memory image of k_conv_strip's weights from Wt[k][n] (k = ci * 9
// + t): tap t, plane c, row n holds channels 8c .. 8c + 7 of W[n][ci * 9 + t]
// (zero past cin and past Np), 16 bytes per (t, c, n).
__global__ void k_pack_strip(int cin, int Nt, int Np, const __nv_bfloat16 *__restrict__ Wt, uint4 *__restrict__ out) {
    const int nplanes = strip_cpad(cin) / 8;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 9 * nplanes * Nt; i += gridDim.x * blockDim.x) {
        const int t = i / (nplanes * Nt), rem = i - t * (nplanes * Nt), c = rem / Nt, n = rem - c * Nt;
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int ci0 = 8 * c + 2 * j, ci1 = ci0 + 1;
            const __nv_bfloat16 z = __float2bfloat16(0.0f);
            const __nv_bfloat16 lo = (n < Np && ci0 < cin) ? Wt[(long long)(ci0 * 9 + t) * Np + n] : z;
            const __nv_bfloat16 hi = (n < Np && ci1 < cin) ? Wt[(long long)(ci1 * 9 + t) * Np + n] : z;
            w[j] = (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
        }
        out[i] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

__global__ void __launch_bounds__(kConvThreads)
    k_conv_strip(int cin, int cout, int H, int W, int Nt, int Np, const float *__restrict__ X,
                 const uint4 *__restrict__ Wimg, const float *__restrict__ bias, float *__restrict__ Y,
                 float *__restrict__ Zp, int relu, int *__restrict__ err, const uint4 *__restrict__ Xh,
                 uint4 *__restrict__ Yh) {
    extern __shared__ uint8_t conv_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)conv_raw + 1023) & ~(uintptr_t)1023);
    const int cpad = strip_cpad(cin), nplanes = cpad / 8;
    constexpr int kPlane = 3 * kStripCols * 16;  // bytes of one 8-channel plane
    uint8_t *halo = base;                                     // nplanes x 3 x 130 x 16 B
    uint8_t *Bs = halo + nplanes * kPlane;                    // 9 taps x (nplanes x Nt x 16 B)
    uint64_t *bar = (uint64_t *)(Bs + 9 * Nt * cpad * 2);     // 8-byte aligned
    uint32_t *tmem_slot = (uint32_t *)(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int M = H * W, y = blockIdx.y, x0 = blockIdx.x * kStripX;
    const int tapB = nplanes * Nt * 16;  // bytes of one tap's weights

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                     "r"(kConvTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 32) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // the weights' shared-memory image, packed once per parameter update (k_pack_strip)
    for (int i = tid; i < 9 * nplanes * Nt; i += kConvThreads) reinterpret_cast<uint4 *>(Bs)[i] = __ldg(Wimg + i);
    // the halo: one cell (plane, row, column) of 8 channels per step, eight
    // channel loads of a column in flight, coalesced along the columns
    for (int i = tid; i < nplanes * 3 * kStripCols; i += kConvThreads) {
        const int c = i / (3 * kStripCols), rem = i - c * 3 * kStripCols, r = rem / kStripCols, q = rem - r * kStripCols;
        const int gy = y - 1 + r, gx = x0 - 1 + q;
        const bool in = gy >= 0 && gy < H && gx >= 0 && gx < W;
        if (Xh) {  // the previous layer's channel-last bf16 copy: the cell is one 16-byte load
            reinterpret_cast<uint4 *>(halo)[i] = in ? __ldg(Xh + (long long)(gy * W + gx) * nplanes + c)
                                                    : make_uint4(0u, 0u, 0u, 0u);
            continue;
        }
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int ci = 8 * c + j;
            v[j] = (in && ci < cin) ? __ldg(X + (long long)ci * M + gy * W + gx) : 0.0f;
        }
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
            w[j] = *reinterpret_cast<const uint32_t *>(&h2);
        }
        *(uint4 *)(halo + (size_t)i * 16) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (tid == 0) {
        const uint32_t idesc = umma_idesc_bf16(kConvRows, Nt);
        const uint32_t h0 = smem_u32(halo), b0 = smem_u32(Bs);
        int issued = 0;
        for (int t = 0; t < 9; t++) {
            const int dy = t / 3, dx = t % 3;
            for (int s = 0; s < cpad / 16; s++) {
                const uint64_t ad = umma_sdesc(h0 + (uint32_t)(2 * s * kPlane + (dy * kStripCols + dx) * 16), kPlane, 128);
                const uint64_t bd = umma_sdesc(b0 + (uint32_t)(t * tapB + 2 * s * Nt * 16), Nt * 16, 128);
                const uint32_t acc = issued > 0;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
                issued++;
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         smem_u32(bar))
                     : "memory");
    }
    const bool done = mbar_wait_bounded(smem_u32(bar), 0);
    if (!done && lane == 0) atomicOr(err, 1);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

    const int q = warp & 3, half = warp >> 2;
    if (done && 16 * half < Nt) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + 16 * half, v);
        const int xx = x0 + 32 * q + lane, m = y * W + xx;
        if (xx < W) {
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int n = 16 * half + j;
                const float raw = v[j];
                v[j] = 0.0f;  // becomes the layer's output (0 past cout)
                if (n < cout) {
                    const float o = raw + bias[n];
                    v[j] = relu ? fmaxf(o, 0.0f) : o;
                    Y[(long long)n * M + m] = v[j];
                    if (Zp) Zp[(long long)m * Np + n] = raw;
                }
            }
            if (Yh) {  // and its channel-last bf16 copy for the next layer's halo: 16 channels, 32 bytes
                uint32_t w[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                    w[j] = *reinterpret_cast<const uint32_t *>(&h2);
                }
                uint4 *dst = Yh + (long long)m * (Nt / 8) + 2 * half;
                dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
                dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kConvTmemCols)
                     : "memory");
    }
}

// ------------------------------------------------------------------ weight gradient on tcgen05
// D[r][n] = sum over positions p of A[r][p] * B[n][p] for the 128 rows r of
// tile blockIdx.y, over the position range of blockIdx.x:
//   A[r][p] = X[ci][p + offset of tap t] (r = ci * 9 + t < 9 cin; zero outside the grid)
//             1 for r == 9 cin (the bias row), 0 beyond
//   B[n][p] = dZ[n][p] (channel-major fp32, already masked by the ReLU derivative)
// Stages of 64 positions (four K = 16 MMAs) are gathered into one of two
// shared-memory buffers while the tensor core consumes the other; each
// buffer's MMAs are committed to its own mbarrier. CTAs split the positions
// (about four per SM, to hide the gathers' latency). The 128 x Nt partial sums
// are added (atomics) into the gradient in parameter layout: g[n][r] for the
// weights, g[cout * 9 cin + n] for the bias.
constexpr int kWgPos = 64;

__host__ __device__ constexpr int wgrad_smem_bytes(int Nt) {
    return 1024 + 2 * (kConvRows * kWgPos * 2) + 2 * (Nt * kWgPos * 2) + 64;
}

__global__ void __launch_bounds__(kConvThreads, 2)
    k_wgrad_tc(int cin, int cout, int H, int W, int Nt, int per_split, const float *__restrict__ X,
               const float *__restrict__ dZ, float *__restrict__ g, int *__restrict__ err) {
    extern __shared__ uint8_t wg_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)wg_raw + 1023) & ~(uintptr_t)1023);
    constexpr int a_bytes = kConvRows * kWgPos * 2;
    const int b_bytes = Nt * kWgPos * 2;
    uint8_t *As0 = base, *Bs0 = base + 2 * a_bytes;                // buffer b at + b * a_bytes / b * b_bytes
    uint64_t *bar = (uint64_t *)(Bs0 + 2 * b_bytes);              // two barriers
    uint32_t *tmem_slot = (uint32_t *)(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int M = H * W, K9 = 9 * cin, r0 = blockIdx.y * kConvRows;
    const int p0 = blockIdx.x * per_split, p1 = min(M, p0 + per_split);
    const int nst = p1 > p0 ? (p1 - p0 + kWgPos - 1) / kWgPos : 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                     "r"(kConvTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 32) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = umma_idesc_bf16(kConvRows, Nt);

    bool ok = true;
    for (int st = 0; st < nst && ok; st++) {
        const int b = st & 1, pb = p0 + st * kWgPos;
        if (st >= 2) {  // buffer b is free once the MMAs of stage st - 2 are done
            ok = __syncthreads_and(mbar_wait_bounded(smem_u32(bar + b), ((st - 2) >> 1) & 1));
            if (!ok) break;
        }
        // A: 128 rows x 8 chunks of 8 positions; item i -> row i % 128, chunk i / 128
        for (int i = tid; i < kConvRows * (kWgPos / 8); i += kConvThreads) {
            const int rr = i & (kConvRows - 1), ch = i >> 7, r = r0 + rr;
            const int p = pb + ch * 8;
            uint32_t w[4] = {0u, 0u, 0u, 0u};
            if (r < K9) {
                const int ci = r / 9, t = r - 9 * ci, dy = t / 3 - 1, dx = t - 3 * (t / 3) - 1;
                int y = p / W, x = p - y * W;
                const float *Xc = X + (long long)ci * M;
                float v[8];
                const int yy = y + dy;
                if (p + 8 <= p1 && x + 8 <= W) {  // one image row: one row check, edge checks at both ends
                    const bool row_ok = yy >= 0 && yy < H;
                    const float *src = Xc + (long long)yy * W + x + dx;
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const int xx = x + j + dx;
                        v[j] = (row_ok && xx >= 0 && xx < W) ? __ldg(src + j) : 0.0f;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const int yj = y + dy, xx = x + dx;
                        v[j] = (p + j < p1 && yj >= 0 && yj < H && xx >= 0 && xx < W) ? __ldg(Xc + yj * W + xx)
                                                                                       : 0.0f;
                        if (++x == W) x = 0, y++;
                    }
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                    w[j] = *reinterpret_cast<const uint32_t *>(&b2);
                }
            } else if (r == K9) {
                const uint32_t one = __bfloat16_as_ushort(__float2bfloat16(1.0f));
#pragma unroll
                for (int j = 0; j < 8; j++)
                    if (p + j < p1) w[j >> 1] |= (j & 1) ? one << 16 : one;
            }
            *(uint4 *)(As0 + b * a_bytes + ch * (kConvRows * 16) + rr * 16) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        // B: Nt rows x 8 chunks
        for (int i = tid; i < Nt * (kWgPos / 8); i += kConvThreads) {
            const int n = i % Nt, ch = i / Nt, p = pb + ch * 8;
            uint32_t w[4] = {0u, 0u, 0u, 0u};
            if (n < cout) {
                const float *dz = dZ + (long long)n * M + p;
                float v[8];
                if (p + 8 <= p1 && ((uintptr_t)dz & 15) == 0) {
                    const float4 a = __ldg((const float4 *)dz), b4 = __ldg((const float4 *)dz + 1);
                    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b4.x, v[5] = b4.y, v[6] = b4.z, v[7] = b4.w;
                } else {
#pragma unroll
                    for (int j = 0; j < 8; j++) v[j] = p + j < p1 ? __ldg(dz + j) : 0.0f;
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                    w[j] = *reinterpret_cast<const uint32_t *>(&b2);
                }
            }
            *(uint4 *)(Bs0 + b * b_bytes + ch * (Nt * 16) + n * 16) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (tid == 0) {
            const uint32_t a0 = smem_u32(As0 + b * a_bytes), b0 = smem_u32(Bs0 + b * b_bytes);
            const uint32_t a_lbo = kConvRows * 16, b_lbo = Nt * 16;
#pragma unroll
            for (int s = 0; s < kWgPos / 16; s++) {
                const uint64_t ad = umma_sdesc(a0 + 2 * s * a_lbo, a_lbo, 128);
                const uint64_t bd = umma_sdesc(b0 + 2 * s * b_lbo, b_lbo, 128);
                const uint32_t acc = (st > 0 || s > 0);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(bar + b))
                         : "memory");
        }
    }
    // the last commit of each buffer (the later one covers every MMA issued)
    if (ok && nst > 1) ok = __syncthreads_and(mbar_wait_bounded(smem_u32(bar + ((nst - 2) & 1)), ((nst - 2) >> 1) & 1));
    if (ok && nst > 0) ok = __syncthreads_and(mbar_wait_bounded(smem_u32(bar + ((nst - 1) & 1)), ((nst - 1) >> 1) & 1));
    if (!ok && tid == 0) atomicOr(err, 1);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

    const int q = warp & 3, half = warp >> 2;
    if (ok && nst > 0 && 16 * half < Nt) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + 16 * half, v);
        const int r = r0 + 32 * q + lane;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int n = 16 * half + j;
            if (n < cout) {
                if (r < K9) atomicAdd(g + (long long)n * K9 + r, v[j]);
                else if (r == K9) atomicAdd(g + (long long)cout * K9 + n, v[j]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kConvTmemCols)
                     : "memory");
    }
}

// ------------------------------------------------------------------ layer pieces
__global__ void k_im2col(int Cin, int H, int W, int Kp, const float *__restrict__ X, __nv_bfloat16 *__restrict__ col) {
    const long long total = (long long)H * W * Kp;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i % Kp);
        const long long m = i / Kp;
        const int y = (int)(m / W), x = (int)(m % W);
        float v = 0.0f;
        if (k < Cin * 9) {
            const int ci = k / 9, r = k % 9, yy = y + r / 3 - 1, xx = x + r % 3 - 1;
            if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = X[((long long)ci * H + yy) * W + xx];
        }
        col[i] = __float2bfloat16(v);
    }
}

// Y[n][m] = act(Z[m][n] + b[n]); keeps Z (pre-activation) for the backward pass
__global__ void k_bias_act(int M, int Cout, int Np, const float *__restrict__ Z, const float *__restrict__ b,
                           float *__restrict__ Y, int relu) {
    const long long total = (long long)M * Cout;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int n = (int)(i / M);
        const long long m = i % M;
        const float v = Z[m * Np + n] + b[n];
        Y[i] = relu ? fmaxf(v, 0.0f) : v;
    }
}

// dY[n][m] = 0 where the layer's ReLU output is 0 (its derivative there)
__global__ void k_relu_mask(long long count, const float *__restrict__ Y, float *__restrict__ dY) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        if (!(Y[i] > 0.0f)) dY[i] = 0.0f;
}

// dY = 2 (Y - T) / count; partial sums of the squared error into loss[0]
__global__ void k_mse(long long count, const float *__restrict__ Y, const float *__restrict__ T,
                      float *__restrict__ dY, float *__restrict__ loss) {
    __shared__ float red[256];
    float s = 0.0f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        const float d = Y[i] - T[i];
        dY[i] = 2.0f * d / (float)count;
        s += d * d;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] / (float)count);
}

// weight layout conversions: W[co][ci][3][3] (f32 master) <-> Wt[k][n] (bf16 GEMM operand)
__global__ void k_pack_w(int Cin, int Cout, int Kp, int Np, const float *__restrict__ Wm,
                         __nv_bfloat16 *__restrict__ Wt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Kp * Np; i += gridDim.x * blockDim.x) {
        const int k = i / Np, n = i % Np;
        const float v = (k < Cin * 9 && n < Cout) ? Wm[n * Cin * 9 + k] : 0.0f;
        Wt[i] = __float2bfloat16(v);
    }
}

// Wf[k][n] (bf16) with k = co * 9 + t, n = ci: W[co][ci][8 - t]
__global__ void k_pack_wflip(int Cin, int Cout, int KpT, int NpT, const float *__restrict__ Wm,
                             __nv_bfloat16 *__restrict__ Wf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < KpT * NpT; i += gridDim.x * blockDim.x) {
        const int k = i / NpT, n = i % NpT;
        const int co = k / 9, t = k % 9;
        const float v = (k < Cout * 9 && n < Cin) ? Wm[(co * Cin + n) * 9 + (8 - t)] : 0.0f;
        Wf[i] = __float2bfloat16(v);
    }
}

__global__ void k_adam(int n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m1,
                       float *__restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        m1[i] = b1 * m1[i] + (1.0f - b1) * gi;
        m2[i] = b2 * m2[i] + (1.0f - b2) * gi * gi;
        p[i] -= lr * (m1[i] / c1) / (sqrtf(m2[i] / c2) + eps);
    }
}

int grid(long long items) {
    long long b = (items + 255) / 256;
    return (int)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

}  // namespace

struct gr_cnn {
    int device = 0, H = 0, W = 0, n_layers = 0;
    int cin[kMaxLayers] = {}, cout[kMaxLayers] = {}, Kp[kMaxLayers] = {}, Np[kMaxLayers] = {};
    int64_t w_ofs[kMaxLayers + 1] = {};  // parameter offsets: weights then bias, per layer
    int64_t n_params = 0;
    float *params = nullptr, *grads = nullptr, *m1 = nullptr, *m2 = nullptr;
    __nv_bfloat16 *wt[kMaxLayers] = {};
    __nv_bfloat16 *wf[kMaxLayers] = {};  // backward operand: Wf[co*9 + t][ci] = W[co][ci][8 - t]
    uint4 *ws[kMaxLayers] = {};   // k_conv_strip's weight image of wt (forward)
    uint4 *wfs[kMaxLayers] = {};  // and of wf (input gradient)
    int KpT[kMaxLayers] = {}, NpT[kMaxLayers] = {};
    float *zero_bias = nullptr;
    float *act[kMaxLayers + 1] = {};  // act[0] = input, act[l+1] = output of layer l
    uint4 *act_h[kMaxLayers + 1] = {};  // act[l] (l >= 1) as channel-last bf16, rounded up to 16 channels
    float *z[kMaxLayers] = {};  // GEMM output of the fallback path
    __nv_bfloat16 *col = nullptr;  // patches of a layer too wide for the tensor-core tile (fallback)
    float *dact = nullptr, *dact2 = nullptr, *loss = nullptr;
    int64_t adam_t = 0;
    int sm_count = 148;
    int *err = nullptr;  // device: set by a convolution whose accumulator wait gave up
    cudaStream_t stream = nullptr;
};

namespace {

int gemm(cudaStream_t s, int M, int N, int K, const __nv_bfloat16 *A, long long sam, long long sak,
         const __nv_bfloat16 *B, long long sbk, long long sbn, float *C, long long scm, long long scn, int splits) {
    int kchunk = round_up((K + splits - 1) / splits, kBK);
    dim3 g((M + kBM - 1) / kBM, (N + kBN - 1) / kBN, (K + kchunk - 1) / kchunk);
    k_gemm<<<g, 128, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, scm, scn, kchunk, g.z > 1 ? 1 : 0);
    CN_CK(cudaGetLastError());
    return GR_OK;
}

int pack_all(gr_cnn *c) {
    for (int l = 0; l < c->n_layers; l++) {
        k_pack_w<<<grid((long long)c->Kp[l] * c->Np[l]), 256, 0, c->stream>>>(c->cin[l], c->cout[l], c->Kp[l], c->Np[l],
                                                                               c->params + c->w_ofs[l], c->wt[l]);
        if (c->ws[l])
            k_pack_strip<<<grid(9LL * strip_cpad(c->cin[l]) / 8 * round_up(c->cout[l], 16)), 256, 0, c->stream>>>(
                c->cin[l], round_up(c->cout[l], 16), c->Np[l], c->wt[l], c->ws[l]);
        if (l > 0) {
            k_pack_wflip<<<grid((long long)c->KpT[l] * c->NpT[l]), 256, 0, c->stream>>>(
                c->cin[l], c->cout[l], c->KpT[l], c->NpT[l], c->params + c->w_ofs[l], c->wf[l]);
            k_pack_strip<<<grid(9LL * strip_cpad(c->cout[l]) / 8 * round_up(c->cin[l], 16)), 256, 0, c->stream>>>(
                c->cout[l], round_up(c->cin[l], 16), c->NpT[l], c->wf[l], c->wfs[l]);
        }
    }
    CN_CK(cudaGetLastError());
    return GR_OK;
}

// tiles of 16 columns x 8 rows

// the tensor-core convolution takes a layer whose tiles fit in shared memory
bool conv_tc_fits(const gr_cnn *c, int l) {
    return strip_smem_bytes(round_up(c->cout[l], 16), c->cin[l]) <= kConvSmemMax && round_up(c->cout[l], 16) <= 32;
}

dim3 strip_grid(const gr_cnn *c) { return dim3((c->W + kStripX - 1) / kStripX, c->H); }

int forward(gr_cnn *c, cudaStream_t s) {
    const int M = c->H * c->W;
    for (int l = 0; l < c->n_layers; l++) {
        const float *bl = c->params + c->w_ofs[l] + (int64_t)c->cout[l] * c->cin[l] * 9;
        if (conv_tc_fits(c, l)) {
            const int Nt = round_up(c->cout[l], 16);
            // the input's channel-last copy when the previous layer (a strip
            // convolution) wrote one; this layer's copy for the next
            const uint4 *xh = (l > 0 && conv_tc_fits(c, l - 1)) ? c->act_h[l] : nullptr;
            uint4 *yh = l + 1 < c->n_layers ? c->act_h[l + 1] : nullptr;
            k_conv_strip<<<strip_grid(c), kConvThreads, strip_smem_bytes(Nt, c->cin[l]), s>>>(
                c->cin[l], c->cout[l], c->H, c->W, Nt, c->Np[l], c->act[l], c->ws[l], bl, c->act[l + 1], nullptr,
                l + 1 < c->n_layers, c->err, xh, yh);
            continue;
        }
        k_im2col<<<grid((long long)M * c->Kp[l]), 256, 0, s>>>(c->cin[l], c->H, c->W, c->Kp[l], c->act[l], c->col);
        int rc = gemm(s, M, c->Np[l], c->Kp[l], c->col, c->Kp[l], 1, c->wt[l], c->Np[l], 1, c->z[l], c->Np[l], 1, 1);
        if (rc) return rc;
        k_bias_act<<<grid((long long)M * c->cout[l]), 256, 0, s>>>(M, c->cout[l], c->Np[l], c->z[l], bl,
                                                                   c->act[l + 1], l + 1 < c->n_layers);
    }
    CN_CK(cudaGetLastError());
    return GR_OK;
}

// gradients of the mean squared error against d_target into c->grads
int backward(gr_cnn *c, const float *d_target) {
    const int M = c->H * c->W, L = c->n_layers;
    cudaStream_t s = c->stream;
    const long long cnt = (long long)c->cout[L - 1] * M;
    CN_CK(cudaMemsetAsync(c->loss, 0, sizeof(float), s));
    k_mse<<<grid(cnt), 256, 0, s>>>(cnt, c->act[L], d_target, c->dact, c->loss);
    float *dY = c->dact, *dX = c->dact2;
    for (int l = L - 1; l >= 0; l--) {
        const int cin = c->cin[l], co = c->cout[l], Nt = round_up(co, 16);
        if (l + 1 < L) k_relu_mask<<<grid((long long)co * M), 256, 0, s>>>((long long)co * M, c->act[l + 1], dY);
        float *g = c->grads + c->w_ofs[l];
        CN_CK(cudaMemsetAsync(g, 0, sizeof(float) * (c->w_ofs[l + 1] - c->w_ofs[l]), s));
        const int ktiles = (9 * cin + 1 + kConvRows - 1) / kConvRows;  // weight rows and the bias row
        const int want = (4 * c->sm_count + ktiles - 1) / ktiles;  // 4 CTAs per SM fit (42 KB, 56 registers)
        const int per = round_up((M + want - 1) / want, kWgPos), splits = (M + per - 1) / per;
        k_wgrad_tc<<<dim3(splits, ktiles), kConvThreads, wgrad_smem_bytes(Nt), s>>>(cin, co, c->H, c->W, Nt, per,
                                                                                   c->act[l], dY, g, c->err);
        if (l > 0) {  // cin = hidden <= 32 and cout <= 32: always within the tensor-core tile
            k_conv_strip<<<strip_grid(c), kConvThreads, strip_smem_bytes(round_up(cin, 16), co), s>>>(co, cin, c->H, c->W, round_up(cin, 16), c->NpT[l], dY, c->wfs[l], c->zero_bias,
                             dX, nullptr, 0, c->err, nullptr, nullptr);
            float *t = dY;
            dY = dX;
            dX = t;
        }
    }
    CN_CK(cudaGetLastError());
    return GR_OK;
}

// waits for the network's stream; a convolution that gave up waiting for its
// accumulator is reported (and the flag cleared)
int finish(gr_cnn *c) {
    int err = 0;
    CN_CK(cudaMemcpyAsync(&err, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CN_CK(cudaStreamSynchronize(c->stream));
    if (err) {
        CN_CK(cudaMemsetAsync(c->err, 0, sizeof(int), c->stream));
        CN_CK(cudaStreamSynchronize(c->stream));
        return GR_ERR_DEVICE;
    }
    return GR_OK;
}

}  // namespace

extern "C" {

int gr_cnn_create(gr_cnn **out, int device, int in_channels, int out_channels, int hidden, int n_layers, int H,
                  int W, uint64_t seed) {
    if (!out || in_channels < 1 || out_channels < 1 || hidden < 1 || hidden > 32 || n_layers < 2 ||
        n_layers > kMaxLayers || H < 1 || W < 1 || out_channels > 32)
        return GR_ERR_ARG;
    *out = nullptr;
    CN_CK(cudaSetDevice(device));
    // the attribute holds for the whole process: one constant value
    CN_CK(cudaFuncSetAttribute(k_conv_strip, cudaFuncAttributeMaxDynamicSharedMemorySize, kConvSmemMax));
    gr_cnn *c = new gr_cnn();
    c->device = device;
    c->H = H;
    c->W = W;
    c->n_layers = n_layers;
    int64_t ofs = 0, kmax = 0, cmax = in_channels;
    for (int l = 0; l < n_layers; l++) {
        c->cin[l] = l == 0 ? in_channels : hidden;
        c->cout[l] = l + 1 == n_layers ? out_channels : hidden;
        c->Kp[l] = round_up(c->cin[l] * 9, 16);
        c->Np[l] = round_up(c->cout[l], 8);
        c->KpT[l] = round_up(c->cout[l] * 9, 16);
        c->NpT[l] = round_up(c->cin[l], 8);
        c->w_ofs[l] = ofs;
        ofs += (int64_t)c->cout[l] * c->cin[l] * 9 + c->cout[l];
        if (!conv_tc_fits(c, l)) kmax = c->Kp[l] > kmax ? c->Kp[l] : kmax;  // fallback patches
        cmax = c->cout[l] > cmax ? c->cout[l] : cmax;
    }
    c->w_ofs[n_layers] = ofs;
    c->n_params = ofs;
    const int64_t M = (int64_t)H * W;
    auto fail = [&](int code) {
        gr_cnn_destroy(c);
        return code;
    };
    bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc(&c->params, sizeof(float) * ofs) == cudaSuccess;
    ok = ok && cudaMalloc(&c->grads, sizeof(float) * ofs) == cudaSuccess;
    ok = ok && cudaMalloc(&c->m1, sizeof(float) * ofs) == cudaSuccess;
    ok = ok && cudaMalloc(&c->m2, sizeof(float) * ofs) == cudaSuccess;
    ok = ok && cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device) == cudaSuccess;
    if (kmax > 0) ok = ok && cudaMalloc(&c->col, sizeof(__nv_bfloat16) * M * kmax) == cudaSuccess;
    // uploads and clears on the network's own (non-blocking) stream: a
    // legacy-stream cudaMemcpy from pageable memory may return before its
    // DMA lands, and nothing orders the legacy stream before this one
    ok = ok && cudaMalloc(&c->zero_bias, sizeof(float) * 64) == cudaSuccess &&
         cudaMemsetAsync(c->zero_bias, 0, sizeof(float) * 64, c->stream) == cudaSuccess;
    ok = ok && cudaMalloc(&c->dact, sizeof(float) * M * cmax) == cudaSuccess;
    ok = ok && cudaMalloc(&c->dact2, sizeof(float) * M * cmax) == cudaSuccess;
    ok = ok && cudaMalloc(&c->loss, sizeof(float) * 2) == cudaSuccess;
    ok = ok && cudaMalloc(&c->err, sizeof(int)) == cudaSuccess &&
         cudaMemsetAsync(c->err, 0, sizeof(int), c->stream) == cudaSuccess;
    for (int l = 0; l <= n_layers && ok; l++)
        ok = cudaMalloc(&c->act[l], sizeof(float) * M * (l == 0 ? in_channels : c->cout[l - 1])) == cudaSuccess;
    for (int l = 1; l < n_layers && ok; l++)
        ok = cudaMalloc(&c->act_h[l], sizeof(uint16_t) * M * round_up(c->cout[l - 1], 16)) == cudaSuccess;
    for (int l = 0; l < n_layers && ok; l++) {
        ok = cudaMalloc(&c->wt[l], sizeof(__nv_bfloat16) * c->Kp[l] * c->Np[l]) == cudaSuccess &&
             cudaMalloc(&c->wf[l], sizeof(__nv_bfloat16) * c->KpT[l] * c->NpT[l]) == cudaSuccess &&
             cudaMalloc(&c->ws[l], sizeof(uint4) * 9 * strip_cpad(c->cin[l]) / 8 * round_up(c->cout[l], 16)) ==
                 cudaSuccess &&
             cudaMalloc(&c->wfs[l], sizeof(uint4) * 9 * strip_cpad(c->cout[l]) / 8 * round_up(c->cin[l], 16)) ==
                 cudaSuccess;
        if (ok && !conv_tc_fits(c, l)) ok = cudaMalloc(&c->z[l], sizeof(float) * M * c->Np[l]) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        return fail(GR_ERR_NOMEM);
    }
    // He-uniform weights from a fixed-seed generator (splitmix64), zero biases
    std::vector<float> h(ofs, 0.0f);
    uint64_t st = seed ? seed : 1;
    auto rnd = [&]() {
        uint64_t z = (st += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) / 9007199254740992.0;
    };
    for (int l = 0; l < n_layers; l++) {
        const double a = std::sqrt(6.0 / (c->cin[l] * 9.0));
        for (int64_t i = 0; i < (int64_t)c->cout[l] * c->cin[l] * 9; i++) h[c->w_ofs[l] + i] = (float)((2 * rnd() - 1) * a);
    }
    if (cudaMemcpyAsync(c->params, h.data(), sizeof(float) * ofs, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->m1, 0, sizeof(float) * ofs, c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->m2, 0, sizeof(float) * ofs, c->stream) != cudaSuccess || pack_all(c) != GR_OK ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return fail(GR_ERR_CUDA);
    *out = c;
    return GR_OK;
}

int gr_cnn_destroy(gr_cnn *c) {
    if (!c) return GR_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (void *p : {(void *)c->params, (void *)c->grads, (void *)c->m1, (void *)c->m2, (void *)c->col,
                    (void *)c->zero_bias, (void *)c->dact, (void *)c->dact2, (void *)c->loss, (void *)c->err})
        cudaFree(p);
    for (int l = 0; l < kMaxLayers; l++) {
        cudaFree(c->wt[l]);
        cudaFree(c->wf[l]);
        cudaFree(c->ws[l]);
        cudaFree(c->wfs[l]);
        cudaFree(c->z[l]);
    }
    for (int l = 0; l <= kMaxLayers; l++) {
        cudaFree(c->act[l]);
        cudaFree(c->act_h[l]);
    }
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return GR_OK;
}

int64_t gr_cnn_num_params(gr_cnn *c) { return c ? c->n_params : -1; }

int gr_cnn_info(gr_cnn *c, int *device, int *in_channels, int *out_channels, int *H, int *W) {
    if (!c) return GR_ERR_ARG;
    if (device) *device = c->device;
    if (in_channels) *in_channels = c->cin[0];
    if (out_channels) *out_channels = c->cout[c->n_layers - 1];
    if (H) *H = c->H;
    if (W) *W = c->W;
    return GR_OK;
}

int gr_cnn_get_params(gr_cnn *c, float *h_out) {
    if (!c || !h_out) return GR_ERR_ARG;
    CN_CK(cudaStreamSynchronize(c->stream));
    CN_CK(cudaMemcpyAsync(h_out, c->params, sizeof(float) * c->n_params, cudaMemcpyDeviceToHost, c->stream));
    CN_CK(cudaStreamSynchronize(c->stream));
    return GR_OK;
}

int gr_cnn_set_params(gr_cnn *c, const float *h_in) {
    if (!c || !h_in) return GR_ERR_ARG;
    CN_CK(cudaStreamSynchronize(c->stream));
    CN_CK(cudaMemcpyAsync(c->params, h_in, sizeof(float) * c->n_params, cudaMemcpyHostToDevice, c->stream));
    int rc = pack_all(c);
    if (rc) return rc;
    CN_CK(cudaStreamSynchronize(c->stream));
    return GR_OK;
}

int gr_cnn_forward(gr_cnn *c, const float *d_in, float *d_out) {
    if (!c || !d_in || !d_out) return GR_ERR_ARG;
    const int64_t M = (int64_t)c->H * c->W;
    CN_CK(cudaMemcpyAsync(c->act[0], d_in, sizeof(float) * M * c->cin[0], cudaMemcpyDeviceToDevice, c->stream));
    int rc = forward(c, c->stream);
    if (rc) return rc;
    CN_CK(cudaMemcpyAsync(d_out, c->act[c->n_layers], sizeof(float) * M * c->cout[c->n_layers - 1],
                          cudaMemcpyDeviceToDevice, c->stream));
    return finish(c);
}

int gr_cnn_forward_async(gr_cnn *c, const float *d_in, float *d_out, void *stream) {
    if (!c || !d_in || !d_out) return GR_ERR_ARG;
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    const int64_t M = (int64_t)c->H * c->W;
    CN_CK(cudaMemcpyAsync(c->act[0], d_in, sizeof(float) * M * c->cin[0], cudaMemcpyDeviceToDevice, s));
    int rc = forward(c, s);
    if (rc) return rc;
    CN_CK(cudaMemcpyAsync(d_out, c->act[c->n_layers], sizeof(float) * M * c->cout[c->n_layers - 1],
                          cudaMemcpyDeviceToDevice, s));
    return GR_OK;
}

int gr_cnn_check(gr_cnn *c) {
    if (!c) return GR_ERR_ARG;
    return finish(c);
}

int gr_cnn_grads(gr_cnn *c, const float *d_in, const float *d_target, float *h_grads, float *h_loss) {
    if (!c || !d_in || !d_target) return GR_ERR_ARG;
    const int64_t M = (int64_t)c->H * c->W;
    CN_CK(cudaMemcpyAsync(c->act[0], d_in, sizeof(float) * M * c->cin[0], cudaMemcpyDeviceToDevice, c->stream));
    int rc = forward(c, c->stream);
    if (!rc) rc = backward(c, d_target);
    if (rc) return rc;
    if (h_grads)
        CN_CK(cudaMemcpyAsync(h_grads, c->grads, sizeof(float) * c->n_params, cudaMemcpyDeviceToHost, c->stream));
    if (h_loss) CN_CK(cudaMemcpyAsync(h_loss, c->loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    return finish(c);
}

int gr_cnn_train_step(gr_cnn *c, const float *d_in, const float *d_target, float lr, float *h_loss) {
    if (!c || !d_in || !d_target || !(lr > 0.0f)) return GR_ERR_ARG;
    const int64_t M = (int64_t)c->H * c->W;
    CN_CK(cudaMemcpyAsync(c->act[0], d_in, sizeof(float) * M * c->cin[0], cudaMemcpyDeviceToDevice, c->stream));
    int rc = forward(c, c->stream);
    if (!rc) rc = backward(c, d_target);
    if (rc) return rc;
    c->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - (float)std::pow((double)b1, (double)c->adam_t);
    const float c2 = 1.0f - (float)std::pow((double)b2, (double)c->adam_t);
    k_adam<<<grid(c->n_params), 256, 0, c->stream>>>((int)c->n_params, c->params, c->grads, c->m1, c->m2, lr, b1, b2,
                                                      1e-8f, c1, c2);
    CN_CK(cudaGetLastError());
    rc = pack_all(c);
    if (rc) return rc;
    if (h_loss) CN_CK(cudaMemcpyAsync(h_loss, c->loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    return finish(c);
}

// test hook: one GEMM C = A * B of row-major bf16 matrices (A: M x K, B: K x N),
// C f32 row-major, with the k range split over `splits` blocks
int gr_cnn_gemm_test(int M, int N, int K, const void *d_a, const void *d_b, float *d_c, int splits) {
    if (M < 1 || N < 1 || K < 1 || !d_a || !d_b || !d_c || splits < 1) return GR_ERR_ARG;
    CN_CK(cudaMemset(d_c, 0, sizeof(float) * M * N));
    int rc = gemm(nullptr, M, N, K, (const __nv_bfloat16 *)d_a, K, 1, (const __nv_bfloat16 *)d_b, N, 1, d_c, N, 1,
                  splits);
    if (rc) return rc;
    CN_CK(cudaDeviceSynchronize());
    return GR_OK;
}

}  // extern "C"
