// lpc.cu - learned Poisson preconditioner: a small convolutional network that maps
// the pressure residual to an error estimate inside flexible CG.
//
// Activations are BF16 in NHWC layout (pixel = MAC cell (i, j) flattened as
// i*W + j with j contiguous, 32 channels innermost); every product is accumulated
// in FP32. The 32 -> 32 channel 3x3 convolutions (the FLOP-heavy layers) are
// implicit GEMMs on the 5th-generation tensor cores: per CTA one or two grid rows of 128
// consecutive pixels (M = 128 per row), N = 32 output channels, K = 9 taps x 32
// input channels = 288, issued as 18 tcgen05.mma per row (kind::f16, BF16 inputs,
// FP32 accumulator in tensor memory) by one thread; the input rows are staged once
// in shared memory in a layout where every tap is a K-major no-swizzle operand
// (8 rows x 16 bytes per core matrix) at its own descriptor offset, so no im2col
// copy is made; the epilogue reads the accumulators with tcgen05.ld and fuses bias,
// skip addition, ReLU and the
// fluid mask. The 1-channel layers, pooling, upsampling and the backward pass run
// on CUDA cores with FP32 accumulation.
//
// This file is compiled without -fmad=false: it is not part of the float64
// parity path.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "lpc.cuh"

namespace cfd {
namespace lpc {

namespace {

constexpr int CH = 32;
constexpr int KDIM = 9 * CH;            // 288
constexpr int TM = 128;                 // pixels per tile
constexpr int CORE_BYTES = 128;         // one core matrix: 8 rows x 16 bytes
constexpr int SBO = (KDIM / 8) * CORE_BYTES;  // 4608 bytes between 8-row groups
constexpr int B_BYTES = (CH / 8) * SBO;       // 18432
constexpr uint32_t kWaitLimit = 1u << 24;

// UMMA instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and B
// BF16 (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bit 17,
// M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(CH >> 3) << 17) |
                            ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor: start address >> 4 (bits 0-13), leading byte
// offset >> 4 (bits 16-29, distance between the two K core matrices of one MMA),
// stride byte offset >> 4 (bits 32-45, distance between 8-row groups), version 1
// (bits 46-47), no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__device__ __forceinline__ float bf2f(__nv_bfloat16 x) { return __bfloat162float(x); }

// Programmatic dependent launch: the network's kernels are launched so that each may
// start while its predecessor finishes. Before pdl_wait() a kernel touches only what
// no predecessor writes (its weights, shared memory, TMEM); pdl_wait() returns once the
// predecessor grid has completed and its memory is visible. pdl_trigger() lets the
// successor start as soon as every CTA of this grid has issued it.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

}  // namespace

// ---------------------------------------------------------------- 32 -> 32 conv (tensor cores)
// y[p][n] = act(bias[n] + sum_{tap, c} w[n][c][tap] * x[p + tap][c] (+ skip[p][n])), masked.
// wpack is the B operand image (N = 32 rows, K = 288) in the shared-memory layout.
//
// One CTA computes ROWS (1 or 2) output rows i0 .. i0+ROWS-1 of one 128-pixel segment
// j0 .. j0+127. The ROWS + 2 input rows it needs, pixels j0-1 .. j0+128 (XP = 130,
// zero outside the grid), are copied once into shared memory, channel-chunk major:
// chunk c (channels 8c .. 8c+7, 16 bytes) of pixel q of staged row r sits at
// r*XROW + c*XCHUNK + q*16. In that layout the A operand of tap (di, dj) for output
// row r is already a K-major no-swizzle matrix: pixel m of the tile is 16 bytes after
// pixel m-1 (8-row groups 128 bytes apart: SBO = 128) and the two 8-channel core
// matrices of one 16-channel MMA step are XCHUNK apart (LBO = XCHUNK), starting at
// (r + di + 1)*XROW + 2h*XCHUNK + (dj + 1)*16. So the nine taps are nine descriptor
// offsets into the same staged rows, with no im2col copy; each output row takes 18
// MMAs into its own 32 TMEM columns, and one commit covers all ROWS*18.
constexpr int XP = TM + 2;
constexpr int XCHUNK = XP * 16;            // 2080
constexpr int XROW = 4 * XCHUNK;           // 8320
constexpr int XB = 13;                     // loads in flight per thread and batch
// Two warpgroups per CTA: both stage operands (twice the loads in flight of one), one
// thread issues the MMAs, and in the epilogue warpgroup g takes rows g, g + 2, ...
// (warp w reads TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31, its 32 pixels).
constexpr int NT = 256;
constexpr int ST_BYTES = TM * 5 * 16;      // epilogue staging of one row: 128 pixels x 80 bytes
__host__ __device__ constexpr int x_bytes(int rows) { return (rows + 2) * XROW; }

template <int ROWS>
__global__ void __launch_bounds__(NT) k_conv32_tc(const __nv_bfloat16* __restrict__ x,
                                                  const uint4* __restrict__ wpack,
                                                  const float* __restrict__ bias,
                                                  const __nv_bfloat16* __restrict__ skip,
                                                  const uint8_t* __restrict__ mask,
                                                  __nv_bfloat16* __restrict__ y, int H, int W,
                                                  int relu, int* __restrict__ err) {
    constexpr int XQ = (ROWS + 2) * XP * 4;    // 16-byte chunks staged per CTA
    constexpr int XPER = (XQ + NT - 1) / NT;   // per thread
    constexpr int BQ = B_BYTES / 16, BPER = (BQ + NT - 1) / NT;
    static_assert(2 * ST_BYTES <= x_bytes(ROWS), "epilogue staging fits in the operand buffer");
    constexpr uint32_t kTmemCols = 32u * ROWS;
    static_assert((kTmemCols & (kTmemCols - 1)) == 0 && kTmemCols >= 32 && kTmemCols <= 512, "TMEM columns");
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* Bs = smem;            // 18432 bytes, offset 0
    uint8_t* Xs = smem + B_BYTES;  // x_bytes(ROWS) bytes, 16-byte aligned
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int ok;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int i0 = blockIdx.y * ROWS;
    const int j0 = blockIdx.x * TM;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        ok = 1;
    }
    // B operand: a straight copy of the prepacked image, all loads of a thread in flight
    {
        uint4 v[BPER];
#pragma unroll
        for (int k = 0; k < BPER; ++k)
            if (tid + k * NT < BQ) v[k] = wpack[tid + k * NT];
#pragma unroll
        for (int k = 0; k < BPER; ++k)
            if (tid + k * NT < BQ) reinterpret_cast<uint4*>(Bs)[tid + k * NT] = v[k];
    }
    // everything below reads what the predecessor kernel wrote
    pdl_trigger();
    pdl_wait();
    // staged input rows: consecutive threads take consecutive 16-byte chunks in global
    // order (chunk fastest, then pixel), so each warp reads 512 contiguous bytes; the
    // loads go out in batches of XB per thread before their shared-memory stores
#pragma unroll
    for (int k0 = 0; k0 < XPER; k0 += XB) {
        uint4 v[XB];
#pragma unroll
        for (int k = 0; k < XB; ++k) {
            const int q = tid + (k0 + k) * NT;
            const int c = q & 3, t = q >> 2;
            const int r = t / XP, px = t - r * XP;
            const int ii = i0 - 1 + r, jj = j0 - 1 + px;
            v[k] = make_uint4(0u, 0u, 0u, 0u);
            if (k0 + k < XPER && q < XQ && ii >= 0 && ii < H && jj >= 0 && jj < W)
                v[k] = reinterpret_cast<const uint4*>(x + ((size_t)ii * W + jj) * CH)[c];
        }
#pragma unroll
        for (int k = 0; k < XB; ++k) {
            const int q = tid + (k0 + k) * NT;
            if (k0 + k < XPER && q < XQ) {
                const int c = q & 3, t = q >> 2;
                const int r = t / XP, px = t - r * XP;
                *reinterpret_cast<uint4*>(Xs + r * XROW + c * XCHUNK + px * 16) = v[k];
            }
        }
    }
    // generic-proxy shared-memory writes become visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    if (tid == 0) {
        const uint32_t x0 = smem_u32(Xs), b0 = smem_u32(Bs);
        for (int r = 0; r < ROWS; ++r) {
#pragma unroll
            for (int s = 0; s < KDIM / 16; ++s) {
                const int tap = s >> 1, h = s & 1;
                const int di = tap / 3, dj = tap % 3;  // di, dj in 0..2 stand for -1..1
                const uint32_t aaddr = x0 + (uint32_t)((r + di) * XROW + 2 * h * XCHUNK + dj * 16);
                const uint64_t ad = umma_desc(aaddr, XCHUNK, CORE_BYTES);
                const uint64_t bd = umma_desc(b0 + s * 2 * CORE_BYTES, CORE_BYTES, SBO);
                const uint32_t acc = s > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + (uint32_t)(32 * r)),
                    "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc));
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&mbar))
                     : "memory");
    }
    // bounded wait for the accumulators
    {
        uint32_t done = 0;
        for (uint32_t spin = 0; spin < kWaitLimit && !done; ++spin) {
            asm volatile(
                "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                "selp.b32 %0, 1, 0, P1;\n\t}\n"
                : "=r"(done)
                : "r"(smem_u32(&mbar)), "r"(0));
        }
        if (!done) {
            ok = 0;
            if (err) atomicExch(err, 1);
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        // The MMAs have finished reading the staged rows, so their buffer stages the
        // epilogue: 128 pixels x 80 bytes per output row and warpgroup (skip input in,
        // result out), read and written in global memory as contiguous 16-byte chunks.
        // Each warpgroup synchronises on its own named barrier (1 or 2).
        const int g = warp >> 2, wq = warp & 3, lt = tid & (TM - 1);
        const int m = wq * 32 + lane;
        const int j = j0 + m;
        const int npx = min(TM, W - j0);
        uint4* st = reinterpret_cast<uint4*>(Xs + g * ST_BYTES);
        const uint4* skip4 = reinterpret_cast<const uint4*>(skip);
        uint4* y4 = reinterpret_cast<uint4*>(y);
        for (int r = g; r < ROWS; r += 2) {
            const int i = i0 + r;
            if (i >= H) break;
            const size_t rowp = (size_t)i * W + j0;
            if (skip) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int q = lt + k * TM, px = q >> 2;
                    if (px < npx) st[px * 5 + (q & 3)] = skip4[(rowp + px) * 4 + (q & 3)];
                }
            }
            asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(TM) : "memory");
            float acc[CH];
#pragma unroll
            for (int c0 = 0; c0 < CH; c0 += 8) {
                uint32_t v[8];
                const uint32_t taddr = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)(32 * r + c0);
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                               "=r"(v[6]), "=r"(v[7])
                             : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int q = 0; q < 8; ++q) acc[c0 + q] = __uint_as_float(v[q]);
            }
            if (j < W) {
                const size_t p = rowp + m;
                const bool fl = mask ? (mask[p] != 0) : true;
                __align__(16) __nv_bfloat16 sk[CH];
                if (skip) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) reinterpret_cast<uint4*>(sk)[q] = st[m * 5 + q];
                }
                __align__(16) __nv_bfloat16 out[CH];
#pragma unroll
                for (int n = 0; n < CH; ++n) {
                    float val = acc[n] + bias[n];
                    if (skip) val += bf2f(sk[n]);
                    if (relu) val = fmaxf(val, 0.0f);
                    out[n] = __float2bfloat16(fl ? val : 0.0f);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) st[m * 5 + q] = reinterpret_cast<const uint4*>(out)[q];
            }
            asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(TM) : "memory");
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int q = lt + k * TM, px = q >> 2;
                if (px < npx) y4[(rowp + px) * 4 + (q & 3)] = st[px * 5 + (q & 3)];
            }
            asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(TM) : "memory");
        }
    } else {
        // The accumulators never arrived: this CTA's output rows are written as zeros
        // (a defined output; the host reads *err and abandons the result), and the
        // MMAs get a second bounded wait before their TMEM columns are freed. TMEM
        // contents are undefined after a timeout.
        const int npx = min(TM, W - j0);
        uint4* y4 = reinterpret_cast<uint4*>(y);
        for (int r = 0; r < ROWS; ++r) {
            const int i = i0 + r;
            if (i >= H) break;
            const size_t rowp = (size_t)i * W + j0;
            for (int q = tid; q < npx * 4; q += NT) y4[rowp * 4 + q] = make_uint4(0u, 0u, 0u, 0u);
        }
        if (tid == 0) {
            uint32_t done = 0;
            for (uint32_t spin = 0; spin < kWaitLimit && !done; ++spin) {
                asm volatile(
                    "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                    "selp.b32 %0, 1, 0, P1;\n\t}\n"
                    : "=r"(done)
                    : "r"(smem_u32(&mbar)), "r"(0));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

// Pack w[n][c][3][3] (float, PyTorch OIHW) into the B operand image.
// adjoint = 1: the image of the data-gradient convolution of the same layer,
// dx[p][c] = sum_{tap, o} w[o][c][tap] dy[p - tap][o], i.e. a forward convolution
// with input and output channels swapped and the taps mirrored (tap -> 8 - tap).
__global__ void k_pack_w32(const float* __restrict__ w, __nv_bfloat16* __restrict__ img, int adjoint) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;  // over n * 288
    if (e >= CH * KDIM) return;
    const int n = e / KDIM, k = e % KDIM;
    const int tap = k / CH, c = k % CH;
    const float v = adjoint ? w[(c * CH + n) * 9 + (8 - tap)] : w[(n * CH + c) * 9 + tap];
    const int off = (n >> 3) * SBO + (k >> 3) * CORE_BYTES + (n & 7) * 16 + (k & 7) * 2;
    img[off / 2] = __float2bfloat16(v);
}

// ---------------------------------------------------------------- generic conv (CUDA cores)
// cin, cout in {1, 32}. Forward: y[p][o] = bias[o] + sum w[o][c][tap] x[p + tap][c].
// transposed (backward data): y[p][c] = sum w[o][c][tap] x[p - tap][o] (x = dy, cin = cout of
// the forward layer). Inputs and outputs are FP32 or BF16 (xbf/ybf).
template <int CIN, int COUT>
__global__ void k_conv_generic(const void* __restrict__ x, int xbf, const float* __restrict__ w,
                               const float* __restrict__ bias, const uint8_t* __restrict__ mask,
                               void* __restrict__ y, int ybf, int H, int W, int relu, int transposed) {
    __shared__ float ws[CIN * COUT * 9];
    for (int e = threadIdx.x; e < CIN * COUT * 9; e += blockDim.x) ws[e] = w[e];
    __syncthreads();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= H * W) return;
    const int i = p / W, j = p % W;
    float acc[COUT];
#pragma unroll
    for (int o = 0; o < COUT; ++o) acc[o] = (bias && !transposed) ? bias[o] : 0.0f;
    for (int tap = 0; tap < 9; ++tap) {
        const int di = tap / 3 - 1, dj = tap % 3 - 1;
        const int ii = transposed ? i - di : i + di, jj = transposed ? j - dj : j + dj;
        if (ii < 0 || ii >= H || jj < 0 || jj >= W) continue;
        const size_t q = (size_t)ii * W + jj;
#pragma unroll 4
        for (int c = 0; c < CIN; ++c) {
            const float xv = xbf ? bf2f(reinterpret_cast<const __nv_bfloat16*>(x)[q * CIN + c])
                                 : reinterpret_cast<const float*>(x)[q * CIN + c];
#pragma unroll
            for (int o = 0; o < COUT; ++o) {
                // forward: w[o][c][tap]; transposed: the forward layer had (cin = COUT, cout = CIN)
                const float wv = transposed ? ws[(c * COUT + o) * 9 + tap] : ws[(o * CIN + c) * 9 + tap];
                acc[o] += wv * xv;
            }
        }
    }
    const bool fl = mask ? (mask[p] != 0) : true;
#pragma unroll
    for (int o = 0; o < COUT; ++o) {
        float v = acc[o];
        if (relu) v = fmaxf(v, 0.0f);
        if (!fl) v = 0.0f;
        if (ybf) reinterpret_cast<__nv_bfloat16*>(y)[(size_t)p * COUT + o] = __float2bfloat16(v);
        else reinterpret_cast<float*>(y)[(size_t)p * COUT + o] = v;
    }
}

// Forward 1 -> 32 layer (FP32 input, BF16 output) and 32 -> 1 layer (BF16 input,
// FP32 output): one thread per pixel (128 consecutive pixels per block), the 288
// weights tap-major in shared memory (16-byte vectors over the channels). The
// 32-channel side goes through shared memory with an 80-byte pixel stride (no bank
// conflicts for 16-byte accesses), so that global memory is read and written in
// contiguous 16-byte chunks by consecutive threads. Taps and channels are summed in
// the same order as k_conv_generic, so both give the same bits.
constexpr int FP = 128;      // pixels per block
constexpr int PSTRIDE = 5;   // uint4 per staged pixel (4 used)

__global__ void __launch_bounds__(FP) k_conv_1to32(const float* __restrict__ x, const float* __restrict__ w,
                                                   const float* __restrict__ bias,
                                                   const uint8_t* __restrict__ mask,
                                                   __nv_bfloat16* __restrict__ y, int H, int W, int relu) {
    __shared__ __align__(16) float ws[9 * CH];
    __shared__ uint4 os[FP * PSTRIDE];
    for (int e = threadIdx.x; e < CH * 9; e += blockDim.x) ws[(e % 9) * CH + e / 9] = w[e];
    pdl_trigger();
    pdl_wait();
    __syncthreads();
    const long long n = (long long)H * W;
    const long long p0 = (long long)blockIdx.x * FP;
    const long long p = p0 + threadIdx.x;
    if (p < n) {
        const int i = (int)(p / W), j = (int)(p - (long long)i * W);
        float acc[CH];
#pragma unroll
        for (int o = 0; o < CH; ++o) acc[o] = bias ? bias[o] : 0.0f;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
            const int ii = i + tap / 3 - 1, jj = j + tap % 3 - 1;
            if (ii < 0 || ii >= H || jj < 0 || jj >= W) continue;
            const float xv = x[(size_t)ii * W + jj];
#pragma unroll
            for (int o = 0; o < CH; ++o) acc[o] += ws[tap * CH + o] * xv;
        }
        const bool fl = mask ? (mask[p] != 0) : true;
        __align__(16) __nv_bfloat16 out[CH];
#pragma unroll
        for (int o = 0; o < CH; ++o) {
            float v = acc[o];
            if (relu) v = fmaxf(v, 0.0f);
            out[o] = __float2bfloat16(fl ? v : 0.0f);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) os[threadIdx.x * PSTRIDE + q] = reinterpret_cast<const uint4*>(out)[q];
    }
    __syncthreads();
    uint4* y4 = reinterpret_cast<uint4*>(y);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int q = threadIdx.x + k * FP;
        const int px = q >> 2, c = q & 3;
        if (p0 + px < n) y4[(p0 + px) * 4 + c] = os[px * PSTRIDE + c];
    }
}

__global__ void __launch_bounds__(FP) k_conv_32to1(const __nv_bfloat16* __restrict__ x,
                                                   const float* __restrict__ w, const float* __restrict__ bias,
                                                   const uint8_t* __restrict__ mask, float* __restrict__ y, int H,
                                                   int W, int relu) {
    constexpr int SP = FP + 2;             // staged pixels per tap row
    constexpr int SQ = 3 * SP * 4;         // staged 16-byte chunks (1560)
    constexpr int SPER = (SQ + FP - 1) / FP;
    __shared__ __align__(16) float ws[9 * CH];
    __shared__ uint4 xs[3 * SP * PSTRIDE];
    for (int e = threadIdx.x; e < CH * 9; e += blockDim.x) ws[(e % 9) * CH + e / 9] = w[e];
    pdl_trigger();
    pdl_wait();
    const long long n = (long long)H * W;
    const long long p0 = (long long)blockIdx.x * FP;
    // tap row d (di = d - 1) holds pixels p0 + di*W - 1 .. p0 + di*W + FP; taps that
    // leave the grid are skipped below, so the clamp to [0, n) only avoids reading
    // outside the array
    const uint4* x4 = reinterpret_cast<const uint4*>(x);
    {
        uint4 v[SPER];
#pragma unroll
        for (int k = 0; k < SPER; ++k) {
            const int q = threadIdx.x + k * FP;
            const int d = q / (SP * 4), rem = q - d * (SP * 4);
            const long long g = p0 + (long long)(d - 1) * W - 1 + (rem >> 2);
            v[k] = make_uint4(0u, 0u, 0u, 0u);
            if (q < SQ && g >= 0 && g < n) v[k] = x4[g * 4 + (rem & 3)];
        }
#pragma unroll
        for (int k = 0; k < SPER; ++k) {
            const int q = threadIdx.x + k * FP;
            const int d = q / (SP * 4), rem = q - d * (SP * 4);
            if (q < SQ) xs[(d * SP + (rem >> 2)) * PSTRIDE + (rem & 3)] = v[k];
        }
    }
    __syncthreads();
    const long long p = p0 + threadIdx.x;
    if (p >= n) return;
    const int i = (int)(p / W), j = (int)(p - (long long)i * W);
    float acc = bias ? bias[0] : 0.0f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
        const int di = tap / 3 - 1, dj = tap % 3 - 1;
        const int ii = i + di, jj = j + dj;
        if (ii < 0 || ii >= H || jj < 0 || jj >= W) continue;
        const uint4* src = xs + ((di + 1) * SP + threadIdx.x + dj + 1) * PSTRIDE;
        uint4 v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = src[q];
        const __nv_bfloat16* xv = reinterpret_cast<const __nv_bfloat16*>(v);
#pragma unroll
        for (int c = 0; c < CH; ++c) acc += ws[tap * CH + c] * bf2f(xv[c]);
    }
    if (relu) acc = fmaxf(acc, 0.0f);
    const bool fl = mask ? (mask[p] != 0) : true;
    y[p] = fl ? acc : 0.0f;
}

// ---------------------------------------------------------------- pooling, upsampling
// coarse (Hc, Wc) = (ceil(H/2), ceil(W/2)): mean of the in-range children; one thread
// per 8 channels of a coarse pixel (one 16-byte vector)
__global__ void k_pool2(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ y, int H, int W) {
    pdl_trigger();
    pdl_wait();
    const int Hc = (H + 1) / 2, Wc = (W + 1) / 2;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Hc * Wc * (CH / 8)) return;
    const int c8 = e & 3, q = e >> 2;
    const int ic = q / Wc, jc = q - (q / Wc) * Wc;
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int n = 0;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            const int i = 2 * ic + a, j = 2 * jc + b;
            if (i < H && j < W) {
                const uint4 v = reinterpret_cast<const uint4*>(x + ((size_t)i * W + j) * CH)[c8];
                const __nv_bfloat16* h = reinterpret_cast<const __nv_bfloat16*>(&v);
#pragma unroll
                for (int k = 0; k < 8; ++k) s[k] += bf2f(h[k]);
                ++n;
            }
        }
    __align__(16) __nv_bfloat16 out[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) out[k] = __float2bfloat16(s[k] / (float)n);
    reinterpret_cast<uint4*>(y)[e] = *reinterpret_cast<const uint4*>(out);
}

// y[p] = coarse[parent(p)] + skip[p]; one thread per 8 channels of a pixel
__global__ void k_upadd(const __nv_bfloat16* __restrict__ coarse, const __nv_bfloat16* __restrict__ skip,
                        __nv_bfloat16* __restrict__ y, int H, int W, float scale) {
    pdl_trigger();
    pdl_wait();
    const int Wc = (W + 1) / 2;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= H * W * (CH / 8)) return;
    const int c8 = e & 3, p = e >> 2;
    const int i = p / W, j = p - (p / W) * W;
    const uint4 cv = reinterpret_cast<const uint4*>(coarse + ((size_t)(i / 2) * Wc + j / 2) * CH)[c8];
    const uint4 sv = reinterpret_cast<const uint4*>(skip)[e];
    const __nv_bfloat16* ch = reinterpret_cast<const __nv_bfloat16*>(&cv);
    const __nv_bfloat16* sh = reinterpret_cast<const __nv_bfloat16*>(&sv);
    __align__(16) __nv_bfloat16 out[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) out[k] = __float2bfloat16(scale * bf2f(ch[k]) + bf2f(sh[k]));
    reinterpret_cast<uint4*>(y)[e] = *reinterpret_cast<const uint4*>(out);
}

// coarse mask: any child fluid
__global__ void k_pool_mask(const uint8_t* __restrict__ m, uint8_t* __restrict__ mc, int H, int W) {
    const int Hc = (H + 1) / 2, Wc = (W + 1) / 2;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Hc * Wc) return;
    const int ic = q / Wc, jc = q % Wc;
    uint8_t v = 0;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            const int i = 2 * ic + a, j = 2 * jc + b;
            if (i < H && j < W) v |= m[(size_t)i * W + j];
        }
    mc[q] = v ? 1 : 0;
}

// ---------------------------------------------------------------- backward helpers
// g = dy * (y > 0) * mask  (ReLU layers) in FP32
__global__ void k_relu_bwd(const float* __restrict__ dy, const __nv_bfloat16* __restrict__ y,
                           const uint8_t* __restrict__ mask, float* __restrict__ g, int npix, int ch,
                           int relu) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= npix * ch) return;
    const int p = e / ch;
    float v = dy[e];
    if (relu && !(bf2f(y[e]) > 0.0f)) v = 0.0f;
    if (mask && !mask[p]) v = 0.0f;
    g[e] = v;
}

// dcoarse[q] = sum over children of dfine[p]  (upsample backward), dfine given FP32
__global__ void k_upadd_bwd(const float* __restrict__ dy, float* __restrict__ dcoarse, int H, int W, float scale) {
    const int Hc = (H + 1) / 2, Wc = (W + 1) / 2;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Hc * Wc * CH) return;
    const int c = e % CH, q = e / CH;
    const int ic = q / Wc, jc = q % Wc;
    float s = 0.0f;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            const int i = 2 * ic + a, j = 2 * jc + b;
            if (i < H && j < W) s += dy[((size_t)i * W + j) * CH + c];
        }
    dcoarse[e] = scale * s;
}

// dfine[p] += dcoarse[parent(p)] / n_children(parent)   (pool backward, accumulating)
__global__ void k_pool_bwd(const float* __restrict__ dcoarse, float* __restrict__ dfine, int H, int W) {
    const int Wc = (W + 1) / 2;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= H * W * CH) return;
    const int c = e % CH, p = e / CH;
    const int i = p / W, j = p % W;
    const int ic = i / 2, jc = j / 2;
    const int na = (2 * ic + 1 < H) ? 2 : 1, nb = (2 * jc + 1 < W) ? 2 : 1;
    dfine[e] += dcoarse[((size_t)ic * Wc + jc) * CH + c] / (float)(na * nb);
}

// Weight gradient of a 3x3 conv: dw[o][c][tap] = sum_p g[p][o] x[p + tap][c], db[o] = sum_p g[p][o].
// Each block reduces a contiguous pixel range into partial sums (deterministic order);
// k_reduce_partials adds the blocks in index order.
template <int CIN, int COUT>
__global__ void k_conv_dw(const void* __restrict__ x, int xbf, const float* __restrict__ g, int H, int W,
                          int pix_per_block, float* __restrict__ partial) {
    constexpr int NW = COUT * CIN * 9;
    const int p0 = blockIdx.x * pix_per_block;
    const int p1 = min(H * W, p0 + pix_per_block);
    for (int e = threadIdx.x; e < NW + COUT; e += blockDim.x) {
        float s = 0.0f;
        if (e < NW) {
            const int o = e / (CIN * 9), c = (e / 9) % CIN, tap = e % 9;
            const int di = tap / 3 - 1, dj = tap % 3 - 1;
            for (int p = p0; p < p1; ++p) {
                const int i = p / W, j = p % W;
                const int ii = i + di, jj = j + dj;
                if (ii < 0 || ii >= H || jj < 0 || jj >= W) continue;
                const size_t q = (size_t)ii * W + jj;
                const float xv = xbf ? bf2f(reinterpret_cast<const __nv_bfloat16*>(x)[q * CIN + c])
                                     : reinterpret_cast<const float*>(x)[q * CIN + c];
                s += g[(size_t)p * COUT + o] * xv;
            }
        } else {
            const int o = e - NW;
            for (int p = p0; p < p1; ++p) s += g[(size_t)p * COUT + o];
        }
        partial[(size_t)blockIdx.x * (NW + COUT) + e] = s;
    }
}

__global__ void k_reduce_partials(const float* __restrict__ partial, int nblocks, int n, float* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    float s = 0.0f;
    for (int b = 0; b < nblocks; ++b) s += partial[(size_t)b * n + e];
    out[e] = s;
}

// ---------------------------------------------------------------- host launchers
namespace {
inline int cdiv(long long a, int b) { return (int)((a + b - 1) / b); }
}  // namespace

size_t conv32_smem_bytes(int rows) { return (size_t)B_BYTES + x_bytes(rows); }

template <int ROWS>
static cudaError_t conv32_launch(const __nv_bfloat16* x, const __nv_bfloat16* wpack, const float* bias,
                                 const __nv_bfloat16* skip, const uint8_t* mask, __nv_bfloat16* y, int H, int W,
                                 int relu, int* err, cudaStream_t s) {
    // the shared-memory opt-in is a per-device attribute of the kernel
    constexpr int kMaxDev = 64;
    static bool configured[kMaxDev];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
    if (!configured[dev]) {
        e = cudaFuncSetAttribute(k_conv32_tc<ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)conv32_smem_bytes(ROWS));
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    dim3 grid(cdiv(W, TM), cdiv(H, ROWS));
    return launch_pdl(k_conv32_tc<ROWS>, grid, dim3(NT), conv32_smem_bytes(ROWS), s, x,
                      reinterpret_cast<const uint4*>(wpack), bias, skip, mask, y, H, W, relu, err);
}

// Rows per CTA: two where that still leaves about six CTAs per SM (two waves at the
// four CTAs of 52 KB that fit), else one, so that the small levels of the network
// spread over the SMs. (Four rows per CTA halve the halo reads but fit only three CTAs
// per SM and measured slower: 36.4 against 32.5 us at 1024 x 512.)
cudaError_t conv32_tc(const __nv_bfloat16* x, const __nv_bfloat16* wpack, const float* bias,
                      const __nv_bfloat16* skip, const uint8_t* mask, __nv_bfloat16* y, int H, int W, int relu,
                      int* err, cudaStream_t s) {
    const long long segs = cdiv(W, TM);
    if (segs * cdiv(H, 2) >= 6 * 148) return conv32_launch<2>(x, wpack, bias, skip, mask, y, H, W, relu, err, s);
    return conv32_launch<1>(x, wpack, bias, skip, mask, y, H, W, relu, err, s);
}

cudaError_t pack_w32(const float* w, __nv_bfloat16* img, int adjoint, cudaStream_t s) {
    k_pack_w32<<<cdiv(CH * KDIM, 256), 256, 0, s>>>(w, img, adjoint);
    return cudaGetLastError();
}

cudaError_t conv_generic(int cin, int cout, const void* x, int xbf, const float* w, const float* bias,
                         const uint8_t* mask, void* y, int ybf, int H, int W, int relu, int transposed,
                         cudaStream_t s) {
    const int n = H * W;
    const int blk = 128;
    if (!transposed && cin == 1 && cout == 32 && !xbf && ybf) {
        return launch_pdl(k_conv_1to32, dim3(cdiv(n, FP)), dim3(FP), 0, s, static_cast<const float*>(x), w, bias,
                          mask, static_cast<__nv_bfloat16*>(y), H, W, relu);
    }
    if (!transposed && cin == 32 && cout == 1 && xbf && !ybf) {
        return launch_pdl(k_conv_32to1, dim3(cdiv(n, FP)), dim3(FP), 0, s, static_cast<const __nv_bfloat16*>(x), w,
                          bias, mask, static_cast<float*>(y), H, W, relu);
    }
    if (cin == 1 && cout == 32)
        k_conv_generic<1, 32><<<cdiv(n, blk), blk, 0, s>>>(x, xbf, w, bias, mask, y, ybf, H, W, relu, transposed);
    else if (cin == 32 && cout == 1)
        k_conv_generic<32, 1><<<cdiv(n, blk), blk, 0, s>>>(x, xbf, w, bias, mask, y, ybf, H, W, relu, transposed);
    else if (cin == 32 && cout == 32)
        k_conv_generic<32, 32><<<cdiv(n, blk), blk, 0, s>>>(x, xbf, w, bias, mask, y, ybf, H, W, relu, transposed);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t pool2(const __nv_bfloat16* x, __nv_bfloat16* y, int H, int W, cudaStream_t s) {
    const int n = ((H + 1) / 2) * ((W + 1) / 2) * (CH / 8);
    cudaError_t e = launch_pdl(k_pool2, dim3(cdiv(n, 256)), dim3(256), 0, s, x, y, H, W);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t pool_mask(const uint8_t* m, uint8_t* mc, int H, int W, cudaStream_t s) {
    const int n = ((H + 1) / 2) * ((W + 1) / 2);
    k_pool_mask<<<cdiv(n, 256), 256, 0, s>>>(m, mc, H, W);
    return cudaGetLastError();
}

cudaError_t upadd(const __nv_bfloat16* coarse, const __nv_bfloat16* skip, __nv_bfloat16* y, int H, int W, float scale,
                  cudaStream_t s) {
    cudaError_t e = launch_pdl(k_upadd, dim3(cdiv((long long)H * W * (CH / 8), 256)), dim3(256), 0, s, coarse, skip,
                               y, H, W, scale);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t relu_bwd(const float* dy, const __nv_bfloat16* y, const uint8_t* mask, float* g, int npix, int ch,
                     int relu, cudaStream_t s) {
    k_relu_bwd<<<cdiv((long long)npix * ch, 256), 256, 0, s>>>(dy, y, mask, g, npix, ch, relu);
    return cudaGetLastError();
}

cudaError_t upadd_bwd(const float* dy, float* dcoarse, int H, int W, float scale, cudaStream_t s) {
    const int n = ((H + 1) / 2) * ((W + 1) / 2) * CH;
    k_upadd_bwd<<<cdiv(n, 256), 256, 0, s>>>(dy, dcoarse, H, W, scale);
    return cudaGetLastError();
}

cudaError_t pool_bwd(const float* dcoarse, float* dfine, int H, int W, cudaStream_t s) {
    k_pool_bwd<<<cdiv((long long)H * W * CH, 256), 256, 0, s>>>(dcoarse, dfine, H, W);
    return cudaGetLastError();
}

size_t conv_dw_partial_floats(int cin, int cout, int H, int W, int pix_per_block) {
    return (size_t)cdiv((long long)H * W, pix_per_block) * (cin * cout * 9 + cout);
}

cudaError_t conv_dw(int cin, int cout, const void* x, int xbf, const float* g, int H, int W, int pix_per_block,
                    float* partial, float* out, cudaStream_t s) {
    const int nb = cdiv((long long)H * W, pix_per_block);
    const int n = cin * cout * 9 + cout;
    if (cin == 1 && cout == 32)
        k_conv_dw<1, 32><<<nb, 256, 0, s>>>(x, xbf, g, H, W, pix_per_block, partial);
    else if (cin == 32 && cout == 1)
        k_conv_dw<32, 1><<<nb, 256, 0, s>>>(x, xbf, g, H, W, pix_per_block, partial);
    else if (cin == 32 && cout == 32)
        k_conv_dw<32, 32><<<nb, 256, 0, s>>>(x, xbf, g, H, W, pix_per_block, partial);
    else
        return cudaErrorInvalidValue;
    k_reduce_partials<<<cdiv(n, 256), 256, 0, s>>>(partial, nb, n, out);
    return cudaGetLastError();
}

}  // namespace lpc
}  // namespace cfd
