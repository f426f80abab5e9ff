// Learned kernel-predicting denoiser (include/ntrace_denoise.h) on the sm_100a tensor cores.
//
// The network's matrix products run in one GEMM kernel built on tcgen05: operand tiles are copied
// global -> shared with cp.async in 16-byte chunks, into the canonical layouts without swizzle (8 x
// 16-byte core matrices), K-major for row-major operands and MN-major for transposed ones, two stages
// deep; one elected thread issues tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulator in tensor
// memory) and commits to the stage's mbarrier, and the epilogue reads the accumulator back with
// tcgen05.ld and applies a fused bias / ReLU / mask / store or atomic reduction.  The forward pass,
// the backward data products and the weight gradients (a reduction over pixels, split across CTAs)
// all use the same kernel.  The rest (features, softmax filters, loss, bias sums, Adam) are plain
// CUDA-core kernels.
#include "ntrace.h"
#include "ntrace_denoise.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace ntrace
{
int report_error(int code, const std::string& message);
}

namespace
{
constexpr int HID = 64;
constexpr int TAPS = 9;
constexpr int RADIUS = 4;
constexpr int MAX_AXES = 5;
// Guides of the cross-bilateral filter: normal, depth and colour distance between a pixel and a tap.
// The network predicts, per screen axis, one log-bandwidth o per guide; the guide's weight on the
// tap logits is GUIDE_SCALE x exp(min(o, BANDWIDTH_MAX)).
constexpr int GUIDES = 3;
constexpr float BANDWIDTH_MAX = 20.0f;
// floats per pixel in the base-feature buffer: n + 10 of them used (n <= 6), the rest zero, so that a
// pixel's features are four aligned 16-byte words
constexpr int BASE_STRIDE = 16;

// ------------------------------------------------------------------------------------------------
// tcgen05 GEMM

constexpr int GM = 128;      // rows per CTA: the MMA's M
constexpr int GK = 64;       // K per shared-memory stage: 4 MMAs of K = 16
constexpr int GTHREADS = 128;
constexpr int SM_SMEM = 233472;  // shared memory per SM (228 KB)

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
        return (uint32_t)__cvta_generic_to_shared(p);
}

// one 16-byte global -> shared copy that does not pass through registers (cp.async, L2 only)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}

// byte offset of element (r, k) of a GK-wide K-major tile: core matrices of 8 rows x 16 bytes, the
// K direction first (leading byte offset 128), then the next 8 rows (stride byte offset GK / 8 x 128)
__device__ __forceinline__ uint32_t tile_off(int r, int k)
{
        return (uint32_t)((r >> 3) * (GK / 8 * 128) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start, leading and stride byte offsets (>> 4), version 1, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
        return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
               ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, N >> 3, M >> 4
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n)
{
        return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// Bounds of the GEMM's completion waits.  withhold = 1 is the failure-detection self-test: the MMAs
// and their commit are not issued, so nothing ever arrives on the barrier and every wait runs out.
struct GemmCtl
{
        unsigned long long wait_ns = 1000000000ull;  // about a second
        int withhold = 0;
};

__device__ __forceinline__ unsigned long long global_ns()
{
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        return t;
}

// Waits for the mbarrier phase `parity` to complete; gives up after limit_ns nanoseconds.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity, unsigned long long limit_ns)
{
        const uint32_t addr = smem_u32(bar);
        const unsigned long long t0 = global_ns();
        while (true)
        {
                uint32_t done;
                asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                        "selp.u32 %0, 1, 0, p;\n\t}"
                        : "=r"(done)
                        : "r"(addr), "r"(parity)
                        : "memory");
                if (done)
                {
                        return true;
                }
                if (global_ns() - t0 > limit_ns)
                {
                        return false;
                }
        }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
        uint32_t r[16];
        asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 16; ++j)
        {
                v[j] = __uint_as_float(r[j]);
        }
}

// byte offset of element (r, k) of a GK-wide MN-major tile: core matrices of 8 k x 16 bytes (eight
// consecutive rows), k fastest (leading byte offset 128 between groups of eight k), then the next
// eight rows (stride byte offset GK x 16)
__device__ __forceinline__ uint32_t tile_off_mn(int r, int k)
{
        return (uint32_t)((r >> 3) * (GK * 16) + k * 16 + (r & 7) * 2);
}

// Copies the GK-wide slice [kc, kc + GK) of rows [r0, r0 + rows) of an operand into a shared-memory
// tile with cp.async, one 16-byte chunk per copy (every chunk of the tile in flight at once); chunks
// outside the operand (row >= rmax or k >= ke) are zeroed.
//  * K-major operands (L::MN_MAJOR false): a chunk is eight consecutive k of one row, and eight
//    consecutive rows go fastest, so that a quarter warp fills one 128-byte block of core-matrix rows
//    (no bank conflicts).
//  * MN-major operands (the transpose of a row-major matrix): a chunk is eight consecutive rows at one
//    k; two threads take sixteen rows (one 32-byte sector), and consecutive pairs consecutive k, so
//    that a warp's 32 chunks spread over all 32 banks.
template <class L>
__device__ __forceinline__ void fill_tile(const L& ld, unsigned char* s, int rows, int r0, int rmax, int kc, int ke)
{
        if constexpr (!L::MN_MAJOR)
        {
                for (int idx = threadIdx.x; idx < rows * (GK / 8); idx += GTHREADS)
                {
                        const int r = (idx & 7) | ((idx / (8 * (GK / 8))) << 3);
                        const int k8 = ((idx >> 3) % (GK / 8)) * 8;
                        unsigned char* dst = s + tile_off(r, k8);
                        if (r0 + r < rmax && kc + k8 < ke)
                        {
                                cp_async16(dst, ld.addr8(r0 + r, kc + k8));
                        }
                        else
                        {
                                *reinterpret_cast<uint4*>(dst) = make_uint4(0u, 0u, 0u, 0u);
                        }
                }
        }
        else
        {
                for (int idx = threadIdx.x; idx < (rows / 8) * GK; idx += GTHREADS)
                {
                        const int k = (idx >> 1) % GK;
                        const int r = ((idx >> 1) / GK) * 16 + (idx & 1) * 8;
                        unsigned char* dst = s + tile_off_mn(r, k);
                        if (r0 + r < rmax && kc + k < ke)
                        {
                                cp_async16(dst, ld.addr8(r0 + r, kc + k));
                        }
                        else
                        {
                                *reinterpret_cast<uint4*>(dst) = make_uint4(0u, 0u, 0u, 0u);
                        }
                }
        }
}

// C[M x N] = sum_k A(m, k) B(n, k) over k in this CTA's K range [blockIdx.y * k_per_cta, ...).
// LA / LB: operand loaders (LoadRows: K-major, LoadCols: MN-major); EPI: epilogue (row, first column,
// 16 values).  N: multiple of 16, at most 256; ncols: tensor-memory columns (power of two >= max(32, N)).
//
// Two shared-memory stages: while the tensor core multiplies chunk i out of one stage, the threads
// copy chunk i + 1 into the other, once the MMAs of chunk i - 1 (which read it) have completed.  Each
// stage has its own mbarrier, to which the MMA thread commits; chunk j's commit completes phase j / 2
// of barrier j % 2.
template <class LA, class LB, class EPI>
__global__ void __launch_bounds__(GTHREADS) k_gemm(const LA la, const LB lb, const EPI epi, int M, int N, int K,
                                                   int k_per_cta, uint32_t ncols, int* err, const GemmCtl ctl)
{
        extern __shared__ __align__(1024) unsigned char g_smem[];
        __shared__ __align__(8) unsigned long long s_bar[2];
        __shared__ uint32_t s_tmem;
        const int tid = threadIdx.x;
        const int warp = tid >> 5;
        const int lane = tid & 31;
        const int m0 = blockIdx.x * GM;
        const int kb = blockIdx.y * k_per_cta;
        const int ke = min(K, kb + k_per_cta);
        const int stage_bytes = (GM + N) * GK * 2;  // A then B; a multiple of 2048 bytes
        const int nk = ke > kb ? (ke - kb + GK - 1) / GK : 0;

        if (warp == 0)
        {
                asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                             "r"(ncols)
                             : "memory");
                asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        if (tid == 0)
        {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_bar[0])) : "memory");
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_bar[1])) : "memory");
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tmem = s_tmem;
        const uint32_t idesc = umma_idesc_bf16(GM, N) | (LA::MN_MAJOR ? 1u << 15 : 0u) | (LB::MN_MAJOR ? 1u << 16 : 0u);
        // both layouts: 128 bytes between groups of eight k, GK x 16 bytes between groups of eight rows
        const uint32_t lbo = 128, sbo = GK * 16;

        if (nk > 0)
        {
                fill_tile(la, g_smem, GM, m0, M, kb, ke);
                fill_tile(lb, g_smem + GM * GK * 2, N, 0, N, kb, ke);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        bool ok = true;
        int issued = 0;  // chunks whose MMAs have been committed
        for (int i = 0; i < nk; ++i)
        {
                const int b = i & 1;
                unsigned char* sA = g_smem + b * stage_bytes;
                unsigned char* sB = sA + GM * GK * 2;
                asm volatile("cp.async.wait_group 0;" ::: "memory");
                // the tensor core reads shared memory through the async proxy
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncthreads();
                if (tid == 0 && !ctl.withhold)
                {
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                        for (int s = 0; s < GK / 16; ++s)
                        {
                                const uint64_t da = umma_desc(smem_u32(sA) + s * 256, lbo, sbo);
                                const uint64_t db = umma_desc(smem_u32(sB) + s * 256, lbo, sbo);
                                const uint32_t accumulate = (i > 0 || s > 0) ? 1u : 0u;
                                asm volatile(
                                        "{\n\t.reg .pred p;\n\t"
                                        "setp.ne.b32 p, %4, 0;\n\t"
                                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                                        "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
                                        : "memory");
                        }
                        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                             smem_u32(&s_bar[b]))
                                     : "memory");
                }
                issued = i + 1;
                if (i + 1 < nk)
                {
                        if (i >= 1)
                        {
                                // the other stage was read by chunk i - 1's MMAs
                                const bool done = mbar_wait(&s_bar[b ^ 1], (uint32_t)(((i - 1) >> 1) & 1), ctl.wait_ns);
                                ok = __syncthreads_and(done) != 0;
                                if (!ok)
                                {
                                        break;
                                }
                        }
                        unsigned char* nA = g_smem + (b ^ 1) * stage_bytes;
                        const int kn = kb + (i + 1) * GK;
                        fill_tile(la, nA, GM, m0, M, kn, ke);
                        fill_tile(lb, nA + GM * GK * 2, N, 0, N, kn, ke);
                        asm volatile("cp.async.commit_group;" ::: "memory");
                }
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        if (issued > 0)
        {
                // the last chunk's MMAs (and with them every earlier one) before the accumulator is read
                // or its columns are given back; after a wait that ran out, once more (bounded)
                const int j = issued - 1;
                const bool done = mbar_wait(&s_bar[j & 1], (uint32_t)((j >> 1) & 1), ctl.wait_ns);
                ok = (__syncthreads_and(done) != 0) && ok;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (ok && issued > 0)
        {
                const int row = m0 + warp * 32 + lane;
                for (int c = 0; c < N; c += 16)
                {
                        float v[16];
                        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
                        if (row < M)
                        {
                                epi(row, c, v);
                        }
                }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (warp == 0)
        {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
        }
        if (!ok && tid == 0 && err)
        {
                atomicOr(err, 1);
        }
}

// ---- operand loaders ----

// A(r, k) = p[r * ld + k], BF16, K-major: eight consecutive k (k a multiple of 8) are one 16-byte
// chunk, which needs p 16-byte aligned and ld a multiple of 8
struct LoadRows
{
        static constexpr bool MN_MAJOR = false;
        const __nv_bfloat16* p;
        int ld;
        __device__ __forceinline__ const void* addr8(int r, int k) const
        {
                return p + (size_t)r * ld + k;
        }
        bool chunks_ok() const
        {
                return ((uintptr_t)p & 15u) == 0 && ld % 8 == 0;
        }
};

// A(r, k) = p[k * ld + r], BF16 (the transpose of a row-major matrix), MN-major: eight consecutive
// rows (r a multiple of 8) are one 16-byte chunk, which needs p 16-byte aligned and ld a multiple of 8
struct LoadCols
{
        static constexpr bool MN_MAJOR = true;
        const __nv_bfloat16* p;
        int ld;
        __device__ __forceinline__ const void* addr8(int r, int k) const
        {
                return p + (size_t)k * ld + r;
        }
        bool chunks_ok() const
        {
                return ((uintptr_t)p & 15u) == 0 && ld % 8 == 0;
        }
};

// The screen and the network's feature stencil.
struct Stencil
{
        int axes;                   // n - 1
        int size[MAX_AXES];
        long long stride[MAX_AXES];
        int nf;                     // base features per pixel
        int stencil_features;       // nf x (2 axes + 1)
        int features;               // stencil_features + 1: the noise level of the input last
        float noise_level;          // 1 / sqrt(samples per pixel)

        // pixel at offset d along axis a from p, clamped to the screen
        __device__ __forceinline__ long long neighbour(long long p, int a, int d) const
        {
                const int x = (int)((p / stride[a]) % size[a]);
                const int y = min(max(x + d, 0), size[a] - 1);
                return p + (long long)(y - x) * stride[a];
        }
};

// Source pixel of stencil slot q of pixel p (slot 0 the pixel, 2a + 1 / 2a + 2 its -1 / +1 neighbour
// along axis a, clamped), in 32-bit arithmetic (at most 2^30 pixels)
__device__ __forceinline__ unsigned slot_source(const Stencil& st, unsigned p, int q)
{
        if (q <= 0 || q > 2 * st.axes)
        {
                return p;
        }
        const int a = (q - 1) >> 1;
        const unsigned stride = (unsigned)st.stride[a];
        const int x = (int)((p / stride) % (unsigned)st.size[a]);
        const int y = min(max(x + ((q & 1) ? -1 : 1), 0), st.size[a] - 1);
        return (unsigned)((int)p + (y - x) * (int)stride);
}

// The network's input matrix X (pixels x padded features, BF16), written once per input: thread
// (pixel, chunk) forms eight consecutive features and stores them as one 16-byte word, so that
// consecutive threads write consecutive chunks of a row.  A chunk spans at most two stencil slots
// (nf > 8), so the thread walks the slots incrementally: one source pixel per slot it touches.
__global__ void k_features(long long P, __grid_constant__ const Stencil st, int Fp, const float* __restrict__ base, __nv_bfloat16* __restrict__ X)
{
        const int chunks = Fp / 8;
        const long long total = P * chunks;
        const int nf = st.nf;
        const int S = 2 * st.axes + 1;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        {
                const unsigned p = (unsigned)(i / chunks);
                const int c = (int)(i - (long long)p * chunks);
                int q = (c * 8) / nf;
                int f = c * 8 - q * nf;
                unsigned src = slot_source(st, p, q);
                __align__(16) __nv_bfloat16 v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j)
                {
                        float x = 0.0f;
                        if (q < S)
                        {
                                x = __ldg(base + (size_t)src * BASE_STRIDE + f);
                        }
                        else if (q == S && f == 0)
                        {
                                x = st.noise_level;
                        }
                        v[j] = __float2bfloat16_rn(x);
                        if (++f == nf)
                        {
                                f = 0;
                                ++q;
                                src = slot_source(st, p, q);
                        }
                }
                *reinterpret_cast<uint4*>(X + (size_t)p * Fp + c * 8) = *reinterpret_cast<const uint4*>(v);
        }
}

// ---- epilogues ----

struct EpiStoreF32
{
        float* out;
        int ld;
        __device__ __forceinline__ void operator()(int row, int c0, const float* v) const
        {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                        out[(size_t)row * ld + c0 + j] = v[j];
                }
        }
};

// The epilogues below store a row's 16 columns as 16-byte words: out 16-byte aligned and ld a
// multiple of 16 (every matrix they write has 64 or outputs_padded columns).
struct EpiBiasF32
{
        const float* bias;
        float* out;
        int ld;
        __device__ __forceinline__ void operator()(int row, int c0, const float* v) const
        {
                float4* o = reinterpret_cast<float4*>(out + (size_t)row * ld + c0);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                        o[j] = make_float4(v[4 * j] + bias[c0 + 4 * j], v[4 * j + 1] + bias[c0 + 4 * j + 1],
                                           v[4 * j + 2] + bias[c0 + 4 * j + 2], v[4 * j + 3] + bias[c0 + 4 * j + 3]);
                }
        }
};

struct EpiBiasReluBF16
{
        const float* bias;
        __nv_bfloat16* out;
        int ld;
        __device__ __forceinline__ void operator()(int row, int c0, const float* v) const
        {
                __align__(16) __nv_bfloat16 h[16];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                        h[j] = __float2bfloat16_rn(fmaxf(v[j] + bias[c0 + j], 0.0f));
                }
                uint4* o = reinterpret_cast<uint4*>(out + (size_t)row * ld + c0);
                o[0] = reinterpret_cast<const uint4*>(h)[0];
                o[1] = reinterpret_cast<const uint4*>(h)[1];
        }
};

// backward through ReLU: keep the gradient where the layer's output was positive
struct EpiMaskBF16
{
        const __nv_bfloat16* act;
        __nv_bfloat16* out;
        int ld;
        __device__ __forceinline__ void operator()(int row, int c0, const float* v) const
        {
                __align__(16) __nv_bfloat16 a[16];
                __align__(16) __nv_bfloat16 h[16];
                const uint4* pa = reinterpret_cast<const uint4*>(act + (size_t)row * ld + c0);
                reinterpret_cast<uint4*>(a)[0] = pa[0];
                reinterpret_cast<uint4*>(a)[1] = pa[1];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                        h[j] = __float2bfloat16_rn(__bfloat162float(a[j]) > 0.0f ? v[j] : 0.0f);
                }
                uint4* o = reinterpret_cast<uint4*>(out + (size_t)row * ld + c0);
                o[0] = reinterpret_cast<const uint4*>(h)[0];
                o[1] = reinterpret_cast<const uint4*>(h)[1];
        }
};

// split-K partial sums added into an FP32 matrix
struct EpiAtomicF32
{
        float* out;
        int ld;
        int ncols;
        __device__ __forceinline__ void operator()(int row, int c0, const float* v) const
        {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                        if (c0 + j < ncols)
                        {
                                atomicAdd(out + (size_t)row * ld + c0 + j, v[j]);
                        }
                }
        }
};

uint32_t tmem_cols(int n)
{
        uint32_t c = 32;
        while ((int)c < n)
        {
                c <<= 1;
        }
        return c;
}

template <class LA, class LB, class EPI>
cudaError_t gemm(const LA& la, const LB& lb, const EPI& epi, int M, int N, int K, int k_per_cta, int* err,
                 cudaStream_t st, const GemmCtl ctl = GemmCtl{})
{
        if (M <= 0 || K <= 0)
        {
                return cudaSuccess;
        }
        if (N <= 0 || N % 16 != 0 || N > 256)
        {
                return cudaErrorInvalidValue;
        }
        // 16-byte operand chunks: a K-major chunk lies wholly inside or outside a CTA's K range when K
        // is a multiple of 8, an MN-major one inside or outside the rows when M (N) is
        if (!la.chunks_ok() || !lb.chunks_ok() || (!LA::MN_MAJOR && K % 8 != 0) || (!LB::MN_MAJOR && K % 8 != 0) ||
            (LA::MN_MAJOR && M % 8 != 0))
        {
                return cudaErrorInvalidValue;
        }
        const uint32_t ncols = tmem_cols(N);
        // at most 512 / ncols CTAs share an SM's tensor memory: ask for enough shared memory that no
        // more are resident (an allocation then never waits)
        const int per_sm = 512 / (int)ncols;
        const size_t need = 2 * (size_t)(GM + N) * GK * 2;  // two stages
        const size_t smem = std::max(need, (size_t)(SM_SMEM / (per_sm + 1) + 1024));
        cudaError_t e = cudaFuncSetAttribute(k_gemm<LA, LB, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
        {
                return e;
        }
        const int kpc = k_per_cta > 0 ? (k_per_cta + GK - 1) / GK * GK : (K + GK - 1) / GK * GK;
        dim3 grid((unsigned)((M + GM - 1) / GM), (unsigned)((K + kpc - 1) / kpc));
        k_gemm<LA, LB, EPI><<<grid, GTHREADS, smem, st>>>(la, lb, epi, M, N, K, kpc, ncols, err, ctl);
        return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// CUDA-core kernels

constexpr int TB = 256;

unsigned blocks_for(long long n)
{
        return (unsigned)std::min<long long>((n + TB - 1) / TB, 148LL * 64);
}

// per-pixel base features: mean (3), standard deviation of the mean (3), normal (n), depth / 10, and
// the spatial noise estimate (3): sqrt of half the mean squared difference of the mean to the 2(n-1)
// axis neighbours (clamped), which for independent noise over a locally constant image is the
// standard deviation of the mean; unlike the per-pixel estimate it exists at one sample per pixel
__global__ void k_base_features(long long P, __grid_constant__ const Stencil st, const float* __restrict__ mean, const float* __restrict__ var,
                                const float* __restrict__ normal, const float* __restrict__ depth, float* __restrict__ out)
{
        const int nf = st.nf;
        const int n = nf - 10;
        const float inv = 1.0f / (float)(4 * st.axes);
        for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x)
        {
                float* o = out + p * BASE_STRIDE;
                float m[3], sq[3] = {0, 0, 0};
                for (int c = 0; c < 3; ++c)
                {
                        m[c] = mean[p * 3 + c];
                        o[c] = m[c];
                        o[3 + c] = sqrtf(fmaxf(var[p * 3 + c], 0.0f));
                }
                for (int k = 0; k < n; ++k)
                {
                        o[6 + k] = normal[p * n + k];
                }
                o[6 + n] = depth[p] * 0.1f;
                for (int a = 0; a < st.axes; ++a)
                {
                        for (int d = -1; d <= 1; d += 2)
                        {
                                const long long q = st.neighbour(p, a, d);
                                for (int c = 0; c < 3; ++c)
                                {
                                        const float t = mean[q * 3 + c] - m[c];
                                        sq[c] += t * t;
                                }
                        }
                }
                for (int c = 0; c < 3; ++c)
                {
                        o[7 + n + c] = sqrtf(sq[c] * inv);
                }
                for (int k = nf; k < BASE_STRIDE; ++k)
                {
                        o[k] = 0.0f;
                }
        }
}

__device__ __forceinline__ void softmax9(const float* z, float* w)
{
        float mx = z[0];
#pragma unroll
        for (int j = 1; j < TAPS; ++j)
        {
                mx = fmaxf(mx, z[j]);
        }
        float s = 0;
#pragma unroll
        for (int j = 0; j < TAPS; ++j)
        {
                w[j] = __expf(z[j] - mx);
                s += w[j];
        }
        const float inv = 1.0f / s;
#pragma unroll
        for (int j = 0; j < TAPS; ++j)
        {
                w[j] *= inv;
        }
}

// base bandwidths: at log-bandwidth 0 an object boundary (squared normal difference about 1) or a
// depth step of a unit costs a tap a few units of logit, the colour term only a clear edge
__device__ __forceinline__ float guide_scale(int g)
{
        return g == 0 ? 4.0f : (g == 1 ? 1.0f : 0.05f);
}

// Guide distances between pixels p and q from the base features (mean 0..2, standard deviation of the
// mean 3..5, normal 6..6+n-1, depth / 10 at 6+n, spatial noise 7+n..9+n): squared normal difference, squared depth
// difference, and the colour distance of non-local-means filtering (Rousselle, Knaus and Zwicker,
// "Adaptive rendering with non-local means filtering", 2012): the squared difference of the means
// less the variance it carries from the noise, over that variance plus a small relative floor,
// averaged over the channels.
__device__ __forceinline__ void load_base(const float* __restrict__ base, long long p, float* b)
{
        const float4* s = reinterpret_cast<const float4*>(base + p * BASE_STRIDE);
#pragma unroll
        for (int i = 0; i < BASE_STRIDE / 4; ++i)
        {
                const float4 t = __ldg(s + i);
                b[4 * i] = t.x;
                b[4 * i + 1] = t.y;
                b[4 * i + 2] = t.z;
                b[4 * i + 3] = t.w;
        }
}

// bp, bq: the two pixels' base features (load_base); n: the space dimension (3..6)
__device__ __forceinline__ void guide_distance(const float* bp, const float* bq, int n, float* D)
{
        float dn = 0;
#pragma unroll
        for (int k = 0; k < 6; ++k)
        {
                if (k < n)
                {
                        const float t = bp[6 + k] - bq[6 + k];
                        dn += t * t;
                }
        }
        // depth / 10 at 6 + n, picked by selects (an index computed from n would send the arrays to
        // local memory)
        const float dp = n == 3 ? bp[9] : (n == 4 ? bp[10] : (n == 5 ? bp[11] : bp[12]));
        const float dq = n == 3 ? bq[9] : (n == 4 ? bq[10] : (n == 5 ? bq[11] : bq[12]));
        const float dd = 10.0f * (dp - dq);
        float dc = 0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
        {
                const float dm = bp[c] - bq[c];
                const float v = bp[3 + c] * bp[3 + c] + bq[3 + c] * bq[3 + c];
                const float mb = 0.5f * (bp[c] + bq[c]);
                dc += fmaxf(dm * dm - v, 0.0f) / (1e-4f + 0.01f * mb * mb + v);
        }
        D[0] = dn;
        D[1] = dd * dd;
        D[2] = dc * (1.0f / 3.0f);
}

// The axis's tap weights at pixel p: softmax over taps of Z[p, a*9 + j] - sum_g s_g D_g(p, tap j),
// s_g = GUIDE_SCALE x exp(min(Z[p, 9 (n-1) + a*3 + g], BANDWIDTH_MAX)).  The taps' pixels q, D, s and
// whether each log-bandwidth lies below its clamp are returned for the backward pass.
__device__ __forceinline__ void tap_weights(const Stencil& st, const float* __restrict__ base, int a, long long p,
                                            const float* __restrict__ Z, int ldz, long long* q, float (*D)[GUIDES],
                                            float* s, bool* open, float* w)
{
        const float* zrow = Z + p * ldz;
#pragma unroll
        for (int g = 0; g < GUIDES; ++g)
        {
                const float o = zrow[st.axes * TAPS + a * GUIDES + g];
                open[g] = o < BANDWIDTH_MAX;
                s[g] = guide_scale(g) * expf(fminf(o, BANDWIDTH_MAX));
        }
        float z[TAPS];
        float bp[BASE_STRIDE];
        load_base(base, p, bp);
#pragma unroll
        for (int j = 0; j < TAPS; ++j)
        {
                q[j] = st.neighbour(p, a, j - RADIUS);
                float bq[BASE_STRIDE];
                load_base(base, q[j], bq);
                guide_distance(bp, bq, st.nf - 10, D[j]);
                z[j] = zrow[a * TAPS + j] - (s[0] * D[j][0] + s[1] * D[j][1] + s[2] * D[j][2]);
        }
        softmax9(z, w);
}

// y_out[p] = sum_j w_j y_in[p + (j - 4) e_a] with the tap weights above
__global__ void k_filter_fwd(long long P, __grid_constant__ const Stencil st, int a, const float* __restrict__ base, const float* __restrict__ Z,
                             int ldz, const float* __restrict__ y_in, float* __restrict__ y_out)
{
        for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x)
        {
                long long q[TAPS];
                float D[TAPS][GUIDES], s[GUIDES], w[TAPS];
                bool open[GUIDES];
                tap_weights(st, base, a, p, Z, ldz, q, D, s, open, w);
                float acc[3] = {0, 0, 0};
#pragma unroll
                for (int j = 0; j < TAPS; ++j)
                {
#pragma unroll
                        for (int c = 0; c < 3; ++c)
                        {
                                acc[c] += w[j] * y_in[q[j] * 3 + c];
                        }
                }
#pragma unroll
                for (int c = 0; c < 3; ++c)
                {
                        y_out[p * 3 + c] = acc[c];
                }
        }
}

// backward of k_filter_fwd: dZ for the axis's tap logits and log-bandwidths (through the softmax) and,
// when g_in is given, dL/dy_in added by atomics
__global__ void k_filter_bwd(long long P, __grid_constant__ const Stencil st, int a, const float* __restrict__ base, const float* __restrict__ Z,
                             int ldz, const float* __restrict__ y_in, const float* __restrict__ g_out, float* g_in,
                             __nv_bfloat16* __restrict__ dZ)
{
        for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x)
        {
                long long q[TAPS];
                float D[TAPS][GUIDES], s[GUIDES], w[TAPS], dw[TAPS];
                bool open[GUIDES];
                tap_weights(st, base, a, p, Z, ldz, q, D, s, open, w);
                const float g0 = g_out[p * 3], g1 = g_out[p * 3 + 1], g2 = g_out[p * 3 + 2];
                float dot = 0;
#pragma unroll
                for (int j = 0; j < TAPS; ++j)
                {
                        const long long qj = q[j];
                        dw[j] = g0 * y_in[qj * 3] + g1 * y_in[qj * 3 + 1] + g2 * y_in[qj * 3 + 2];
                        dot += w[j] * dw[j];
                        if (g_in)
                        {
                                atomicAdd(g_in + qj * 3, w[j] * g0);
                                atomicAdd(g_in + qj * 3 + 1, w[j] * g1);
                                atomicAdd(g_in + qj * 3 + 2, w[j] * g2);
                        }
                }
                float ds[GUIDES] = {0, 0, 0};
#pragma unroll
                for (int j = 0; j < TAPS; ++j)
                {
                        const float gl = w[j] * (dw[j] - dot);
                        dZ[p * ldz + a * TAPS + j] = __float2bfloat16_rn(gl);
#pragma unroll
                        for (int g = 0; g < GUIDES; ++g)
                        {
                                ds[g] -= gl * D[j][g];
                        }
                }
                // d logit_j / d o_g = -s_g D_g(j), zero where the log-bandwidth is clamped
#pragma unroll
                for (int g = 0; g < GUIDES; ++g)
                {
                        dZ[p * ldz + st.axes * TAPS + a * GUIDES + g] = __float2bfloat16_rn(open[g] ? ds[g] * s[g] : 0.0f);
                }
        }
}

__device__ __forceinline__ double block_sum(double v, double* s_red)
{
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
                v += __shfl_down_sync(0xffffffffu, v, o);
        }
        if ((threadIdx.x & 31) == 0)
        {
                s_red[threadIdx.x >> 5] = v;
        }
        __syncthreads();
        double t = 0;
        if (threadIdx.x == 0)
        {
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
                {
                        t += s_red[w];
                }
        }
        __syncthreads();
        return t;
}

// sums[0] += sum((noisy - target)^2), the squared error of the input
__global__ void k_energy(long long n3, const float* __restrict__ noisy, const float* __restrict__ target, double* sums)
{
        __shared__ double s_red[TB / 32];
        double acc = 0;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
        {
                const double t = (double)noisy[i] - (double)target[i];
                acc += t * t;
        }
        const double b = block_sum(acc, s_red);
        if (threadIdx.x == 0)
        {
                atomicAdd(sums, b);
        }
}

// sums[1] += sum((out - target)^2) / sums[0]; g = 2 (out - target) / sums[0]
__global__ void k_loss_grad(long long n3, const float* __restrict__ out, const float* __restrict__ target, double* sums,
                            float* __restrict__ g)
{
        __shared__ double s_red[TB / 32];
        const double inv = sums[0] > 0 ? 1.0 / sums[0] : 0.0;
        double acc = 0;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
        {
                const double d = (double)out[i] - (double)target[i];
                acc += d * d;
                g[i] = (float)(2.0 * d * inv);
        }
        const double b = block_sum(acc, s_red);
        if (threadIdx.x == 0)
        {
                atomicAdd(sums + 1, b * inv);
        }
}

// out[c] += sum over rows of m[row, c] (c < cols)
__global__ void k_colsum(long long rows, int cols, int ld, const __nv_bfloat16* __restrict__ m, float* out)
{
        const int c = threadIdx.x % 64;
        const int rg = threadIdx.x / 64;
        const int groups = blockDim.x / 64;
        if (c >= cols)
        {
                return;
        }
        float acc = 0;
        for (long long r = blockIdx.x * (long long)groups + rg; r < rows; r += (long long)gridDim.x * groups)
        {
                acc += __bfloat162float(m[r * ld + c]);
        }
        atomicAdd(out + c, acc);
}

__global__ void k_adam(long long count, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float c1, float c2)
{
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x)
        {
                const float gi = g[i];
                const float mi = b1 * m[i] + (1 - b1) * gi;
                const float vi = b2 * v[i] + (1 - b2) * gi * gi;
                m[i] = mi;
                v[i] = vi;
                w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        }
}

// flat FP32 parameters -> padded BF16 weight matrices and FP32 biases for the GEMMs
__global__ void k_pack(const float* __restrict__ w, int F, int Fp, int O, int Op, __nv_bfloat16* W1, float* b1,
                       __nv_bfloat16* W2, float* b2, __nv_bfloat16* W3, float* b3)
{
        const float* w1 = w;
        const float* pb1 = w1 + HID * F;
        const float* w2 = pb1 + HID;
        const float* pb2 = w2 + HID * HID;
        const float* w3 = pb2 + HID;
        const float* pb3 = w3 + O * HID;
        const int total = HID * Fp + HID + HID * HID + HID + Op * HID + Op;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
        {
                int k = i;
                if (k < HID * Fp)
                {
                        const int r = k / Fp, c = k % Fp;
                        W1[k] = __float2bfloat16_rn(c < F ? w1[r * F + c] : 0.0f);
                        continue;
                }
                k -= HID * Fp;
                if (k < HID)
                {
                        b1[k] = pb1[k];
                        continue;
                }
                k -= HID;
                if (k < HID * HID)
                {
                        W2[k] = __float2bfloat16_rn(w2[k]);
                        continue;
                }
                k -= HID * HID;
                if (k < HID)
                {
                        b2[k] = pb2[k];
                        continue;
                }
                k -= HID;
                if (k < Op * HID)
                {
                        const int r = k / HID;
                        W3[k] = __float2bfloat16_rn(r < O ? w3[k] : 0.0f);
                        continue;
                }
                k -= Op * HID;
                b3[k] = k < O ? pb3[k] : 0.0f;
        }
}

// padded FP32 gradients -> flat gradient in the parameter order
__global__ void k_unpack(int F, int Fp, int O, const float* gW1, const float* gb1, const float* gW2, const float* gb2,
                         const float* gW3, const float* gb3, float* __restrict__ g)
{
        const int total = HID * F + HID + HID * HID + HID + O * HID + O;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
        {
                int k = i;
                if (k < HID * F)
                {
                        g[i] = gW1[(k / F) * Fp + k % F];
                        continue;
                }
                k -= HID * F;
                if (k < HID)
                {
                        g[i] = gb1[k];
                        continue;
                }
                k -= HID;
                if (k < HID * HID)
                {
                        g[i] = gW2[k];
                        continue;
                }
                k -= HID * HID;
                if (k < HID)
                {
                        g[i] = gb2[k];
                        continue;
                }
                k -= HID;
                if (k < O * HID)
                {
                        g[i] = gW3[k];
                        continue;
                }
                k -= O * HID;
                g[i] = gb3[k];
        }
}

// ------------------------------------------------------------------------------------------------
// host side

struct DError
{
        int code;
        std::string msg;
};

void ck(cudaError_t e, const char* what)
{
        if (e != cudaSuccess)
        {
                throw DError{e == cudaErrorMemoryAllocation ? NT_ENOMEM : NT_ECUDA,
                             std::string(what) + ": " + cudaGetErrorString(e)};
        }
}

template <typename F>
int guard(F&& f)
{
        try
        {
                f();
                return NT_OK;
        }
        catch (const DError& e)
        {
                return ntrace::report_error(e.code, e.msg);
        }
        catch (const std::bad_alloc&)
        {
                return ntrace::report_error(NT_ENOMEM, "host allocation failed");
        }
}

struct Buf
{
        void* p = nullptr;
        size_t bytes = 0;
        ~Buf()
        {
                if (p)
                {
                        cudaFree(p);
                }
        }
        void ensure(size_t b)
        {
                if (b <= bytes)
                {
                        return;
                }
                if (p)
                {
                        cudaFree(p);
                        p = nullptr;
                        bytes = 0;
                }
                ck(cudaMalloc(&p, b), "cudaMalloc");
                bytes = b;
        }
        template <typename T>
        T* as() const
        {
                return static_cast<T*>(p);
        }
};

uint64_t splitmix(uint64_t& s)
{
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
}
}

struct nt_denoiser
{
        int n = 0;
        int nf = 0, F = 0, Fp = 0, O = 0, Op = 0;
        long long nparams = 0;
        long long P = 0;
        Stencil st{};
        cudaStream_t own = nullptr;
        cudaStream_t st_use = nullptr;
        long long adam_t = 0;
        // parameters and optimiser state (flat FP32), packed weights
        Buf w, g, m, v;
        Buf W1, b1, W2, b2, W3, b3;
        // padded FP32 gradients in one block (cleared together): gW1 | gb1 | gW2 | gb2 | gW3 | gb3
        Buf gblock;
        float *gW1 = nullptr, *gb1 = nullptr, *gW2 = nullptr, *gb2 = nullptr, *gW3 = nullptr, *gb3 = nullptr;
        // per-image workspace
        Buf base, X, H1, H2, Z, Y, G, dZ, dH1, dH2, sums, err;
        bool packed = false;

        size_t gbytes() const
        {
                return sizeof(float) * (size_t)(HID * Fp + HID + HID * HID + HID + Op * HID + Op);
        }
};

namespace
{
void pack(nt_denoiser* d)
{
        k_pack<<<64, TB, 0, d->st_use>>>(d->w.as<float>(), d->F, d->Fp, d->O, d->Op, d->W1.as<__nv_bfloat16>(),
                                         d->b1.as<float>(), d->W2.as<__nv_bfloat16>(), d->b2.as<float>(),
                                         d->W3.as<__nv_bfloat16>(), d->b3.as<float>());
        ck(cudaGetLastError(), "pack");
        d->packed = true;
}

void check_err(nt_denoiser* d)
{
        int h = 0;
        ck(cudaMemcpyAsync(&h, d->err.p, sizeof(int), cudaMemcpyDeviceToHost, d->st_use), "error flag");
        ck(cudaStreamSynchronize(d->st_use), "sync");
        if (h)
        {
                throw DError{NT_ETIMEOUT, "tensor-core GEMM: an MMA completion wait ran out"};
        }
}

// forward pass of the current input: Y[n-1] is the denoised image
void forward(nt_denoiser* d)
{
        if (d->P <= 0)
        {
                throw DError{NT_ESTATE, "no input set"};
        }
        if (!d->packed)
        {
                pack(d);
        }
        const long long P = d->P;
        const int P32 = (int)P;
        cudaStream_t s = d->st_use;
        int* err = d->err.as<int>();
        ck(gemm(LoadRows{d->X.as<__nv_bfloat16>(), d->Fp}, LoadRows{d->W1.as<__nv_bfloat16>(), d->Fp},
                EpiBiasReluBF16{d->b1.as<float>(), d->H1.as<__nv_bfloat16>(), HID}, P32, HID, d->Fp, 0, err, s),
           "gemm 1");
        ck(gemm(LoadRows{d->H1.as<__nv_bfloat16>(), HID}, LoadRows{d->W2.as<__nv_bfloat16>(), HID},
                EpiBiasReluBF16{d->b2.as<float>(), d->H2.as<__nv_bfloat16>(), HID}, P32, HID, HID, 0, err, s),
           "gemm 2");
        ck(gemm(LoadRows{d->H2.as<__nv_bfloat16>(), HID}, LoadRows{d->W3.as<__nv_bfloat16>(), HID},
                EpiBiasF32{d->b3.as<float>(), d->Z.as<float>(), d->Op}, P32, d->Op, HID, 0, err, s),
           "gemm 3");
        for (int a = 0; a < d->n - 1; ++a)
        {
                k_filter_fwd<<<blocks_for(P), TB, 0, s>>>(P, d->st, a, d->base.as<float>(), d->Z.as<float>(), d->Op,
                                                            d->Y.as<float>() + (size_t)a * P * 3,
                                                            d->Y.as<float>() + (size_t)(a + 1) * P * 3);
        }
        ck(cudaGetLastError(), "filter");
}

// loss and gradients (padded, in gW*/gb*) against target
double backward(nt_denoiser* d, const float* target)
{
        const long long P = d->P;
        const int P32 = (int)P;
        cudaStream_t s = d->st_use;
        int* err = d->err.as<int>();
        const int A = d->n - 1;
        ck(cudaMemsetAsync(d->sums.p, 0, 2 * sizeof(double), s), "memset");
        k_energy<<<blocks_for(P * 3), TB, 0, s>>>(P * 3, d->Y.as<float>(), target, d->sums.as<double>());
        float* G0 = d->G.as<float>();
        float* G1 = G0 + (size_t)P * 3;
        k_loss_grad<<<blocks_for(P * 3), TB, 0, s>>>(P * 3, d->Y.as<float>() + (size_t)A * P * 3, target,
                                                       d->sums.as<double>(), G0);
        ck(cudaMemsetAsync(d->dZ.p, 0, (size_t)P * d->Op * sizeof(__nv_bfloat16), s), "memset");
        float* gout = G0;
        float* gin = G1;
        for (int a = A - 1; a >= 0; --a)
        {
                if (a > 0)
                {
                        ck(cudaMemsetAsync(gin, 0, (size_t)P * 3 * sizeof(float), s), "memset");
                }
                k_filter_bwd<<<blocks_for(P), TB, 0, s>>>(P, d->st, a, d->base.as<float>(), d->Z.as<float>(), d->Op,
                                                            d->Y.as<float>() + (size_t)a * P * 3, gout, a > 0 ? gin : nullptr,
                                                            d->dZ.as<__nv_bfloat16>());
                std::swap(gout, gin);
        }
        ck(cudaGetLastError(), "filter backward");
        // backward data products
        ck(gemm(LoadRows{d->dZ.as<__nv_bfloat16>(), d->Op}, LoadCols{d->W3.as<__nv_bfloat16>(), HID},
                EpiMaskBF16{d->H2.as<__nv_bfloat16>(), d->dH2.as<__nv_bfloat16>(), HID}, P32, HID, d->Op, 0, err, s),
           "gemm dH2");
        ck(gemm(LoadRows{d->dH2.as<__nv_bfloat16>(), HID}, LoadCols{d->W2.as<__nv_bfloat16>(), HID},
                EpiMaskBF16{d->H1.as<__nv_bfloat16>(), d->dH1.as<__nv_bfloat16>(), HID}, P32, HID, HID, 0, err, s),
           "gemm dH1");
        // weight gradients: reductions over pixels, split across CTAs, about four per SM (the products
        // are skinny and HBM-bound, so their copies need the CTAs in flight)
        ck(cudaMemsetAsync(d->gblock.p, 0, d->gbytes(), s), "memset");
        int dev = 0, sms = 148;
        ck(cudaGetDevice(&dev), "device");
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "device attribute");
        const long long ctas = 4LL * std::max(1, sms);
        const int kpc = (int)std::max<long long>(GK, ((long long)P32 + ctas - 1) / ctas);
        ck(gemm(LoadCols{d->dZ.as<__nv_bfloat16>(), d->Op}, LoadCols{d->H2.as<__nv_bfloat16>(), HID},
                EpiAtomicF32{d->gW3, HID, HID}, d->Op, HID, P32, kpc, err, s),
           "gemm dW3");
        ck(gemm(LoadCols{d->dH2.as<__nv_bfloat16>(), HID}, LoadCols{d->H1.as<__nv_bfloat16>(), HID},
                EpiAtomicF32{d->gW2, HID, HID}, HID, HID, P32, kpc, err, s),
           "gemm dW2");
        ck(gemm(LoadCols{d->dH1.as<__nv_bfloat16>(), HID}, LoadCols{d->X.as<__nv_bfloat16>(), d->Fp},
                EpiAtomicF32{d->gW1, d->Fp, d->Fp}, HID, d->Fp, P32, kpc, err, s),
           "gemm dW1");
        const unsigned cb = (unsigned)std::min<long long>((P + 3) / 4, 1024);
        k_colsum<<<cb, TB, 0, s>>>(P, d->Op, d->Op, d->dZ.as<__nv_bfloat16>(), d->gb3);
        k_colsum<<<cb, TB, 0, s>>>(P, HID, HID, d->dH2.as<__nv_bfloat16>(), d->gb2);
        k_colsum<<<cb, TB, 0, s>>>(P, HID, HID, d->dH1.as<__nv_bfloat16>(), d->gb1);
        k_unpack<<<64, TB, 0, s>>>(d->F, d->Fp, d->O, d->gW1, d->gb1, d->gW2,
                                   d->gb2, d->gW3, d->gb3, d->g.as<float>());
        ck(cudaGetLastError(), "gradients");
        double sums[2];
        ck(cudaMemcpyAsync(sums, d->sums.p, sizeof(sums), cudaMemcpyDeviceToHost, s), "loss");
        check_err(d);
        return sums[1];
}
}

extern "C" {

int nt_denoiser_create(int n, uint64_t seed, nt_denoiser** out)
{
        return guard([&]() {
                if (!out || n < 3 || n > 6)
                {
                        throw DError{NT_EINVAL, "n must be 3..6"};
                }
                auto d = std::make_unique<nt_denoiser>();
                d->n = n;
                d->nf = n + 10;
                d->F = d->nf * (2 * (n - 1) + 1) + 1;
                d->Fp = (d->F + 15) / 16 * 16;
                d->O = (TAPS + GUIDES) * (n - 1);
                d->Op = (d->O + 15) / 16 * 16;
                d->nparams = (long long)HID * d->F + HID + HID * HID + HID + (long long)d->O * HID + d->O;
                ck(cudaStreamCreateWithFlags(&d->own, cudaStreamNonBlocking), "cudaStreamCreate");
                d->st_use = d->own;
                const size_t pb = sizeof(float) * (size_t)d->nparams;
                d->w.ensure(pb);
                d->g.ensure(pb);
                d->m.ensure(pb);
                d->v.ensure(pb);
                ck(cudaMemsetAsync(d->m.p, 0, pb, d->own), "memset");
                ck(cudaMemsetAsync(d->v.p, 0, pb, d->own), "memset");
                d->W1.ensure(sizeof(__nv_bfloat16) * HID * d->Fp);
                d->b1.ensure(sizeof(float) * HID);
                d->W2.ensure(sizeof(__nv_bfloat16) * HID * HID);
                d->b2.ensure(sizeof(float) * HID);
                d->W3.ensure(sizeof(__nv_bfloat16) * d->Op * HID);
                d->b3.ensure(sizeof(float) * d->Op);
                d->gblock.ensure(d->gbytes());
                d->gW1 = d->gblock.as<float>();
                d->gb1 = d->gW1 + HID * d->Fp;
                d->gW2 = d->gb1 + HID;
                d->gb2 = d->gW2 + HID * HID;
                d->gW3 = d->gb2 + HID;
                d->gb3 = d->gW3 + d->Op * HID;
                d->sums.ensure(2 * sizeof(double));
                d->err.ensure(sizeof(int));
                ck(cudaMemsetAsync(d->err.p, 0, sizeof(int), d->own), "memset");
                // initial weights: Kaiming-uniform hidden layers, a small output layer, zero biases
                std::vector<float> h((size_t)d->nparams, 0.0f);
                uint64_t s = seed;
                auto uni = [&](float bound) {
                        const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
                        return (float)((2 * u - 1) * bound);
                };
                size_t k = 0;
                const float bw1 = std::sqrt(6.0f / d->F), bw2 = std::sqrt(6.0f / HID), bw3 = 0.1f * std::sqrt(6.0f / HID);
                for (int i = 0; i < HID * d->F; ++i)
                {
                        h[k++] = uni(bw1);
                }
                k += HID;
                for (int i = 0; i < HID * HID; ++i)
                {
                        h[k++] = uni(bw2);
                }
                k += HID;
                for (int i = 0; i < d->O * HID; ++i)
                {
                        h[k++] = uni(bw3);
                }
                ck(cudaMemcpyAsync(d->w.p, h.data(), pb, cudaMemcpyHostToDevice, d->own), "upload");
                ck(cudaStreamSynchronize(d->own), "sync");
                *out = d.release();
        });
}

int nt_denoiser_destroy(nt_denoiser* d)
{
        if (!d)
        {
                return NT_OK;
        }
        if (d->own)
        {
                cudaStreamSynchronize(d->own);
                cudaStreamDestroy(d->own);
        }
        delete d;
        return NT_OK;
}

int nt_denoiser_get_layout(nt_denoiser* d, nt_denoiser_layout* out)
{
        return guard([&]() {
                if (!d || !out)
                {
                        throw DError{NT_EINVAL, "null argument"};
                }
                out->n = d->n;
                out->base_features = d->nf;
                out->features = d->F;
                out->features_padded = d->Fp;
                out->hidden = HID;
                out->outputs = d->O;
                out->outputs_padded = d->Op;
                out->param_count = d->nparams;
        });
}

int nt_denoiser_get_params(nt_denoiser* d, float* params)
{
        return guard([&]() {
                if (!d || !params)
                {
                        throw DError{NT_EINVAL, "null argument"};
                }
                ck(cudaMemcpyAsync(params, d->w.p, sizeof(float) * d->nparams, cudaMemcpyDeviceToHost, d->st_use), "copy");
                ck(cudaStreamSynchronize(d->st_use), "sync");
        });
}

int nt_denoiser_set_params(nt_denoiser* d, const float* params)
{
        return guard([&]() {
                if (!d || !params)
                {
                        throw DError{NT_EINVAL, "null argument"};
                }
                ck(cudaMemcpyAsync(d->w.p, params, sizeof(float) * d->nparams, cudaMemcpyHostToDevice, d->st_use), "copy");
                ck(cudaStreamSynchronize(d->st_use), "sync");
                d->packed = false;
        });
}

int nt_denoiser_set_input(nt_denoiser* d, const int32_t* screen, int samples_per_pixel, const float* d_mean,
                          const float* d_var, const float* d_normal, const float* d_depth, void* stream)
{
        return guard([&]() {
                if (!d || !screen || !d_mean || !d_var || !d_normal || !d_depth)
                {
                        throw DError{NT_EINVAL, "null argument"};
                }
                if (samples_per_pixel < 1)
                {
                        throw DError{NT_EINVAL, "samples_per_pixel must be positive"};
                }
                Stencil st{};
                st.axes = d->n - 1;
                long long P = 1;
                for (int a = 0; a < st.axes; ++a)
                {
                        if (screen[a] < 1)
                        {
                                throw DError{NT_EINVAL, "screen sizes must be positive"};
                        }
                        st.size[a] = screen[a];
                        st.stride[a] = P;
                        P *= screen[a];
                }
                if (P > (1LL << 30))
                {
                        throw DError{NT_EINVAL, "too many pixels for the denoiser"};
                }
                st.nf = d->nf;
                st.stencil_features = d->F - 1;
                st.features = d->F;
                st.noise_level = (float)(1.0 / std::sqrt((double)samples_per_pixel));
                d->st = st;
                d->P = P;
                d->st_use = stream ? (cudaStream_t)stream : d->own;
                d->base.ensure(sizeof(float) * (size_t)P * BASE_STRIDE);
                d->X.ensure(sizeof(__nv_bfloat16) * (size_t)P * d->Fp);
                d->H1.ensure(sizeof(__nv_bfloat16) * (size_t)P * HID);
                d->H2.ensure(sizeof(__nv_bfloat16) * (size_t)P * HID);
                d->dH1.ensure(sizeof(__nv_bfloat16) * (size_t)P * HID);
                d->dH2.ensure(sizeof(__nv_bfloat16) * (size_t)P * HID);
                d->Z.ensure(sizeof(float) * (size_t)P * d->Op);
                d->dZ.ensure(sizeof(__nv_bfloat16) * (size_t)P * d->Op);
                d->Y.ensure(sizeof(float) * (size_t)P * 3 * d->n);
                d->G.ensure(sizeof(float) * (size_t)P * 3 * 2);
                k_base_features<<<blocks_for(P), TB, 0, d->st_use>>>(P, st, d_mean, d_var, d_normal, d_depth,
                                                                      d->base.as<float>());
                k_features<<<blocks_for(P * (d->Fp / 8)), TB, 0, d->st_use>>>(P, st, d->Fp, d->base.as<float>(),
                                                                              d->X.as<__nv_bfloat16>());
                ck(cudaGetLastError(), "features");
                ck(cudaMemcpyAsync(d->Y.p, d_mean, sizeof(float) * (size_t)P * 3, cudaMemcpyDeviceToDevice, d->st_use),
                   "copy");
        });
}

int nt_denoiser_apply(nt_denoiser* d, float* d_out)
{
        return guard([&]() {
                if (!d || !d_out)
                {
                        throw DError{NT_EINVAL, "null argument"};
                }
                forward(d);
                ck(cudaMemcpyAsync(d_out, d->Y.as<float>() + (size_t)(d->n - 1) * d->P * 3, sizeof(float) * (size_t)d->P * 3,
                                   cudaMemcpyDeviceToDevice, d->st_use),
                   "copy");
                check_err(d);
        });
}

int nt_denoiser_gradient(nt_denoiser* d, const float* d_target, float* grad, double* loss)
{
        return guard([&]() {
                if (!d || !d_target)
                {
                        throw DError{NT_EINVAL, "null argument"};
                }
                forward(d);
                const double l = backward(d, d_target);
                if (grad)
                {
                        ck(cudaMemcpyAsync(grad, d->g.p, sizeof(float) * d->nparams, cudaMemcpyDeviceToHost, d->st_use),
                           "copy");
                        ck(cudaStreamSynchronize(d->st_use), "sync");
                }
                if (loss)
                {
                        *loss = l;
                }
        });
}

int nt_denoiser_train_step(nt_denoiser* d, const float* d_target, float lr, double* loss)
{
        return guard([&]() {
                if (!d || !d_target || !(lr > 0))
                {
                        throw DError{NT_EINVAL, "bad argument"};
                }
                forward(d);
                const double l = backward(d, d_target);
                ++d->adam_t;
                const float c1 = 1.0f - std::pow(0.9f, (float)d->adam_t);
                const float c2 = 1.0f - std::pow(0.999f, (float)d->adam_t);
                k_adam<<<blocks_for(d->nparams), TB, 0, d->st_use>>>(d->nparams, d->w.as<float>(), d->g.as<float>(),
                                                                     d->m.as<float>(), d->v.as<float>(), lr, c1, c2);
                ck(cudaGetLastError(), "adam");
                pack(d);
                if (loss)
                {
                        *loss = l;
                }
        });
}

int nt_tc_gemm_wait_selftest(void* stream)
{
        return guard([&]() {
                cudaStream_t s = (cudaStream_t)stream;
                Buf a, b, c, err;
                const int m = 128, n = 16, k = 64;
                a.ensure((size_t)m * k * 2);
                b.ensure((size_t)n * k * 2);
                c.ensure((size_t)m * n * 4);
                err.ensure(sizeof(int));
                ck(cudaMemsetAsync(a.p, 0, (size_t)m * k * 2, s), "memset");
                ck(cudaMemsetAsync(b.p, 0, (size_t)n * k * 2, s), "memset");
                ck(cudaMemsetAsync(err.p, 0, sizeof(int), s), "memset");
                GemmCtl ctl;
                ctl.wait_ns = 20000000ull;  // 20 ms
                ctl.withhold = 1;
                ck(gemm(LoadRows{a.as<const __nv_bfloat16>(), k}, LoadRows{b.as<const __nv_bfloat16>(), k}, EpiStoreF32{c.as<float>(), n},
                        m, n, k, 0, err.as<int>(), s, ctl),
                   "gemm");
                int h = 0;
                ck(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, s), "copy");
                ck(cudaStreamSynchronize(s), "sync");
                if (h)
                {
                        throw DError{NT_ETIMEOUT, "tensor-core GEMM: an MMA completion wait ran out"};
                }
        });
}

int nt_tc_gemm_bf16(const uint16_t* d_a, const uint16_t* d_b, float* d_c, int m, int n, int k, void* stream)
{
        return guard([&]() {
                if (!d_a || !d_b || !d_c || m < 1 || n < 16 || n > 256 || n % 16 || k < 16 || k % 16)
                {
                        throw DError{NT_EINVAL, "nt_tc_gemm_bf16: bad arguments"};
                }
                cudaStream_t s = (cudaStream_t)stream;
                Buf err;
                err.ensure(sizeof(int));
                ck(cudaMemsetAsync(err.p, 0, sizeof(int), s), "memset");
                ck(gemm(LoadRows{(const __nv_bfloat16*)d_a, k}, LoadRows{(const __nv_bfloat16*)d_b, k}, EpiStoreF32{d_c, n},
                        m, n, k, 0, err.as<int>(), s),
                   "gemm");
                int h = 0;
                ck(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, s), "copy");
                ck(cudaStreamSynchronize(s), "sync");
                if (h)
                {
                        throw DError{NT_ETIMEOUT, "tensor-core GEMM: an MMA completion wait ran out"};
                }
        });
}

int nt_tc_gemm_bf16_t(const uint16_t* d_at, const uint16_t* d_bt, float* d_c, int m, int n, int k, int k_per_cta,
                      void* stream)
{
        return guard([&]() {
                if (!d_at || !d_bt || !d_c || m < 8 || m % 8 || n < 16 || n > 256 || n % 16 || k < 1 || k_per_cta < 0)
                {
                        throw DError{NT_EINVAL, "nt_tc_gemm_bf16_t: bad arguments"};
                }
                cudaStream_t s = (cudaStream_t)stream;
                Buf err;
                err.ensure(sizeof(int));
                ck(cudaMemsetAsync(err.p, 0, sizeof(int), s), "memset");
                ck(cudaMemsetAsync(d_c, 0, (size_t)m * n * sizeof(float), s), "memset");
                ck(gemm(LoadCols{(const __nv_bfloat16*)d_at, m}, LoadCols{(const __nv_bfloat16*)d_bt, n},
                        EpiAtomicF32{d_c, n, n}, m, n, k, k_per_cta, err.as<int>(), s),
                   "gemm");
                int h = 0;
                ck(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, s), "copy");
                ck(cudaStreamSynchronize(s), "sync");
                if (h)
                {
                        throw DError{NT_ETIMEOUT, "tensor-core GEMM: an MMA completion wait ran out"};
                }
        });
}
}
