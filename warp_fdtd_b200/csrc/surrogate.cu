// Kernels of the CNN surrogate: a 2-D encoder-decoder that maps a design
// density to modal transmission at several wavelengths and to the
// transmission-gradient map.  It has no counterpart in the reference (the
// reference optimises with the adjoint only); the optimisation loop uses it to
// propose design updates that a full FDTD forward then accepts or rejects.
//
// Every 3x3 convolution runs as conv-as-GEMM on the fifth-generation tensor
// cores: fdtd_sg_gemm stages bf16 operand tiles with TMA into a shared-memory
// ring, one thread issues tcgen05.mma (kind::f16, bf16 inputs) into a float32
// accumulator in tensor memory, and the four warps read it back with
// tcgen05.ld for a fused bias / ReLU / bf16-rounding epilogue.  Forward,
// input-gradient and weight-gradient products are all this one GEMM
// C[M, N] = A[M, K] . B[N, K]^T with both operands K-contiguous; the kernels
// below supply the layouts (im2col, transposes, col2im), pooling, upsampling,
// the two heads, the loss and the optimiser.
//
// Layouts: activations are NHWC, pixel p = (b*H + y)*W + x, channel fastest,
// with a row stride (ld) so a layer can write into a channel slice of a
// concatenation buffer.  im2col column k = tap*C + c with tap = (dy+1)*3 +
// (dx+1), dy the row and dx the column offset.  Weights are [Cout, 9*Cin] in
// the same k order.
#include <cuda_bf16.h>

#include <mutex>

#include "common.cuh"
#include "tma_util.cuh"

namespace wfb {
namespace sg {

typedef __nv_bfloat16 bf16;

// Set to 1 by a GEMM whose bounded wait on an mbarrier ran out; read and
// cleared through fdtd_sg_status.
__device__ int g_status;

constexpr long WAIT_LIMIT = 1L << 24;  // polls (>= 1 s with the back-off)

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Whole warp: allocate `ncols` tensor-memory columns (power of two >= 32),
// address written to shared memory.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, int ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

// D[tmem] (+)= A[smem] . B[smem]^T, one 128 x N x 16 step.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, int accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive on `bar` once every tcgen05.mma issued so far by this thread is done.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

// Warp-wide: 16 consecutive float32 columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// Shared-memory matrix descriptors of K-major operand tiles (the version
// field, bit 46, is 1 on sm_100).
// * Interleaved (no swizzle): core matrices of 8 rows x 16 bytes stored
//   contiguously (128 B); `lbo` bytes between the two core matrices along K
//   of one MMA, `sbo` bytes between 8-row groups.
// * 128-byte swizzle (layout type 2): rows of 64 bf16 (128 B), the 16-byte
//   chunk c of row r stored at chunk c ^ (r % 8) inside 1024-byte atoms of 8
//   rows; sbo = 1024 between atoms, lbo unused (16); a K step of 16 elements
//   advances the start address by 32 bytes inside the atom.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo,
                                              uint32_t layout = 0) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}

// Instruction descriptor of kind::f16: bf16 A and B, both K-major, float32 D.
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

// ---------------------------------------------------------------- the GEMM
constexpr int BM = 128;  // rows of A per tile (TMEM lanes)
constexpr int BK = 64;   // K per pipeline stage: 8 core-matrix columns

template <int BN>
struct GemmCfg {
    static constexpr int STAGES = BN == 128 ? 3 : 4;
    static constexpr int A_BYTES = BM * BK * 2;
    static constexpr int B_BYTES = BN * BK * 2;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 + 256;
    static constexpr int TMEM_COLS = BN < 32 ? 32 : BN;
};

struct GemmParams {
    void *C;
    int ldc, c_bf16;
    const float *bias;
    int M, N, K;
    int chunks_per_split, nchunks;
    long long split_stride;
    int accumulate, relu;
};

// One 128 x BN output tile over the K chunks of split blockIdx.z.  Warp 0
// lane 0 streams A and B chunks with TMA: with SW, one 64 x rows box per
// operand through the tensor map's 128-byte swizzle; without, eight boxes of
// 8 K-elements, which land directly in the interleaved core-matrix layout;
// warp 1 lane 0 issues four K=16 MMAs per chunk and commits each stage back to
// the producer; all four warps then drain tensor memory.  Out-of-range rows
// and K columns are zero-filled by TMA.  Every wait is bounded; a wait that
// runs out sets g_status and the tile's epilogue is skipped.
template <int BN, bool SW>
__global__ void __launch_bounds__(128) gemm_kernel(const __grid_constant__ CUtensorMap ta,
                                                   const __grid_constant__ CUtensorMap tb,
                                                   const GemmParams p) {
    using CF = GemmCfg<BN>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    unsigned char *sa = smem;
    unsigned char *sb = smem + CF::STAGES * CF::A_BYTES;
    uint64_t *full = (uint64_t *)(sb + CF::STAGES * CF::B_BYTES);
    uint64_t *empty = full + CF::STAGES;
    uint64_t *done = empty + CF::STAGES;
    uint32_t *tmem_slot = (uint32_t *)(done + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM, z = blockIdx.z;
    const int c_begin = z * p.chunks_per_split;
    const int nk = min(p.chunks_per_split, p.nchunks - c_begin);

    if (threadIdx.x == 0) {
        for (int s = 0; s < CF::STAGES; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(tmem_slot, CF::TMEM_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            for (int i = 0; i < nk; ++i) {
                const int s = i % CF::STAGES;
                if (i >= CF::STAGES &&
                    !mbar_wait_bounded(empty + s, ((i / CF::STAGES) - 1) & 1, WAIT_LIMIT)) {
                    atomicExch(&g_status, 1);
                    break;
                }
                mbar_expect_tx(full + s, CF::STAGE_BYTES);
                const int k0 = (c_begin + i) * BK;
                if (SW) {
                    tma_load_2d(sa + s * CF::A_BYTES, &ta, k0, m0, full + s);
                    tma_load_2d(sb + s * CF::B_BYTES, &tb, k0, n0, full + s);
                } else {
#pragma unroll
                    for (int j = 0; j < BK / 8; ++j) {
                        tma_load_2d(sa + s * CF::A_BYTES + j * BM * 16, &ta, k0 + 8 * j, m0,
                                    full + s);
                        tma_load_2d(sb + s * CF::B_BYTES + j * BN * 16, &tb, k0 + 8 * j, n0,
                                    full + s);
                    }
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = instr_desc(BM, BN);
            int i = 0;
            for (; i < nk; ++i) {
                const int s = i % CF::STAGES;
                if (!mbar_wait_bounded(full + s, (i / CF::STAGES) & 1, WAIT_LIMIT)) {
                    atomicExch(&g_status, 1);
                    break;
                }
                tc_fence_after();
                const uint32_t a0 = smem_u32(sa + s * CF::A_BYTES);
                const uint32_t b0 = smem_u32(sb + s * CF::B_BYTES);
#pragma unroll
                for (int kk = 0; kk < BK / 16; ++kk) {
                    uint64_t ad, bd;
                    if (SW) {
                        ad = smem_desc(a0 + kk * 32, 16, 1024, 2);
                        bd = smem_desc(b0 + kk * 32, 16, 1024, 2);
                    } else {
                        ad = smem_desc(a0 + kk * 2 * BM * 16, BM * 16, 128);
                        bd = smem_desc(b0 + kk * 2 * BN * 16, BN * 16, 128);
                    }
                    mma_bf16(tmem, ad, bd, idesc, (i > 0 || kk > 0) ? 1 : 0);
                }
                mma_commit(empty + s);
            }
            if (i == nk) mma_commit(done);
        }
        __syncwarp();
    }

    const bool have = mbar_wait_bounded(done, 0, WAIT_LIMIT);
    if (!have) atomicExch(&g_status, 1);
    __syncwarp();
    tc_fence_after();
    if (__all_sync(0xffffffffu, have)) {
        const int row = m0 + warp * 32 + lane;
        const bool row_ok = row < p.M;
        for (int c0 = 0; c0 < BN && n0 + c0 < p.N; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (!row_ok) continue;
            const int nb = n0 + c0;
            const bool whole = nb + 16 <= p.N;
            if (p.c_bf16) {
                bf16 *c = (bf16 *)p.C + (i64)row * p.ldc + nb;
                __align__(16) bf16 o[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    float x = v[j];
                    if (p.bias && nb + j < p.N) x = x + p.bias[nb + j];
                    if (p.relu) x = fmaxf(x, 0.0f);
                    o[j] = __float2bfloat16_rn(x);
                }
                if (whole && ((uintptr_t)c & 15) == 0) {
                    ((uint4 *)c)[0] = ((const uint4 *)o)[0];
                    ((uint4 *)c)[1] = ((const uint4 *)o)[1];
                } else {
                    for (int j = 0; j < 16 && nb + j < p.N; ++j) c[j] = o[j];
                }
            } else {
                float *c = (float *)p.C + (i64)z * p.split_stride + (i64)row * p.ldc + nb;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    if (p.bias && nb + j < p.N) v[j] = v[j] + p.bias[nb + j];
                }
                if (p.accumulate) {
                    for (int j = 0; j < 16 && nb + j < p.N; ++j) v[j] = c[j] + v[j];
                }
                if (p.relu) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j], 0.0f);
                }
                if (whole && ((uintptr_t)c & 15) == 0) {
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        ((float4 *)c)[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2],
                                                       v[4 * j + 3]);
                } else {
                    for (int j = 0; j < 16 && nb + j < p.N; ++j) c[j] = v[j];
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, CF::TMEM_COLS);
}

// ---------------------------------------------------------------- layouts
__global__ void im2col_vec_kernel(const bf16 *__restrict__ x, int ldx, int B, int H, int W,
                                  int C, bf16 *__restrict__ col, int ldcol) {
    const int c8 = C >> 3;
    const i64 total = (i64)B * H * W * 9 * c8;
    const i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int cc = (int)(idx % c8);
    const i64 t = idx / c8;
    const int tap = (int)(t % 9);
    const i64 p = t / 9;
    const int xw = (int)(p % W);
    const i64 q = p / W;
    const int yh = (int)(q % H);
    const i64 b = q / H;
    const int yy = yh + tap / 3 - 1, xx = xw + tap % 3 - 1;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (yy >= 0 && yy < H && xx >= 0 && xx < W)
        v = *(const uint4 *)(x + ((b * H + yy) * W + xx) * ldx + cc * 8);
    *(uint4 *)(col + p * ldcol + tap * C + cc * 8) = v;
}

__global__ void im2col_kernel(const bf16 *__restrict__ x, int ldx, int B, int H, int W, int C,
                              bf16 *__restrict__ col, int ldcol) {
    const i64 total = (i64)B * H * W * 9 * C;
    const i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = (int)(idx % C);
    const i64 t = idx / C;
    const int tap = (int)(t % 9);
    const i64 p = t / 9;
    const int xw = (int)(p % W);
    const i64 q = p / W;
    const int yh = (int)(q % H);
    const i64 b = q / H;
    const int yy = yh + tap / 3 - 1, xx = xw + tap % 3 - 1;
    bf16 v = __float2bfloat16_rn(0.0f);
    if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = x[((b * H + yy) * W + xx) * ldx + c];
    col[p * ldcol + tap * C + c] = v;
}

// dst[c, r] = src[r, c] for a rows x cols bf16 matrix, 32 x 32 tiles.
__global__ void transpose_kernel(const bf16 *__restrict__ src, int lds, i64 rows, int cols,
                                 bf16 *__restrict__ dst, i64 ldd) {
    __shared__ unsigned short tile[32][33];
    const i64 r0 = (i64)blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    const unsigned short *s = (const unsigned short *)src;
    unsigned short *d = (unsigned short *)dst;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const i64 r = r0 + j;
        const int c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[j][threadIdx.x] = s[r * lds + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int c = c0 + j;
        const i64 r = r0 + threadIdx.x;
        if (r < rows && c < cols) d[(i64)c * ldd + r] = tile[threadIdx.x][j];
    }
}

// Input gradient of a 3x3 convolution from the column gradient: dx[p, c] =
// sum over taps of dcol[p - offset(tap), tap*C + c], taps in ascending order.
__global__ void col2im_kernel(const float *__restrict__ dcol, int ldd, int B, int H, int W, int C,
                              float *__restrict__ dx, int ldx, int accumulate) {
    const i64 total = (i64)B * H * W * C;
    const i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = (int)(idx % C);
    const i64 p = idx / C;
    const int xw = (int)(p % W);
    const i64 q = p / W;
    const int yh = (int)(q % H);
    const i64 b = q / H;
    float s = 0.0f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
        const int oy = yh - (tap / 3 - 1), ox = xw - (tap % 3 - 1);
        if (oy >= 0 && oy < H && ox >= 0 && ox < W)
            s = s + dcol[((b * H + oy) * W + ox) * ldd + tap * C + c];
    }
    float *o = dx + p * ldx + c;
    *o = accumulate ? *o + s : s;
}

// ReLU backward: dz = bf16(y > 0 ? dy : 0), and per-group column sums of the
// same masked float values (the bias gradient, first stage).  Block (32, 8)
// over 32 channels; group g = blockIdx.y takes rows g*8 + ty + k*8*G.
__global__ void relu_backward_kernel(const float *__restrict__ dy, int lddy,
                                     const bf16 *__restrict__ y, int ldy, i64 P, int C,
                                     bf16 *__restrict__ dz, int ldz, float *__restrict__ part,
                                     int G) {
    __shared__ float red[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    float s = 0.0f;
    if (c < C) {
        for (i64 r = (i64)blockIdx.y * 8 + threadIdx.y; r < P; r += (i64)8 * G) {
            const float m = __bfloat162float(y[r * ldy + c]) > 0.0f ? dy[r * lddy + c] : 0.0f;
            dz[r * ldz + c] = __float2bfloat16_rn(m);
            s = s + m;
        }
    }
    red[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < C) {
        float t = red[0][threadIdx.x];
        for (int j = 1; j < 8; ++j) t = t + red[j][threadIdx.x];
        part[(i64)blockIdx.y * C + c] = t;
    }
}

// part[g, c] = sum over the rows r of group g of w[r] * x[r, c] (x bf16; a
// null x stands for ones), same grouping as relu_backward_kernel.
__global__ void rowdot_kernel(const float *__restrict__ w, const bf16 *__restrict__ x, int ldx,
                              i64 P, int C, float *__restrict__ part, int G) {
    __shared__ float red[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    float s = 0.0f;
    if (c < C) {
        for (i64 r = (i64)blockIdx.y * 8 + threadIdx.y; r < P; r += (i64)8 * G) {
            const float xv = x ? __bfloat162float(x[r * ldx + c]) : 1.0f;
            s = s + w[r] * xv;
        }
    }
    red[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < C) {
        float t = red[0][threadIdx.x];
        for (int j = 1; j < 8; ++j) t = t + red[j][threadIdx.x];
        part[(i64)blockIdx.y * C + c] = t;
    }
}

// out[c] = sum_g part[g, c] in group order.
__global__ void colsum_final_kernel(const float *__restrict__ part, int G, int C,
                                    float *__restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    float t = part[c];
    for (int g = 1; g < G; ++g) t = t + part[(i64)g * C + c];
    out[c] = t;
}

// 2 x 2 average pool: y[b, i, j, c] = 0.25 * ((x00 + x01) + (x10 + x11)).
__global__ void pool_kernel(const bf16 *__restrict__ x, int ldx, int B, int H, int W, int C,
                            bf16 *__restrict__ y, int ldy) {
    const int h = H / 2, w = W / 2;
    const i64 total = (i64)B * h * w * C;
    const i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = (int)(idx % C);
    const i64 q = idx / C;
    const int j = (int)(q % w);
    const i64 t = q / w;
    const int i = (int)(t % h);
    const i64 b = t / h;
    const i64 r = (b * H + 2 * i) * W + 2 * j;
    const float a = __bfloat162float(x[r * ldx + c]) + __bfloat162float(x[(r + 1) * ldx + c]);
    const float d =
        __bfloat162float(x[(r + W) * ldx + c]) + __bfloat162float(x[(r + W + 1) * ldx + c]);
    y[q * ldy + c] = __float2bfloat16_rn(0.25f * (a + d));
}

__global__ void pool_backward_kernel(const float *__restrict__ dy, int lddy, int B, int H, int W,
                                     int C, float *__restrict__ dx, int ldx, int accumulate) {
    const i64 total = (i64)B * H * W * C;
    const i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = (int)(idx % C);
    const i64 p = idx / C;
    const int xw = (int)(p % W);
    const i64 q = p / W;
    const int yh = (int)(q % H);
    const i64 b = q / H;
    const float g = 0.25f * dy[((b * (H / 2) + yh / 2) * (W / 2) + xw / 2) * lddy + c];
    float *o = dx + p * ldx + c;
    *o = accumulate ? *o + g : g;
}

// Nearest 2x upsample of an H x W map.
__global__ void upsample_kernel(const bf16 *__restrict__ x, int ldx, int B, int H, int W, int C,
                                bf16 *__restrict__ y, int ldy) {
    const i64 total = (i64)B * 4 * H * W * C;
    const i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = (int)(idx % C);
    const i64 q = idx / C;
    const int j = (int)(q % (2 * W));
    const i64 t = q / (2 * W);
    const int i = (int)(t % (2 * H));
    const i64 b = t / (2 * H);
    y[q * ldy + c] = x[((b * H + i / 2) * W + j / 2) * ldx + c];
}

__global__ void upsample_backward_kernel(const float *__restrict__ dy, int lddy, int B, int H,
                                         int W, int C, float *__restrict__ dx, int ldx,
                                         int accumulate) {
    const i64 total = (i64)B * H * W * C;
    const i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = (int)(idx % C);
    const i64 p = idx / C;
    const int j = (int)(p % W);
    const i64 t = p / W;
    const int i = (int)(t % H);
    const i64 b = t / H;
    const i64 r = (b * 2 * H + 2 * i) * (2 * W) + 2 * j;
    const float g = (dy[r * lddy + c] + dy[(r + 1) * lddy + c]) +
                    (dy[(r + 2 * W) * lddy + c] + dy[(r + 2 * W + 1) * lddy + c]);
    float *o = dx + p * ldx + c;
    *o = accumulate ? *o + g : g;
}

// Transmission head: feat[b, c] = mean over the npix pixels of x[b, :, c];
// out[b, k] = bl[k] + sum_c feat[b, c] * Wl[k, c].  One block per instance.
__global__ void gap_linear_kernel(const bf16 *__restrict__ x, int ldx, int npix, int C,
                                  const float *__restrict__ Wl, const float *__restrict__ bl,
                                  int K, float *__restrict__ feat, float *__restrict__ out) {
    extern __shared__ float sf[];
    const int b = blockIdx.x;
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        float s = 0.0f;
        for (int p = 0; p < npix; ++p) s = s + __bfloat162float(x[((i64)b * npix + p) * ldx + c]);
        const float f = s / (float)npix;
        sf[c] = f;
        feat[(i64)b * C + c] = f;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        float s = bl[k];
        for (int c = 0; c < C; ++c) s = s + sf[c] * Wl[(i64)k * C + c];
        out[(i64)b * K + k] = s;
    }
}

// dWl[k, c] = sum_b dout[b, k] * feat[b, c]; dbl[k] = sum_b dout[b, k].
__global__ void gap_linear_wgrad_kernel(const float *__restrict__ dout,
                                        const float *__restrict__ feat, int B, int C, int K,
                                        float *__restrict__ dWl, float *__restrict__ dbl) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= K * C) return;
    const int k = idx / C, c = idx % C;
    float s = 0.0f, t = 0.0f;
    for (int b = 0; b < B; ++b) {
        s = s + dout[(i64)b * K + k] * feat[(i64)b * C + c];
        t = t + dout[(i64)b * K + k];
    }
    dWl[idx] = s;
    if (c == 0) dbl[k] = t;
}

// dx[b, p, c] (+)= (sum_k dout[b, k] * Wl[k, c]) / npix.
__global__ void gap_linear_dgrad_kernel(const float *__restrict__ dout,
                                        const float *__restrict__ Wl, int B, int npix, int C,
                                        int K, float *__restrict__ dx, int ldx, int accumulate) {
    const i64 total = (i64)B * npix * C;
    const i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = (int)(idx % C);
    const i64 p = idx / C;
    const i64 b = p / npix;
    float g = 0.0f;
    for (int k = 0; k < K; ++k) g = g + dout[b * K + k] * Wl[(i64)k * C + c];
    g = g / (float)npix;
    float *o = dx + p * ldx + c;
    *o = accumulate ? *o + g : g;
}

// Gradient-map head (1 x 1 convolution to one channel): out[p] = bg +
// sum_c x[p, c] * wg[c].
__global__ void head_kernel(const bf16 *__restrict__ x, int ldx, i64 P, int C,
                            const float *__restrict__ wg, const float *__restrict__ bg,
                            float *__restrict__ out) {
    const i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (p >= P) return;
    float s = bg[0];
    for (int c = 0; c < C; ++c) s = s + __bfloat162float(x[p * ldx + c]) * wg[c];
    out[p] = s;
}

__global__ void head_dgrad_kernel(const float *__restrict__ dout, i64 P, int C,
                                  const float *__restrict__ wg, float *__restrict__ dx, int ldx) {
    const i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= P * C) return;
    const int c = (int)(idx % C);
    const i64 p = idx / C;
    dx[p * ldx + c] = dout[p] * wg[c];
}

// Squared-error loss term: grad[i] = scale * 2 * (pred[i] - target[i]);
// part[block] = sum of (pred - target)^2 over the block's elements.
__global__ void mse_kernel(const float *__restrict__ pred, const float *__restrict__ target,
                           i64 n, float scale, float *__restrict__ grad,
                           float *__restrict__ part) {
    __shared__ float red[256];
    const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    float d2 = 0.0f;
    if (i < n) {
        const float d = pred[i] - target[i];
        grad[i] = scale * (2.0f * d);
        d2 = d * d;
    }
    red[threadIdx.x] = d2;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Adam (Kingma & Ba 2015) with bias corrections c1 = 1 - b1^t, c2 = 1 - b2^t.
__global__ void adam_kernel(float *__restrict__ w, const float *__restrict__ g,
                            float *__restrict__ m, float *__restrict__ v, i64 n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
    const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * (gi * gi);
    m[i] = mi;
    v[i] = vi;
    w[i] = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// bf16 copies of a float32 [cout, kw] weight: wb [cout, ldw] and its
// transpose wt [kw, cout].
__global__ void cast_weights_kernel(const float *__restrict__ w, int cout, int kw,
                                    bf16 *__restrict__ wb, int ldw, bf16 *__restrict__ wt) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= cout * kw) return;
    const int co = idx / kw, k = idx % kw;
    const bf16 v = __float2bfloat16_rn(w[idx]);
    wb[(i64)co * ldw + k] = v;
    if (wt) wt[(i64)k * cout + co] = v;
}

// out[m, n] (or out[n, m] when transpose) = sum_z part[z][m, n], z ascending.
__global__ void splitk_reduce_kernel(const float *__restrict__ part, int splits, i64 stride,
                                     int M, int N, int ldp, float *__restrict__ out, int ldo,
                                     int transpose) {
    const i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= (i64)M * N) return;
    const int n = (int)(idx % N), m = (int)(idx / N);
    float s = part[(i64)m * ldp + n];
    for (int z = 1; z < splits; ++z) s = s + part[z * stride + (i64)m * ldp + n];
    if (transpose)
        out[(i64)n * ldo + m] = s;
    else
        out[(i64)m * ldo + n] = s;
}

__global__ void to_bf16_kernel(const float *__restrict__ x, bf16 *__restrict__ y, i64 n) {
    const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

// ---------------------------------------------------------------- host side
static inline unsigned nblocks(i64 n, int threads) {
    return (unsigned)((n + threads - 1) / threads);
}

static inline cudaStream_t st(void *s) { return (cudaStream_t)s; }

static bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

template <int BN, bool SW>
static int launch_gemm(const fdtd_sg_gemm_args *g, int splits, int per, int nchunks,
                       cudaStream_t stream) {
    using CF = GemmCfg<BN>;
    // the shared-memory opt-in is per device: set it once on each
    static std::mutex mu;
    static bool ready[64] = {};
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err == cudaSuccess) {
        std::lock_guard<std::mutex> lock(mu);
        if (dev < 0 || dev >= 64 || !ready[dev]) {
            err = cudaFuncSetAttribute(gemm_kernel<BN, SW>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, CF::SMEM);
            if (err == cudaSuccess && dev >= 0 && dev < 64) ready[dev] = true;
        }
    }
    if (err != cudaSuccess) {
        set_error("fdtd_sg_gemm: %s", cudaGetErrorString(err));
        return FDTD_ERR_CUDA;
    }
    CUtensorMap ta, tb;
    int rc = get_encoder();
    if (rc) return rc;
    const cuuint64_t adims[2] = {(cuuint64_t)g->K, (cuuint64_t)g->M};
    const cuuint64_t astr[1] = {(cuuint64_t)g->lda * 2};
    const cuuint32_t kbox = SW ? BK : 8;
    const cuuint32_t abox[2] = {kbox, BM};
    const cuuint64_t bdims[2] = {(cuuint64_t)g->K, (cuuint64_t)g->N};
    const cuuint64_t bstr[1] = {(cuuint64_t)g->ldb * 2};
    const cuuint32_t bbox[2] = {kbox, BN};
    const CUtensorMapSwizzle swz = SW ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE;
    if ((rc = encode(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, g->A, adims, astr, abox, swz)))
        return rc;
    if ((rc = encode(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, g->B, bdims, bstr, bbox, swz)))
        return rc;
    GemmParams p;
    p.C = g->C;
    p.ldc = g->ldc;
    p.c_bf16 = g->c_bf16;
    p.bias = g->bias;
    p.M = g->M;
    p.N = g->N;
    p.K = g->K;
    p.chunks_per_split = per;
    p.nchunks = nchunks;
    p.split_stride = g->split_stride;
    p.accumulate = g->accumulate;
    p.relu = g->relu;
    dim3 grid((g->N + BN - 1) / BN, (g->M + BM - 1) / BM, splits);
    gemm_kernel<BN, SW><<<grid, 128, CF::SMEM, stream>>>(ta, tb, p);
    return launch_status("fdtd_sg_gemm");
}

}  // namespace sg
}  // namespace wfb

using namespace wfb;
using namespace wfb::sg;

extern "C" {

int fdtd_sg_gemm(const fdtd_sg_gemm_args *g, void *stream) {
    if (!g || !g->A || !g->B || !g->C) {
        set_error("fdtd_sg_gemm: null argument");
        return FDTD_ERR_ARG;
    }
    if (g->M < 1 || g->N < 1 || g->K < 1 || g->lda < g->K || g->ldb < g->K || g->ldc < g->N ||
        (g->lda & 7) || (g->ldb & 7) || !aligned16(g->A) || !aligned16(g->B)) {
        set_error("fdtd_sg_gemm: need M, N, K >= 1, lda, ldb >= K and multiples of 8, ldc >= N, "
                  "16-byte aligned A and B");
        return FDTD_ERR_ARG;
    }
    const int nchunks = (g->K + BK - 1) / BK;
    int splits = g->splits < 1 ? 1 : g->splits;
    if (splits > nchunks) splits = nchunks;
    const int per = (nchunks + splits - 1) / splits;
    splits = (nchunks + per - 1) / per;  // every split holds at least one chunk
    if (splits > 65535) {
        set_error("fdtd_sg_gemm: too many K splits");
        return FDTD_ERR_ARG;
    }
    if (splits > 1 && (g->c_bf16 || g->bias || g->relu || g->accumulate ||
                       g->split_stride < (long long)(g->M - 1) * g->ldc + g->N)) {
        set_error("fdtd_sg_gemm: split K writes plain float32 partials (no bias, relu, "
                  "accumulate) at least M*ldc apart");
        return FDTD_ERR_ARG;
    }
    if (g->c_bf16 && g->accumulate) {
        set_error("fdtd_sg_gemm: accumulate needs a float32 C");
        return FDTD_ERR_ARG;
    }
    if ((long long)((g->M + BM - 1) / BM) > 65535) {
        set_error("fdtd_sg_gemm: M too large");
        return FDTD_ERR_ARG;
    }
    if (g->layout != 0 && g->layout != 1) {
        set_error("fdtd_sg_gemm: layout must be 0 (128-byte swizzle) or 1 (interleaved)");
        return FDTD_ERR_ARG;
    }
    cudaStream_t s = st(stream);
    if (g->layout == 0) {
        if (g->N <= 32) return launch_gemm<32, true>(g, splits, per, nchunks, s);
        if (g->N <= 64) return launch_gemm<64, true>(g, splits, per, nchunks, s);
        return launch_gemm<128, true>(g, splits, per, nchunks, s);
    }
    if (g->N <= 32) return launch_gemm<32, false>(g, splits, per, nchunks, s);
    if (g->N <= 64) return launch_gemm<64, false>(g, splits, per, nchunks, s);
    return launch_gemm<128, false>(g, splits, per, nchunks, s);
}

int fdtd_sg_gemm_splits(const fdtd_sg_gemm_args *g) {
    if (!g || g->K < 1) return 0;
    const int nchunks = (g->K + BK - 1) / BK;
    int splits = g->splits < 1 ? 1 : g->splits;
    if (splits > nchunks) splits = nchunks;
    const int per = (nchunks + splits - 1) / splits;
    return (nchunks + per - 1) / per;
}

int fdtd_sg_status(int *out, int reset) {
    if (!out) {
        set_error("fdtd_sg_status: null out");
        return FDTD_ERR_ARG;
    }
    cudaError_t e = cudaMemcpyFromSymbol(out, g_status, sizeof(int));
    if (e == cudaSuccess && reset) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(g_status, &zero, sizeof(int));
    }
    if (e != cudaSuccess) {
        set_error("fdtd_sg_status: %s", cudaGetErrorString(e));
        return FDTD_ERR_CUDA;
    }
    return FDTD_OK;
}

int fdtd_sg_im2col(const void *x, int ldx, int B, int H, int W, int C, void *col, int ldcol,
                   void *stream) {
    if (!x || !col || B < 1 || H < 1 || W < 1 || C < 1 || ldx < C || ldcol < 9 * C) {
        set_error("fdtd_sg_im2col: bad argument");
        return FDTD_ERR_ARG;
    }
    const bf16 *xp = (const bf16 *)x;
    bf16 *cp = (bf16 *)col;
    if ((C & 7) == 0 && (ldx & 7) == 0 && (ldcol & 7) == 0 && aligned16(x) && aligned16(col)) {
        const i64 n = (i64)B * H * W * 9 * (C / 8);
        im2col_vec_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>(xp, ldx, B, H, W, C, cp,
                                                                    ldcol);
    } else {
        const i64 n = (i64)B * H * W * 9 * C;
        im2col_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>(xp, ldx, B, H, W, C, cp, ldcol);
    }
    return launch_status("fdtd_sg_im2col");
}

int fdtd_sg_transpose(const void *src, int lds, long long rows, int cols, void *dst,
                      long long ldd, void *stream) {
    if (!src || !dst || rows < 1 || cols < 1 || lds < cols || ldd < rows) {
        set_error("fdtd_sg_transpose: bad argument");
        return FDTD_ERR_ARG;
    }
    if ((rows + 31) / 32 > 0x7fffffffLL || (cols + 31) / 32 > 65535) {
        set_error("fdtd_sg_transpose: matrix too large");
        return FDTD_ERR_ARG;
    }
    dim3 grid((unsigned)((rows + 31) / 32), (unsigned)((cols + 31) / 32));
    transpose_kernel<<<grid, dim3(32, 8), 0, st(stream)>>>((const bf16 *)src, lds, rows, cols,
                                                           (bf16 *)dst, ldd);
    return launch_status("fdtd_sg_transpose");
}

int fdtd_sg_col2im(const float *dcol, int ldd, int B, int H, int W, int C, float *dx, int ldx,
                   int accumulate, void *stream) {
    if (!dcol || !dx || B < 1 || H < 1 || W < 1 || C < 1 || ldd < 9 * C || ldx < C) {
        set_error("fdtd_sg_col2im: bad argument");
        return FDTD_ERR_ARG;
    }
    const i64 n = (i64)B * H * W * C;
    col2im_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>(dcol, ldd, B, H, W, C, dx, ldx,
                                                            accumulate);
    return launch_status("fdtd_sg_col2im");
}

// Row groups of the two-stage column reductions: one group per 256 rows, at
// most SG_GROUPS_MAX (the scratch holds SG_GROUPS_MAX * C floats).
#define SG_GROUPS_MAX 1024
static int sg_groups(long long P) {
    long long g = (P + 255) / 256;
    return (int)(g < 1 ? 1 : (g > SG_GROUPS_MAX ? SG_GROUPS_MAX : g));
}

int fdtd_sg_relu_backward(const float *dy, int lddy, const void *y, int ldy, long long P, int C,
                          void *dz, int ldz, float *bias_grad, float *scratch, void *stream) {
    if (!dy || !y || !dz || !bias_grad || !scratch || P < 1 || C < 1 || lddy < C || ldy < C ||
        ldz < C) {
        set_error("fdtd_sg_relu_backward: bad argument");
        return FDTD_ERR_ARG;
    }
    const int G = sg_groups(P);
    dim3 grid((C + 31) / 32, G);
    relu_backward_kernel<<<grid, dim3(32, 8), 0, st(stream)>>>(
        dy, lddy, (const bf16 *)y, ldy, P, C, (bf16 *)dz, ldz, scratch, G);
    colsum_final_kernel<<<nblocks(C, 128), 128, 0, st(stream)>>>(scratch, G, C, bias_grad);
    return launch_status("fdtd_sg_relu_backward");
}

int fdtd_sg_pool(const void *x, int ldx, int B, int H, int W, int C, void *y, int ldy,
                 void *stream) {
    if (!x || !y || B < 1 || H < 2 || W < 2 || (H & 1) || (W & 1) || C < 1 || ldx < C ||
        ldy < C) {
        set_error("fdtd_sg_pool: bad argument (H and W even)");
        return FDTD_ERR_ARG;
    }
    const i64 n = (i64)B * (H / 2) * (W / 2) * C;
    pool_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>((const bf16 *)x, ldx, B, H, W, C,
                                                         (bf16 *)y, ldy);
    return launch_status("fdtd_sg_pool");
}

int fdtd_sg_pool_backward(const float *dy, int lddy, int B, int H, int W, int C, float *dx,
                          int ldx, int accumulate, void *stream) {
    if (!dy || !dx || B < 1 || H < 2 || W < 2 || (H & 1) || (W & 1) || C < 1 || lddy < C ||
        ldx < C) {
        set_error("fdtd_sg_pool_backward: bad argument (H and W even)");
        return FDTD_ERR_ARG;
    }
    const i64 n = (i64)B * H * W * C;
    pool_backward_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>(dy, lddy, B, H, W, C, dx, ldx,
                                                                   accumulate);
    return launch_status("fdtd_sg_pool_backward");
}

int fdtd_sg_upsample(const void *x, int ldx, int B, int H, int W, int C, void *y, int ldy,
                     void *stream) {
    if (!x || !y || B < 1 || H < 1 || W < 1 || C < 1 || ldx < C || ldy < C) {
        set_error("fdtd_sg_upsample: bad argument");
        return FDTD_ERR_ARG;
    }
    const i64 n = (i64)B * 4 * H * W * C;
    upsample_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>((const bf16 *)x, ldx, B, H, W, C,
                                                             (bf16 *)y, ldy);
    return launch_status("fdtd_sg_upsample");
}

int fdtd_sg_upsample_backward(const float *dy, int lddy, int B, int H, int W, int C, float *dx,
                              int ldx, int accumulate, void *stream) {
    if (!dy || !dx || B < 1 || H < 1 || W < 1 || C < 1 || lddy < C || ldx < C) {
        set_error("fdtd_sg_upsample_backward: bad argument");
        return FDTD_ERR_ARG;
    }
    const i64 n = (i64)B * H * W * C;
    upsample_backward_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>(dy, lddy, B, H, W, C, dx,
                                                                       ldx, accumulate);
    return launch_status("fdtd_sg_upsample_backward");
}

int fdtd_sg_gap_linear(const void *x, int ldx, int B, int npix, int C, const float *Wl,
                       const float *bl, int K, float *feat, float *out, void *stream) {
    if (!x || !Wl || !bl || !feat || !out || B < 1 || npix < 1 || C < 1 || C > 4096 || K < 1 ||
        ldx < C) {
        set_error("fdtd_sg_gap_linear: bad argument");
        return FDTD_ERR_ARG;
    }
    gap_linear_kernel<<<B, 256, C * sizeof(float), st(stream)>>>((const bf16 *)x, ldx, npix, C,
                                                                 Wl, bl, K, feat, out);
    return launch_status("fdtd_sg_gap_linear");
}

int fdtd_sg_gap_linear_backward(const float *dout, const float *feat, const float *Wl, int B,
                                int npix, int C, int K, float *dWl, float *dbl, float *dx,
                                int ldx, int accumulate, void *stream) {
    if (!dout || !feat || !Wl || !dWl || !dbl || !dx || B < 1 || npix < 1 || C < 1 || K < 1 ||
        ldx < C) {
        set_error("fdtd_sg_gap_linear_backward: bad argument");
        return FDTD_ERR_ARG;
    }
    gap_linear_wgrad_kernel<<<nblocks((i64)K * C, 256), 256, 0, st(stream)>>>(dout, feat, B, C,
                                                                              K, dWl, dbl);
    const i64 n = (i64)B * npix * C;
    gap_linear_dgrad_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>(dout, Wl, B, npix, C, K, dx,
                                                                      ldx, accumulate);
    return launch_status("fdtd_sg_gap_linear_backward");
}

int fdtd_sg_head(const void *x, int ldx, long long P, int C, const float *wg, const float *bg,
                 float *out, void *stream) {
    if (!x || !wg || !bg || !out || P < 1 || C < 1 || ldx < C) {
        set_error("fdtd_sg_head: bad argument");
        return FDTD_ERR_ARG;
    }
    head_kernel<<<nblocks(P, 256), 256, 0, st(stream)>>>((const bf16 *)x, ldx, P, C, wg, bg, out);
    return launch_status("fdtd_sg_head");
}

int fdtd_sg_head_backward(const float *dout, const void *x, int ldx, long long P, int C,
                          const float *wg, float *dx, int lddx, float *dwg, float *dbg,
                          float *scratch, void *stream) {
    if (!dout || !x || !wg || !dx || !dwg || !dbg || !scratch || P < 1 || C < 1 || ldx < C ||
        lddx < C) {
        set_error("fdtd_sg_head_backward: bad argument");
        return FDTD_ERR_ARG;
    }
    cudaStream_t s = st(stream);
    const int G = sg_groups(P);
    head_dgrad_kernel<<<nblocks(P * C, 256), 256, 0, s>>>(dout, P, C, wg, dx, lddx);
    rowdot_kernel<<<dim3((C + 31) / 32, G), dim3(32, 8), 0, s>>>(dout, (const bf16 *)x, ldx, P,
                                                                  C, scratch, G);
    colsum_final_kernel<<<nblocks(C, 128), 128, 0, s>>>(scratch, G, C, dwg);
    rowdot_kernel<<<dim3(1, G), dim3(32, 8), 0, s>>>(dout, nullptr, 0, P, 1, scratch, G);
    colsum_final_kernel<<<1, 128, 0, s>>>(scratch, G, 1, dbg);
    return launch_status("fdtd_sg_head_backward");
}

int fdtd_sg_mse(const float *pred, const float *target, long long n, float scale, float *grad,
                float *partial, void *stream) {
    if (!pred || !target || !grad || !partial || n < 1) {
        set_error("fdtd_sg_mse: bad argument");
        return FDTD_ERR_ARG;
    }
    mse_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>(pred, target, n, scale, grad, partial);
    return launch_status("fdtd_sg_mse");
}

int fdtd_sg_adam(float *w, const float *g, float *m, float *v, long long n, float lr, float b1,
                 float b2, float eps, int step, void *stream) {
    if (!w || !g || !m || !v || n < 1 || step < 1) {
        set_error("fdtd_sg_adam: bad argument");
        return FDTD_ERR_ARG;
    }
    const float c1 = (float)(1.0 - pow((double)b1, step));
    const float c2 = (float)(1.0 - pow((double)b2, step));
    adam_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return launch_status("fdtd_sg_adam");
}

int fdtd_sg_cast_weights(const float *w, int cout, int kw, void *wb, int ldw, void *wt,
                         void *stream) {
    if (!w || !wb || cout < 1 || kw < 1 || ldw < kw) {
        set_error("fdtd_sg_cast_weights: bad argument");
        return FDTD_ERR_ARG;
    }
    cast_weights_kernel<<<nblocks((i64)cout * kw, 256), 256, 0, st(stream)>>>(
        w, cout, kw, (bf16 *)wb, ldw, (bf16 *)wt);
    return launch_status("fdtd_sg_cast_weights");
}

int fdtd_sg_splitk_reduce(const float *part, int splits, long long stride, int M, int N, int ldp,
                          float *out, int ldo, int transpose, void *stream) {
    if (!part || !out || splits < 1 || M < 1 || N < 1 || ldp < N ||
        (splits > 1 && stride < (long long)(M - 1) * ldp + N) || ldo < (transpose ? M : N)) {
        set_error("fdtd_sg_splitk_reduce: bad argument");
        return FDTD_ERR_ARG;
    }
    splitk_reduce_kernel<<<nblocks((i64)M * N, 256), 256, 0, st(stream)>>>(
        part, splits, stride, M, N, ldp, out, ldo, transpose);
    return launch_status("fdtd_sg_splitk_reduce");
}

int fdtd_sg_to_bf16(const float *x, void *y, long long n, void *stream) {
    if (!x || !y || n < 1) {
        set_error("fdtd_sg_to_bf16: bad argument");
        return FDTD_ERR_ARG;
    }
    to_bf16_kernel<<<nblocks(n, 256), 256, 0, st(stream)>>>(x, (bf16 *)y, n);
    return launch_status("fdtd_sg_to_bf16");
}

}  // extern "C"
