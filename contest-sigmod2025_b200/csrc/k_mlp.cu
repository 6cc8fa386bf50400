// Kernels of the learned cardinality estimator: a three-layer MLP (features
// -> 256 -> 256 -> 1, ReLU) with BF16 weights and FP32 accumulation, trained
// on the device. No reference counterpart: it stands in for the reference's
// sampling estimator (engine/query/QueryPlan.cpp:719-746) inside join
// ordering.
//
// The matrix products run on the tensor cores through mma.sync m16n8k16
// (BF16 in, FP32 accumulate): a CTA of four warps computes a 64 x 64 tile of
// C = A B, staging 64 x 32 slices of A and B in shared memory (k contiguous,
// rows padded to 80 bytes so ldmatrix reads are free of bank conflicts),
// each warp a 32 x 32 quarter as 2 x 4 MMA tiles. A and B may each be stored
// with either dimension contiguous (the backward pass reads the forward
// operands transposed); the fused epilogues are bias + ReLU (forward), the
// ReLU mask of the layer's activation (backward) and a plain FP32 store
// (weight gradients).
#include "launch.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace bj {
namespace {

constexpr int kBM = 64, kBN = 64, kBK = 32, kPad = 8;
constexpr int kLd = kBK + kPad;  // shared row stride in bf16 elements (80 bytes)

__device__ __forceinline__ float bf2f(uint16_t v) { return __uint_as_float(uint32_t(v) << 16); }
__device__ __forceinline__ uint16_t f2bf(float f) {
    __nv_bfloat16 b = __float2bfloat16_rn(f);
    return *reinterpret_cast<uint16_t*>(&b);
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3, const void* p) {
    const uint32_t a = uint32_t(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(a));
}

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Loads the 64 x 32 slice [r0, r0+64) x [k0, k0+32) of an operand into s[r][k]
// (rows beyond `rows` are zero). Element (r, k) is at p[r * rs + k * ks];
// one of rs, ks is 1 and the other a multiple of 8, so 16-byte loads run
// along the contiguous dimension.
__device__ __forceinline__ void load_slice(uint16_t (*s)[kLd], const uint16_t* p, long rs, long ks, int r0, int rows,
                                           int k0) {
    const int t = threadIdx.x;
    if (ks == 1) {
        // 64 rows x 4 chunks of 8 k: two chunks per thread.
        for (int c = t; c < kBM * (kBK / 8); c += blockDim.x) {
            const int r = c >> 2, kc = (c & 3) * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (r0 + r < rows) v = *reinterpret_cast<const uint4*>(p + long(r0 + r) * rs + (k0 + kc));
            *reinterpret_cast<uint4*>(&s[r][kc]) = v;
        }
    } else {
        // 32 k x 8 chunks of 8 rows: two chunks per thread, stored transposed.
        for (int c = t; c < kBK * (kBM / 8); c += blockDim.x) {
            const int k = c >> 3, rc = (c & 7) * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (r0 + rc < rows) v = *reinterpret_cast<const uint4*>(p + long(k0 + k) * ks + (r0 + rc));
            const uint16_t* e = reinterpret_cast<const uint16_t*>(&v);
#pragma unroll
            for (int i = 0; i < 8; i++) s[rc + i][k] = (r0 + rc + i < rows) ? e[i] : uint16_t(0);
        }
    }
}

__global__ void __launch_bounds__(128) k_gemm_bf16(GemmArgs g) {
    __shared__ __align__(16) uint16_t sA[kBM][kLd];
    __shared__ __align__(16) uint16_t sB[kBN][kLd];
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4] = {};
    for (int k0 = 0; k0 < g.K; k0 += kBK) {
        load_slice(sA, g.A, g.a_rs, g.a_cs, m0, g.M, k0);
        // B(k, n): rows of the slice are n, so the "row stride" is b_cs.
        load_slice(sB, g.B, g.b_cs, g.b_rs, n0, g.N, k0);
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBK; kk += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; i++)
                ldmatrix_x4(a[i][0], a[i][1], a[i][2], a[i][3], &sA[wm + i * 16 + (lane & 15)][kk + (lane >> 4) * 8]);
#pragma unroll
            for (int j = 0; j < 4; j += 2)
                ldmatrix_x4(b[j][0], b[j][1], b[j + 1][0], b[j + 1][1],
                            &sB[wn + j * 8 + (lane & 7) + (lane >> 4) * 8][kk + ((lane >> 3) & 1) * 8]);
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], a[i], b[j][0], b[j][1]);
        }
        __syncthreads();
    }
    // Epilogue: acc[i][j] covers rows wm + 16 i + lane / 4 (+ 8) and columns
    // wn + 8 j + 2 (lane % 4) (+ 1).
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int m = m0 + wm + i * 16 + (lane >> 2) + h * 8;
                const int n = n0 + wn + j * 8 + (lane & 3) * 2;
                if (m >= g.M || n >= g.N) continue;
                float v0 = acc[i][j][2 * h], v1 = acc[i][j][2 * h + 1];
                const long o = long(m) * g.ldc + n;
                if (g.epi == kEpiBiasRelu) {
                    v0 = fmaxf(v0 + bf2f(g.bias[n]), 0.f);
                    v1 = fmaxf(v1 + bf2f(g.bias[n + 1]), 0.f);
                } else if (g.epi == kEpiReluMask) {
                    if (bf2f(g.mask[o]) <= 0.f) v0 = 0.f;
                    if (bf2f(g.mask[o + 1]) <= 0.f) v1 = 0.f;
                }
                if (g.epi == kEpiStoreF32) {
                    *reinterpret_cast<float2*>(g.Cf + o) = make_float2(v0, v1);
                } else {
                    const uint32_t packed = uint32_t(f2bf(v0)) | (uint32_t(f2bf(v1)) << 16);
                    *reinterpret_cast<uint32_t*>(g.Cb + o) = packed;
                }
            }
}

// Output layer and its gradient, one CTA of 256 threads per batch row:
// y = H2 . w3 + b3; with targets, loss += (y - t)^2, dy = 2 (y - t) / n_real,
// dH2 = bf16(dy * w3 * [H2 > 0]); rows at or beyond n_real get dy = 0.
__global__ void __launch_bounds__(256) k_mlp_head(MlpHeadArgs a) {
    const int m = blockIdx.x, n = threadIdx.x;
    const float h = bf2f(a.H2[long(m) * kMlpHidden + n]);
    const float w = bf2f(a.w3[n]);
    float p = h * w;
    for (int o = 16; o > 0; o >>= 1) p += __shfl_down_sync(0xffffffffu, p, o);
    __shared__ float part[8];
    __shared__ float dy_s;
    if ((n & 31) == 0) part[n >> 5] = p;
    __syncthreads();
    if (n == 0) {
        float y = bf2f(a.b3[0]);
        for (int i = 0; i < 8; i++) y += part[i];
        if (a.y) a.y[m] = y;
        float dy = 0.f;
        if (a.t && m < a.n_real) {
            const float d = y - a.t[m];
            atomicAdd(a.loss, d * d);
            dy = 2.f * d / float(a.n_real);
        }
        if (a.dy) a.dy[m] = dy;
        dy_s = dy;
    }
    __syncthreads();
    if (a.dH2) a.dH2[long(m) * kMlpHidden + n] = f2bf(h > 0.f ? dy_s * w : 0.f);
}

// Column sums: out[n] = sum over rows m of X[m][n] (bf16 X, or the product of
// bf16 H2 and fp32 dy when dy is given). One thread per column, rows split
// over blockIdx.y and combined with atomics (out zero before).
__global__ void k_colsum(const uint16_t* X, const float* dy, int rows, int cols, float* out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= cols) return;
    const int per = (rows + gridDim.y - 1) / gridDim.y;
    const int r0 = blockIdx.y * per, r1 = min(rows, r0 + per);
    float s = 0.f;
    for (int m = r0; m < r1; m++) s += bf2f(X[long(m) * cols + n]) * (dy ? dy[m] : 1.f);
    if (r1 > r0) atomicAdd(&out[n], s);
}

__global__ void k_sum(const float* v, int n, float* out) {
    float s = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// Adam (Kingma & Ba 2015) over every parameter; the BF16 copy the products
// read is refreshed from the FP32 master.
__global__ void k_adam(AdamArgs a) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < a.n; i += long(gridDim.x) * blockDim.x) {
        const float g = a.grad[i];
        const float m = a.beta1 * a.m[i] + (1.f - a.beta1) * g;
        const float v = a.beta2 * a.v[i] + (1.f - a.beta2) * g * g;
        a.m[i] = m;
        a.v[i] = v;
        const float mh = m / a.bc1, vh = v / a.bc2;
        const float p = a.w[i] - a.lr * mh / (sqrtf(vh) + a.eps);
        a.w[i] = p;
        a.wb[i] = f2bf(p);
    }
}

__global__ void k_f32_to_bf16(const float* in, uint16_t* out, long n) {
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        out[i] = f2bf(in[i]);
}

// Gathers rows idx[0..n) of a bf16 matrix (cols wide) into dst, and their
// targets; rows of dst beyond n up to n_pad are zero.
__global__ void k_gather_rows(const uint16_t* src, const float* tsrc, const uint32_t* idx, int n, int n_pad, int cols,
                              uint16_t* dst, float* tdst) {
    const int r = blockIdx.x;
    if (r >= n_pad) return;
    const uint4* s = r < n ? reinterpret_cast<const uint4*>(src + long(idx[r]) * cols) : nullptr;
    uint4* d = reinterpret_cast<uint4*>(dst + long(r) * cols);
    for (int c = threadIdx.x; c < cols / 8; c += blockDim.x) d[c] = s ? s[c] : make_uint4(0, 0, 0, 0);
    if (threadIdx.x == 0 && tdst) tdst[r] = r < n ? tsrc[idx[r]] : 0.f;
}

} // namespace

int gemm_bf16(const GemmArgs& g, cudaStream_t st) {
    dim3 grid((g.N + kBN - 1) / kBN, (g.M + kBM - 1) / kBM);
    if (!grid.x || !grid.y) return 0;
    k_gemm_bf16<<<grid, 128, 0, st>>>(g);
    return 1;
}

int mlp_head(const MlpHeadArgs& a, int rows, cudaStream_t st) {
    if (rows <= 0) return 0;
    k_mlp_head<<<rows, kMlpHidden, 0, st>>>(a);
    return 1;
}

int colsum(const uint16_t* X, const float* dy, int rows, int cols, float* out, cudaStream_t st) {
    dim3 grid((cols + 127) / 128, std::max(1, std::min(64, rows / 32)));
    k_colsum<<<grid, 128, 0, st>>>(X, dy, rows, cols, out);
    return 1;
}

int sum_f32(const float* v, int n, float* out, cudaStream_t st) {
    k_sum<<<1, 256, 0, st>>>(v, n, out);
    return 1;
}

int adam_step(const AdamArgs& a, cudaStream_t st) {
    k_adam<<<592, 256, 0, st>>>(a);
    return 1;
}

int f32_to_bf16(const float* in, uint16_t* out, long n, cudaStream_t st) {
    k_f32_to_bf16<<<592, 256, 0, st>>>(in, out, n);
    return 1;
}

int gather_rows(const uint16_t* src, const float* tsrc, const uint32_t* idx, int n, int n_pad, int cols, uint16_t* dst,
                float* tdst, cudaStream_t st) {
    if (n_pad <= 0) return 0;
    k_gather_rows<<<n_pad, 128, 0, st>>>(src, tsrc, idx, n, n_pad, cols, dst, tdst);
    return 1;
}

} // namespace bj
