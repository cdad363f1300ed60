// mlp.cu -- the learned warm start: canonical pair features, a BF16 tensor-core GEMM,
// the MLP's elementwise steps, Adam, and the penalty solver started from a prediction.
//
// The network maps a canonicalised triangle pair (18 coordinates) to the four barycentric
// weights (x0, x1 of P on A; x2, x3 of Q on B) that penaltySolver iterates on
// (penalty.cpp:353-356 starts them at 0.33).  Labels come from the FP64 bfSolver result.
// Matrices are row-major; GEMMs are C = op(A) op(B) in BF16 with FP32 accumulation on
// the tensor cores (mma.sync m16n8k16).
#include <cuda_bf16.h>

#include <algorithm>

#include "internal.h"
#include "tri_learned.cuh"
#include "tri_ref.cuh"

namespace delta {

namespace {

// ---------------------------------------------------------------------------------------
// canonical features and labels
// ---------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __halves2bfloat162(__float2bfloat16(lo), __float2bfloat16(hi));
  return *reinterpret_cast<const uint32_t *>(&v);
}

// Frame of triangle A: origin at its centroid, x along A1-A0, z along its normal, unit
// scale = its longest edge.  Features: the 6 vertices in that frame (18 values).  FP64
// with every operation rounded once (xf64), so the features are reproducible bit for bit;
// ok is false for a degenerate A.
__device__ __forceinline__ void canon_pair(const double *__restrict__ a, const double *__restrict__ b, int64_t ld,
                                           int64_t i, xf64 A[3][3], xf64 B[3][3], float f[18], bool &ok) {
  for (int v = 0; v < 3; ++v)
    for (int k = 0; k < 3; ++k) {
      A[v][k] = xf64(a[(3 * v + k) * ld + i]);
      B[v][k] = xf64(b[(3 * v + k) * ld + i]);
    }
  xf64 c[3], E0[3], E1[3], E2[3], E3[3], nr[3];
  for (int k = 0; k < 3; ++k) {
    c[k] = ((A[0][k] + A[1][k]) + A[2][k]) / xf64(3.0);
    E0[k] = A[1][k] - A[0][k];
    E1[k] = A[2][k] - A[0][k];
    E2[k] = A[2][k] - A[1][k];
    E3[k] = A[0][k] - A[2][k];
  }
  nr[0] = E0[1] * E1[2] - E0[2] * E1[1];
  nr[1] = E0[2] * E1[0] - E0[0] * E1[2];
  nr[2] = E0[0] * E1[1] - E0[1] * E1[0];
  const xf64 l0 = sqrt_(dot3(E0, E0)), l1 = sqrt_(dot3(E2, E2)), l2 = sqrt_(dot3(E3, E3));
  const xf64 ln = sqrt_(dot3(nr, nr));
  xf64 emax = l0;
  if (l1 > emax) emax = l1;
  if (l2 > emax) emax = l2;
  ok = l0 > xf64(0.0) && ln > xf64(0.0);
  xf64 e1[3], e3[3], e2[3];
  for (int k = 0; k < 3; ++k) {
    e1[k] = ok ? E0[k] / l0 : xf64(0.0);
    e3[k] = ok ? nr[k] / ln : xf64(0.0);
  }
  e2[0] = e3[1] * e1[2] - e3[2] * e1[1];
  e2[1] = e3[2] * e1[0] - e3[0] * e1[2];
  e2[2] = e3[0] * e1[1] - e3[1] * e1[0];
  const xf64 s = ok ? xf64(1.0) / emax : xf64(0.0);
  for (int v = 0; v < 6; ++v) {
    const xf64 *X = v < 3 ? A[v] : B[v - 3];
    const xf64 d[3] = {X[0] - c[0], X[1] - c[1], X[2] - c[2]};
    f[3 * v + 0] = (float)(s * dot3(d, e1)).v;
    f[3 * v + 1] = (float)(s * dot3(d, e2)).v;
    f[3 * v + 2] = (float)(s * dot3(d, e3)).v;
  }
}

// Features (rows of 32 BF16, 18 used) and, when P, Q are given, the targets: barycentric
// weights of P on A and Q on B from the 2x2 normal equations; rows with a degenerate
// triangle are marked invalid.
__global__ void k_canon(int64_t n, const double *__restrict__ a, const double *__restrict__ b, int64_t ld,
                        const double *__restrict__ p, const double *__restrict__ q, __nv_bfloat16 *feat,
                        float *target, uint8_t *valid) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  xf64 A[3][3], B[3][3];
  float f[18];
  bool ok;
  canon_pair(a, b, ld, i, A, B, f, ok);
  // the 64-byte row as four 16-byte stores
  uint32_t w[16];
  for (int k = 0; k < 9; ++k) w[k] = pack_bf16(f[2 * k], f[2 * k + 1]);
  for (int k = 9; k < 16; ++k) w[k] = 0u;
  uint4 *row = reinterpret_cast<uint4 *>(feat + 32 * i);
  for (int k = 0; k < 4; ++k) row[k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
  if (p && q) {
    // P = A0 + x0 (A1-A0) + x1 (A2-A0); Q = B0 + x2 (B1-B0) + x3 (B2-B0)
    xf64 x[4];
    for (int t = 0; t < 2; ++t) {
      const xf64(*T)[3] = t == 0 ? A : B;
      const double *src = t == 0 ? p : q;
      xf64 U[3], V[3], W[3];
      for (int k = 0; k < 3; ++k) {
        U[k] = T[1][k] - T[0][k];
        V[k] = T[2][k] - T[0][k];
        W[k] = xf64(src[k * ld + i]) - T[0][k];
      }
      const xf64 uu = dot3(U, U), uv = dot3(U, V), vv = dot3(V, V), wu = dot3(W, U), wv = dot3(W, V);
      const xf64 det = uu * vv - uv * uv;
      if (!(det > xf64(1e-12) * uu * vv)) ok = false;
      x[2 * t] = (wu * vv - wv * uv) / det;
      x[2 * t + 1] = (wv * uu - wu * uv) / det;
    }
    reinterpret_cast<float4 *>(target)[i] = ok ? make_float4((float)x[0].v, (float)x[1].v, (float)x[2].v, (float)x[3].v)
                                               : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (valid) valid[i] = ok ? 1 : 0;
}

// ---------------------------------------------------------------------------------------
// BF16 GEMM on the tensor cores: C[M,N] (+)= op(A)[M,K] op(B)[K,N], FP32 accumulate.
// A is stored [M,K] (trans_a = 0) or [K,M]; B is stored [K,N] (trans_b = 0) or [N,K].
// CTA tile 64x64x32, 4 warps of 32x32, split-K over gridDim.z with FP32 atomics.
// ---------------------------------------------------------------------------------------
constexpr int BM = 64, BN = 64, BK = 32, PAD = 8;

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const __nv_bfloat16 *__restrict__ A, int lda,
                                              int trans_a, const __nv_bfloat16 *__restrict__ B, int ldb, int trans_b,
                                              float *__restrict__ Cm, int ldc, int accumulate, int k_per_split) {
  __shared__ __align__(16) __nv_bfloat16 As[BM][BK + PAD];  // [m][k]
  __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + PAD];  // [n][k]
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kb = blockIdx.z * k_per_split, ke = min(K, kb + k_per_split);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  float acc[2][4][4] = {};
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  for (int k0 = kb; k0 < ke; k0 += BK) {
    for (int e = tid; e < BM * BK; e += 128) {
      const int r = e / BK, c = e % BK, m = m0 + r, k = k0 + c;
      __nv_bfloat16 v = zero;
      if (m < M && k < ke) v = trans_a ? A[(int64_t)k * lda + m] : A[(int64_t)m * lda + k];
      As[r][c] = v;
    }
    for (int e = tid; e < BN * BK; e += 128) {
      const int r = e / BK, c = e % BK, nn = n0 + r, k = k0 + c;
      __nv_bfloat16 v = zero;
      if (nn < N && k < ke) v = trans_b ? B[(int64_t)nn * ldb + k] : B[(int64_t)k * ldb + nn];
      Bs[r][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        const int r = wm + mi * 16 + g;
        af[mi][0] = *reinterpret_cast<const uint32_t *>(&As[r][kk + 2 * t]);
        af[mi][1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][kk + 2 * t]);
        af[mi][2] = *reinterpret_cast<const uint32_t *>(&As[r][kk + 2 * t + 8]);
        af[mi][3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        const int cidx = wn + ni * 8 + g;
        bfr[ni][0] = *reinterpret_cast<const uint32_t *>(&Bs[cidx][kk + 2 * t]);
        bfr[ni][1] = *reinterpret_cast<const uint32_t *>(&Bs[cidx][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) mma_bf16(acc[mi][ni], af[mi], bfr[ni]);
    }
    __syncthreads();
  }
  const bool atomic = gridDim.z > 1 || accumulate;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const int m = m0 + wm + mi * 16 + g + (h >= 2 ? 8 : 0);
        const int nn = n0 + wn + ni * 8 + 2 * t + (h & 1);
        if (m < M && nn < N) {
          float *dst = Cm + (int64_t)m * ldc + nn;
          if (atomic) atomicAdd(dst, acc[mi][ni][h]);
          else *dst = acc[mi][ni][h];
        }
      }
}

// ---------------------------------------------------------------------------------------
// elementwise steps
// ---------------------------------------------------------------------------------------
// GELU, tanh form (Hendrycks & Gimpel 2016), with the hardware tanh (tanh.approx.f32,
// relative error about 2^-11, below the BF16 rounding that follows).
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kGeluK = 0.7978845608028654f;  // sqrt(2/pi)
constexpr float kGeluC = 0.044715f;
__device__ __forceinline__ float gelu(float x) {
  const float u = x * fmaf(kGeluC * kGeluK, x * x, kGeluK);
  const float h = 0.5f * x;
  return fmaf(h, tanh_hw(u), h);
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float x2 = x * x;
  const float th = tanh_hw(x * fmaf(kGeluC * kGeluK, x2, kGeluK));
  return 0.5f * (1.f + th) + 0.5f * x * (1.f - th * th) * kGeluK * fmaf(3.f * kGeluC, x2, 1.f);
}

// Z[M,N] += bias; H = bf16(gelu(Z)) (or bf16(Z) when act == 0); Z keeps the pre-activation.
__global__ void k_bias_act(int64_t M, int N, float *Z, const float *bias, __nv_bfloat16 *H, int act) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M * N) return;
  const float z = Z[e] + bias[e % N];
  Z[e] = z;
  if (H) H[e] = __float2bfloat16(act ? gelu(z) : z);
}

// MSE over valid rows: dY = 2 (Y - T) / n_valid (bf16), loss accumulated into *loss.
__global__ void k_mse(int64_t M, const float *Y, const float *T, const uint8_t *valid, float inv_n,
                      __nv_bfloat16 *dY, float *loss) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (e < M * 4) {
    const bool v = valid[e / 4] != 0;
    const float d = v ? Y[e] - T[e] : 0.f;
    dY[e] = __float2bfloat16(2.f * d * inv_n);
    l = d * d * inv_n;
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l);
}

// dZ = bf16(dH * gelu'(Z))
__global__ void k_act_grad(int64_t M, int N, const float *dH, const float *Z, __nv_bfloat16 *dZ) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M * N) return;
  dZ[e] = __float2bfloat16(dH[e] * gelu_grad(Z[e]));
}

// Row-tiled forms of the three element-wise kernels for N dividing 4 * 256 (N a power of
// two, at most 1024): thread t of a block owns 4 consecutive columns (N4 = N / 4 groups of
// them per row) of rows t / N4, t / N4 + 256 / N4, ..., so a warp moves whole row segments
// with 16-byte loads and the column needs no 64-bit division.  Same arithmetic as the
// scalar kernels above.
__global__ void k_bias_act4(int64_t M, int N4, float *__restrict__ Z, const float *__restrict__ bias,
                            __nv_bfloat16 *__restrict__ H, int act) {
  const int c4 = threadIdx.x % N4, rows = blockDim.x / N4;
  const float b0 = bias[4 * c4], b1 = bias[4 * c4 + 1], b2 = bias[4 * c4 + 2], b3 = bias[4 * c4 + 3];
  for (int64_t m = (int64_t)blockIdx.x * rows + threadIdx.x / N4; m < M; m += (int64_t)gridDim.x * rows) {
    float4 *zp = reinterpret_cast<float4 *>(Z + m * 4 * N4) + c4;
    float4 z = *zp;
    z.x += b0;
    z.y += b1;
    z.z += b2;
    z.w += b3;
    *zp = z;
    if (H) {
      const __nv_bfloat162 h0 = act ? __floats2bfloat162_rn(gelu(z.x), gelu(z.y)) : __floats2bfloat162_rn(z.x, z.y);
      const __nv_bfloat162 h1 = act ? __floats2bfloat162_rn(gelu(z.z), gelu(z.w)) : __floats2bfloat162_rn(z.z, z.w);
      uint2 v;
      v.x = *reinterpret_cast<const uint32_t *>(&h0);
      v.y = *reinterpret_cast<const uint32_t *>(&h1);
      reinterpret_cast<uint2 *>(H + m * 4 * N4)[c4] = v;
    }
  }
}

__global__ void k_act_grad4(int64_t M, int N4, const float *__restrict__ dH, const float *__restrict__ Z,
                            __nv_bfloat16 *__restrict__ dZ) {
  const int c4 = threadIdx.x % N4, rows = blockDim.x / N4;
  for (int64_t m = (int64_t)blockIdx.x * rows + threadIdx.x / N4; m < M; m += (int64_t)gridDim.x * rows) {
    const float4 d = reinterpret_cast<const float4 *>(dH + m * 4 * N4)[c4];
    const float4 z = reinterpret_cast<const float4 *>(Z + m * 4 * N4)[c4];
    const __nv_bfloat162 h0 = __floats2bfloat162_rn(d.x * gelu_grad(z.x), d.y * gelu_grad(z.y));
    const __nv_bfloat162 h1 = __floats2bfloat162_rn(d.z * gelu_grad(z.z), d.w * gelu_grad(z.w));
    uint2 v;
    v.x = *reinterpret_cast<const uint32_t *>(&h0);
    v.y = *reinterpret_cast<const uint32_t *>(&h1);
    reinterpret_cast<uint2 *>(dZ + m * 4 * N4)[c4] = v;
  }
}

// db[n] += column sums of dZ: thread t sums column t % N over rows t / N, t / N + 256 / N,
// ... (a warp reads whole row segments), the block combines its row partials per column
// in shared memory and adds them to db.
__global__ void k_colsum_rows(int64_t M, int N, const __nv_bfloat16 *__restrict__ dZ, float *db) {
  __shared__ float part[256];
  const int c = threadIdx.x % N, rows = blockDim.x / N;
  float s = 0.f;
  for (int64_t m = (int64_t)blockIdx.x * rows + threadIdx.x / N; m < M; m += (int64_t)gridDim.x * rows)
    s += __bfloat162float(dZ[m * N + c]);
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < N) {
    float t = 0.f;
    for (int r = 0; r < rows; ++r) t += part[r * N + threadIdx.x];
    atomicAdd(&db[threadIdx.x], t);
  }
}

// db[n] += sum over rows of dZ[:, n]
__global__ void k_colsum(int64_t M, int N, const __nv_bfloat16 *dZ, float *db) {
  const int n = blockIdx.x;
  float s = 0.f;
  for (int64_t m = threadIdx.x + (int64_t)blockIdx.y * blockDim.x; m < M; m += (int64_t)blockDim.x * gridDim.y)
    s += __bfloat162float(dZ[m * N + n]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ float part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    atomicAdd(&db[n], t);
  }
}

// Adam (Kingma & Ba 2015) on FP32 master weights; refreshes the BF16 copy.
__global__ void k_adam(int64_t n, float *w, const float *g, float *m, float *v, float lr, float b1, float b2,
                       float eps, float c1, float c2, __nv_bfloat16 *wb) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16(wi);
}

__global__ void k_f32_to_bf16(int64_t n, const float *x, __nv_bfloat16 *y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16(x[i]);
}

// ---------------------------------------------------------------------------------------
// fused inference: the four layers on rows of canonical features, one kernel.  Weights
// stay in shared memory for the CTA's lifetime; each warp owns 16 pairs at a time and
// keeps their activations in registers: the FP32 accumulator fragment of one layer
// (m16n8 tiles) is, packed to BF16 pairs, exactly the A fragment (m16k16) of the next.
// The MMAs run in the same order as k_gemm's and the epilogue is k_bias_act's, so the
// output equals the layer-by-layer path bit for bit.
// ---------------------------------------------------------------------------------------
constexpr int kIn = 32, kHid = 128, kOut = 4;
constexpr int64_t kOffW1 = 0, kOffB1 = kOffW1 + kHid * kIn, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
                  kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kHid, kOffW4 = kOffB3 + kHid,
                  kOffB4 = kOffW4 + kOut * kHid, kNumParams = (kOffB4 + kOut + 7) / 8 * 8;
constexpr int kIP = kIn + 8, kHP = kHid + 8;  // padded row pitches (bf16): conflict-free ldmatrix
constexpr int kInferWarps = 8;

struct InferSmem {
  __nv_bfloat16 w1[kHid][kIP];
  __nv_bfloat16 w2[kHid][kHP];
  __nv_bfloat16 w3[kHid][kHP];
  __nv_bfloat16 w4[8][kHP];  // rows 4..7 zero
  float bias[3 * kHid + 8];
};

__device__ __forceinline__ void ldmatrix_x4(uint32_t r[4], const void *row_addr) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(row_addr);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(s));
}
__device__ __forceinline__ void ldmatrix_x2(uint32_t r[2], const void *row_addr) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(row_addr);
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r[0]), "=r"(r[1]) : "r"(s));
}

// acc[NT][4] = H . W^T for 16 rows: H as A fragments a[KS][4] in registers, W rows
// 0..8*NT-1 (row pitch wp) in shared memory, B fragments by ldmatrix (row addresses
// 16-byte aligned: pitches of 80 and 272 bytes, column offsets of 16 bytes).
template <int KS, int NT>
__device__ __forceinline__ void warp_layer(const uint32_t a[KS][4], const __nv_bfloat16 *W, int wp,
                                           float acc[NT][4]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
  // B is stored [n][k]: lanes 0-7 address rows n0..n0+7 at k, 8-15 the same rows at k+8,
  // 16-23 rows n0+8.. at k, 24-31 those at k+8
  const __nv_bfloat16 *brow = W + ((lane & 7) + ((lane >> 4) << 3)) * wp + ((lane >> 3) & 1) * 8;
#pragma unroll
  for (int ks = 0; ks < KS; ++ks) {
    const int kk = 16 * ks;
    if constexpr (NT == 1) {
      uint32_t bf[2];
      ldmatrix_x2(bf, brow + kk);
      mma_bf16(acc[0], a[ks], bf);
    } else {
#pragma unroll
      for (int nt = 0; nt < NT; nt += 2) {
        uint32_t r[4];
        ldmatrix_x4(r, brow + 8 * nt * wp + kk);
        const uint32_t b0[2] = {r[0], r[1]}, b1[2] = {r[2], r[3]};
        mma_bf16(acc[nt], a[ks], b0);
        mma_bf16(acc[nt + 1], a[ks], b1);
      }
    }
  }
}

// GELU(acc + bias) packed to BF16 as the next layer's A fragments: k-tile kt takes output
// n-tiles 2kt (k 0..7) and 2kt+1 (k 8..15); rows g (regs 0, 2) and g+8 (regs 1, 3).
__device__ __forceinline__ void warp_gelu_to_a(const float acc[16][4], const float *bias, uint32_t a[8][4]) {
  const int t = threadIdx.x & 3;
#pragma unroll
  for (int kt = 0; kt < 8; ++kt) {
#pragma unroll
    for (int hlf = 0; hlf < 2; ++hlf) {
      const int nt = 2 * kt + hlf, col = 8 * nt + 2 * t;
      const float b0 = bias[col], b1 = bias[col + 1];
      a[kt][2 * hlf] = pack_bf16(gelu(acc[nt][0] + b0), gelu(acc[nt][1] + b1));
      a[kt][2 * hlf + 1] = pack_bf16(gelu(acc[nt][2] + b0), gelu(acc[nt][3] + b1));
    }
  }
}

__global__ void __launch_bounds__(32 * kInferWarps, 2)
    k_mlp_infer(int64_t n, const __nv_bfloat16 *__restrict__ feat, const float *__restrict__ params,
                const __nv_bfloat16 *__restrict__ wb, float *__restrict__ x0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  InferSmem &sm = *reinterpret_cast<InferSmem *>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // weights (BF16) and biases (FP32) into shared memory, once per CTA
  for (int e = tid; e < kHid * (kIn / 2); e += blockDim.x) {
    const int r = e / (kIn / 2), c = 2 * (e % (kIn / 2));
    *reinterpret_cast<uint32_t *>(&sm.w1[r][c]) = *reinterpret_cast<const uint32_t *>(wb + kOffW1 + r * kIn + c);
  }
  for (int e = tid; e < kHid * (kHid / 2); e += blockDim.x) {
    const int r = e / (kHid / 2), c = 2 * (e % (kHid / 2));
    *reinterpret_cast<uint32_t *>(&sm.w2[r][c]) = *reinterpret_cast<const uint32_t *>(wb + kOffW2 + r * kHid + c);
    *reinterpret_cast<uint32_t *>(&sm.w3[r][c]) = *reinterpret_cast<const uint32_t *>(wb + kOffW3 + r * kHid + c);
  }
  for (int e = tid; e < 8 * (kHid / 2); e += blockDim.x) {
    const int r = e / (kHid / 2), c = 2 * (e % (kHid / 2));
    *reinterpret_cast<uint32_t *>(&sm.w4[r][c]) =
        r < kOut ? *reinterpret_cast<const uint32_t *>(wb + kOffW4 + r * kHid + c) : 0u;
  }
  for (int e = tid; e < kHid; e += blockDim.x) {
    sm.bias[e] = params[kOffB1 + e];
    sm.bias[kHid + e] = params[kOffB2 + e];
    sm.bias[2 * kHid + e] = params[kOffB3 + e];
  }
  if (tid < 8) sm.bias[3 * kHid + tid] = tid < kOut ? params[kOffB4 + tid] : 0.f;
  __syncthreads();

  const int g = lane >> 2, t = lane & 3;
  const int64_t tiles = (n + 15) / 16;
  for (int64_t tile = (int64_t)blockIdx.x * kInferWarps + warp; tile < tiles;
       tile += (int64_t)gridDim.x * kInferWarps) {
    const int64_t row0 = tile * 16;
    // layer-1 A fragments straight from the feature rows (32 BF16 = 16 words per row)
    uint32_t a1[2][4];
    {
      const int64_t r0 = row0 + g, r1 = row0 + g + 8;
      const uint32_t *f0 = reinterpret_cast<const uint32_t *>(feat + 32 * (r0 < n ? r0 : n - 1));
      const uint32_t *f1 = reinterpret_cast<const uint32_t *>(feat + 32 * (r1 < n ? r1 : n - 1));
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        a1[ks][0] = __ldg(f0 + 8 * ks + t);
        a1[ks][1] = __ldg(f1 + 8 * ks + t);
        a1[ks][2] = __ldg(f0 + 8 * ks + 4 + t);
        a1[ks][3] = __ldg(f1 + 8 * ks + 4 + t);
      }
    }
    float acc[16][4];
    uint32_t h[8][4];
    warp_layer<2, 16>(a1, &sm.w1[0][0], kIP, acc);
    warp_gelu_to_a(acc, sm.bias, h);
    warp_layer<8, 16>(h, &sm.w2[0][0], kHP, acc);
    warp_gelu_to_a(acc, sm.bias + kHid, h);
    warp_layer<8, 16>(h, &sm.w3[0][0], kHP, acc);
    warp_gelu_to_a(acc, sm.bias + 2 * kHid, h);
    float out[1][4];
    warp_layer<8, 1>(h, &sm.w4[0][0], kHP, out);
    if (t < 2) {
      const float b0 = sm.bias[3 * kHid + 2 * t], b1 = sm.bias[3 * kHid + 2 * t + 1];
      if (row0 + g < n)
        *reinterpret_cast<float2 *>(x0 + 4 * (row0 + g) + 2 * t) = make_float2(out[0][0] + b0, out[0][1] + b1);
      if (row0 + g + 8 < n)
        *reinterpret_cast<float2 *>(x0 + 4 * (row0 + g + 8) + 2 * t) = make_float2(out[0][2] + b0, out[0][3] + b1);
    }
  }
}

// ---------------------------------------------------------------------------------------
// fused inference on the 5th-generation tensor cores (tcgen05, accumulators in TMEM).
// One CTA = 8 warps = 256 threads works on tiles of 128 pairs: pair r of the tile is row r
// of every layer's M=128 MMA and TMEM lane r of its accumulator; warps w and w+4 both read
// lanes 32(w%4)..32(w%4)+31 (the TMEM lanes a warp may access), w < 4 columns 0..63 and
// w >= 4 columns 64..127.  Two CTAs fit on an SM, so one's MMAs overlap the other's
// epilogue.
// Operands live in shared memory in the canonical K-major layout without swizzle:
// element (r, k) of a [rows][K] BF16 matrix sits at (r/8)*SBO + (k/8)*128 + (r%8)*16 +
// (k%8)*2 bytes (8x8 core matrices of 128 bytes; LBO = 128 between K neighbours, SBO =
// 16*K between row groups).  One thread issues the MMAs of a layer (K/16 of them,
// 128x128x16 or 128x16x16), commits them to an mbarrier, and every thread then reads its
// row of the accumulator with tcgen05.ld, adds the bias, applies GELU and writes the BF16
// row back as the next layer's A operand.  Waits on the mbarrier are bounded: on time-out
// the kernel records it in *err, stops, and frees its TMEM.
// ---------------------------------------------------------------------------------------
constexpr int kTcRows = 128;          // pairs per tile = MMA M
constexpr uint32_t kTmemCols = 128;   // FP32 accumulator columns (N of the hidden layers)
constexpr int kTcW4Rows = 16;         // W4 padded to N = 16
constexpr uint32_t kTcSpin = 1u << 22;  // mbarrier polls before giving up

struct TcSmem {
  __nv_bfloat16 w1[kHid * kIn];         // 8 KB   (N=128, K=32)
  __nv_bfloat16 w2[kHid * kHid];        // 32 KB  (N=128, K=128)
  __nv_bfloat16 w3[kHid * kHid];        // 32 KB
  __nv_bfloat16 w4[kTcW4Rows * kHid];   // 4 KB   (N=16, K=128; rows 4..15 zero)
  __nv_bfloat16 ah[kTcRows * kHid];     // 32 KB  A operand: layer-1 input (K=32) or hidden (K=128)
  float bias[3 * kHid + kTcW4Rows];
  uint64_t mbar;
  uint32_t tmem_base;
  int abort;
};

// byte offset of the 16-byte chunk (row r, k-chunk kc) in a canonical K-major tile
__device__ __forceinline__ uint32_t tc_chunk(int r, int kc, int K) {
  return (uint32_t)((r >> 3) * (16 * K) + kc * 128 + (r & 7) * 16);
}

__device__ __forceinline__ uint64_t tc_desc(uint32_t smem_addr, uint32_t sbo) {
  // start address >> 4 [0,14), LBO >> 4 [16,30) = 128 B, SBO >> 4 [32,46), version 1 at
  // bit 46, base offset 0, no swizzle
  return (uint64_t)((smem_addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: F32 accumulator, BF16 A and B, both K-major, M x N
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint64_t *mbar) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(mbar);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(a) : "memory");
}

// bounded wait for the mbarrier phase with parity `phase`; false on time-out
__device__ __forceinline__ bool tc_wait(uint64_t *mbar, uint32_t phase, uint32_t spin) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(mbar);
  for (uint32_t it = 0; it < spin; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float v[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// copy a row-major [rows][K] BF16 matrix (global, 16-byte aligned rows) into the canonical
// layout; rows at or beyond `valid_rows` are zero
__device__ __forceinline__ void tc_stage(__nv_bfloat16 *dst, const __nv_bfloat16 *src, int rows, int valid_rows,
                                         int K) {
  const int chunks = K / 8;
  for (int e = threadIdx.x; e < rows * chunks; e += blockDim.x) {
    const int r = e / chunks, kc = e % chunks;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (r < valid_rows) v = __ldg(reinterpret_cast<const uint4 *>(src + (size_t)r * K + kc * 8));
    *reinterpret_cast<uint4 *>(reinterpret_cast<char *>(dst) + tc_chunk(r, kc, K)) = v;
  }
}

// one layer: the elected thread issues K/16 MMAs into TMEM and commits; everyone waits
// (at most `spin` polls).  Returns false (and sets the CTA's abort flag) when the wait
// timed out.  `withhold` (the time-out test only) issues neither the MMAs nor the commit,
// so the barrier never completes and the wait runs out with nothing in flight.
__device__ __forceinline__ bool tc_layer(TcSmem &sm, const __nv_bfloat16 *A, const __nv_bfloat16 *W, int K, int N,
                                         uint32_t &phase, uint32_t spin = kTcSpin, bool withhold = false) {
  // make the generic-proxy stores of A visible to the tensor cores, then synchronise
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (threadIdx.x == 0) {
    const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(A), w0 = (uint32_t)__cvta_generic_to_shared(W);
    const uint32_t idesc = tc_idesc(kTcRows, N);
    if (!withhold) {
      for (int s = 0; s < K / 16; ++s)
        tc_mma(sm.tmem_base, tc_desc(a0 + 256u * s, 16u * K), tc_desc(w0 + 256u * s, 16u * K), idesc, s > 0 ? 1u : 0u);
      tc_commit(&sm.mbar);
    }
    if (!tc_wait(&sm.mbar, phase, spin)) sm.abort = 1;
  }
  __syncthreads();
  phase ^= 1u;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return sm.abort == 0;
}

constexpr int kTcThreads = 2 * kTcRows;

__global__ void __launch_bounds__(kTcThreads, 2)
    k_mlp_infer_tc(int64_t n, const __nv_bfloat16 *__restrict__ feat, const float *__restrict__ params,
                   const __nv_bfloat16 *__restrict__ wb, float *__restrict__ x0, int *__restrict__ err,
                   uint32_t spin, int withhold) {
  extern __shared__ __align__(128) unsigned char tc_smem_raw[];
  TcSmem &sm = *reinterpret_cast<TcSmem *>(tc_smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  tc_stage(sm.w1, wb + kOffW1, kHid, kHid, kIn);
  tc_stage(sm.w2, wb + kOffW2, kHid, kHid, kHid);
  tc_stage(sm.w3, wb + kOffW3, kHid, kHid, kHid);
  tc_stage(sm.w4, wb + kOffW4, kTcW4Rows, kOut, kHid);
  for (int e = tid; e < kHid; e += blockDim.x) {
    sm.bias[e] = params[kOffB1 + e];
    sm.bias[kHid + e] = params[kOffB2 + e];
    sm.bias[2 * kHid + e] = params[kOffB3 + e];
  }
  if (tid < kTcW4Rows) sm.bias[3 * kHid + tid] = tid < kOut ? params[kOffB4 + tid] : 0.f;
  if (tid == 0) {
    sm.abort = 0;
    const unsigned a = (unsigned)__cvta_generic_to_shared(&sm.mbar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(&sm.tmem_base);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const int r = tid & (kTcRows - 1), half = tid >> 7;  // row of the tile, column half
  // this thread's TMEM lane (row) in bits 16..31 of the address, column in bits 0..15
  const uint32_t tlane = sm.tmem_base + ((uint32_t)((warp & 3) * 32) << 16);
  uint32_t phase = 0;
  const int64_t tiles = (n + kTcRows - 1) / kTcRows;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t row = tile * kTcRows + r;
    // layer-1 input: two of the row's four 16-byte feature chunks per thread
    {
      const uint4 *src = reinterpret_cast<const uint4 *>(feat + 32 * (row < n ? row : n - 1));
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int kc = 2 * half + q;
        *reinterpret_cast<uint4 *>(reinterpret_cast<char *>(sm.ah) + tc_chunk(r, kc, kIn)) = __ldg(src + kc);
      }
    }
    int K = kIn;
    const __nv_bfloat16 *Ws[3] = {sm.w1, sm.w2, sm.w3};
    bool ok = true;
    for (int l = 0; l < 3; ++l) {
      ok = tc_layer(sm, sm.ah, Ws[l], K, kHid, phase, spin, withhold != 0 && l == 0);
      if (!ok) break;
      // bias + GELU of this thread's 64 columns of its row, into the hidden A tile
#pragma unroll 1
      for (int c = 64 * half; c < 64 * half + 64; c += 32) {
        float v[32];
        tc_ld32(tlane + (uint32_t)c, v);
        uint32_t w[16];
#pragma unroll
        for (int k = 0; k < 16; ++k)
          w[k] = pack_bf16(gelu(v[2 * k] + sm.bias[l * kHid + c + 2 * k]),
                           gelu(v[2 * k + 1] + sm.bias[l * kHid + c + 2 * k + 1]));
        char *dst = reinterpret_cast<char *>(sm.ah);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          *reinterpret_cast<uint4 *>(dst + tc_chunk(r, c / 8 + q, kHid)) =
              make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
      }
      K = kHid;
    }
    if (!ok) break;
    if (!tc_layer(sm, sm.ah, sm.w4, kHid, kTcW4Rows, phase, spin)) break;
    if (half == 0) {
      float v[16];
      tc_ld16(tlane, v);
      if (row < n)
        *reinterpret_cast<float4 *>(x0 + 4 * row) =
            make_float4(v[0] + sm.bias[3 * kHid], v[1] + sm.bias[3 * kHid + 1], v[2] + sm.bias[3 * kHid + 2],
                        v[3] + sm.bias[3 * kHid + 3]);
    }
  }
  if (sm.abort && tid == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sm.tmem_base), "r"(kTmemCols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------------------
// the training GEMM on the 5th-generation tensor cores: C[M,N] (+)= op(A)[M,K] op(B)[K,N]
// with BF16 operands and an FP32 TMEM accumulator.  A CTA of 256 threads owns a 128 x 128
// output tile (M rows = TMEM lanes, N columns) and a K range, taken in chunks of 64 through
// two shared-memory buffers: the threads stage chunk i+1 (16-byte loads spread over the
// shared-memory banks; an operand stored the other way is loaded as half 8 x 8 blocks and
// transposed in registers) while the tensor core runs chunk i's K/16 MMAs, issued by one
// thread and committed to the buffer's mbarrier (bounded waits).  The TMEM accumulator
// carries the sum over the CTA's K range.  The epilogue goes through shared memory so that
// every warp store writes 128 contiguous bytes of one output row.  With split-K each CTA writes its partial tile to a workspace
// and k_gemm_reduce adds the partials in split order, so the result does not depend on
// scheduling (no atomics).
// ---------------------------------------------------------------------------------------
constexpr int kGtRows = 128, kGtK = 64, kGtThreads = 256;
constexpr int kGtTile = kGtRows * kGtK;             // elements of one operand chunk (16 KB)
constexpr int kGtSmem = 2 * 2 * kGtTile * 2;        // two buffers of (A, B): 64 KB
constexpr int kGtEpi = 33;                          // floats per staged output row (no bank conflicts)
constexpr int kGtEpiBytes = (kGtThreads / 32) * 32 * kGtEpi * 4;  // one 32 x 32 tile per warp
constexpr int kGtSmem1 = kGtSmem / 2 > kGtEpiBytes ? kGtSmem / 2 : kGtEpiBytes;  // one-chunk CTAs
static_assert(kGtEpiBytes <= kGtSmem, "epilogue staging fits in the operand buffers");

// 4 x 8 transpose of 16-bit elements: in[i] holds row i (8 elements), out[j] column j
// (4 elements)
__device__ __forceinline__ void gt_transpose4x8(const uint4 in[4], uint2 out[8]) {
  const uint32_t *w = reinterpret_cast<const uint32_t *>(in);  // w[4*i + q] = (in[i][2q], in[i][2q+1])
  uint32_t *o = reinterpret_cast<uint32_t *>(out);              // o[2*j + p] = (in[2p][j], in[2p+1][j])
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t lo = w[4 * (2 * p) + q], hi = w[4 * (2 * p + 1) + q];
      o[2 * (2 * q) + p] = __byte_perm(lo, hi, 0x5410);
      o[2 * (2 * q + 1) + p] = __byte_perm(lo, hi, 0x7632);
    }
}

// Stages rows [r0, r0+128) x k [k0, k0+64) of X into the canonical K-major tile dst, where
// element (r, k) is X[r*ld + k] (trans = 0) or X[k*ld + r] (trans = 1); rows >= rmax and
// k >= kend are zero.
__device__ __forceinline__ void gt_stage(__nv_bfloat16 *dst, const __nv_bfloat16 *__restrict__ X, int ld, int trans,
                                         int r0, int rmax, int k0, int kend) {
  const int tid = threadIdx.x;
  char *d = reinterpret_cast<char *>(dst);
  const bool aligned = (ld % 8 == 0) && ((reinterpret_cast<uintptr_t>(X) & 15) == 0);
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  if (!trans && aligned) {
    // 16-byte chunks along k: 128 rows x 8 chunks.  A warp takes 8 rows (one 8-row group)
    // x 4 chunks: its loads are 8 runs of 64 contiguous bytes, and its stores fall in the
    // 8 bank groups of the 8 rows, 4 threads each (the 4 wavefronts that 512 bytes take)
    for (int e = tid; e < kGtRows * (kGtK / 8); e += kGtThreads) {
      const int w = e >> 5, l = e & 31;
      const int r = 8 * (w >> 1) + (l & 7), kc = (l >> 3) + 4 * (w & 1), gr = r0 + r, gk = k0 + 8 * kc;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gr < rmax && gk < kend) {
        if (gk + 8 <= kend) {
          v = __ldg(reinterpret_cast<const uint4 *>(X + (int64_t)gr * ld + gk));
        } else {
          __nv_bfloat16 t[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) t[j] = gk + j < kend ? X[(int64_t)gr * ld + gk + j] : zero;
          v = *reinterpret_cast<const uint4 *>(t);
        }
      }
      *reinterpret_cast<uint4 *>(d + tc_chunk(r, kc, kGtK)) = v;
    }
  } else if (aligned) {
    // half of an 8 (k) x 8 (r) block per thread: 4 loads of 8 consecutive r (k rows
    // 4h .. 4h+3 of the block), transposed in registers into the 8-byte halves h of 8
    // chunks of 8 consecutive k.  A warp holds one k block (kb): 16 r blocks x 2 halves;
    // 16 threads read 256 contiguous bytes per load.  Each thread stores its 8 chunks
    // starting at row (rb mod 8) of the 8-row group, so that the 32 stores of a warp fall
    // in 16 different 16-byte bank groups and halves (2 wavefronts for 256 bytes)
    static_assert(kGtThreads == 256, "the transposed staging maps 256 threads onto 16 x 8 x 2 half blocks");
    const int h = tid & 1, rb = (tid >> 1) & 15, kb = tid >> 5, gr = r0 + 8 * rb;
    uint4 in[4];
    uint2 out[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int gk = k0 + 8 * kb + 4 * h + i;
      in[i] = make_uint4(0u, 0u, 0u, 0u);
      if (gk < kend && gr < rmax) {
        const __nv_bfloat16 *src = X + (int64_t)gk * ld + gr;
        if (gr + 8 <= rmax) {
          in[i] = __ldg(reinterpret_cast<const uint4 *>(src));
        } else {
          __nv_bfloat16 t[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) t[j] = gr + j < rmax ? src[j] : zero;
          in[i] = *reinterpret_cast<const uint4 *>(t);
        }
      }
    }
    gt_transpose4x8(in, out);
    // rotate out[] left by rot = rb mod 8 (three conditional stages of register moves)
    const int rot = rb & 7;
#pragma unroll
    for (int b = 1; b < 8; b <<= 1) {
      uint2 t[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) t[j] = out[(j + b) & 7];
      if (rot & b) {
#pragma unroll
        for (int j = 0; j < 8; ++j) out[j] = t[j];
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      *reinterpret_cast<uint2 *>(d + tc_chunk(8 * rb + ((j + rot) & 7), kb, kGtK) + 8 * h) = out[j];
  } else {
    // unaligned operand: pairs (k, k+1) of one row per thread, 4-byte stores
    for (int e = tid; e < kGtRows * (kGtK / 2); e += kGtThreads) {
      const int r = e & (kGtRows - 1), k = 2 * (e >> 7), gr = r0 + r;
      __nv_bfloat16 v0 = zero, v1 = zero;
      if (gr < rmax) {
        const int g0 = k0 + k, g1 = g0 + 1;
        if (g0 < kend) v0 = trans ? X[(int64_t)g0 * ld + gr] : X[(int64_t)gr * ld + g0];
        if (g1 < kend) v1 = trans ? X[(int64_t)g1 * ld + gr] : X[(int64_t)gr * ld + g1];
      }
      __nv_bfloat162 pr;
      pr.x = v0;
      pr.y = v1;
      *reinterpret_cast<__nv_bfloat162 *>(d + tc_chunk(r, k >> 3, kGtK) + (k & 7) * 2) = pr;
    }
  }
}

__global__ void __launch_bounds__(kGtThreads) k_gemm_tc(int M, int N, int K, const __nv_bfloat16 *__restrict__ A,
                                                        int lda, int trans_a, const __nv_bfloat16 *__restrict__ B,
                                                        int ldb, int trans_b, float *__restrict__ Cm, int ldc,
                                                        int accumulate, int k_per_split, float *__restrict__ part,
                                                        int *__restrict__ err, uint32_t spin) {
  extern __shared__ __align__(1024) unsigned char gsm[];
  __shared__ uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  __nv_bfloat16 *bufs = reinterpret_cast<__nv_bfloat16 *>(gsm);  // [2 buffers][A, B][kGtTile]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n0 = blockIdx.x * kGtRows, m0 = blockIdx.y * kGtRows;
  const int kb = blockIdx.z * k_per_split, ke = min(K, kb + k_per_split);
  const int nvalid = min(kGtRows, N - n0), ntile = (nvalid + 15) / 16 * 16;
  if (tid == 0) {
    abort_flag = 0;
    for (int b = 0; b < 2; ++b) {
      const unsigned a = (unsigned)__cvta_generic_to_shared(&mbar[b]);
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(&tmem_base);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  uint32_t ph[2] = {0u, 0u};  // parity of the next phase of each buffer's mbarrier (thread 0)
  int pending = -1;           // buffer whose last commit has not been waited for (thread 0)
  int chunks = 0;
  for (int k0 = kb; k0 < ke; k0 += kGtK, ++chunks) {
    if (abort_flag) break;  // set by thread 0 before the last barrier: the same for all
    const int s = chunks & 1;
    __nv_bfloat16 *sa = bufs + (2 * s) * kGtTile, *sb = sa + kGtTile;
    // buffer s was last read by chunk i-2's MMAs, waited for at the end of chunk i-1
    gt_stage(sa, A, lda, trans_a, m0, M, k0, ke);
    gt_stage(sb, B, ldb, !trans_b, n0, N, k0, ke);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(sa), b0 = (uint32_t)__cvta_generic_to_shared(sb);
      const uint32_t idesc = tc_idesc(kGtRows, ntile);
      const int steps = (min(kGtK, ke - k0) + 15) / 16;
      for (int st = 0; st < steps; ++st)
        tc_mma(tmem_base, tc_desc(a0 + 256u * st, 16u * kGtK), tc_desc(b0 + 256u * st, 16u * kGtK), idesc,
               (chunks > 0 || st > 0) ? 1u : 0u);
      tc_commit(&mbar[s]);
      // the previous chunk's MMAs (buffer s^1) must be done before the next chunk is staged
      if (pending >= 0) {
        if (!tc_wait(&mbar[pending], ph[pending], spin)) abort_flag = 1;
        ph[pending] ^= 1u;
      }
      pending = s;
    }
    __syncthreads();
  }
  // the last commit (it tracks every earlier MMA of this thread too): also after a
  // time-out, bounded, so that no MMA is left in flight when the TMEM is freed
  if (tid == 0 && pending >= 0) {
    if (!tc_wait(&mbar[pending], ph[pending], spin)) abort_flag = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // epilogue: warps w and w+4 read TMEM lanes 32(w%4).. (their rows), the first the
  // column chunks 0, 64, the second 32, 96, 32 columns at a time; each stages its 32 x 32
  // tile in shared memory row by row and writes each row's 32 columns with one store
  const bool ok = !abort_flag;
  const bool issued = chunks > 0;
  const int quad = warp & 3;
  float *stg = reinterpret_cast<float *>(gsm) + warp * 32 * kGtEpi;
  const uint32_t tlane = tmem_base + ((uint32_t)(quad * 32) << 16);
  for (int c = (warp >> 2) * 32; c < ntile; c += 64) {
    float v[32];
    if (issued && ok) {
      tc_ld32(tlane + (uint32_t)c, v);
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = ok ? 0.f : __int_as_float(0x7fc00000);
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) stg[lane * kGtEpi + j] = v[j];
    __syncwarp();
    const int n = n0 + c + lane;
    const bool col_ok = c + lane < nvalid;
    for (int rr = 0; rr < 32; ++rr) {
      const int row = quad * 32 + rr, m = m0 + row;
      if (m < M && col_ok) {
        const float x = stg[rr * kGtEpi + lane];
        if (part) {
          part[((int64_t)blockIdx.z * M + m) * N + n] = x;
        } else {
          float *dst = Cm + (int64_t)m * ldc + n;
          *dst = accumulate ? *dst + x : x;
        }
      }
    }
    __syncwarp();
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kTmemCols)
                 : "memory");
  }
}

// C[m][n] = (accumulate ? C[m][n] : 0) + the sum of the split partials part[s][m][n], in a
// fixed order: a block of 8 warps takes 32 consecutive elements, warp w adds splits w,
// w + 8, ... in order, and warp 0 adds the 8 warp sums in order (deterministic, and every
// load is 128 contiguous bytes).
__global__ void __launch_bounds__(256) k_gemm_reduce(int M, int N, int splits, const float *__restrict__ part,
                                                     float *__restrict__ Cm, int ldc, int accumulate) {
  __shared__ float ws[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t e = (int64_t)blockIdx.x * 32 + lane, mn = (int64_t)M * N;
  float s = 0.f;
  if (e < mn)
    for (int j = w; j < splits; j += 8) s += part[(int64_t)j * mn + e];
  ws[w][lane] = s;
  __syncthreads();
  if (w == 0 && e < mn) {
    float t = ws[0][lane];
#pragma unroll
    for (int k = 1; k < 8; ++k) t += ws[k][lane];
    const int m = (int)(e / N), n = (int)(e % N);
    float *dst = Cm + (int64_t)m * ldc + n;
    *dst = accumulate ? *dst + t : t;
  }
}

// penaltySolver (penalty.cpp:434-582, adaptive, FP64 reference arithmetic) started from
// x0 (4 floats per pair) instead of 0.33; iterations written to iters.
__global__ void k_penalty_warm(int64_t n, const double *a, const double *b, int64_t ld, const float *x0,
                               double max_error, double *p, double *q, double *dist, uint8_t *iters) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  xf64 A[3][3], B[3][3], pq[6];
  for (int v = 0; v < 3; ++v)
    for (int k = 0; k < 3; ++k) {
      A[v][k] = xf64(a[(3 * v + k) * ld + i]);
      B[v][k] = xf64(b[(3 * v + k) * ld + i]);
    }
  xf64 start[4];
  for (int k = 0; k < 4; ++k) start[k] = x0 ? xf64((double)x0[4 * i + k]) : xf64(0.33);
  int it = 16;  // 16: did not meet the tolerance within MaxNumberOfNewtonIterations
  penalty_ref_from(A, B, xf64(max_error), true, pq, it, start);
  for (int k = 0; k < 3; ++k) {
    p[k * ld + i] = pq[k].v;
    q[k * ld + i] = pq[3 + k].v;
  }
  dist[i] = pq_distance(pq).v;
  iters[i] = (uint8_t)it;
}

// Learned hybrid solver, one pair per thread.  From the warm start x0 (barycentric
// weights of P on A and Q on B; centroids when x0 is null), `sweeps` FP32 alternating
// projections (Q <- closest point of B to P, P <- closest point of A to Q) locate the
// closest points roughly.  CAND bfSolver features are then evaluated in FP32: 3 = read off
// the projections (B's vertex nearest Q against face A, A's vertex nearest P against face
// B, the edge pair nearest (P, Q)); 7 = all six vertex-face features and that edge pair;
// 11 = all six vertex-face features and the six edge pairs that contain A's or B's
// nearest edge; 15 = all features.  The one bfSolver's rule (bf.cpp:1102: first minimum in feature order
// within each family, the edge pair only when strictly closer) picks on FP32 distances is
// evaluated in FP64 with the reference arithmetic (bf.cpp:586-697 or 920-1090), so a
// pair whose closest feature was found gets bfSolver's points bit for bit.
// FP64 certificate: with r = P - Q, every plane normal to r bounds the distance below by
// (min_i r.A_i - max_j r.B_j)/|r|; the result is certified when
// |r|^2 - (min_i r.A_i - max_j r.B_j) + slack |r| <= rel_tol |r|^2, i.e. the distance is
// within rel_tol of the true one; slack = 1e-14 max|coordinate| covers the rounding of the
// dot products.  Intersecting triangles have no separating plane and are never certified.
// With `list`, uncertified pairs are appended to list[*count] (one atomicAdd per block,
// in pair order within the block; with `stage`, their 18 coordinates too, at
// stage_at(list position, c)) and their
// outputs left for the exact solver; flags then read 1 (certified) or 2 (listed).
template <int CAND>
__global__ void __launch_bounds__(128, 8) k_learned_refine(int64_t n, const double *__restrict__ a,
                                                        const double *__restrict__ b, int64_t ld,
                                                        const float *__restrict__ x0, int sweeps, double rel_tol,
                                                        double *__restrict__ p, double *__restrict__ q,
                                                        double *__restrict__ dist, uint8_t *__restrict__ flags,
                                                        uint32_t *__restrict__ list, uint32_t *__restrict__ count,
                                                        double *__restrict__ stage) {
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid0 = i0 < n;
  bool edge0;      // the chosen feature is an edge pair
  unsigned code0;  // edge pair: ea | eb << 2; vertex-face: vtx | faceB << 2
  // the block's FP64 coordinates, kept in shared memory for the FP64 stage (which takes
  // the block's pairs in another order) instead of in registers through the FP32 search:
  // [plane 3 * vertex + coordinate][pair of the block]
  __shared__ double s_a[9][128], s_b[9][128];
  {
    const int64_t ii = valid0 ? i0 : n - 1;
    // FP32 copies relative to A0 (the distance is translation invariant)
    float Af[3][3], Bf[3][3];
    {
      double A0[3];
#pragma unroll
      for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double xa = __ldg(a + (3 * v + k) * ld + ii), xb = __ldg(b + (3 * v + k) * ld + ii);
          s_a[3 * v + k][threadIdx.x] = xa;
          s_b[3 * v + k][threadIdx.x] = xb;
          if (v == 0) A0[k] = xa;
          // A0 is the origin (a non-finite A0 fails the FP64 certificate all the same)
          Af[v][k] = v == 0 ? 0.f : (float)(xa - A0[k]);
          Bf[v][k] = (float)(xb - A0[k]);
        }
    }
    float s = 1.f / 3.f, t = 1.f / 3.f, u = 1.f / 3.f, w = 1.f / 3.f;
    if (x0) {
      const float4 x = reinterpret_cast<const float4 *>(x0)[ii];
      // project the prediction into the parameter triangles
      s = fmaxf(x.x, 0.f); t = fmaxf(x.y, 0.f); u = fmaxf(x.z, 0.f); w = fmaxf(x.w, 0.f);
      const float st = s + t, uw = u + w;
      if (st > 1.f) { s /= st; t /= st; }
      if (uw > 1.f) { u /= uw; w /= uw; }
    }
    // each triangle's constants once, for the sweeps and the vertex-face distances
    const TriFrame FA = tri_frame(Af), FB = tri_frame(Bf);
    for (int it = 0; it < sweeps; ++it) {
      float P[3];
      for (int k = 0; k < 3; ++k) P[k] = Af[0][k] + s * FA.e0[k] + t * FA.e1[k];
      closest_on_frame(Bf[0], FB, P, u, w);
      float Q[3];
      for (int k = 0; k < 3; ++k) Q[k] = Bf[0][k] + u * FB.e0[k] + w * FB.e1[k];
      closest_on_frame(Af[0], FA, Q, s, t);
    }
    // features read off the barycentric weights lA = (1-s-t, s, t), lB = (1-u-w, u, w)
    const int iA = argmax3(1.f - s - t, s, t), jB = argmax3(1.f - u - w, u, w);
    const int kA = argmin3(1.f - s - t, s, t), kB = argmin3(1.f - u - w, u, w);
    // bf's vertex-face features: B's vertex jB on face A (feature 9 + jB), A's vertex iA
    // on face B (12 + iA); edge-edge feature 3 ea + eb joins vertices ea, ea+1 (the edge
    // opposite vertex ea+2).  Operands are selected, not indexed, so all lanes run the
    // same code whichever features they picked.
    int ea = (kA + 1) % 3, eb = (kB + 1) % 3;
    float HA[3], TA[3], HB[3], TB[3];
    bool faceB;  // chosen vertex-face feature: A's vertex vtx on face B, else B's vertex vtx on face A
    int vtx;
    float dpt, de;  // squared FP32 distances of the picked vertex-face and edge features
    if constexpr (CAND == 3) {
      float X1[3], X2[3];
      pick_vertex(Bf, jB, X1);
      pick_vertex(Af, iA, X2);
      const float d1 = pt_dist2_frame(Af[0], FA, X1);
      const float d2 = pt_dist2_frame(Bf[0], FB, X2);
      faceB = d2 < d1;
      vtx = faceB ? iA : jB;
      dpt = faceB ? d2 : d1;
    } else {
      // all six vertex-face features in bfSolver's order, first minimum kept
      dpt = 1e30f;
      faceB = false;
      vtx = 0;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const float dj = j < 3 ? pt_dist2_frame(Af[0], FA, Bf[j]) : pt_dist2_frame(Bf[0], FB, Af[j - 3]);
        if (dj < dpt) { dpt = dj; faceB = j >= 3; vtx = j % 3; }
      }
    }
    if constexpr (CAND == 15) {
      // all nine edge pairs, first minimum kept
      de = 1e30f;
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        const float dj = seg_seg_dist2_32(Af[j / 3], Af[(j / 3 + 1) % 3], Bf[j % 3], Bf[(j % 3 + 1) % 3]);
        if (dj < de) { de = dj; ea = j / 3; eb = j % 3; }
      }
    } else if constexpr (CAND == 11) {
      // the edge pairs that contain A's nearest edge or B's nearest edge; the minimum in
      // feature order (distance, then index 3 ea + eb)
      const int ean = ea, ebn = eb;
      de = 1e30f;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const int xa = j < 3 ? ean : j - 3, xb = j < 3 ? j : ebn;
        pick_vertex(Af, xa, HA);
        pick_vertex(Af, (xa + 1) % 3, TA);
        pick_vertex(Bf, xb, HB);
        pick_vertex(Bf, (xb + 1) % 3, TB);
        const float dj = seg_seg_dist2_32(HA, TA, HB, TB);
        if (dj < de || (dj == de && 3 * xa + xb < 3 * ea + eb)) { de = dj; ea = xa; eb = xb; }
      }
    } else {
      other_two(Af, kA, HA, TA);  // edge ea of A
      other_two(Bf, kB, HB, TB);  // edge eb of B
      de = seg_seg_dist2_32(HA, TA, HB, TB);
    }
    edge0 = dpt > de;
    code0 = edge0 ? (unsigned)(ea | (eb << 2)) : (unsigned)(vtx | (faceB ? 4 : 0));
  }
  // Regroup the block's pairs by family before the FP64 stage: an edge pair and a
  // vertex-face pair run different FP64 code, so edge pairs go first and vertex-face pairs
  // after them (each family in pair order), and thread t continues with item t.  A warp
  // then runs one family's code, except the warp whose items straddle the boundary.
  __shared__ uint16_t s_item[128];
  __shared__ int s_cnt[2][4];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const unsigned be = __ballot_sync(0xffffffffu, valid0 && edge0), bv = __ballot_sync(0xffffffffu, valid0 && !edge0);
  if (lane == 0) {
    s_cnt[0][wid] = __popc(be);
    s_cnt[1][wid] = __popc(bv);
  }
  __syncthreads();
  int nE = 0, nV = 0, preE = 0, preV = 0;
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    const int ce = s_cnt[0][w], cv = s_cnt[1][w];
    preE += w < wid ? ce : 0;
    preV += w < wid ? cv : 0;
    nE += ce;
    nV += cv;
  }
  if (valid0) {
    const int pos = edge0 ? preE + __popc(be & lt) : nE + preV + __popc(bv & lt);
    s_item[pos] = (uint16_t)(tid | (edge0 ? 128u : 0u) | (code0 << 8));
  }
  __syncthreads();
  // threads past the block's pairs (last block only) repeat item 0 and write nothing
  const bool has = tid < nE + nV;
  const unsigned item = s_item[has ? tid : 0];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + (item & 127);
  const bool edge = (item & 128u) != 0;
  const int ea = (item >> 8) & 3, eb = (item >> 10) & 3, vtx = (item >> 8) & 3;
  const bool faceB = ((item >> 10) & 1) != 0;
  // FP64 stage: only the chosen feature's vertices are read (from the block's shared
  // copies), then the six vertices stream through the certificate one at a time
  const int it = (int)(item & 127);  // the pair's slot in the block's shared copies
  auto vtx64 = [&](const double (*T)[128], int v, xf64 out[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = xf64(T[3 * v + k][it]);
  };
  xf64 pq[6];
  if (edge) {
    xf64 HA[3], TA[3], HB[3], TB[3], sc, tc;
    vtx64(s_a, ea, HA);
    vtx64(s_a, (ea + 1) % 3, TA);
    vtx64(s_b, eb, HB);
    vtx64(s_b, (eb + 1) % 3, TB);
    seg_seg_ref(HA, TA, HB, TB, sc, tc);
#pragma unroll
    for (int k = 0; k < 3; ++k) {  // bf.cpp:715-879 (seg_seg_points)
      pq[k] = TA[k] + ((HA[k] - TA[k]) * sc);
      pq[3 + k] = TB[k] + ((HB[k] - TB[k]) * tc);
    }
  } else {
    // face of A with B's vertex vtx, or face of B with A's vertex vtx
    const double(*face)[128] = faceB ? s_b : s_a;
    const double(*pnt)[128] = faceB ? s_a : s_b;
    xf64 T0[3], T1[3], T2[3], X[3], sf, tf;
    vtx64(face, 0, T0);
    vtx64(face, 1, T1);
    vtx64(face, 2, T2);
    vtx64(pnt, vtx, X);
    pt_tri_ref(T0, T1, T2, X, sf, tf);
#pragma unroll
    for (int k = 0; k < 3; ++k) {  // bf.cpp:1104-1177 (pt_tri_points)
      const xf64 fp = T0[k] + ((T2[k] - T0[k]) * tf) + ((T1[k] - T0[k]) * sf);
      pq[k] = faceB ? X[k] : fp;
      pq[3 + k] = faceB ? fp : X[k];
    }
  }
  const double d = pq_distance(pq).v;
  bool ok = false;
  if (d > 0) {
    const double r[3] = {pq[0].v - pq[3].v, pq[1].v - pq[4].v, pq[2].v - pq[5].v};
    double amin = 1e300, bmax = -1e300, scale = 0.0;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      xf64 VA[3], VB[3];
      vtx64(s_a, v, VA);
      vtx64(s_b, v, VB);
      amin = fmin(amin, VA[0].v * r[0] + VA[1].v * r[1] + VA[2].v * r[2]);
      bmax = fmax(bmax, VB[0].v * r[0] + VB[1].v * r[1] + VB[2].v * r[2]);
#pragma unroll
      for (int k = 0; k < 3; ++k) scale = fmax(scale, fmax(fabs(VA[k].v), fabs(VB[k].v)));
    }
    const double d2r = d * d;
    ok = d2r - (amin - bmax) + 1e-14 * scale * d <= rel_tol * d2r;
  }
  if (has && (ok || !list)) {
    for (int k = 0; k < 3; ++k) {
      p[k * ld + i] = pq[k].v;
      q[k * ld + i] = pq[3 + k].v;
    }
    dist[i] = d;
  }
  if (has && flags) flags[i] = list ? (ok ? 1 : 2) : (ok ? 1 : 0);
  if (!list) return;
  // The uncertified pairs are appended by their own threads, in pair order within the
  // block, so the list (and the exact solver's reads and writes through it) keeps the
  // pairs' order block by block. One atomicAdd per block on the shared counter: appends
  // from every warp to one address serialise in L2 (the counter's slice may sit on the
  // other die), which cost up to a fifth of the pipeline's time.
  __shared__ uint8_t s_bad[128];
  __shared__ uint32_t s_wcount[4], s_base;
  if (has) s_bad[item & 127] = ok ? 0 : 1;
  __syncthreads();
  const bool bad = valid0 && s_bad[tid];
  const unsigned bad_mask = __ballot_sync(0xffffffffu, bad);
  if (lane == 0) s_wcount[wid] = __popc(bad_mask);
  __syncthreads();
  if (tid == 0) {
    const uint32_t total = s_wcount[0] + s_wcount[1] + s_wcount[2] + s_wcount[3];
    s_base = total ? atomicAdd(count, total) : 0u;
  }
  __syncthreads();
  if (bad) {
    uint32_t slot = s_base + __popc(bad_mask & lt);
    for (int w = 0; w < wid; ++w) slot += s_wcount[w];
    list[slot] = (uint32_t)i0;
    if (stage) {
      // the pair's coordinates, compact at its list position, for the exact solver
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        stage[stage_at(slot, c)] = s_a[c][tid];
        stage[stage_at(slot, 9 + c)] = s_b[c][tid];
      }
    }
  }
}

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t > 0 ? (n + t - 1) / t : 1); }

// Features into scratch, then the network on `engine`; with the tcgen05 engine *err_out
// receives the device time-out flag (zeroed here, set by the kernel).
delta_status mlp_infer_launch(delta_ctx *ctx, int engine, int64_t n, const double *a, const double *b, int64_t ld,
                              const float *params, const void *params_bf16, float *x0, int **err_out,
                              uint32_t spin = kTcSpin, int withhold = 0) {
  void *fbuf;
  delta_status st = ctx_scratch(ctx, 15, sizeof(__nv_bfloat16) * 32 * (size_t)n, &fbuf);
  if (st != DELTA_OK) return st;
  __nv_bfloat16 *feat = static_cast<__nv_bfloat16 *>(fbuf);
  k_canon<<<nblk(n), 256, 0, ctx->stream>>>(n, a, b, ld, nullptr, nullptr, feat, nullptr, nullptr);
  ctx->launches += 1;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "mlp features");
  const __nv_bfloat16 *wb = static_cast<const __nv_bfloat16 *>(params_bf16);
  if (engine == DELTA_MLP_TCGEN05) {
    void *ebuf;
    if ((st = ctx_scratch(ctx, 16, sizeof(int), &ebuf)) != DELTA_OK) return st;
    int *err = static_cast<int *>(ebuf);
    if ((e = cudaMemsetAsync(err, 0, sizeof(int), ctx->stream)) != cudaSuccess) return cuda_error(e, "mlp flag");
    static thread_local int configured_device = -1;
    if (configured_device != ctx->device) {
      e = cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem));
      if (e != cudaSuccess) return cuda_error(e, "mlp tcgen05: shared memory attribute");
      configured_device = ctx->device;
    }
    const int64_t tiles = (n + kTcRows - 1) / kTcRows;
    const unsigned grid = (unsigned)std::min<int64_t>(tiles, 2 * kNumSMs);
    k_mlp_infer_tc<<<grid, kTcThreads, sizeof(TcSmem), ctx->stream>>>(n, feat, params, wb, x0, err, spin, withhold);
    if (err_out) *err_out = err;
  } else {
    static thread_local int configured_device = -1;
    if (configured_device != ctx->device) {
      e = cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(InferSmem));
      if (e != cudaSuccess) return cuda_error(e, "mlp mma: shared memory attribute");
      configured_device = ctx->device;
    }
    const int64_t tiles = (n + 15) / 16;
    const int64_t want = (tiles + kInferWarps - 1) / kInferWarps;
    const unsigned grid = (unsigned)std::min<int64_t>(want, 2 * kNumSMs);
    k_mlp_infer<<<grid, 32 * kInferWarps, sizeof(InferSmem), ctx->stream>>>(n, feat, params, wb, x0);
    if (err_out) *err_out = nullptr;
  }
  ctx->launches += 1;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "mlp network");
  return DELTA_OK;
}

// Synchronises and reports the tcgen05 kernel's time-out flag (err may be null).
delta_status mlp_check_error(delta_ctx *ctx, const int *err) {
  if (!err) return DELTA_OK;
  void *pin;
  delta_status st = ctx_pinned(ctx, sizeof(int), &pin);
  if (st != DELTA_OK) return st;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(pin, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
    return cuda_error(e, "mlp status");
  if (*static_cast<int *>(pin))
    return set_error(DELTA_ERR_TIMEOUT, "tcgen05 inference: bounded wait for the tensor cores gave up");
  return DELTA_OK;
}

// The learned pipeline enqueued on the context stream: network (when params are given),
// refine with the device list of uncertified pairs, exact fallback over that list.
// *count_out: device count of listed pairs; *err_out: the network's time-out flag or null.
delta_status learned_enqueue(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                             const float *params, const void *params_bf16, int sweeps, int features, double rel_tol,
                             double *p, double *q, double *dist, uint8_t *flags, uint32_t **count_out,
                             int **err_out);

void launch_refine(int features, cudaStream_t s, int64_t n, const double *a, const double *b, int64_t ld,
                   const float *x0, int sweeps, double rel_tol, double *p, double *q, double *dist, uint8_t *flags,
                   uint32_t *list, uint32_t *count, double *stage = nullptr) {
  const unsigned g = nblk(n, 128);
  if (features == 11) k_learned_refine<11><<<g, 128, 0, s>>>(n, a, b, ld, x0, sweeps, rel_tol, p, q, dist, flags, list, count, stage);
  else if (features == 15) k_learned_refine<15><<<g, 128, 0, s>>>(n, a, b, ld, x0, sweeps, rel_tol, p, q, dist, flags, list, count, stage);
  else if (features == 7) k_learned_refine<7><<<g, 128, 0, s>>>(n, a, b, ld, x0, sweeps, rel_tol, p, q, dist, flags, list, count, stage);
  else k_learned_refine<3><<<g, 128, 0, s>>>(n, a, b, ld, x0, sweeps, rel_tol, p, q, dist, flags, list, count, stage);
}

delta_status learned_enqueue(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                             const float *params, const void *params_bf16, int sweeps, int features, double rel_tol,
                             double *p, double *q, double *dist, uint8_t *flags, uint32_t **count_out,
                             int **err_out) {
  delta_status st;
  float *x0 = nullptr;
  *err_out = nullptr;
  if (params) {
    void *buf;
    if ((st = ctx_scratch(ctx, 13, sizeof(float) * 4 * (size_t)n, &buf)) != DELTA_OK) return st;
    x0 = static_cast<float *>(buf);
    if ((reinterpret_cast<uintptr_t>(params_bf16) & 15))
      return set_error(DELTA_ERR_INVALID, "learned pipeline: params_bf16 must be 16-byte aligned");
    if ((st = mlp_infer_launch(ctx, ctx->mlp_engine, n, a, b, ld, params, params_bf16, x0, err_out)) != DELTA_OK)
      return st;
  }
  void *lbuf;
  if ((st = ctx_scratch(ctx, 14, 256 + sizeof(uint32_t) * (size_t)n, &lbuf)) != DELTA_OK) return st;
  uint32_t *count = static_cast<uint32_t *>(lbuf);
  uint32_t *list = reinterpret_cast<uint32_t *>(static_cast<char *>(lbuf) + 256);
  // compact copies of the uncertified pairs' coordinates (tiles of 32) for the exact solver
  void *sbuf;
  if ((st = ctx_scratch(ctx, 25, sizeof(double) * stage_doubles(n), &sbuf)) != DELTA_OK) return st;
  double *stage = static_cast<double *>(sbuf);
  cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint32_t), ctx->stream);
  if (e != cudaSuccess) return cuda_error(e, "learned pipeline: memset");
  launch_refine(features, ctx->stream, n, a, b, ld, x0, sweeps, rel_tol, p, q, dist, flags, list, count, stage);
  ctx->launches += 1;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "learned pipeline: refine");
  const PairLaunch cfg = ctx->pair_launch_set[DELTA_BF_CERT][0] ? ctx->pair_launch[DELTA_BF_CERT][0]
                                                                : default_pair_launch(DELTA_BF_CERT);
  e = launch_cert_indexed(ctx->stream, count, n, list, a, b, ld, p, q, dist, cfg, stage);
  ctx->launches += 1;
  if (e != cudaSuccess) return cuda_error(e, "learned pipeline: exact fallback");
  *count_out = count;
  return DELTA_OK;
}

}  // namespace

}  // namespace delta

using namespace delta;

extern "C" {

delta_status delta_mlp_features(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                const double *p, const double *q, void *features_bf16, float *targets,
                                uint8_t *valid) {
  if (!ctx || n < 0 || ld < n || (n > 0 && (!a || !b || !features_bf16)) || ((p == nullptr) != (q == nullptr)) ||
      (p && !targets))
    return set_error(DELTA_ERR_INVALID, "delta_mlp_features: bad argument");
  if ((reinterpret_cast<uintptr_t>(features_bf16) & 15) || (reinterpret_cast<uintptr_t>(targets) & 15))
    return set_error(DELTA_ERR_INVALID, "delta_mlp_features: features and targets must be 16-byte aligned");
  if (n == 0) return DELTA_OK;
  k_canon<<<nblk(n), 256, 0, ctx->stream>>>(n, a, b, ld, p, q, (__nv_bfloat16 *)features_bf16, targets, valid);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_mlp_features");
}

delta_status delta_gemm_bf16(delta_ctx *ctx, int M, int N, int K, const void *A, int lda, int trans_a,
                             const void *B, int ldb, int trans_b, float *C, int ldc, int accumulate, int split_k) {
  if (!ctx || M < 0 || N < 0 || K < 0 || !A || !B || !C || split_k < 1)
    return set_error(DELTA_ERR_INVALID, "delta_gemm_bf16: bad argument");
  if (M == 0 || N == 0) return DELTA_OK;
  cudaError_t e = cudaSuccess;
  if (ctx->mlp_engine == DELTA_MLP_TCGEN05) {
    if (!ctx->gemm_err) {
      if ((e = cudaMalloc(&ctx->gemm_err, sizeof(int))) != cudaSuccess) return cuda_error(e, "gemm flag");
      if ((e = cudaMemsetAsync(ctx->gemm_err, 0, sizeof(int), ctx->stream)) != cudaSuccess)
        return cuda_error(e, "gemm flag");
    }
    int per = (K + split_k - 1) / split_k;
    per = (per + kGtK - 1) / kGtK * kGtK;
    if (per <= 0) per = kGtK;
    const int splits = K > 0 ? (K + per - 1) / per : 1;
    float *part = nullptr;
    if (splits > 1) {
      void *buf;
      delta_status st = ctx_scratch(ctx, 28, sizeof(float) * (size_t)splits * M * N, &buf);
      if (st != DELTA_OK) return st;
      part = static_cast<float *>(buf);
    }
    if ((e = cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kGtSmem)) != cudaSuccess)
      return cuda_error(e, "gemm shared memory");
    // a CTA with one K chunk uses one buffer: half the shared memory, twice the CTAs per SM
    const int smem = per <= kGtK ? kGtSmem1 : kGtSmem;
    dim3 grid((N + kGtRows - 1) / kGtRows, (M + kGtRows - 1) / kGtRows, splits);
    k_gemm_tc<<<grid, kGtThreads, smem, ctx->stream>>>(M, N, K, (const __nv_bfloat16 *)A, lda, trans_a,
                                                    (const __nv_bfloat16 *)B, ldb, trans_b, C, ldc, accumulate, per,
                                                    part, ctx->gemm_err, kTcSpin);
    ctx->launches += 1;
    if (splits > 1) {
      k_gemm_reduce<<<(unsigned)(((int64_t)M * N + 31) / 32), 256, 0, ctx->stream>>>(M, N, splits, part, C, ldc,
                                                                                     accumulate);
      ctx->launches += 1;
    }
    return cuda_error(cudaGetLastError(), "delta_gemm_bf16 (tcgen05)");
  }
  if (!accumulate && (split_k > 1)) e = cudaMemsetAsync(C, 0, sizeof(float) * (size_t)M * ldc, ctx->stream);
  if (e != cudaSuccess) return cuda_error(e, "gemm memset");
  int per = (K + split_k - 1) / split_k;
  per = (per + BK - 1) / BK * BK;
  const int splits = per > 0 ? (K + per - 1) / per : 1;
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, splits > 0 ? splits : 1);
  k_gemm<<<grid, 128, 0, ctx->stream>>>(M, N, K, (const __nv_bfloat16 *)A, lda, trans_a, (const __nv_bfloat16 *)B,
                                        ldb, trans_b, C, ldc, accumulate, per > 0 ? per : BK);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_gemm_bf16");
}

// The row-tiled element-wise kernels take N a power of two from 4 to 1024 and 16-byte
// aligned FP32 rows (8-byte aligned BF16 rows follow).
static bool rows_tiled(int N, const void *f32, const void *bf16) {
  return N >= 4 && N <= 1024 && (N & (N - 1)) == 0 && (reinterpret_cast<uintptr_t>(f32) & 15) == 0 &&
         (reinterpret_cast<uintptr_t>(bf16) & 7) == 0;
}
static unsigned tiled_blocks(int64_t M, int rows) {
  const int64_t b = (M + rows - 1) / rows, cap = (int64_t)kNumSMs * 8;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

delta_status delta_mlp_bias_act(delta_ctx *ctx, int64_t M, int N, float *Z, const float *bias, void *H_bf16,
                                int gelu_on) {
  if (!ctx || !Z || !bias || M < 0 || N <= 0) return set_error(DELTA_ERR_INVALID, "delta_mlp_bias_act");
  if (M == 0) return DELTA_OK;
  if (rows_tiled(N, Z, H_bf16)) {
    const int rows = 256 / (N / 4);
    k_bias_act4<<<tiled_blocks(M, rows), 256, 0, ctx->stream>>>(M, N / 4, Z, bias, (__nv_bfloat16 *)H_bf16, gelu_on);
  } else {
    k_bias_act<<<nblk(M * N), 256, 0, ctx->stream>>>(M, N, Z, bias, (__nv_bfloat16 *)H_bf16, gelu_on);
  }
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_mlp_bias_act");
}

delta_status delta_mlp_mse(delta_ctx *ctx, int64_t M, const float *Y, const float *T, const uint8_t *valid,
                           float inv_n, void *dY_bf16, float *loss) {
  if (!ctx || !Y || !T || !valid || !dY_bf16 || !loss) return set_error(DELTA_ERR_INVALID, "delta_mlp_mse");
  if (M == 0) return DELTA_OK;
  k_mse<<<nblk(M * 4), 256, 0, ctx->stream>>>(M, Y, T, valid, inv_n, (__nv_bfloat16 *)dY_bf16, loss);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_mlp_mse");
}

delta_status delta_mlp_act_grad(delta_ctx *ctx, int64_t M, int N, const float *dH, const float *Z, void *dZ_bf16) {
  if (!ctx || !dH || !Z || !dZ_bf16) return set_error(DELTA_ERR_INVALID, "delta_mlp_act_grad");
  if (M == 0) return DELTA_OK;
  if (rows_tiled(N, dH, dZ_bf16) && (reinterpret_cast<uintptr_t>(Z) & 15) == 0) {
    const int rows = 256 / (N / 4);
    k_act_grad4<<<tiled_blocks(M, rows), 256, 0, ctx->stream>>>(M, N / 4, dH, Z, (__nv_bfloat16 *)dZ_bf16);
  } else {
    k_act_grad<<<nblk(M * N), 256, 0, ctx->stream>>>(M, N, dH, Z, (__nv_bfloat16 *)dZ_bf16);
  }
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_mlp_act_grad");
}

delta_status delta_mlp_colsum(delta_ctx *ctx, int64_t M, int N, const void *dZ_bf16, float *db) {
  if (!ctx || !dZ_bf16 || !db) return set_error(DELTA_ERR_INVALID, "delta_mlp_colsum");
  if (M == 0) return DELTA_OK;
  if (N <= 256 && (N & (N - 1)) == 0) {
    k_colsum_rows<<<tiled_blocks(M, 256 / N), 256, 0, ctx->stream>>>(M, N, (const __nv_bfloat16 *)dZ_bf16, db);
  } else {
    const int ys = (int)std::min<int64_t>(64, (M + 255) / 256);
    k_colsum<<<dim3(N, ys > 0 ? ys : 1), 256, 0, ctx->stream>>>(M, N, (const __nv_bfloat16 *)dZ_bf16, db);
  }
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_mlp_colsum");
}

delta_status delta_adam(delta_ctx *ctx, int64_t n, float *w, const float *g, float *m, float *v, float lr, float b1,
                        float b2, float eps, int64_t step, void *w_bf16) {
  if (!ctx || !w || !g || !m || !v || step < 1) return set_error(DELTA_ERR_INVALID, "delta_adam");
  if (n == 0) return DELTA_OK;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<nblk(n), 256, 0, ctx->stream>>>(n, w, g, m, v, lr, b1, b2, eps, c1, c2, (__nv_bfloat16 *)w_bf16);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_adam");
}

delta_status delta_to_bf16(delta_ctx *ctx, int64_t n, const float *x, void *y_bf16) {
  if (!ctx || (n > 0 && (!x || !y_bf16))) return set_error(DELTA_ERR_INVALID, "delta_to_bf16");
  if (n == 0) return DELTA_OK;
  k_f32_to_bf16<<<nblk(n), 256, 0, ctx->stream>>>(n, x, (__nv_bfloat16 *)y_bf16);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_to_bf16");
}

delta_status delta_mlp_layout(int64_t offsets[9]) {
  if (!offsets) return set_error(DELTA_ERR_INVALID, "delta_mlp_layout: null");
  const int64_t o[9] = {kOffW1, kOffB1, kOffW2, kOffB2, kOffW3, kOffB3, kOffW4, kOffB4, kNumParams};
  for (int k = 0; k < 9; ++k) offsets[k] = o[k];
  return DELTA_OK;
}

delta_status delta_mlp_set_engine(delta_ctx *ctx, int engine) {
  if (!ctx || (engine != DELTA_MLP_TCGEN05 && engine != DELTA_MLP_MMA_SYNC))
    return set_error(DELTA_ERR_INVALID, "delta_mlp_set_engine: unknown engine");
  ctx->mlp_engine = engine;
  return DELTA_OK;
}

delta_status delta_mlp_infer(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                             const float *params, const void *params_bf16, float *x0) {
  if (!ctx || n < 0 || ld < n || (n > 0 && (!a || !b || !params || !params_bf16 || !x0)))
    return set_error(DELTA_ERR_INVALID, "delta_mlp_infer: bad argument");
  if ((reinterpret_cast<uintptr_t>(params_bf16) & 15) || (reinterpret_cast<uintptr_t>(x0) & 15))
    return set_error(DELTA_ERR_INVALID, "delta_mlp_infer: params_bf16 and x0 must be 16-byte aligned");
  if (n == 0) return DELTA_OK;
  return mlp_infer_launch(ctx, DELTA_MLP_MMA_SYNC, n, a, b, ld, params, params_bf16, x0, nullptr);
}

delta_status delta_mlp_infer_tcgen05(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                     const float *params, const void *params_bf16, float *x0) {
  if (!ctx || n < 0 || ld < n || (n > 0 && (!a || !b || !params || !params_bf16 || !x0)))
    return set_error(DELTA_ERR_INVALID, "delta_mlp_infer_tcgen05: bad argument");
  if ((reinterpret_cast<uintptr_t>(params_bf16) & 15) || (reinterpret_cast<uintptr_t>(x0) & 15))
    return set_error(DELTA_ERR_INVALID, "delta_mlp_infer_tcgen05: params_bf16 and x0 must be 16-byte aligned");
  if (n == 0) return DELTA_OK;
  int *err = nullptr;
  delta_status st = mlp_infer_launch(ctx, DELTA_MLP_TCGEN05, n, a, b, ld, params, params_bf16, x0, &err);
  if (st != DELTA_OK) return st;
  return mlp_check_error(ctx, err);
}

delta_status delta_mlp_infer_tcgen05_wait_test(delta_ctx *ctx, int64_t n, const double *a, const double *b,
                                               int64_t ld, const float *params, const void *params_bf16, float *x0,
                                               uint32_t polls) {
  if (!ctx || n <= 0 || ld < n || !a || !b || !params || !params_bf16 || !x0 || polls < 1 || polls > kTcSpin)
    return set_error(DELTA_ERR_INVALID, "delta_mlp_infer_tcgen05_wait_test: bad argument");
  if ((reinterpret_cast<uintptr_t>(params_bf16) & 15) || (reinterpret_cast<uintptr_t>(x0) & 15))
    return set_error(DELTA_ERR_INVALID, "delta_mlp_infer_tcgen05_wait_test: params_bf16 and x0 must be 16-byte aligned");
  int *err = nullptr;
  delta_status st = mlp_infer_launch(ctx, DELTA_MLP_TCGEN05, n, a, b, ld, params, params_bf16, x0, &err, polls, 1);
  if (st != DELTA_OK) return st;
  return mlp_check_error(ctx, err);
}

delta_status delta_penalty_warm(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                const float *x0, double max_error, double *p, double *q, double *dist,
                                uint8_t *iterations) {
  if (!ctx || n < 0 || ld < n || (n > 0 && (!a || !b || !p || !q || !dist || !iterations)))
    return set_error(DELTA_ERR_INVALID, "delta_penalty_warm: bad argument");
  if (n == 0) return DELTA_OK;
  k_penalty_warm<<<nblk(n, 128), 128, 0, ctx->stream>>>(n, a, b, ld, x0, max_error, p, q, dist, iterations);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_penalty_warm");
}

delta_status delta_learned_refine(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                  const float *x0, int32_t sweeps, int32_t features, double rel_tol, double *p,
                                  double *q, double *dist, uint8_t *certified) {
  if (!ctx || n < 0 || ld < n || sweeps < 0 || (features != 3 && features != 7 && features != 11 && features != 15) ||
      (n > 0 && (!a || !b || !p || !q || !dist || !certified)))
    return set_error(DELTA_ERR_INVALID, "delta_learned_refine: bad argument");
  if (reinterpret_cast<uintptr_t>(x0) & 15)
    return set_error(DELTA_ERR_INVALID, "delta_learned_refine: x0 must be 16-byte aligned");
  if (n == 0) return DELTA_OK;
  launch_refine(features, ctx->stream, n, a, b, ld, x0, sweeps, rel_tol, p, q, dist, certified, nullptr, nullptr);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_learned_refine");
}

delta_status delta_pairs_run_learned(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                     const float *params, const void *params_bf16, int32_t sweeps, int32_t features,
                                     double rel_tol, double *p, double *q, double *dist, uint8_t *flags,
                                     int64_t *n_fallback) {
  if (!ctx || n < 0 || ld < n || sweeps < 0 || n > (int64_t)UINT32_MAX ||
      (features != 3 && features != 7 && features != 11 && features != 15) ||
      (n > 0 && (!a || !b || !p || !q || !dist)) || ((params == nullptr) != (params_bf16 == nullptr)))
    return set_error(DELTA_ERR_INVALID, "delta_pairs_run_learned: bad argument");
  if (n_fallback) *n_fallback = 0;
  if (n == 0) return DELTA_OK;
  uint32_t *count = nullptr;
  int *mlp_err = nullptr;
  delta_status st = learned_enqueue(ctx, n, a, b, ld, params, params_bf16, sweeps, features, rel_tol, p, q, dist,
                                    flags, &count, &mlp_err);
  if (st != DELTA_OK || !n_fallback) return st;
  void *pin;
  if ((st = ctx_pinned(ctx, sizeof(uint32_t), &pin)) != DELTA_OK) return st;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(pin, count, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
    return cuda_error(e, "delta_pairs_run_learned: count");
  *n_fallback = *static_cast<uint32_t *>(pin);
  // the warm start only steers the search (every result is certified or exact), but a
  // tensor-core time-out is still reported
  return mlp_check_error(ctx, mlp_err);
}

delta_status delta_pairs_run_learned_host(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                          const float *params, const void *params_bf16, int32_t sweeps,
                                          int32_t features, double rel_tol, double *p, double *q, double *dist,
                                          uint8_t *flags, int64_t *n_fallback) {
  if (!ctx || n < 0 || ld < n || sweeps < 0 || n > (int64_t)UINT32_MAX ||
      (features != 3 && features != 7 && features != 11 && features != 15) ||
      (n > 0 && (!a || !b || !p || !q || !dist)) || ((params == nullptr) != (params_bf16 == nullptr)))
    return set_error(DELTA_ERR_INVALID, "delta_pairs_run_learned_host: bad argument");
  if (n_fallback) *n_fallback = 0;
  if (n == 0) return DELTA_OK;
  // per chunk: fallback count and network time-out flag, gathered on the device
  void *sbuf;
  delta_status st = ctx_scratch(ctx, 24, 64 * sizeof(uint32_t), &sbuf);
  if (st != DELTA_OK) return st;
  uint32_t *tally = static_cast<uint32_t *>(sbuf);
  cudaError_t e = cudaMemsetAsync(tally, 0, 64 * sizeof(uint32_t), ctx->stream);
  if (e != cudaSuccess) return cuda_error(e, "learned host: tally");
  uint32_t *count = nullptr;
  int *mlp_err = nullptr;
  int chunks = 0;
  st = host_pipeline(
      ctx, n, a, b, ld, p, q, dist, flags,
      [&](int64_t, int64_t nc, const double *da, const double *db, int64_t ldd, double *dp, double *dq, double *dd,
          uint8_t *df) {
        return learned_enqueue(ctx, nc, da, db, ldd, params, params_bf16, sweeps, features, rel_tol, dp, dq, dd, df,
                               &count, &mlp_err);
      },
      [&](int k) {
        cudaError_t ce = cudaMemcpyAsync(tally + 2 * k, count, sizeof(uint32_t), cudaMemcpyDeviceToDevice, ctx->stream);
        if (ce == cudaSuccess && mlp_err)
          ce = cudaMemcpyAsync(tally + 2 * k + 1, mlp_err, sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream);
        chunks = k + 1;
        return cuda_error(ce, "learned host: tally");
      });
  if (st != DELTA_OK) return st;
  uint32_t h[64];
  if ((e = cudaMemcpy(h, tally, sizeof(uint32_t) * 2 * chunks, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return cuda_error(e, "learned host: tally read");
  int64_t total = 0;
  bool timeout = false;
  for (int k = 0; k < chunks; ++k) {
    total += h[2 * k];
    timeout |= h[2 * k + 1] != 0;
  }
  if (n_fallback) *n_fallback = total;
  if (timeout) return set_error(DELTA_ERR_TIMEOUT, "tcgen05 inference: bounded wait for the tensor cores gave up");
  return DELTA_OK;
}

}  // extern "C"
