// Neural-operator warm start (no SLEPc counterpart): a small spectral neural
// operator that maps the coefficient field of a diffusion operator to a block
// of approximate eigenvectors, used as the initial space of EPSSolve
// (EPSSetInitialSpace, src/eps/interface/epssetup.c:613; the LOBPCG block and
// the Krylov-Schur start vector).  Training and inference run on the GPU in
// these kernels, forward and backward, FP32.
//
// Network, on an N x N cell grid (P = N^2 points, row-major), batch B:
//   features F[b] (3 x P: log kappa, x, y)
//   V_0 = Pw F + Pb                                        (lift to W channels)
//   for l < L:  U_l = S (R_l . (S^T V_l S)) S^T + W_l V_l + b_l
//               V_{l+1} = gelu(U_l)  (l < L-1),  U_l  (l = L-1)
//   Z = Q1 V_L + q1,  H = gelu(Z),  Y = Q2 H + q2          (K output fields)
// S (N x M) is the orthonormal Dirichlet sine basis S[i][k] = sqrt(2/(N+1))
// sin(pi (i+1)(k+1)/(N+1)); S^T V S keeps the M x M lowest sine modes of each
// channel, and R_l mixes the W channels separately for every kept mode (the
// spectral convolution of a Fourier neural operator, written as GEMMs against
// the mode basis).  Loss, per sample b and output k with target eigenvector
// u_k (unit norm): 1 - (y_k . u_k)^2 / (y_k . y_k), averaged over b and k
// (invariant to the sign and scale of y_k).  Adam updates the parameters.
//
// Every contraction is one call of the strided, batched tensor-core GEMM of
// tcgemm.cu (tcgen05 TF32 MMAs, three products per step for FP32-level
// accuracy, FP32 accumulation in TMEM; long reductions split across CTAs and
// summed in a fixed order); elementwise kernels add biases and apply gelu and
// its derivative; reductions (bias gradients, the loss) use fixed orders.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "kernels.h"

struct b200_neural_op_s {
  int N = 0, P = 0, W = 0, M = 0, L = 0, H = 0, K = 0;
  static constexpr int Cin = 3;
  cudaStream_t stream = nullptr;
  size_t nparams = 0;
  float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  long long step = 0;
  float *S = nullptr;  // N x M sine basis
  // offsets of the parameter tensors inside params / grads
  size_t oPw = 0, oPb = 0, oQ1 = 0, oq1 = 0, oQ2 = 0, oq2 = 0;
  std::vector<size_t> oR, oW, ob;
  // activations and scratch for up to cap batch samples
  int cap = 0;
  float *act = nullptr;
  size_t act_len = 0;
  float *loss_bk = nullptr;  // B x K per-output losses
  std::vector<float> hloss;
  float *ws = nullptr;       // split-depth partial products of the GEMMs
  size_t ws_len = 0;
  int *dev_err = nullptr;    // device error bits of the GEMMs (bounded waits)
};

namespace b200 {
namespace {

struct MView {
  const float *p;
  long long rs, cs, bs;  // element (i, j) of matrix z at p + z*bs + i*rs + j*cs
};

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// U[b][c][p] += bias[c]; V = act ? gelu(U) : U
__global__ void bias_act_kernel(float *U, const float *__restrict__ bias, float *V, int C, int P, long long total,
                                int act) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)((t / P) % C);
    const float u = U[t] + bias[c];
    U[t] = u;
    if (V) V[t] = act ? gelu(u) : u;
  }
}

// dU = dV * gelu'(U)
__global__ void gelu_bwd_kernel(const float *__restrict__ dV, const float *__restrict__ U, float *dU, long long total) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x)
    dU[t] = dV[t] * gelu_grad(U[t]);
}

// db[c] = sum over b and p of D[b][c][p] in two fixed-order stages: block (c, s) sums its slice
// s of the B * P entries of channel c into part[c * S + s]; bias_final_kernel adds the S slices.
constexpr int kBiasSlices = 64;
__global__ void bias_grad_kernel(const float *__restrict__ D, int B, int C, int P, float *part) {
  __shared__ float red[256];
  const int c = blockIdx.x, sl = blockIdx.y;
  const long long total = (long long)B * P, per = (total + kBiasSlices - 1) / kBiasSlices;
  const long long e0 = sl * per, e1 = min(total, e0 + per);
  float s = 0.f;
  for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const long long b = e / P, p = e - b * P;
    s += D[(b * C + c) * P + p];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(size_t)c * kBiasSlices + sl] = red[0];
}
__global__ void bias_final_kernel(const float *__restrict__ part, int C, float *db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float s = 0.f;
  for (int q = 0; q < kBiasSlices; ++q) s += part[(size_t)c * kBiasSlices + q];
  db[c] = s;
}

// Per (k, b): l = 1 - (y.u)^2/(y.y) and dY = (-2 (y.u)/(y.y) u + 2 (y.u)^2/(y.y)^2 y) * scale
__global__ void loss_kernel(const float *__restrict__ Y, const float *__restrict__ T, int K, int P, float scale,
                            float *loss_bk, float *dY) {
  __shared__ float r1[256], r2[256];
  const int k = blockIdx.x, b = blockIdx.y;
  const long long base = ((long long)b * K + k) * P;
  float yu = 0.f, yy = 0.f;
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    const float y = Y[base + p], u = T[base + p];
    yu = fmaf(y, u, yu);
    yy = fmaf(y, y, yy);
  }
  r1[threadIdx.x] = yu;
  r2[threadIdx.x] = yy;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      r1[threadIdx.x] += r1[threadIdx.x + w];
      r2[threadIdx.x] += r2[threadIdx.x + w];
    }
    __syncthreads();
  }
  yu = r1[0];
  yy = fmaxf(r2[0], 1e-30f);
  if (threadIdx.x == 0) loss_bk[b * K + k] = 1.f - yu * yu / yy;
  if (dY) {
    const float cu = -2.f * yu / yy * scale, cy = 2.f * yu * yu / (yy * yy) * scale;
    for (int p = threadIdx.x; p < P; p += blockDim.x) dY[base + p] = cu * T[base + p] + cy * Y[base + p];
  }
}

__global__ void adam_kernel(float *p, const float *__restrict__ g, float *m, float *v, long long n, float lr,
                            float b1, float b2, float c1, float c2, float eps) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const float gi = g[t];
    const float mi = b1 * m[t] + (1.f - b1) * gi;
    const float vi = b2 * v[t] + (1.f - b2) * gi * gi;
    m[t] = mi;
    v[t] = vi;
    p[t] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

unsigned grid_len(long long len) {
  const long long g = (len + 255) / 256;
  return (unsigned)(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

// Every contraction of the network: the tensor-core GEMM of tcgemm.cu with the operator's split-depth
// workspace and device error word.
cudaError_t gemm(b200_neural_op op, int batch, int m, int n, int k, float alpha, MView A, MView B, float beta,
                 float *C, long long rsc, long long csc, long long bsc, bool sum_batch = false) {
  return tc_sgemm(op->stream, batch, m, n, k, alpha, A.p, A.rs, A.cs, A.bs, B.p, B.rs, B.cs, B.bs, beta, C, rsc, csc,
                  bsc, op->dev_err, op->ws, op->ws_len, sum_batch);
}

}  // namespace
}  // namespace b200

using namespace b200;

namespace {

// Activation layout for batch cap: offsets (in floats) into op->act
struct Acts {
  float *F, *V, *U, *Ch, *T1, *Dh, *T2, *Z, *Hh, *Y;  // forward
  float *dY, *dH, *dV0, *dV1, *dU, *dDh, *dCh;        // backward
};

Acts carve(b200_neural_op op, size_t *len) {
  const size_t B = op->cap, P = op->P, W = op->W, L = op->L, M2 = (size_t)op->M * op->M, NM = (size_t)op->N * op->M;
  size_t off = 0;
  Acts a{};
  auto take = [&](size_t n) {
    float *p = op->act ? op->act + off : nullptr;
    off += (n + 63) / 64 * 64;
    return p;
  };
  a.F = take(B * 3 * P);
  a.V = take((L + 1) * B * W * P);
  a.U = take(L * B * W * P);
  a.Ch = take(L * B * W * M2);
  a.T1 = take(B * W * NM);
  a.Dh = take(B * W * M2);
  a.T2 = take(B * W * NM);
  a.Z = take(B * op->H * P);
  a.Hh = take(B * op->H * P);
  a.Y = take(B * op->K * P);
  a.dY = take(B * op->K * P);
  a.dH = take(B * op->H * P);
  a.dV0 = take(B * W * P);
  a.dV1 = take(B * W * P);
  a.dU = take(B * W * P);
  a.dDh = take(B * W * M2);
  a.dCh = take(B * W * M2);
  *len = off;
  return a;
}

b200_status reserve(b200_neural_op op, int B) {
  if (B <= op->cap && op->act) return B200_OK;
  cudaFree(op->act);
  cudaFree(op->loss_bk);
  op->act = nullptr;
  op->loss_bk = nullptr;
  op->cap = B;
  size_t len = 0;
  carve(op, &len);
  if (cudaMalloc(&op->act, sizeof(float) * len) != cudaSuccess ||
      cudaMalloc(&op->loss_bk, sizeof(float) * (size_t)B * op->K) != cudaSuccess) {
    cudaFree(op->act);
    op->act = nullptr;
    op->cap = 0;
    b200_set_last_error(__FILE__, __LINE__, "cudaMalloc failed for the neural-operator activations");
    return B200_ERR_NOMEM;
  }
  op->act_len = len;
  // split-depth workspace: the widest summed weight gradient over the batch, four depth splits
  const size_t W = op->W, mn = std::max({W * 3, W * W, (size_t)op->H * W, (size_t)op->K * op->H});
  const size_t ws_len = std::max<size_t>(mn * (size_t)B * 4, (size_t)1 << 22);
  if (ws_len > op->ws_len) {
    cudaFree(op->ws);
    op->ws = nullptr;
    op->ws_len = 0;
    if (cudaMalloc(&op->ws, sizeof(float) * ws_len) != cudaSuccess) {
      b200_set_last_error(__FILE__, __LINE__, "cudaMalloc failed for the neural-operator GEMM workspace");
      return B200_ERR_NOMEM;
    }
    op->ws_len = ws_len;
  }
  return B200_OK;
}

// Reads and clears the GEMMs' device error bits (the stream is synchronised by the caller); bits
// that a training step's backward pass sets are reported by the next call that reads them.
b200_status gemm_status(b200_neural_op op) {
  int e = 0;
  B200_CUDA_CHECK(cudaMemcpy(&e, op->dev_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    B200_CUDA_CHECK(cudaMemset(op->dev_err, 0, sizeof(int)));
    b200_set_last_error(__FILE__, __LINE__, "a tensor-core GEMM gave up a bounded wait");
    return B200_ERR_CUDA;
  }
  return B200_OK;
}

float *prm(b200_neural_op op, size_t off) { return op->params + off; }
float *grd(b200_neural_op op, size_t off) { return op->grads + off; }

// Channel mix Out[b] (Co x P) = Wt (Co x Ci) In[b] (Ci x P) (+ beta Out)
cudaError_t mix(b200_neural_op op, int B, int Co, int Ci, const float *Wt, const float *In, float *Out, float beta) {
  const long long P = op->P;
  return gemm(op, B, Co, (int)P, Ci, 1.f, MView{Wt, Ci, 1, 0}, MView{In, P, 1, (long long)Ci * P}, beta, Out,
              P, 1, (long long)Co * P);
}
// Transposed mix Out[b] (Ci x P) = Wt^T (Ci x Co) In[b] (Co x P)
cudaError_t mix_t(b200_neural_op op, int B, int Co, int Ci, const float *Wt, const float *In, float *Out, float beta) {
  const long long P = op->P;
  return gemm(op, B, Ci, (int)P, Co, 1.f, MView{Wt, 1, Ci, 0}, MView{In, P, 1, (long long)Co * P}, beta, Out,
              P, 1, (long long)Ci * P);
}
// Weight gradient dWt (Co x Ci) = sum_b D[b] (Co x P) X[b]^T (P x Ci): one product summed over b
cudaError_t mix_grad(b200_neural_op op, int B, int Co, int Ci, const float *D, const float *X, float *dWt) {
  const long long P = op->P;
  return gemm(op, B, Co, Ci, (int)P, 1.f, MView{D, P, 1, (long long)Co * P}, MView{X, 1, P, (long long)Ci * P}, 0.f,
              dWt, Ci, 1, 0, true);
}
cudaError_t bias_act(b200_neural_op op, int B, int C, float *U, const float *bias, float *V, int act) {
  const long long total = (long long)B * C * op->P;
  bias_act_kernel<<<grid_len(total), 256, 0, op->stream>>>(U, bias, V, C, op->P, total, act);
  count_launch();
  return cudaGetLastError();
}
cudaError_t bias_grad(b200_neural_op op, int B, int C, const float *D, float *db) {
  // the slices go to the GEMM workspace (free between GEMMs on the same stream)
  bias_grad_kernel<<<dim3(C, kBiasSlices), 256, 0, op->stream>>>(D, B, C, op->P, op->ws);
  count_launch();
  bias_final_kernel<<<(C + 127) / 128, 128, 0, op->stream>>>(op->ws, C, db);
  count_launch();
  return cudaGetLastError();
}
cudaError_t gelu_bwd(b200_neural_op op, long long total, const float *dV, const float *U, float *dU) {
  gelu_bwd_kernel<<<grid_len(total), 256, 0, op->stream>>>(dV, U, dU, total);
  count_launch();
  return cudaGetLastError();
}
// Mode coefficients C[z] (M x M) = S^T X[z] S for z < nz fields (N x N each)
cudaError_t to_modes(b200_neural_op op, int nz, const float *X, float *T1, float *C) {
  const int N = op->N, M = op->M;
  const long long P = op->P, NM = (long long)N * M, M2 = (long long)M * M;
  cudaError_t e = gemm(op, nz, M, N, N, 1.f, MView{op->S, 1, M, 0}, MView{X, N, 1, P}, 0.f, T1, N, 1, NM);
  if (e != cudaSuccess) return e;
  return gemm(op, nz, M, M, N, 1.f, MView{T1, N, 1, NM}, MView{op->S, M, 1, 0}, 0.f, C, M, 1, M2);
}
// Fields X[z] (N x N) = S C[z] S^T (+ beta X)
cudaError_t from_modes(b200_neural_op op, int nz, const float *C, float *T2, float *X, float beta) {
  const int N = op->N, M = op->M;
  const long long P = op->P, NM = (long long)N * M, M2 = (long long)M * M;
  cudaError_t e = gemm(op, nz, N, M, M, 1.f, MView{op->S, M, 1, 0}, MView{C, M, 1, M2}, 0.f, T2, M, 1, NM);
  if (e != cudaSuccess) return e;
  return gemm(op, nz, N, N, M, 1.f, MView{T2, M, 1, NM}, MView{op->S, 1, M, 0}, beta, X, N, 1, P);
}

b200_status forward(b200_neural_op op, int B, const float *feat, Acts &a) {
  const int W = op->W, L = op->L, M = op->M;
  const long long P = op->P, M2 = (long long)M * M, WP = (long long)W * P;
  B200_CUDA_CHECK(cudaMemcpyAsync(a.F, feat, sizeof(float) * (size_t)B * 3 * P, cudaMemcpyDeviceToDevice, op->stream));
  // lift
  B200_CUDA_CHECK(mix(op, B, W, 3, prm(op, op->oPw), a.F, a.V, 0.f));
  B200_CUDA_CHECK(bias_act(op, B, W, a.V, prm(op, op->oPb), nullptr, 0));
  for (int l = 0; l < L; ++l) {
    float *Vl = a.V + (size_t)l * B * WP, *Ul = a.U + (size_t)l * B * WP, *Cl = a.Ch + (size_t)l * B * W * M2;
    B200_CUDA_CHECK(to_modes(op, B * W, Vl, a.T1, Cl));
    // per mode q: Dh_q (B x W_o) = C_q (B x W_c) R_q^T (W_c x W_o)
    const float *R = prm(op, op->oR[l]);
    B200_CUDA_CHECK(gemm(op, (int)M2, B, W, W, 1.f, MView{Cl, W * M2, M2, 1}, MView{R, M2, W * M2, 1}, 0.f,
                         a.Dh, W * M2, M2, 1));
    B200_CUDA_CHECK(from_modes(op, B * W, a.Dh, a.T2, Ul, 0.f));
    B200_CUDA_CHECK(mix(op, B, W, W, prm(op, op->oW[l]), Vl, Ul, 1.f));
    B200_CUDA_CHECK(bias_act(op, B, W, Ul, prm(op, op->ob[l]), a.V + (size_t)(l + 1) * B * WP, l < L - 1));
  }
  // projection
  float *VL = a.V + (size_t)L * B * WP;
  B200_CUDA_CHECK(mix(op, B, op->H, W, prm(op, op->oQ1), VL, a.Z, 0.f));
  B200_CUDA_CHECK(bias_act(op, B, op->H, a.Z, prm(op, op->oq1), a.Hh, 1));
  B200_CUDA_CHECK(mix(op, B, op->K, op->H, prm(op, op->oQ2), a.Hh, a.Y, 0.f));
  B200_CUDA_CHECK(bias_act(op, B, op->K, a.Y, prm(op, op->oq2), nullptr, 0));
  return B200_OK;
}

b200_status backward(b200_neural_op op, int B, Acts &a) {
  const int W = op->W, L = op->L, M = op->M, H = op->H, K = op->K;
  const long long P = op->P, M2 = (long long)M * M, WP = (long long)W * P;
  // output layer
  B200_CUDA_CHECK(mix_grad(op, B, K, H, a.dY, a.Hh, grd(op, op->oQ2)));
  B200_CUDA_CHECK(bias_grad(op, B, K, a.dY, grd(op, op->oq2)));
  B200_CUDA_CHECK(mix_t(op, B, K, H, prm(op, op->oQ2), a.dY, a.dH, 0.f));
  B200_CUDA_CHECK(gelu_bwd(op, (long long)B * H * P, a.dH, a.Z, a.dH));
  B200_CUDA_CHECK(mix_grad(op, B, H, W, a.dH, a.V + (size_t)L * B * WP, grd(op, op->oQ1)));
  B200_CUDA_CHECK(bias_grad(op, B, H, a.dH, grd(op, op->oq1)));
  float *dV = a.dV0, *dVn = a.dV1;  // dV holds the gradient of V_{l+1}
  B200_CUDA_CHECK(mix_t(op, B, H, W, prm(op, op->oQ1), a.dH, dV, 0.f));
  for (int l = L - 1; l >= 0; --l) {
    float *Vl = a.V + (size_t)l * B * WP, *Ul = a.U + (size_t)l * B * WP, *Cl = a.Ch + (size_t)l * B * W * M2;
    const float *dU = dV;
    if (l < L - 1) {
      B200_CUDA_CHECK(gelu_bwd(op, (long long)B * WP, dV, Ul, a.dU));
      dU = a.dU;
    }
    B200_CUDA_CHECK(bias_grad(op, B, W, dU, grd(op, op->ob[l])));
    B200_CUDA_CHECK(mix_grad(op, B, W, W, dU, Vl, grd(op, op->oW[l])));
    B200_CUDA_CHECK(mix_t(op, B, W, W, prm(op, op->oW[l]), dU, dVn, 0.f));
    // spectral path: dDh = S^T dU S; dR_q = dDh_q^T C_q; dC_q = dDh_q R_q; dV += S dC S^T
    B200_CUDA_CHECK(to_modes(op, B * W, dU, a.T1, a.dDh));
    const float *R = prm(op, op->oR[l]);
    B200_CUDA_CHECK(gemm(op, (int)M2, W, W, B, 1.f, MView{a.dDh, M2, W * M2, 1}, MView{Cl, W * M2, M2, 1}, 0.f,
                         grd(op, op->oR[l]), W * M2, M2, 1));
    B200_CUDA_CHECK(gemm(op, (int)M2, B, W, W, 1.f, MView{a.dDh, W * M2, M2, 1}, MView{R, W * M2, M2, 1}, 0.f,
                         a.dCh, W * M2, M2, 1));
    B200_CUDA_CHECK(from_modes(op, B * W, a.dCh, a.T2, dVn, 1.f));
    float *t = dV;
    dV = dVn;
    dVn = t;
  }
  // lift
  B200_CUDA_CHECK(mix_grad(op, B, W, 3, dV, a.F, grd(op, op->oPw)));
  B200_CUDA_CHECK(bias_grad(op, B, W, dV, grd(op, op->oPb)));
  return B200_OK;
}

b200_status loss(b200_neural_op op, int B, const float *targets, Acts &a, bool want_grad, float *loss_out) {
  const float scale = 1.f / (float)(B * op->K);
  loss_kernel<<<dim3(op->K, B), 256, 0, op->stream>>>(a.Y, targets, op->K, op->P, scale, op->loss_bk,
                                                      want_grad ? a.dY : nullptr);
  count_launch();
  B200_CUDA_CHECK(cudaGetLastError());
  op->hloss.resize((size_t)B * op->K);
  B200_CUDA_CHECK(cudaMemcpyAsync(op->hloss.data(), op->loss_bk, sizeof(float) * op->hloss.size(),
                                  cudaMemcpyDeviceToHost, op->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(op->stream));
  B200_CHECK(gemm_status(op));
  double s = 0.0;
  for (float v : op->hloss) s += v;
  if (loss_out) *loss_out = (float)(s / (double)op->hloss.size());
  return B200_OK;
}

}  // namespace

extern "C" b200_status b200_neural_op_create(int N, int width, int modes, int layers, int hidden, int nout,
                                             void *stream, b200_neural_op *out) {
  B200_ARG_CHECK(out && N >= 2 && width > 0 && modes > 0 && modes <= N && layers > 0 && hidden > 0 && nout > 0,
                 "invalid neural-operator sizes");
  B200_ARG_CHECK((long long)N * N <= (1ll << 24) && width <= 256 && modes <= 64 && layers <= 16 && hidden <= 1024 &&
                     nout <= 256,
                 "neural-operator sizes out of range");
  b200_neural_op op = new b200_neural_op_s;
  op->N = N;
  op->P = N * N;
  op->W = width;
  op->M = modes;
  op->L = layers;
  op->H = hidden;
  op->K = nout;
  op->stream = (cudaStream_t)stream;
  size_t off = 0;
  auto take = [&](size_t n) {
    const size_t o = off;
    off += n;
    return o;
  };
  const size_t W = width, M2 = (size_t)modes * modes;
  op->oPw = take(W * 3);
  op->oPb = take(W);
  for (int l = 0; l < layers; ++l) {
    op->oR.push_back(take(W * W * M2));
    op->oW.push_back(take(W * W));
    op->ob.push_back(take(W));
  }
  op->oQ1 = take((size_t)hidden * W);
  op->oq1 = take(hidden);
  op->oQ2 = take((size_t)nout * hidden);
  op->oq2 = take(nout);
  op->nparams = off;
  bool ok = cudaMalloc(&op->params, sizeof(float) * off) == cudaSuccess &&
            cudaMalloc(&op->grads, sizeof(float) * off) == cudaSuccess &&
            cudaMalloc(&op->adam_m, sizeof(float) * off) == cudaSuccess &&
            cudaMalloc(&op->adam_v, sizeof(float) * off) == cudaSuccess &&
            cudaMalloc(&op->S, sizeof(float) * (size_t)N * modes) == cudaSuccess &&
            cudaMalloc(&op->dev_err, sizeof(int)) == cudaSuccess;
  if (ok) {
    std::vector<float> S((size_t)N * modes);
    const double c = std::sqrt(2.0 / (N + 1));
    for (int i = 0; i < N; ++i)
      for (int k = 0; k < modes; ++k) S[(size_t)i * modes + k] = (float)(c * std::sin(M_PI * (i + 1) * (k + 1) / (N + 1)));
    ok = cudaMemcpyAsync(op->S, S.data(), sizeof(float) * S.size(), cudaMemcpyHostToDevice, op->stream) == cudaSuccess &&
         cudaMemsetAsync(op->params, 0, sizeof(float) * off, op->stream) == cudaSuccess &&
         cudaMemsetAsync(op->adam_m, 0, sizeof(float) * off, op->stream) == cudaSuccess &&
         cudaMemsetAsync(op->adam_v, 0, sizeof(float) * off, op->stream) == cudaSuccess &&
         cudaMemsetAsync(op->dev_err, 0, sizeof(int), op->stream) == cudaSuccess &&
         cudaStreamSynchronize(op->stream) == cudaSuccess;
  }
  if (!ok) {
    b200_neural_op_destroy(op);
    b200_set_last_error(__FILE__, __LINE__, "cudaMalloc failed for the neural operator");
    return B200_ERR_NOMEM;
  }
  *out = op;
  return B200_OK;
}

extern "C" b200_status b200_neural_op_destroy(b200_neural_op op) {
  if (!op) return B200_OK;
  cudaFree(op->params);
  cudaFree(op->grads);
  cudaFree(op->adam_m);
  cudaFree(op->adam_v);
  cudaFree(op->S);
  cudaFree(op->act);
  cudaFree(op->loss_bk);
  cudaFree(op->ws);
  cudaFree(op->dev_err);
  delete op;
  return B200_OK;
}

extern "C" b200_status b200_neural_op_num_params(b200_neural_op op, int64_t *n) {
  B200_ARG_CHECK(op && n, "null argument");
  *n = (int64_t)op->nparams;
  return B200_OK;
}

extern "C" b200_status b200_neural_op_set_params(b200_neural_op op, const float *host) {
  B200_ARG_CHECK(op && host, "null argument");
  B200_CUDA_CHECK(cudaMemcpyAsync(op->params, host, sizeof(float) * op->nparams, cudaMemcpyHostToDevice, op->stream));
  B200_CUDA_CHECK(cudaMemsetAsync(op->adam_m, 0, sizeof(float) * op->nparams, op->stream));
  B200_CUDA_CHECK(cudaMemsetAsync(op->adam_v, 0, sizeof(float) * op->nparams, op->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(op->stream));
  op->step = 0;
  return B200_OK;
}

extern "C" b200_status b200_neural_op_get_params(b200_neural_op op, float *host) {
  B200_ARG_CHECK(op && host, "null argument");
  B200_CUDA_CHECK(cudaMemcpyAsync(host, op->params, sizeof(float) * op->nparams, cudaMemcpyDeviceToHost, op->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(op->stream));
  return B200_OK;
}

extern "C" b200_status b200_neural_op_forward(b200_neural_op op, int batch, const float *features_dev, float *out_dev) {
  B200_ARG_CHECK(op && batch > 0 && features_dev && out_dev, "invalid forward arguments");
  B200_CHECK(reserve(op, batch));
  size_t len;
  Acts a = carve(op, &len);
  B200_CHECK(forward(op, batch, features_dev, a));
  B200_CUDA_CHECK(cudaMemcpyAsync(out_dev, a.Y, sizeof(float) * (size_t)batch * op->K * op->P,
                                  cudaMemcpyDeviceToDevice, op->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(op->stream));
  return gemm_status(op);
}

extern "C" b200_status b200_neural_op_loss_grad(b200_neural_op op, int batch, const float *features_dev,
                                                const float *targets_dev, float *loss_out, float *grads_host) {
  B200_ARG_CHECK(op && batch > 0 && features_dev && targets_dev, "invalid loss arguments");
  B200_CHECK(reserve(op, batch));
  size_t len;
  Acts a = carve(op, &len);
  B200_CHECK(forward(op, batch, features_dev, a));
  B200_CHECK(loss(op, batch, targets_dev, a, true, loss_out));
  B200_CHECK(backward(op, batch, a));
  if (grads_host) {
    B200_CUDA_CHECK(
        cudaMemcpyAsync(grads_host, op->grads, sizeof(float) * op->nparams, cudaMemcpyDeviceToHost, op->stream));
    B200_CUDA_CHECK(cudaStreamSynchronize(op->stream));
    return gemm_status(op);
  }
  return B200_OK;
}

extern "C" b200_status b200_neural_op_train_step(b200_neural_op op, int batch, const float *features_dev,
                                                 const float *targets_dev, float lr, float *loss_out) {
  B200_CHECK(b200_neural_op_loss_grad(op, batch, features_dev, targets_dev, loss_out, nullptr));
  op->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)op->step), c2 = 1.f - std::pow(b2, (float)op->step);
  adam_kernel<<<grid_len((long long)op->nparams), 256, 0, op->stream>>>(op->params, op->grads, op->adam_m, op->adam_v,
                                                                       (long long)op->nparams, lr, b1, b2, c1, c2,
                                                                       1e-8f);
  count_launch();
  B200_CUDA_CHECK(cudaGetLastError());
  return B200_OK;
}

extern "C" b200_status b200_neural_op_loss(b200_neural_op op, int batch, const float *features_dev,
                                           const float *targets_dev, float *loss_out) {
  B200_ARG_CHECK(op && batch > 0 && features_dev && targets_dev && loss_out, "invalid loss arguments");
  B200_CHECK(reserve(op, batch));
  size_t len;
  Acts a = carve(op, &len);
  B200_CHECK(forward(op, batch, features_dev, a));
  return loss(op, batch, targets_dev, a, false, loss_out);
}
