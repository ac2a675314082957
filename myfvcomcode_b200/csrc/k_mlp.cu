// k_mlp.cu - the network of the learned vertical closure: an MLP 8 -> 64 -> 64 -> 3 with
// GELU (tanh form) on the two hidden layers, trained in FP32 by the kernels in this file (mean-squared
// error, Adam).  Inference in BF16 on the tensor cores is in k_closure.cu; the FP32
// forward pass here is its reference.
//
// Parameters are one FP32 vector: W1 (64x8, row j = hidden unit j), b1 (64), W2 (64x64),
// b2 (64), W3 (3x64), b3 (3).
//
// Training step over a batch of B samples: k_mlp_fwd_bwd runs one block per T=64
// samples.  Each thread carries one sample forward and backward (the activations and
// their gradients of the block live in shared memory, [unit][T+1] so the 32 lanes of a
// warp touch 32 banks); then the threads switch to weight elements and form the block's
// weight gradient as sums over its samples, in sample order.  k_mlp_adam sums the blocks'
// gradients in block order and applies Adam.  The gradient is thus deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "fvg_model.h"

namespace {

constexpr int MI = 8, MH = 64, MO = 3;
constexpr int OW1 = 0, OB1 = OW1 + MH * MI, OW2 = OB1 + MH, OB2 = OW2 + MH * MH, OW3 = OB2 + MH,
              OB3 = OW3 + MO * MH, NPAR = OB3 + MO;
constexpr int T = 64;        // samples per block
constexpr int TS = T + 1;    // padded stride of the activation planes

// GELU in its tanh form, 0.5 z (1 + tanh(c (z + 0.044715 z^3))), c = sqrt(2/pi), and its
// derivative.
constexpr float kGc = 0.79788456080286536f, kGa = 0.044715f;
__device__ inline float gelu(float z) { return 0.5f * z * (1.0f + tanhf(kGc * (z + kGa * z * z * z))); }
__device__ inline float gelu_d(float z) {
  const float t = tanhf(kGc * (z + kGa * z * z * z));
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGc * (1.0f + 3.0f * kGa * z * z);
}

// Shared-memory layout of k_mlp_fwd_bwd (floats).
constexpr int SM_W = 0;                    // parameters
constexpr int SM_X = SM_W + NPAR;          // x   [MI][TS]
constexpr int SM_Z1 = SM_X + MI * TS;      // z1, then dz1 [MH][TS]
constexpr int SM_H1 = SM_Z1 + MH * TS;     // h1  [MH][TS]
constexpr int SM_Z2 = SM_H1 + MH * TS;     // z2, then dz2 [MH][TS]
constexpr int SM_H2 = SM_Z2 + MH * TS;     // h2  [MH][TS]
constexpr int SM_DY = SM_H2 + MH * TS;     // dy  [MO][TS]
constexpr int SM_TOTAL = SM_DY + MO * TS;

// x: row-major [n][MI] inputs, y: [n][MO] targets, idx: optional sample order (the
// batch is idx[b0 .. b0+nb-1]).  part: [gridDim.x][NPAR] gradients, lpart: [gridDim.x]
// summed squared errors.  scale = 1/(number of batch samples * MO).
__global__ void __launch_bounds__(T) k_mlp_fwd_bwd(const float* __restrict__ par, const float* __restrict__ x,
                                                   const float* __restrict__ y, const int* __restrict__ idx,
                                                   int b0, int nb, float scale, float* part, float* lpart) {
  extern __shared__ float sm[];
  float* w = sm + SM_W;
  const int t = threadIdx.x;
  for (int p = t; p < NPAR; p += T) w[p] = par[p];
  const int r = blockIdx.x * T + t;
  const bool live = r < nb;
  const int row = live ? (idx ? idx[b0 + r] : b0 + r) : 0;
  for (int k = 0; k < MI; ++k) sm[SM_X + k * TS + t] = live ? x[(size_t)row * MI + k] : 0.f;
  __syncthreads();
  float err2 = 0.f;
  // forward
  for (int j = 0; j < MH; ++j) {
    float z = w[OB1 + j];
    for (int k = 0; k < MI; ++k) z += w[OW1 + j * MI + k] * sm[SM_X + k * TS + t];
    sm[SM_Z1 + j * TS + t] = z;
    sm[SM_H1 + j * TS + t] = gelu(z);
  }
  float out[MO];
  for (int o = 0; o < MO; ++o) out[o] = w[OB3 + o];
  for (int j = 0; j < MH; ++j) {
    float z = w[OB2 + j];
    for (int k = 0; k < MH; ++k) z += w[OW2 + j * MH + k] * sm[SM_H1 + k * TS + t];
    sm[SM_Z2 + j * TS + t] = z;
    float h = gelu(z);
    sm[SM_H2 + j * TS + t] = h;
    for (int o = 0; o < MO; ++o) out[o] += w[OW3 + o * MH + j] * h;
  }
  float dy[MO];
  for (int o = 0; o < MO; ++o) {
    float e = live ? out[o] - y[(size_t)row * MO + o] : 0.f;
    err2 += e * e;
    dy[o] = 2.f * e * scale;
    sm[SM_DY + o * TS + t] = dy[o];
  }
  // backward through the units of this sample
  for (int j = 0; j < MH; ++j) {
    float dh = 0.f;
    for (int o = 0; o < MO; ++o) dh += w[OW3 + o * MH + j] * dy[o];
    float z = sm[SM_Z2 + j * TS + t];
    sm[SM_Z2 + j * TS + t] = dh * gelu_d(z);
  }
  for (int k = 0; k < MH; ++k) {
    float dh = 0.f;
    for (int j = 0; j < MH; ++j) dh += w[OW2 + j * MH + k] * sm[SM_Z2 + j * TS + t];
    float z = sm[SM_Z1 + k * TS + t];
    sm[SM_Z1 + k * TS + t] = dh * gelu_d(z);
  }
  __syncthreads();
  // weight gradients of the block: thread t takes elements p = t, t+T, ...
  float* gp = part + (size_t)blockIdx.x * NPAR;
  for (int p = t; p < NPAR; p += T) {
    const float *a, *b = nullptr;
    if (p < OB1) { a = sm + SM_Z1 + (p / MI) * TS; b = sm + SM_X + (p % MI) * TS; }
    else if (p < OW2) { a = sm + SM_Z1 + (p - OB1) * TS; }
    else if (p < OB2) { int q = p - OW2; a = sm + SM_Z2 + (q / MH) * TS; b = sm + SM_H1 + (q % MH) * TS; }
    else if (p < OW3) { a = sm + SM_Z2 + (p - OB2) * TS; }
    else if (p < OB3) { int q = p - OW3; a = sm + SM_DY + (q / MH) * TS; b = sm + SM_H2 + (q % MH) * TS; }
    else { a = sm + SM_DY + (p - OB3) * TS; }
    float s = 0.f;
    if (b)
      for (int u = 0; u < T; ++u) s += a[u] * b[u];
    else
      for (int u = 0; u < T; ++u) s += a[u];
    gp[p] = s;
  }
  // squared error of the block, in sample order
  __shared__ float e2[T];
  e2[t] = err2;
  __syncthreads();
  if (t == 0) {
    float s = 0.f;
    for (int u = 0; u < T; ++u) s += e2[u];
    lpart[blockIdx.x] = s;
  }
}

// Sum of the blocks' gradients (block order) and, when step > 0, one Adam update.
__global__ void k_mlp_adam(float* par, float* m, float* v, const float* part, int nblk, float* grad_out,
                           const float* lpart, float* loss_acc, int step, float lr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0) {
    float s = 0.f;
    for (int b = 0; b < nblk; ++b) s += lpart[b];
    *loss_acc += s;
  }
  if (p >= NPAR) return;
  float g = 0.f;
  for (int b = 0; b < nblk; ++b) g += part[(size_t)b * NPAR + p];
  if (grad_out) grad_out[p] = g;
  if (step <= 0) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float mm = b1 * m[p] + (1.f - b1) * g;
  float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  float mh = mm / (1.f - powf(b1, (float)step));
  float vh = vv / (1.f - powf(b2, (float)step));
  par[p] -= lr * mh / (sqrtf(vh) + eps);
}

// FP32 forward pass, one thread per sample (the reference of the tensor-core kernel).
__global__ void k_mlp_forward(const float* __restrict__ par, const float* __restrict__ x, int n, float* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  float xi[MI], h1[MH];
  for (int k = 0; k < MI; ++k) xi[k] = x[(size_t)r * MI + k];
  for (int j = 0; j < MH; ++j) {
    float z = par[OB1 + j];
    for (int k = 0; k < MI; ++k) z += par[OW1 + j * MI + k] * xi[k];
    h1[j] = gelu(z);
  }
  float o3[MO];
  for (int o = 0; o < MO; ++o) o3[o] = par[OB3 + o];
  for (int j = 0; j < MH; ++j) {
    float z = par[OB2 + j];
    for (int k = 0; k < MH; ++k) z += par[OW2 + j * MH + k] * h1[k];
    float h = gelu(z);
    for (int o = 0; o < MO; ++o) o3[o] += par[OW3 + o * MH + j] * h;
  }
  for (int o = 0; o < MO; ++o) out[(size_t)r * MO + o] = o3[o];
}

}  // namespace

struct fvg_mlp {
  float *par = nullptr, *m = nullptr, *v = nullptr, *part = nullptr, *lpart = nullptr, *grad = nullptr;
  float* loss = nullptr;
  int* idx = nullptr;
  int idx_cap = 0, part_blocks = 0, step = 0;
  cudaStream_t stream = nullptr;
  std::string err;
};

static int mlp_cuda(fvg_mlp* q, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FVG_OK;
  q->err = std::string(what) + ": " + cudaGetErrorString(e);
  return FVG_ERR_CUDA;
}
#define MK(call) do { int rc_ = mlp_cuda(q, (call), #call); if (rc_) return rc_; } while (0)

static int mlp_parts(fvg_mlp* q, int nblk) {
  if (nblk <= q->part_blocks) return FVG_OK;
  if (q->part) cudaFree(q->part);
  if (q->lpart) cudaFree(q->lpart);
  q->part = nullptr;
  q->lpart = nullptr;
  MK(cudaMalloc(&q->part, (size_t)nblk * NPAR * sizeof(float)));
  MK(cudaMalloc(&q->lpart, (size_t)nblk * sizeof(float)));
  q->part_blocks = nblk;
  return FVG_OK;
}

// One pass of forward/backward over samples b0..b0+nb-1 of the order idx (or the rows
// in order), gradient summed into q->grad; an Adam step when step > 0.
static int mlp_pass(fvg_mlp* q, const float* x, const float* y, const int* idx, int b0, int nb, int step,
                    float lr, float scale) {
  const int nblk = (nb + T - 1) / T;
  int rc = mlp_parts(q, nblk);
  if (rc) return rc;
  k_mlp_fwd_bwd<<<nblk, T, SM_TOTAL * sizeof(float), q->stream>>>(q->par, x, y, idx, b0, nb, scale, q->part,
                                                                    q->lpart);
  k_mlp_adam<<<(NPAR + 255) / 256, 256, 0, q->stream>>>(q->par, q->m, q->v, q->part, nblk, q->grad, q->lpart,
                                                         q->loss, step, lr);
  MK(cudaGetLastError());
  return FVG_OK;
}

extern "C" {

int fvg_mlp_create(uint64_t seed, fvg_mlp** out) {
  if (!out) return FVG_ERR_ARG;
  *out = nullptr;
  fvg_mlp* q = new fvg_mlp();
  auto fail = [&](int rc) { fvg_mlp_destroy(q); return rc; };
  if (cudaFuncSetAttribute(k_mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(SM_TOTAL * sizeof(float))) != cudaSuccess)
    return fail(FVG_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(FVG_ERR_CUDA);
  for (float** p : {&q->par, &q->m, &q->v, &q->grad})
    if (cudaMalloc(p, NPAR * sizeof(float)) != cudaSuccess) return fail(FVG_ERR_NOMEM);
  if (cudaMalloc(&q->loss, sizeof(float)) != cudaSuccess) return fail(FVG_ERR_NOMEM);
  // He-style initialisation scaled by fan-in, biases zero.
  std::vector<float> h(NPAR, 0.f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (int p = OW1; p < OB1; ++p) h[p] = nd(rng) * std::sqrt(2.f / MI);
  for (int p = OW2; p < OB2; ++p) h[p] = nd(rng) * std::sqrt(2.f / MH);
  for (int p = OW3; p < OB3; ++p) h[p] = nd(rng) * std::sqrt(1.f / MH);
  if (cudaMemcpy(q->par, h.data(), NPAR * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(q->m, 0, NPAR * sizeof(float)) != cudaSuccess || cudaMemset(q->v, 0, NPAR * sizeof(float)) != cudaSuccess)
    return fail(FVG_ERR_CUDA);
  *out = q;
  return FVG_OK;
}

void fvg_mlp_destroy(fvg_mlp* q) {
  if (!q) return;
  if (q->stream) cudaStreamSynchronize(q->stream);
  for (float* p : {q->par, q->m, q->v, q->part, q->lpart, q->grad, q->loss})
    if (p) cudaFree(p);
  if (q->idx) cudaFree(q->idx);
  if (q->stream) cudaStreamDestroy(q->stream);
  delete q;
}

const char* fvg_mlp_last_error(const fvg_mlp* q) { return q ? q->err.c_str() : "null network"; }

int32_t fvg_mlp_num_params(void) { return NPAR; }

int fvg_mlp_get_params(fvg_mlp* q, float* host, int32_t n) {
  if (!q || !host || n != NPAR) return FVG_ERR_ARG;
  MK(cudaStreamSynchronize(q->stream));
  MK(cudaMemcpy(host, q->par, NPAR * sizeof(float), cudaMemcpyDeviceToHost));
  return FVG_OK;
}

int fvg_mlp_set_params(fvg_mlp* q, const float* host, int32_t n) {
  if (!q || !host || n != NPAR) return FVG_ERR_ARG;
  MK(cudaStreamSynchronize(q->stream));
  MK(cudaMemcpy(q->par, host, NPAR * sizeof(float), cudaMemcpyHostToDevice));
  MK(cudaMemset(q->m, 0, NPAR * sizeof(float)));
  MK(cudaMemset(q->v, 0, NPAR * sizeof(float)));
  q->step = 0;
  return FVG_OK;
}

int fvg_mlp_loss_grad(fvg_mlp* q, const float* x, const float* y, int32_t n, float* loss, float* grad) {
  if (!q || !x || !y || n < 1 || !loss || !grad) return FVG_ERR_ARG;
  MK(cudaMemsetAsync(q->loss, 0, sizeof(float), q->stream));
  int rc = mlp_pass(q, x, y, nullptr, 0, n, 0, 0.f, 1.f / ((float)n * MO));
  if (rc) return rc;
  MK(cudaMemcpyAsync(grad, q->grad, NPAR * sizeof(float), cudaMemcpyDeviceToHost, q->stream));
  MK(cudaMemcpyAsync(loss, q->loss, sizeof(float), cudaMemcpyDeviceToHost, q->stream));
  MK(cudaStreamSynchronize(q->stream));
  *loss /= (float)n * MO;
  return FVG_OK;
}

int fvg_mlp_train(fvg_mlp* q, const float* x, const float* y, int32_t n, int32_t epochs, int32_t batch,
                  float lr, uint64_t seed, float* epoch_loss) {
  if (!q || !x || !y || n < 1 || epochs < 1 || batch < 1 || batch > n) return FVG_ERR_ARG;
  if (n > q->idx_cap) {
    if (q->idx) cudaFree(q->idx);
    q->idx = nullptr;
    MK(cudaMalloc(&q->idx, (size_t)n * sizeof(int)));
    q->idx_cap = n;
  }
  std::vector<int> order(n);
  std::mt19937_64 rng(seed);
  for (int e = 0; e < epochs; ++e) {
    for (int i = 0; i < n; ++i) order[i] = i;
    std::shuffle(order.begin(), order.end(), rng);
    MK(cudaStreamSynchronize(q->stream));
    MK(cudaMemcpyAsync(q->idx, order.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, q->stream));
    MK(cudaMemsetAsync(q->loss, 0, sizeof(float), q->stream));
    const int nbat = n / batch;
    for (int b = 0; b < nbat; ++b) {
      q->step += 1;
      int rc = mlp_pass(q, x, y, q->idx, b * batch, batch, q->step, lr, 1.f / ((float)batch * MO));
      if (rc) return rc;
    }
    float l = 0.f;
    MK(cudaMemcpyAsync(&l, q->loss, sizeof(float), cudaMemcpyDeviceToHost, q->stream));
    MK(cudaStreamSynchronize(q->stream));
    if (epoch_loss) epoch_loss[e] = l / ((float)nbat * batch * MO);
  }
  return FVG_OK;
}

int fvg_mlp_forward(fvg_mlp* q, const float* x, int32_t n, float* out) {
  if (!q || !x || !out || n < 1) return FVG_ERR_ARG;
  k_mlp_forward<<<(n + 127) / 128, 128, 0, q->stream>>>(q->par, x, n, out);
  MK(cudaGetLastError());
  MK(cudaStreamSynchronize(q->stream));
  return FVG_OK;
}

const float* fvg_mlp_device_params(const fvg_mlp* q) { return q ? q->par : nullptr; }

int fvg_mlp_forward_bf16(fvg_mlp* q, const float* x, int32_t n, float* out) {
  if (!q || !x || !out || n < 1) return FVG_ERR_ARG;
  if (fvg::closure_setup_attrs()) { q->err = "cannot configure the tensor-core kernel"; return FVG_ERR_CUDA; }
  std::vector<float> h(NPAR);
  MK(cudaStreamSynchronize(q->stream));
  MK(cudaMemcpy(h.data(), q->par, NPAR * sizeof(float), cudaMemcpyDeviceToHost));
  std::vector<uint8_t> img;
  std::vector<float> bias;
  fvg::closure_weight_image(h.data(), img, bias);
  void* dimg = nullptr;
  float* dbias = nullptr;
  int* derr = nullptr;
  int rc = FVG_OK;
  auto cleanup = [&]() {
    if (dimg) cudaFree(dimg);
    if (dbias) cudaFree(dbias);
    if (derr) cudaFree(derr);
  };
  if (cudaMalloc(&dimg, img.size()) != cudaSuccess || cudaMalloc(&dbias, bias.size() * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&derr, sizeof(int)) != cudaSuccess) {
    cleanup();
    return FVG_ERR_NOMEM;
  }
  cudaMemcpy(dimg, img.data(), img.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(dbias, bias.data(), bias.size() * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(derr, 0, sizeof(int));
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int tiles = (n + 127) / 128;
  fvg::launch_mlp_tc_forward(dimg, dbias, x, n, out, derr, tiles < 2 * nsm ? tiles : 2 * nsm, q->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(q->stream);
  int herr = 0;
  if (e == cudaSuccess) cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
  cleanup();
  if (e != cudaSuccess) { q->err = cudaGetErrorString(e); return FVG_ERR_CUDA; }
  if (herr) { q->err = "a tensor-core wait ran out"; rc = FVG_ERR_TIMEOUT; }
  return rc;
}

}  // extern "C"
