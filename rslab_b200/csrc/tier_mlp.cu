// Precision-tier network: a 8 -> 64 -> 64 -> 3 MLP (ReLU, softmax) that picks
// the refined factor's precision tier (FP64 / FP32 / TF32x3) from a matrix's
// size, fill, norm and diagonal-dominance features.  Training (weighted
// cross-entropy, full-batch Adam) and inference run in these kernels; the
// host only moves data.  FP32 CUDA-core arithmetic: at 4,931 parameters and
// a few thousand samples the whole epoch is a few microseconds of work, far
// below what would pay for tensor-core tiles.
//
// Parameter layout (floats): W1[64][8], b1[64], W2[64][64], b2[64], W3[3][64],
// b3[3] (row = output unit).  Per-block gradient partials are summed over
// blocks in block order, so a gradient and a training run are reproducible
// bit for bit on a given launch configuration.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/rslab_b200.h"

namespace rslab {
void set_last_error(const std::string& msg);
}

namespace {

constexpr int IN = RSLAB_TIER_FEATURES, HID = RSLAB_TIER_HIDDEN, OUT = RSLAB_TIER_COUNT;
constexpr int O_W1 = 0, O_B1 = O_W1 + HID * IN, O_W2 = O_B1 + HID, O_B2 = O_W2 + HID * HID, O_W3 = O_B2 + HID,
              O_B3 = O_W3 + OUT * HID, NPARAM = O_B3 + OUT;
static_assert(NPARAM == RSLAB_TIER_MLP_PARAMS, "parameter count");
constexpr int SPB = 32;            // samples per block
constexpr int LD1 = IN + 1;        // padded smem row strides (bank-conflict free row reads)
constexpr int LD2 = HID + 1;

struct Smem {
  float w1[HID * LD1], b1[HID], w2[HID * LD2], b2[HID], w3[OUT * HID], b3[OUT];
  float xs[IN], h1[HID], h2[HID], z[OUT], dz[OUT], dh2[HID];
};

// One block of HID threads handles up to SPB samples one after another:
// thread j owns hidden unit j of both layers (and column j of W3), so every
// gradient it accumulates is its own row; partials go to gpart[block].
// probs (m x OUT) and gpart are optional; lpart[block] = sum_s w_s CE_s.
__global__ void __launch_bounds__(HID) k_tier_fwd_grad(const float* __restrict__ p, const float* __restrict__ x,
                                                      const int32_t* __restrict__ y, const float* __restrict__ w,
                                                      long long m, float inv_wsum, float* __restrict__ probs,
                                                      float* __restrict__ gpart, float* __restrict__ lpart) {
  __shared__ Smem S;
  const int j = threadIdx.x;
  for (int i = j; i < HID * IN; i += HID) S.w1[(i / IN) * LD1 + i % IN] = p[O_W1 + i];
  for (int i = j; i < HID * HID; i += HID) S.w2[(i / HID) * LD2 + i % HID] = p[O_W2 + i];
  for (int i = j; i < OUT * HID; i += HID) S.w3[i] = p[O_W3 + i];
  S.b1[j] = p[O_B1 + j];
  S.b2[j] = p[O_B2 + j];
  if (j < OUT) S.b3[j] = p[O_B3 + j];
  const bool grad = gpart != nullptr;
  float g1[IN], g2[HID], g3[OUT], gb1 = 0.f, gb2 = 0.f, gb3[OUT];
#pragma unroll
  for (int k = 0; k < IN; ++k) g1[k] = 0.f;
#pragma unroll
  for (int k = 0; k < HID; ++k) g2[k] = 0.f;
#pragma unroll
  for (int k = 0; k < OUT; ++k) g3[k] = gb3[k] = 0.f;
  float loss = 0.f;
  const long long s0 = (long long)blockIdx.x * SPB;
  const long long s1 = s0 + SPB < m ? s0 + SPB : m;
  __syncthreads();
  for (long long s = s0; s < s1; ++s) {
    if (j < IN) S.xs[j] = x[s * IN + j];
    __syncthreads();
    float a = S.b1[j];
#pragma unroll
    for (int k = 0; k < IN; ++k) a = fmaf(S.w1[j * LD1 + k], S.xs[k], a);
    const float h1 = fmaxf(a, 0.f);
    S.h1[j] = h1;
    __syncthreads();
    a = S.b2[j];
#pragma unroll 16
    for (int k = 0; k < HID; ++k) a = fmaf(S.w2[j * LD2 + k], S.h1[k], a);
    const float h2 = fmaxf(a, 0.f);
    S.h2[j] = h2;
    __syncthreads();
    if (j < OUT) {
      float t = S.b3[j];
      for (int k = 0; k < HID; ++k) t = fmaf(S.w3[j * HID + k], S.h2[k], t);
      S.z[j] = t;
    }
    __syncthreads();
    if (j == 0) {
      float zmax = S.z[0];
      for (int k = 1; k < OUT; ++k) zmax = fmaxf(zmax, S.z[k]);
      float e[OUT], sum = 0.f;
      for (int k = 0; k < OUT; ++k) {
        e[k] = expf(S.z[k] - zmax);
        sum += e[k];
      }
      const int lab = y ? y[s] : -1;
      const float ws = w ? w[s] : 1.f;
      for (int k = 0; k < OUT; ++k) {
        const float pk = e[k] / sum;
        if (probs) probs[s * OUT + k] = pk;
        S.dz[k] = ws * inv_wsum * (pk - (k == lab ? 1.f : 0.f));
      }
      if (lab >= 0 && lab < OUT) loss += ws * (logf(sum) - (S.z[lab] - zmax));
    }
    __syncthreads();
    if (grad) {
      float d = 0.f;
#pragma unroll
      for (int k = 0; k < OUT; ++k) {
        g3[k] = fmaf(S.dz[k], h2, g3[k]);
        d = fmaf(S.w3[k * HID + j], S.dz[k], d);
      }
      if (j == 0)
        for (int k = 0; k < OUT; ++k) gb3[k] += S.dz[k];
      const float dh2 = h2 > 0.f ? d : 0.f;
      S.dh2[j] = dh2;
      gb2 += dh2;
#pragma unroll
      for (int k = 0; k < HID; ++k) g2[k] = fmaf(dh2, S.h1[k], g2[k]);
      __syncthreads();
      float d1 = 0.f;
#pragma unroll 16
      for (int i = 0; i < HID; ++i) d1 = fmaf(S.w2[i * LD2 + j], S.dh2[i], d1);
      const float dh1 = h1 > 0.f ? d1 : 0.f;
      gb1 += dh1;
#pragma unroll
      for (int k = 0; k < IN; ++k) g1[k] = fmaf(dh1, S.xs[k], g1[k]);
    }
    __syncthreads();
  }
  if (grad) {
    float* g = gpart + (size_t)blockIdx.x * NPARAM;
#pragma unroll
    for (int k = 0; k < IN; ++k) g[O_W1 + j * IN + k] = g1[k];
    g[O_B1 + j] = gb1;
#pragma unroll
    for (int k = 0; k < HID; ++k) g[O_W2 + j * HID + k] = g2[k];
    g[O_B2 + j] = gb2;
#pragma unroll
    for (int k = 0; k < OUT; ++k) g[O_W3 + k * HID + j] = g3[k];
    if (j == 0)
      for (int k = 0; k < OUT; ++k) g[O_B3 + k] = gb3[k];
  }
  if (j == 0 && lpart) lpart[blockIdx.x] = loss;
}

// grad[i] = sum over blocks (in block order) of gpart[b][i]; with Adam state
// given, also one Adam step on params.  Thread 0 of block 0 sums the loss
// partials (block order) into *loss.
__global__ void k_tier_reduce(const float* __restrict__ gpart, int nblk, const float* __restrict__ lpart,
                              float inv_wsum, float* __restrict__ grad, float* __restrict__ loss,
                              float* __restrict__ params, float* __restrict__ mom, float* __restrict__ vel,
                              float lr, float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && loss) {
    float l = 0.f;
    for (int b = 0; b < nblk; ++b) l += lpart[b];
    *loss = l * inv_wsum;
  }
  if (i >= NPARAM) return;
  float g = 0.f;
  for (int b = 0; b < nblk; ++b) g += gpart[(size_t)b * NPARAM + i];
  if (grad) grad[i] = g;
  if (params) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float mi = b1 * mom[i] + (1.f - b1) * g;
    const float vi = b2 * vel[i] + (1.f - b2) * g * g;
    mom[i] = mi;
    vel[i] = vi;
    params[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

struct Err {
  std::string msg;
};
#define TK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) throw Err{std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

// Device copies of the caller's arrays (or the caller's device pointers).
struct Dev {
  std::vector<void*> owned;
  cudaStream_t st = nullptr;
  Dev() { TK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)); }
  ~Dev() {
    if (st) cudaStreamSynchronize(st);
    for (void* q : owned) cudaFree(q);
    if (st) cudaStreamDestroy(st);
  }
  template <typename T>
  T* alloc(size_t count) {
    void* q = nullptr;
    TK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
    owned.push_back(q);
    return (T*)q;
  }
  template <typename T>
  const T* in(const T* src, size_t count, bool on_device) {
    if (!src || on_device) return src;
    T* d = alloc<T>(count);
    TK(cudaMemcpyAsync(d, src, count * sizeof(T), cudaMemcpyHostToDevice, st));
    return d;
  }
  template <typename T>
  void out(T* dst, const T* dev, size_t count, bool on_device) {
    if (!dst || on_device) return;
    TK(cudaMemcpyAsync(dst, dev, count * sizeof(T), cudaMemcpyDeviceToHost, st));
  }
};

int fail_msg(const std::string& m) {
  rslab::set_last_error(m);
  return RSLAB_INVALID_INPUT;
}

int check_args(const void* params, const void* x, int64_t m) {
  if (!params || (!x && m > 0)) return fail_msg("tier network: null params or features");
  if (m < 0) return fail_msg("tier network: negative sample count");
  return RSLAB_OK;
}

// sum of weights (host or device array), 1 per sample when w is NULL
float weight_sum(Dev& D, const float* w, int64_t m, bool on_device) {
  if (!w) return (float)m;
  std::vector<float> h(m);
  if (on_device) {
    TK(cudaMemcpyAsync(h.data(), w, m * sizeof(float), cudaMemcpyDeviceToHost, D.st));
    TK(cudaStreamSynchronize(D.st));
  } else {
    std::copy(w, w + m, h.begin());
  }
  double s = 0;
  for (float v : h) {
    if (!(v >= 0.f) || !std::isfinite(v)) throw Err{"tier network: sample weights must be finite and >= 0"};
    s += v;
  }
  if (!(s > 0)) throw Err{"tier network: sample weights sum to zero"};
  return (float)s;
}

void check_labels(Dev& D, const int32_t* y, int64_t m, bool on_device) {
  std::vector<int32_t> h(m);
  if (on_device) {
    TK(cudaMemcpyAsync(h.data(), y, m * sizeof(int32_t), cudaMemcpyDeviceToHost, D.st));
    TK(cudaStreamSynchronize(D.st));
  } else {
    std::copy(y, y + m, h.begin());
  }
  for (int32_t v : h)
    if (v < 0 || v >= OUT) throw Err{"tier network: labels must be 0, 1 or 2"};
}

}  // namespace

extern "C" {

int rslab_tier_mlp_forward(const float* params, const float* x, int64_t m, float* probs, int on_device) {
  if (int rc = check_args(params, x, m)) return rc;
  if (!probs) return fail_msg("tier network: null probs");
  if (m == 0) return RSLAB_OK;
  try {
    Dev D;
    const bool od = on_device != 0;
    const float* p = D.in(params, NPARAM, od);
    const float* xd = D.in(x, (size_t)m * IN, od);
    float* pr = od ? probs : D.alloc<float>((size_t)m * OUT);
    const int nblk = (int)((m + SPB - 1) / SPB);
    k_tier_fwd_grad<<<nblk, HID, 0, D.st>>>(p, xd, nullptr, nullptr, m, 1.f, pr, nullptr, nullptr);
    TK(cudaGetLastError());
    D.out(probs, pr, (size_t)m * OUT, od);
    TK(cudaStreamSynchronize(D.st));
    return RSLAB_OK;
  } catch (const Err& e) {
    return fail_msg(e.msg);
  }
}

int rslab_tier_mlp_grad(const float* params, const float* x, const int32_t* y, const float* w, int64_t m,
                        float* grad, float* loss, int on_device) {
  if (int rc = check_args(params, x, m)) return rc;
  if (!y || !grad || !loss) return fail_msg("tier network: null labels, grad or loss");
  if (m == 0) return fail_msg("tier network: no samples");
  try {
    Dev D;
    const bool od = on_device != 0;
    check_labels(D, y, m, od);
    const float inv = 1.f / weight_sum(D, w, m, od);
    const float* p = D.in(params, NPARAM, od);
    const float* xd = D.in(x, (size_t)m * IN, od);
    const int32_t* yd = D.in(y, (size_t)m, od);
    const float* wd = D.in(w, (size_t)m, od);
    const int nblk = (int)((m + SPB - 1) / SPB);
    float* gpart = D.alloc<float>((size_t)nblk * NPARAM);
    float* lpart = D.alloc<float>(nblk);
    float* gd = od ? grad : D.alloc<float>(NPARAM);
    float* ld = od ? loss : D.alloc<float>(1);
    k_tier_fwd_grad<<<nblk, HID, 0, D.st>>>(p, xd, yd, wd, m, inv, nullptr, gpart, lpart);
    k_tier_reduce<<<(NPARAM + 255) / 256, 256, 0, D.st>>>(gpart, nblk, lpart, inv, gd, ld, nullptr, nullptr,
                                                          nullptr, 0.f, 1.f, 1.f);
    TK(cudaGetLastError());
    D.out(grad, gd, NPARAM, od);
    D.out(loss, ld, 1, od);
    TK(cudaStreamSynchronize(D.st));
    return RSLAB_OK;
  } catch (const Err& e) {
    return fail_msg(e.msg);
  }
}

int rslab_tier_mlp_train(float* params, const float* x, const int32_t* y, const float* w, int64_t m, int64_t epochs,
                         float lr, float* loss_curve, int on_device) {
  if (int rc = check_args(params, x, m)) return rc;
  if (!y) return fail_msg("tier network: null labels");
  if (m == 0) return fail_msg("tier network: no samples");
  if (epochs < 0 || !(lr > 0.f)) return fail_msg("tier network: epochs >= 0 and lr > 0 required");
  try {
    Dev D;
    const bool od = on_device != 0;
    check_labels(D, y, m, od);
    const float inv = 1.f / weight_sum(D, w, m, od);
    float* p = od ? params : D.alloc<float>(NPARAM);
    if (!od) TK(cudaMemcpyAsync(p, params, NPARAM * sizeof(float), cudaMemcpyHostToDevice, D.st));
    const float* xd = D.in(x, (size_t)m * IN, od);
    const int32_t* yd = D.in(y, (size_t)m, od);
    const float* wd = D.in(w, (size_t)m, od);
    const int nblk = (int)((m + SPB - 1) / SPB);
    float* gpart = D.alloc<float>((size_t)nblk * NPARAM);
    float* lpart = D.alloc<float>(nblk);
    float* mom = D.alloc<float>(NPARAM);
    float* vel = D.alloc<float>(NPARAM);
    TK(cudaMemsetAsync(mom, 0, NPARAM * sizeof(float), D.st));
    TK(cudaMemsetAsync(vel, 0, NPARAM * sizeof(float), D.st));
    float* lc = nullptr;
    if (loss_curve) lc = od ? loss_curve : D.alloc<float>((size_t)std::max<int64_t>(epochs, 1));
    double bc1 = 1.0, bc2 = 1.0;
    for (int64_t e = 0; e < epochs; ++e) {
      bc1 *= 0.9;
      bc2 *= 0.999;
      k_tier_fwd_grad<<<nblk, HID, 0, D.st>>>(p, xd, yd, wd, m, inv, nullptr, gpart, lpart);
      k_tier_reduce<<<(NPARAM + 255) / 256, 256, 0, D.st>>>(gpart, nblk, lpart, inv, nullptr, lc ? lc + e : nullptr,
                                                            p, mom, vel, lr, (float)(1.0 - bc1), (float)(1.0 - bc2));
    }
    TK(cudaGetLastError());
    if (!od) TK(cudaMemcpyAsync(params, p, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, D.st));
    if (loss_curve && !od) D.out(loss_curve, lc, (size_t)epochs, false);
    TK(cudaStreamSynchronize(D.st));
    return RSLAB_OK;
  } catch (const Err& e) {
    return fail_msg(e.msg);
  }
}

}  // extern "C"
