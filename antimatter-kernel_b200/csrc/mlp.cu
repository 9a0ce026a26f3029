// Learned far-field correction: a 35 -> 128 -> 128 -> 128 -> 3 MLP with GELU
// activations, BF16 weights and FP32 accumulation (no reference
// counterpart).
//
// Inference runs on the 5th-generation tensor cores: a persistent CTA keeps
// all weights in shared memory (BF16, the canonical K-major no-swizzle
// layout of 8-row x 16-byte core matrices), stages each 128-particle tile of
// features as BF16, and issues tcgen05.mma (M = 128, K = 16 per
// instruction) from one thread into an FP32 accumulator in tensor memory;
// the four warps read their 32 rows back with tcgen05.ld, add the bias,
// apply GELU and write the next layer's BF16 operand. Completion of each
// layer is tracked by tcgen05.commit on an mbarrier whose waits are
// bounded (a timeout sets an error flag and the kernel returns).
//
// Training (forward with stored activations, backward, Adam) runs in FP32
// on the CUDA cores with the same BF16-rounded weights: it is small next to
// inference and is checked against an FP64 CPU implementation.
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "amk_internal.cuh"
#include "philox.cuh"
#include "tcgen05.cuh"

namespace amk {

constexpr int kMlpIn = 35;      // features
constexpr int kMlpInPad = 48;   // K of layer 1 (multiple of 16)
constexpr int kMlpHidden = 128;
constexpr int kMlpOut = 3;
constexpr int kMlpOutPad = 16;  // N of layer 4

// FP32 master parameters, flat: W1[128][35] b1[128] W2[128][128] b2 W3 b3 W4[3][128] b4[3]
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpHidden * kMlpHidden;
constexpr int kOffW4 = kOffB3 + kMlpHidden;
constexpr int kOffB4 = kOffW4 + kMlpOut * kMlpHidden;
constexpr int kMlpParams = kOffB4 + kMlpOut;

struct Mlp {
  DevBuf master, grad, adam_m, adam_v;  // FP32, kMlpParams each
  DevBuf packed;                         // BF16 weights in the tensor-core smem image + FP32 biases
  DevBuf status;                         // int error flag
  long adam_step = 0;
  bool packed_valid = false;
  bool initialized = false;
};

namespace {

// ---------------------------------------------------------------- layout
using namespace tc;  // op_offset: the K-major no-swizzle operand layout

// smem image of the weights (built once on the host side of every update)
constexpr uint32_t kImgW1 = 0;                                            // 128 x 48
constexpr uint32_t kImgW2 = kImgW1 + kMlpHidden * kMlpInPad * 2;          // 128 x 128
constexpr uint32_t kImgW3 = kImgW2 + kMlpHidden * kMlpHidden * 2;
constexpr uint32_t kImgW4 = kImgW3 + kMlpHidden * kMlpHidden * 2;         // 16 x 128
constexpr uint32_t kImgBias = kImgW4 + kMlpOutPad * kMlpHidden * 2;       // FP32: 128*3 + 16
constexpr uint32_t kImgBytes = kImgBias + (3 * kMlpHidden + kMlpOutPad) * 4;
constexpr uint32_t kActBytes = kMlpHidden * kMlpHidden * 2;               // 128 x 128 BF16 operand
constexpr uint32_t kSmemBytes = kImgBytes + kActBytes + 64;               // + mbarrier, TMEM slot

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.3989422804014327f * expf(-0.5f * x * x);
}

// 8 FP32 values -> 8 BF16 packed in 16 bytes
__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 u;
  u.x = (static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(v[1]))) << 16) |
        __bfloat16_as_ushort(__float2bfloat16_rn(v[0]));
  u.y = (static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(v[3]))) << 16) |
        __bfloat16_as_ushort(__float2bfloat16_rn(v[2]));
  u.z = (static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(v[5]))) << 16) |
        __bfloat16_as_ushort(__float2bfloat16_rn(v[4]));
  u.w = (static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(v[7]))) << 16) |
        __bfloat16_as_ushort(__float2bfloat16_rn(v[6]));
  return u;
}

constexpr long kWaitLimit = 1L << 26;  // polls before an mbarrier wait gives up

// Tensor-core inference: y[n][3] = MLP(x[n][35]). One CTA of 128 threads per
// SM walks 128-row tiles. status[0] is set to 1 if a wait times out.
__global__ void __launch_bounds__(128, 1)
mlp_forward_tc_kernel(const unsigned char* __restrict__ img, const float* __restrict__ x, long n,
                      float* __restrict__ y, int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* w_img = sm;
  unsigned char* act = sm + kImgBytes;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + kImgBytes + kActBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kImgBytes + kActBytes + 16);
  const int tid = threadIdx.x, warp = tid >> 5;

  // weights + biases -> smem (16-byte copies)
  for (uint32_t o = tid * 16; o < kImgBytes; o += 128 * 16)
    *reinterpret_cast<uint4*>(w_img + o) = *reinterpret_cast<const uint4*>(img + o);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const float* bias = reinterpret_cast<const float*>(w_img + kImgBias);
  const uint32_t a_base = smem_u32(act), w_base = smem_u32(w_img);
  const uint32_t mbar_a = smem_u32(mbar);
  uint32_t phase = 0;
  bool failed = false;
  const long tiles = (n + 127) / 128;

  auto run_layer = [&](uint32_t w_off, int k_steps, int n_out, int w_rows) -> bool {
    // operands written by all threads are complete and visible to the async proxy
    fence_proxy_async();
    fence_before();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      const uint32_t idesc = make_idesc(n_out);
      for (int s = 0; s < k_steps; ++s) {
        const uint64_t ad = make_sdesc(a_base + s * 128 * 32);
        const uint64_t bd = make_sdesc(w_base + w_off + s * w_rows * 32);
        mma_bf16(tmem, ad, bd, idesc, s > 0);
      }
      mma_commit(mbar_a);
    }
    long spins = 0;
    bool ok = true;
    while (!mbar_try_wait(mbar_a, phase)) {
      if (++spins > kWaitLimit) {
        ok = false;
        break;
      }
    }
    phase ^= 1u;
    fence_after();
    return __syncthreads_and(ok) != 0;  // every thread takes the same decision
  };

  for (long tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
    const long row = tile * 128 + tid;
    // ---- features -> BF16 operand (K padded to 48 with zeros)
    {
      float f[kMlpInPad];
#pragma unroll
      for (int k = 0; k < kMlpInPad; ++k) f[k] = 0.f;
      if (row < n)
        for (int k = 0; k < kMlpIn; ++k) f[k] = x[row * kMlpIn + k];
#pragma unroll
      for (int c = 0; c < kMlpInPad / 8; ++c)
        *reinterpret_cast<uint4*>(act + op_offset(tid, c * 8, 128)) = pack8(f + c * 8);
    }
    // ---- three hidden layers
    const uint32_t w_offs[3] = {kImgW1, kImgW2, kImgW3};
    const int ksteps[3] = {kMlpInPad / 16, kMlpHidden / 16, kMlpHidden / 16};
    for (int l = 0; l < 3 && !failed; ++l) {
      if (!run_layer(w_offs[l], ksteps[l], kMlpHidden, kMlpHidden)) {
        failed = true;
        break;
      }
      const float* b = bias + l * kMlpHidden;
      for (int c0 = 0; c0 < kMlpHidden; c0 += 32) {
        float v[32];
        tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, v);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = gelu(v[i] + b[c0 + i]);
#pragma unroll
        for (int c = 0; c < 4; ++c)
          *reinterpret_cast<uint4*>(act + op_offset(tid, c0 + c * 8, 128)) = pack8(v + c * 8);
      }
    }
    if (failed) break;
    // ---- output layer (N = 16, first 3 used)
    if (!run_layer(kImgW4, kMlpHidden / 16, kMlpOutPad, kMlpOutPad)) {
      failed = true;
      break;
    }
    {
      float v[16];
      tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16), v);
      const float* b = bias + 3 * kMlpHidden;
      if (row < n)
        for (int o = 0; o < kMlpOut; ++o) y[row * kMlpOut + o] = v[o] + b[o];
    }
  }
  if (failed && tid == 0) atomicExch(status, 1);
  fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
}

// Packs FP32 masters into the BF16 shared-memory image + FP32 biases.
__global__ void mlp_pack_kernel(const float* __restrict__ p, unsigned char* __restrict__ img) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  auto put = [&](uint32_t base, int rows, int r, int k, float v) {
    *reinterpret_cast<__nv_bfloat16*>(img + base + op_offset(r, k, rows)) = __float2bfloat16_rn(v);
  };
  if (i < kMlpHidden * kMlpInPad) {  // W1 (K padded)
    const int r = i / kMlpInPad, k = i % kMlpInPad;
    put(kImgW1, kMlpHidden, r, k, k < kMlpIn ? p[kOffW1 + r * kMlpIn + k] : 0.f);
  }
  if (i < kMlpHidden * kMlpHidden) {
    const int r = i / kMlpHidden, k = i % kMlpHidden;
    put(kImgW2, kMlpHidden, r, k, p[kOffW2 + i]);
    put(kImgW3, kMlpHidden, r, k, p[kOffW3 + i]);
  }
  if (i < kMlpOutPad * kMlpHidden) {  // W4 (N padded)
    const int r = i / kMlpHidden, k = i % kMlpHidden;
    put(kImgW4, kMlpOutPad, r, k, r < kMlpOut ? p[kOffW4 + r * kMlpHidden + k] : 0.f);
  }
  float* bias = reinterpret_cast<float*>(img + kImgBias);
  if (i < kMlpHidden) {
    bias[i] = p[kOffB1 + i];
    bias[kMlpHidden + i] = p[kOffB2 + i];
    bias[2 * kMlpHidden + i] = p[kOffB3 + i];
  }
  if (i < kMlpOutPad) bias[3 * kMlpHidden + i] = i < kMlpOut ? p[kOffB4 + i] : 0.f;
}

// ---------------------------------------------------------------- training (FP32)
__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// Z = W_bf16 X + b for a batch: one thread per (sample, output unit).
__global__ void mlp_dense_kernel(const float* __restrict__ p, int w_off, int b_off, int in, int out,
                                 const float* __restrict__ xin, long batch, float* __restrict__ z,
                                 float* __restrict__ h, bool act) {
  const long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (t >= batch * out) return;
  const long s = t / out;
  const int o = static_cast<int>(t - s * out);
  const float* w = p + w_off + o * in;
  const float* xi = xin + s * in;
  float acc = 0.f;
  for (int k = 0; k < in; ++k) acc = fmaf(bf16r(w[k]), xi[k], acc);
  acc += p[b_off + o];
  z[t] = acc;
  if (h) h[t] = act ? gelu(acc) : acc;
}

// dX[s][k] = sum_o dZ[s][o] W[o][k]
__global__ void mlp_back_input_kernel(const float* __restrict__ p, int w_off, int in, int out,
                                      const float* __restrict__ dz, long batch, const float* __restrict__ zprev,
                                      float* __restrict__ dzprev) {
  const long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (t >= batch * in) return;
  const long s = t / in;
  const int k = static_cast<int>(t - s * in);
  float acc = 0.f;
  for (int o = 0; o < out; ++o) acc = fmaf(dz[s * out + o], bf16r(p[w_off + o * in + k]), acc);
  dzprev[t] = acc * gelu_grad(zprev[t]);
}

// dW[o][k] = sum_s dZ[s][o] X[s][k], db[o] = sum_s dZ[s][o] (fixed summation order)
__global__ void mlp_back_weight_kernel(int w_off, int b_off, int in, int out, const float* __restrict__ dz,
                                       const float* __restrict__ xin, long batch, float* __restrict__ g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < out * in) {
    const int o = t / in, k = t % in;
    float acc = 0.f;
    for (long s = 0; s < batch; ++s) acc = fmaf(dz[s * out + o], xin[s * in + k], acc);
    g[w_off + t] = acc;
  }
  if (t < out) {
    float acc = 0.f;
    for (long s = 0; s < batch; ++s) acc += dz[s * out + t];
    g[b_off + t] = acc;
  }
}

// loss = mean over batch and outputs of (y - target)^2; dY = 2 (y - target) / (batch * 3)
__global__ void mlp_loss_kernel(const float* __restrict__ yhat, const float* __restrict__ target, long batch,
                                float* __restrict__ dy, float* __restrict__ loss_part) {
  __shared__ float sh[256];
  float acc = 0.f;
  const long total = batch * kMlpOut;
  for (long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long>(gridDim.x) * blockDim.x) {
    const float d = yhat[t] - target[t];
    dy[t] = 2.f * d / static_cast<float>(total);
    acc += d * d;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = sh[0];
}

__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1,
                                float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void mlp_init_kernel(float* __restrict__ p, uint32_t seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams) return;
  int fan_in = 0;
  bool bias = false;
  if (i < kOffB1) fan_in = kMlpIn;
  else if (i < kOffW2) bias = true;
  else if (i < kOffB2) fan_in = kMlpHidden;
  else if (i < kOffW3) bias = true;
  else if (i < kOffB3) fan_in = kMlpHidden;
  else if (i < kOffW4) bias = true;
  else if (i < kOffB4) fan_in = kMlpHidden;
  else bias = true;
  if (bias) {
    p[i] = 0.f;
    return;
  }
  const Philox4 w = philox4x32(seed, 0x3A71u, static_cast<uint32_t>(i), 0u, 0u, 0u);
  const float u = static_cast<float>(u01(w.w[0])) * 2.f - 1.f;  // U(-1, 1)
  p[i] = u * sqrtf(3.f / static_cast<float>(fan_in));           // variance 1 / fan_in
}

}  // namespace

// ---------------------------------------------------------------- host side
static int mlp_get(amk_ctx* c, Mlp** out) {
  if (!c->mlp) c->mlp = new Mlp();
  Mlp* m = c->mlp;
  if (!m->initialized) {
    const size_t pb = kMlpParams * sizeof(float);
    AMK_TRY(m->master.reserve(pb));
    AMK_TRY(m->grad.reserve(pb));
    AMK_TRY(m->adam_m.reserve(pb));
    AMK_TRY(m->adam_v.reserve(pb));
    AMK_TRY(m->packed.reserve(kImgBytes));
    AMK_TRY(m->status.reserve(16));
    AMK_CUDA_TRY(cudaMemsetAsync(m->adam_m.ptr, 0, pb, c->stream));
    AMK_CUDA_TRY(cudaMemsetAsync(m->adam_v.ptr, 0, pb, c->stream));
    AMK_CUDA_TRY(cudaMemsetAsync(m->packed.ptr, 0, kImgBytes, c->stream));
    mlp_init_kernel<<<(kMlpParams + 255) / 256, 256, 0, c->stream>>>(m->master.as<float>(), 12345u);
    AMK_TRY(check_launch(c, "mlp_init_kernel"));
    m->initialized = true;
    m->packed_valid = false;
  }
  *out = m;
  return AMK_OK;
}

static int mlp_pack(amk_ctx* c, Mlp* m) {
  if (m->packed_valid) return AMK_OK;
  mlp_pack_kernel<<<(kMlpHidden * kMlpHidden + 255) / 256, 256, 0, c->stream>>>(m->master.as<float>(),
                                                                                 m->packed.as<unsigned char>());
  AMK_TRY(check_launch(c, "mlp_pack_kernel"));
  m->packed_valid = true;
  return AMK_OK;
}

// Device-side inference on device buffers (used by the learned FMM).
int mlp_forward_device(amk_ctx* c, const float* x, long n, float* y) {
  if (n <= 0) return AMK_OK;
  Mlp* m = nullptr;
  AMK_TRY(mlp_get(c, &m));
  AMK_TRY(mlp_pack(c, m));
  static bool attr_set = false;
  if (!attr_set) {
    AMK_CUDA_TRY(cudaFuncSetAttribute(mlp_forward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kSmemBytes)));
    attr_set = true;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  const long tiles = (n + 127) / 128;
  const int grid = static_cast<int>(std::min<long>(tiles, sms));
  AMK_CUDA_TRY(cudaMemsetAsync(m->status.ptr, 0, sizeof(int), c->stream));
  AMK_TRY(phase_begin(c, AMK_PHASE_MLP));
  mlp_forward_tc_kernel<<<grid, 128, kSmemBytes, c->stream>>>(m->packed.as<unsigned char>(), x, n, y,
                                                              m->status.as<int>());
  AMK_TRY(check_launch(c, "mlp_forward_tc_kernel"));
  AMK_TRY(phase_end(c, AMK_PHASE_MLP));
  return AMK_OK;
}

int mlp_check_status(amk_ctx* c) {
  if (!c->mlp) return AMK_OK;
  int st = 0;
  AMK_CUDA_TRY(cudaMemcpyAsync(&st, c->mlp->status.ptr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (st) return fail(AMK_ERR_TIMEOUT, "tensor-core MLP: an mbarrier wait timed out");
  return AMK_OK;
}

// FP32 forward + backward on a device batch; fills m->grad, returns the loss.
int mlp_gradients_device(amk_ctx* c, const float* x, const float* target, long batch, float* loss_host,
                         float* yhat_out) {
  Mlp* m = nullptr;
  AMK_TRY(mlp_get(c, &m));
  int rc = AMK_OK;
  const long H = kMlpHidden;
  // activations: z1 h1 z2 h2 z3 h3 (batch x 128), z4 (batch x 3), dz buffers
  float* buf = slot<float>(c, kSlotMlp0, static_cast<size_t>(batch) * (6 * H + 2 * kMlpOut + 2 * H) + 1024, &rc);
  AMK_TRY(rc);
  float *z1 = buf, *h1 = z1 + batch * H, *z2 = h1 + batch * H, *h2 = z2 + batch * H, *z3 = h2 + batch * H,
        *h3 = z3 + batch * H, *y = h3 + batch * H, *dy = y + batch * kMlpOut, *da = dy + batch * kMlpOut,
        *db = da + batch * H;
  float* lp = slot<float>(c, kSlotMlp1, 256, &rc);
  AMK_TRY(rc);
  const float* p = m->master.as<float>();
  float* g = m->grad.as<float>();
  auto grid = [](long work) { return static_cast<unsigned>((work + 255) / 256); };
  mlp_dense_kernel<<<grid(batch * H), 256, 0, c->stream>>>(p, kOffW1, kOffB1, kMlpIn, H, x, batch, z1, h1, true);
  mlp_dense_kernel<<<grid(batch * H), 256, 0, c->stream>>>(p, kOffW2, kOffB2, H, H, h1, batch, z2, h2, true);
  mlp_dense_kernel<<<grid(batch * H), 256, 0, c->stream>>>(p, kOffW3, kOffB3, H, H, h2, batch, z3, h3, true);
  mlp_dense_kernel<<<grid(batch * kMlpOut), 256, 0, c->stream>>>(p, kOffW4, kOffB4, H, kMlpOut, h3, batch, y,
                                                                 nullptr, false);
  AMK_TRY(check_launch(c, "mlp_dense_kernel"));
  const int lblocks = 128;
  mlp_loss_kernel<<<lblocks, 256, 0, c->stream>>>(y, target, batch, dy, lp);
  AMK_TRY(check_launch(c, "mlp_loss_kernel"));
  // layer 4
  mlp_back_weight_kernel<<<grid(kMlpOut * H), 256, 0, c->stream>>>(kOffW4, kOffB4, H, kMlpOut, dy, h3, batch, g);
  mlp_back_input_kernel<<<grid(batch * H), 256, 0, c->stream>>>(p, kOffW4, H, kMlpOut, dy, batch, z3, da);
  // layer 3
  mlp_back_weight_kernel<<<grid(H * H), 256, 0, c->stream>>>(kOffW3, kOffB3, H, H, da, h2, batch, g);
  mlp_back_input_kernel<<<grid(batch * H), 256, 0, c->stream>>>(p, kOffW3, H, H, da, batch, z2, db);
  // layer 2
  mlp_back_weight_kernel<<<grid(H * H), 256, 0, c->stream>>>(kOffW2, kOffB2, H, H, db, h1, batch, g);
  mlp_back_input_kernel<<<grid(batch * H), 256, 0, c->stream>>>(p, kOffW2, H, H, db, batch, z1, da);
  // layer 1
  mlp_back_weight_kernel<<<grid(H * kMlpIn), 256, 0, c->stream>>>(kOffW1, kOffB1, kMlpIn, H, da, x, batch, g);
  AMK_TRY(check_launch(c, "mlp_backward"));
  if (yhat_out) AMK_CUDA_TRY(cudaMemcpyAsync(yhat_out, y, batch * kMlpOut * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
  if (loss_host) {
    float h[lblocks];
    AMK_CUDA_TRY(cudaMemcpyAsync(h, lp, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    double s = 0.0;
    for (int b = 0; b < lblocks; ++b) s += h[b];
    *loss_host = static_cast<float>(s / static_cast<double>(batch * kMlpOut));
  }
  return AMK_OK;
}

int mlp_adam_step(amk_ctx* c, float lr) {
  Mlp* m = nullptr;
  AMK_TRY(mlp_get(c, &m));
  m->adam_step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, static_cast<float>(m->adam_step));
  const float c2 = 1.f - std::pow(b2, static_cast<float>(m->adam_step));
  mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, c->stream>>>(m->master.as<float>(), m->grad.as<float>(),
                                                                   m->adam_m.as<float>(), m->adam_v.as<float>(),
                                                                   kMlpParams, lr, b1, b2, 1e-8f, c1, c2);
  AMK_TRY(check_launch(c, "mlp_adam_kernel"));
  m->packed_valid = false;
  return AMK_OK;
}

// Minibatch Adam over a device dataset: batches are consecutive windows of
// the data (wrapping), so a run is deterministic.
int mlp_train_device(amk_ctx* c, const float* x, const float* target, long n, int steps, long batch, float lr,
                     float* final_loss) {
  batch = std::min(batch, n);
  float loss = 0.f;
  for (int s = 0; s < steps; ++s) {
    const long start = (static_cast<long>(s) * batch) % std::max(1L, n - batch + 1);
    const bool last = s + 1 == steps;
    AMK_TRY(mlp_gradients_device(c, x + start * kMlpIn, target + start * kMlpOut, batch, last ? &loss : nullptr,
                                 nullptr));
    AMK_TRY(mlp_adam_step(c, lr));
  }
  if (final_loss) *final_loss = loss;
  return AMK_OK;
}

}  // namespace amk

using namespace amk;

void mlp_destroy(amk_ctx* c) {
  delete c->mlp;
  c->mlp = nullptr;
}

extern "C" int amk_mlp_num_params(void) { return kMlpParams; }

extern "C" int amk_mlp_set_params(amk_ctx* c, const float* params, long n) {
  if (!c || !params || n != kMlpParams) return fail(AMK_ERR_INVALID, "amk_mlp_set_params: expected %d floats", kMlpParams);
  Mlp* m = nullptr;
  AMK_TRY(mlp_get(c, &m));
  AMK_CUDA_TRY(cudaMemcpyAsync(m->master.ptr, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  AMK_CUDA_TRY(cudaMemsetAsync(m->adam_m.ptr, 0, kMlpParams * sizeof(float), c->stream));
  AMK_CUDA_TRY(cudaMemsetAsync(m->adam_v.ptr, 0, kMlpParams * sizeof(float), c->stream));
  m->adam_step = 0;
  m->packed_valid = false;
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

extern "C" int amk_mlp_get_params(amk_ctx* c, float* params, long n) {
  if (!c || !params || n != kMlpParams) return fail(AMK_ERR_INVALID, "amk_mlp_get_params: expected %d floats", kMlpParams);
  Mlp* m = nullptr;
  AMK_TRY(mlp_get(c, &m));
  AMK_CUDA_TRY(cudaMemcpyAsync(params, m->master.ptr, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

extern "C" int amk_mlp_forward(amk_ctx* c, const float* x, long n, float* y) {
  if (!c || n < 0 || (n > 0 && (!x || !y))) return fail(AMK_ERR_INVALID, "amk_mlp_forward: bad argument");
  if (n == 0) return AMK_OK;
  int rc = AMK_OK;
  float* dx = slot<float>(c, kSlotMlp2, static_cast<size_t>(n) * kMlpIn, &rc);
  AMK_TRY(rc);
  float* dy = slot<float>(c, kSlotMlp3, static_cast<size_t>(n) * kMlpOut, &rc);
  AMK_TRY(rc);
  AMK_CUDA_TRY(cudaMemcpyAsync(dx, x, n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  AMK_TRY(mlp_forward_device(c, dx, n, dy));
  AMK_TRY(mlp_check_status(c));
  AMK_CUDA_TRY(cudaMemcpyAsync(y, dy, n * kMlpOut * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

extern "C" int amk_mlp_gradients(amk_ctx* c, const float* x, const float* target, long n, float* grad,
                                 float* loss, float* yhat) {
  if (!c || n <= 0 || !x || !target) return fail(AMK_ERR_INVALID, "amk_mlp_gradients: bad argument");
  int rc = AMK_OK;
  float* dx = slot<float>(c, kSlotMlp2, static_cast<size_t>(n) * kMlpIn, &rc);
  AMK_TRY(rc);
  float* dt = slot<float>(c, kSlotMlp3, static_cast<size_t>(n) * kMlpOut, &rc);
  AMK_TRY(rc);
  float* dyh = slot<float>(c, kSlotMlp4, static_cast<size_t>(n) * kMlpOut, &rc);
  AMK_TRY(rc);
  AMK_CUDA_TRY(cudaMemcpyAsync(dx, x, n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(dt, target, n * kMlpOut * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  float l = 0.f;
  AMK_TRY(mlp_gradients_device(c, dx, dt, n, &l, dyh));
  if (loss) *loss = l;
  if (grad)
    AMK_CUDA_TRY(cudaMemcpyAsync(grad, c->mlp->grad.ptr, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  if (yhat) AMK_CUDA_TRY(cudaMemcpyAsync(yhat, dyh, n * kMlpOut * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

extern "C" int amk_mlp_train(amk_ctx* c, const float* x, const float* target, long n, int steps, long batch,
                             float lr, float* final_loss) {
  if (!c || n <= 0 || !x || !target || steps < 0 || batch <= 0)
    return fail(AMK_ERR_INVALID, "amk_mlp_train: bad argument");
  int rc = AMK_OK;
  float* dx = slot<float>(c, kSlotMlp2, static_cast<size_t>(n) * kMlpIn, &rc);
  AMK_TRY(rc);
  float* dt = slot<float>(c, kSlotMlp3, static_cast<size_t>(n) * kMlpOut, &rc);
  AMK_TRY(rc);
  AMK_CUDA_TRY(cudaMemcpyAsync(dx, x, n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(dt, target, n * kMlpOut * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  return mlp_train_device(c, dx, dt, n, steps, batch, lr, final_loss);
}

