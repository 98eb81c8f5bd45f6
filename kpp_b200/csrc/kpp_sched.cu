// Learned cell scheduler (include/kpp_sched.h): feature extraction, a BF16
// tensor-core MLP with its training kernels (backward, Adam), and the
// scheduling pass that turns the network's predictions into per-cell Hstart
// and a cost-sorted work-queue order for kpp_b200_rosenbrock_chain.
//
// Every matrix product goes through one kernel, gemm_kernel: C = A * B^T over
// BF16 operands with FP32 accumulation on mma.sync.m16n8k16, operands read
// through arbitrary (row, k) strides so that the same kernel serves the
// forward pass (X W^T), the input gradient (dZ W) and the weight gradient
// (dZ^T X, split over the batch), with fused epilogues: bias + GELU, bias,
// GELU' scaling, plain FP32 partials, and the scheduling epilogue.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "kpp_ratelaws.cuh"
#include "kpp_sched.h"

namespace {

using bf16 = __nv_bfloat16;

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int launch_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(KPP_SCHED_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return KPP_SCHED_OK;
}

int cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) return fail(KPP_SCHED_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return KPP_SCHED_OK;
}

// ---------------------------------------------------------------- activations
__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}

__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// ---------------------------------------------------------------- GEMM
constexpr int kTM = 64, kTN = 64, kTK = 32, kKPad = 8, kGemmThreads = 128;

enum Epilogue : int {
  kEpiF32 = 0,       // C[z][m][n] = acc (split-K partials)
  kEpiBiasGelu = 1,  // pre = acc + bias (to C if given); Cb = bf16(gelu(pre))
  kEpiBias = 2,      // C = acc + bias
  kEpiGeluGrad = 3,  // g = acc * gelu'(pre); C = g (if given), Cb = bf16(g)
  kEpiPlan = 4,      // outputs -> Hstart, cost bin, histogram
};

struct PlanArgs {
  float out_mu0, out_sd0, out_mu1, out_sd1;
  double hmin, hmax;
  double* hstart;
  int* bin;
  int* hist;
  int nbins;
  float lnn_lo, lnn_hi;
};

struct Gemm {
  int M, N, K;
  const bf16* A;
  long a_sm, a_sk;  // A(m, k) = A[m * a_sm + k * a_sk]
  const bf16* B;
  long b_sn, b_sk;  // B(n, k) = B[n * b_sn + k * b_sk]
  int epi;
  const float* bias;
  float* C;
  long ldc;
  bf16* Cb;
  long ldcb;
  const float* pre;
  long ldpre;
  int ksplit;         // > 0: grid.z slices of ksplit rows of K (kEpiF32)
  long split_stride;  // C offset between slices
  PlanArgs plan;
};

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4],
                                         const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ void plan_row(const Gemm& g, int row, float v0, float v1) {
  const PlanArgs& p = g.plan;
  const float o0 = v0 + g.bias[0], o1 = v1 + g.bias[1];
  const float lh = o0 * p.out_sd0 + p.out_mu0;  // log10 Hstart
  const float ln = o1 * p.out_sd1 + p.out_mu1;  // ln Nstp
  if (g.C) {
    g.C[(long)row * g.ldc] = lh;
    g.C[(long)row * g.ldc + 1] = ln;
  }
  double h = exp10((double)lh);
  h = h < p.hmin ? p.hmin : (h > p.hmax ? p.hmax : h);
  p.hstart[row] = h;
  float f = (p.lnn_hi - ln) / (p.lnn_hi - p.lnn_lo) * (float)p.nbins;
  int b = f < 0.0f ? 0 : (f >= (float)p.nbins ? p.nbins - 1 : (int)f);
  p.bin[row] = b;
  atomicAdd(&p.hist[b], 1);
}

// C tile 64 x 64 per CTA, 4 warps of 32 x 32 (2 x 4 mma tiles), K in steps of
// 32 staged through shared memory with the k index fastest (rows padded by 8
// BF16 so the fragment loads of a warp hit 32 distinct banks).
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(const Gemm g) {
  __shared__ __align__(16) bf16 As[kTM][kTK + kKPad];
  __shared__ __align__(16) bf16 Bs[kTN][kTK + kKPad];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int gq = lane >> 2, tq = lane & 3;
  const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
  int k_begin = 0, k_end = g.K;
  if (g.ksplit > 0) {
    k_begin = blockIdx.z * g.ksplit;
    k_end = min(g.K, k_begin + g.ksplit);
  }
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int r = 0; r < 4; r++) acc[i][j][r] = 0.0f;

  const bool a_kfast = g.a_sk == 1, b_kfast = g.b_sk == 1;
  const bf16 zero = __float2bfloat16(0.0f);
  for (int k0 = k_begin; k0 < k_end; k0 += kTK) {
    for (int i = tid; i < kTM * kTK; i += kGemmThreads) {
      const int mm = a_kfast ? i / kTK : i % kTM;
      const int kk = a_kfast ? i % kTK : i / kTM;
      const int m = m0 + mm, k = k0 + kk;
      As[mm][kk] = (m < g.M && k < k_end) ? g.A[(long)m * g.a_sm + (long)k * g.a_sk] : zero;
    }
    for (int i = tid; i < kTN * kTK; i += kGemmThreads) {
      const int nn = b_kfast ? i / kTK : i % kTN;
      const int kk = b_kfast ? i % kTK : i / kTN;
      const int n = n0 + nn, k = k0 + kk;
      Bs[nn][kk] = (n < g.N && k < k_end) ? g.B[(long)n * g.b_sn + (long)k * g.b_sk] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < kTK; ks += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; mt++) {
        const int r = wm * 32 + mt * 16 + gq;
        af[mt][0] = *reinterpret_cast<const uint32_t*>(&As[r][ks + 2 * tq]);
        af[mt][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + 2 * tq]);
        af[mt][2] = *reinterpret_cast<const uint32_t*>(&As[r][ks + 2 * tq + 8]);
        af[mt][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + 2 * tq + 8]);
      }
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        const int c = wn * 32 + nt * 8 + gq;
        bfr[nt][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][ks + 2 * tq]);
        bfr[nt][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][ks + 2 * tq + 8]);
      }
#pragma unroll
      for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++) mma_bf16(acc[mt][nt], af[mt], bfr[nt]);
    }
    __syncthreads();
  }

  if (g.epi == kEpiPlan) {
    // both outputs of a row sit in the thread with tq == 0 of n-tile 0
    if (n0 == 0 && wn == 0 && tq == 0) {
#pragma unroll
      for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int half = 0; half < 2; half++) {
          const int row = m0 + wm * 32 + mt * 16 + gq + half * 8;
          if (row < g.M) plan_row(g, row, acc[mt][0][half * 2], acc[mt][0][half * 2 + 1]);
        }
    }
    return;
  }
#pragma unroll
  for (int mt = 0; mt < 2; mt++)
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int row = m0 + wm * 32 + mt * 16 + gq + (r >> 1) * 8;
        const int col = n0 + wn * 32 + nt * 8 + 2 * tq + (r & 1);
        if (row >= g.M || col >= g.N) continue;
        const float v = acc[mt][nt][r];
        switch (g.epi) {
          case kEpiF32:
            g.C[blockIdx.z * g.split_stride + (long)row * g.ldc + col] = v;
            break;
          case kEpiBiasGelu: {
            const float p = v + g.bias[col];
            if (g.C) g.C[(long)row * g.ldc + col] = p;
            g.Cb[(long)row * g.ldcb + col] = __float2bfloat16(gelu(p));
            break;
          }
          case kEpiBias:
            g.C[(long)row * g.ldc + col] = v + g.bias[col];
            break;
          case kEpiGeluGrad: {
            const float d = v * gelu_grad(g.pre[(long)row * g.ldpre + col]);
            if (g.C) g.C[(long)row * g.ldc + col] = d;
            g.Cb[(long)row * g.ldcb + col] = __float2bfloat16(d);
            break;
          }
        }
      }
}

int run_gemm(const Gemm& g, int splits, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0) return KPP_SCHED_OK;
  dim3 grid((g.N + kTN - 1) / kTN, (g.M + kTM - 1) / kTM, splits > 0 ? splits : 1);
  gemm_kernel<<<grid, kGemmThreads, 0, s>>>(g);
  return launch_check("gemm_kernel");
}

// out[i] = sum over slices of part[z * count + i], slices in order.
__global__ void reduce_splits_kernel(const float* part, int splits, long count, float* out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float s = 0.0f;
  for (int z = 0; z < splits; z++) s += part[(long)z * count + i];
  out[i] = s;
}

// db[n] = sum_b d[b][n], rows in order.
__global__ void colsum_kernel(const float* d, int rows, int cols, long ld, float* out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= cols) return;
  float s = 0.0f;
  for (int b = 0; b < rows; b++) s += d[(long)b * ld + n];
  out[n] = s;
}

// Mean squared error and its gradient d = 2 (o - y) / (rows * cols); one
// block, fixed summation order.
__global__ void __launch_bounds__(1024) mse_kernel(const float* o, const float* y, long count,
                                                   float* d32, bf16* d16, float* loss) {
  __shared__ float red[1024];
  const float scale = 2.0f / (float)count;
  float s = 0.0f;
  for (long i = threadIdx.x; i < count; i += blockDim.x) {
    const float e = o[i] - y[i];
    s += e * e;
    const float d = scale * e;
    d32[i] = d;
    d16[i] = __float2bfloat16(d);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = red[0] / (float)count;
}

__global__ void adam_kernel(float* w, const float* g, float* m, float* v, bf16* w16, long count,
                            float lr, float b1, float b2, float eps, float bc1, float bc2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / bc1, vh = vi / bc2;
  const float wi = w[i] - lr * mh / (sqrtf(vh) + eps);
  w[i] = wi;
  w16[i] = __float2bfloat16(wi);
}

__global__ void to_bf16_kernel(const float* w, bf16* w16, long count) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) w16[i] = __float2bfloat16(w[i]);
}

__global__ void gather_columns_kernel(int nrows, int n, const int* idx, const bf16* src,
                                      long ld_src, bf16* dst, long ld_dst) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const long j = idx[c];
  for (int r = 0; r < nrows; r++) dst[(long)r * ld_dst + c] = src[(long)r * ld_src + j];
}

// One thread per cell; reads the ABI arrays coalesced (cell index fastest)
// and writes the feature column of the cell (feature-major, coalesced).
__global__ void features_kernel(int ncells, int ld, int nvar, const double* var,
                                const double* temp, const double* cfactor, const double* sun,
                                const double* tstart, const double* tend, double dt,
                                const float* mu, const float* isd, bf16* x, long ld_x) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  for (int i = 0; i < nvar; i++) {
    const double v = var[(long)i * ld + c];
    const float f = (float)log10(v > 1e-20 ? v : 1e-20);
    x[(long)i * ld_x + c] = __float2bfloat16((f - mu[i]) * isd[i]);
  }
  const double t0 = tstart[c];
  const double step = tend ? tend[c] - t0 : dt;
  float extra[4];
  extra[0] = (float)temp[c];
  extra[1] = cfactor ? (float)log(cfactor[c]) : 0.0f;
  extra[2] = sun ? (float)sun[c] : (float)kpp_update_sun(t0);
  extra[3] = (float)log(step > 1e-30 ? step : 1e-30);
#pragma unroll
  for (int j = 0; j < 4; j++)
    x[(long)(nvar + j) * ld_x + c] = __float2bfloat16((extra[j] - mu[nvar + j]) * isd[nvar + j]);
}

// Exclusive scan of the bin counts into cursors (one thread; nbins small).
__global__ void scan_bins_kernel(const int* hist, int nbins, int* cursor) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int s = 0;
  for (int b = 0; b < nbins; b++) {
    cursor[b] = s;
    s += hist[b];
  }
}

__global__ void scatter_bins_kernel(int ncells, const int* bin, int* cursor, int* order) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  order[atomicAdd(&cursor[bin[c]], 1)] = c;
}

inline int blocks_for(long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------- the network
struct kpp_sched_mlp {
  int nin = 0, width = 0, nhidden = 0, nout = 0, max_batch = 0;
  int nlayers = 0;
  std::vector<int> fin, fout;
  std::vector<long> w_off, b_off;
  long nparam = 0;
  float *w32 = nullptr, *g32 = nullptr, *m32 = nullptr, *v32 = nullptr;
  bf16* w16 = nullptr;
  float *in_mu = nullptr, *in_isd = nullptr;
  float out_mu[2] = {0.0f, 0.0f}, out_sd[2] = {1.0f, 1.0f};
  long adam_t = 0;
  // training buffers, max_batch rows
  std::vector<float*> pre, dpf;
  std::vector<bf16*> act, dpb;
  float *out = nullptr, *dout32 = nullptr, *split = nullptr;
  bf16* dout16 = nullptr;
  int nsplit = 1;
  // inference buffers, kInferRows rows per chunk
  bf16 *ia = nullptr, *ib = nullptr, *ix = nullptr;
  int *hist = nullptr, *cursor = nullptr, *bins = nullptr;
  long bins_cap = 0;
  std::vector<void*> allocs;

  static constexpr int kInferRows = 1 << 17;
  static constexpr int kMaxBins = 4096;

  template <class T>
  int alloc(T** p, size_t count) {
    void* q = nullptr;
    int rc = cuda_check(cudaMalloc(&q, count * sizeof(T)), "cudaMalloc(scheduler)");
    if (rc) return rc;
    allocs.push_back(q);
    *p = (T*)q;
    return KPP_SCHED_OK;
  }

  ~kpp_sched_mlp() {
    for (void* p : allocs) cudaFree(p);
  }
};

namespace {

// Forward through all layers for `rows` rows of x; hidden activations into
// act (and pre-activations into pre when given), outputs via the last
// layer's epilogue.
int forward_layers(kpp_sched_mlp* m, int rows, const bf16* x, long ld_x, bf16* const* act,
                   float* const* pre, Gemm last, cudaStream_t s) {
  for (int l = 0; l < m->nlayers; l++) {
    Gemm g{};
    g.M = rows;
    g.N = m->fout[l];
    g.K = m->fin[l];
    if (l == 0) {
      g.A = x;
      g.a_sm = 1;
      g.a_sk = ld_x;
    } else {
      g.A = act[l - 1];
      g.a_sm = m->width;
      g.a_sk = 1;
    }
    g.B = m->w16 + m->w_off[l];
    g.b_sn = m->fin[l];
    g.b_sk = 1;
    g.bias = m->w32 + m->b_off[l];
    if (l + 1 < m->nlayers) {
      g.epi = kEpiBiasGelu;
      g.C = pre ? pre[l] : nullptr;
      g.ldc = m->width;
      g.Cb = act[l];
      g.ldcb = m->width;
    } else {
      g.epi = last.epi;
      g.C = last.C;
      g.ldc = last.ldc;
      g.plan = last.plan;
    }
    int rc = run_gemm(g, 1, s);
    if (rc) return rc;
  }
  return KPP_SCHED_OK;
}

}  // namespace

extern "C" {

const char* kpp_sched_last_error(void) { return g_err.c_str(); }

kpp_sched_mlp* kpp_sched_mlp_create(int nin, int width, int nhidden, int nout, int max_batch) {
  if (nin < 1 || width < 1 || nhidden < 1 || nout < 1 || max_batch < 1) {
    fail(KPP_SCHED_EINVAL, "kpp_sched_mlp_create: sizes must be positive");
    return nullptr;
  }
  auto* m = new kpp_sched_mlp;
  m->nin = nin;
  m->width = width;
  m->nhidden = nhidden;
  m->nout = nout;
  m->max_batch = max_batch;
  m->nlayers = nhidden + 1;
  long off = 0;
  for (int l = 0; l < m->nlayers; l++) {
    const int fi = l == 0 ? nin : width, fo = l + 1 < m->nlayers ? width : nout;
    m->fin.push_back(fi);
    m->fout.push_back(fo);
    m->w_off.push_back(off);
    off += (long)fi * fo;
    m->b_off.push_back(off);
    off += fo;
  }
  m->nparam = off;
  // weight gradients are split over the batch in slices of 512 rows
  m->nsplit = (max_batch + 511) / 512;
  const long wmax = (long)width * (nin > width ? nin : width);
  int rc = 0;
  rc |= m->alloc(&m->w32, m->nparam);
  rc |= m->alloc(&m->g32, m->nparam);
  rc |= m->alloc(&m->m32, m->nparam);
  rc |= m->alloc(&m->v32, m->nparam);
  rc |= m->alloc(&m->w16, m->nparam);
  rc |= m->alloc(&m->in_mu, nin);
  rc |= m->alloc(&m->in_isd, nin);
  m->pre.resize(nhidden);
  m->act.resize(nhidden);
  m->dpf.resize(nhidden);
  m->dpb.resize(nhidden);
  for (int l = 0; l < nhidden; l++) {
    rc |= m->alloc(&m->pre[l], (size_t)max_batch * width);
    rc |= m->alloc(&m->act[l], (size_t)max_batch * width);
    rc |= m->alloc(&m->dpf[l], (size_t)max_batch * width);
    rc |= m->alloc(&m->dpb[l], (size_t)max_batch * width);
  }
  rc |= m->alloc(&m->out, (size_t)max_batch * nout);
  rc |= m->alloc(&m->dout32, (size_t)max_batch * nout);
  rc |= m->alloc(&m->dout16, (size_t)max_batch * nout);
  rc |= m->alloc(&m->split, (size_t)m->nsplit * wmax);
  rc |= m->alloc(&m->ia, (size_t)kpp_sched_mlp::kInferRows * width);
  rc |= m->alloc(&m->ib, (size_t)kpp_sched_mlp::kInferRows * width);
  rc |= m->alloc(&m->ix, (size_t)kpp_sched_mlp::kInferRows * nin);
  rc |= m->alloc(&m->hist, kpp_sched_mlp::kMaxBins);
  rc |= m->alloc(&m->cursor, kpp_sched_mlp::kMaxBins);
  if (rc) {
    delete m;
    return nullptr;
  }
  std::vector<float> ones(nin, 1.0f), zeros(nin, 0.0f);
  cudaMemcpy(m->in_mu, zeros.data(), nin * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(m->in_isd, ones.data(), nin * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(m->w32, 0, m->nparam * sizeof(float));
  cudaMemset(m->g32, 0, m->nparam * sizeof(float));
  cudaMemset(m->m32, 0, m->nparam * sizeof(float));
  cudaMemset(m->v32, 0, m->nparam * sizeof(float));
  cudaMemset(m->w16, 0, m->nparam * sizeof(bf16));
  if (cuda_check(cudaDeviceSynchronize(), "kpp_sched_mlp_create")) {
    delete m;
    return nullptr;
  }
  return m;
}

void kpp_sched_mlp_destroy(kpp_sched_mlp* m) { delete m; }

long kpp_sched_mlp_param_count(const kpp_sched_mlp* m) { return m ? m->nparam : 0; }

int kpp_sched_mlp_set_params(kpp_sched_mlp* m, const float* host_params) {
  if (!m || !host_params) return fail(KPP_SCHED_EINVAL, "null argument");
  int rc = cuda_check(cudaMemcpy(m->w32, host_params, m->nparam * sizeof(float),
                                 cudaMemcpyHostToDevice), "set_params");
  if (rc) return rc;
  to_bf16_kernel<<<blocks_for(m->nparam, 256), 256>>>(m->w32, m->w16, m->nparam);
  cudaMemset(m->m32, 0, m->nparam * sizeof(float));
  cudaMemset(m->v32, 0, m->nparam * sizeof(float));
  m->adam_t = 0;
  return cuda_check(cudaDeviceSynchronize(), "set_params");
}

int kpp_sched_mlp_get_params(const kpp_sched_mlp* m, float* host_params) {
  if (!m || !host_params) return fail(KPP_SCHED_EINVAL, "null argument");
  return cuda_check(cudaMemcpy(host_params, m->w32, m->nparam * sizeof(float),
                               cudaMemcpyDeviceToHost), "get_params");
}

int kpp_sched_mlp_get_params_bf16(const kpp_sched_mlp* m, float* host_params) {
  if (!m || !host_params) return fail(KPP_SCHED_EINVAL, "null argument");
  std::vector<bf16> w(m->nparam);
  int rc = cuda_check(cudaMemcpy(w.data(), m->w16, m->nparam * sizeof(bf16),
                                 cudaMemcpyDeviceToHost), "get_params_bf16");
  if (rc) return rc;
  rc = kpp_sched_mlp_get_params(m, host_params);
  if (rc) return rc;
  for (int l = 0; l < m->nlayers; l++)
    for (long i = m->w_off[l]; i < m->b_off[l]; i++) host_params[i] = __bfloat162float(w[i]);
  return KPP_SCHED_OK;
}

int kpp_sched_mlp_get_grads(const kpp_sched_mlp* m, float* host_grads) {
  if (!m || !host_grads) return fail(KPP_SCHED_EINVAL, "null argument");
  return cuda_check(cudaMemcpy(host_grads, m->g32, m->nparam * sizeof(float),
                               cudaMemcpyDeviceToHost), "get_grads");
}

int kpp_sched_mlp_set_scaling(kpp_sched_mlp* m, const float* in_mu, const float* in_sd,
                              const float* out_mu, const float* out_sd) {
  if (!m || !in_mu || !in_sd || !out_mu || !out_sd) return fail(KPP_SCHED_EINVAL, "null argument");
  std::vector<float> isd(m->nin);
  for (int i = 0; i < m->nin; i++) {
    if (!(in_sd[i] > 0.0f)) return fail(KPP_SCHED_EINVAL, "input scale must be positive");
    isd[i] = 1.0f / in_sd[i];
  }
  for (int j = 0; j < m->nout && j < 2; j++) {
    m->out_mu[j] = out_mu[j];
    m->out_sd[j] = out_sd[j];
  }
  int rc = cuda_check(cudaMemcpy(m->in_mu, in_mu, m->nin * sizeof(float), cudaMemcpyHostToDevice),
                      "set_scaling");
  if (rc) return rc;
  return cuda_check(cudaMemcpy(m->in_isd, isd.data(), m->nin * sizeof(float),
                               cudaMemcpyHostToDevice), "set_scaling");
}

int kpp_sched_mlp_forward(kpp_sched_mlp* m, int batch, const void* x, long ld_x, float* out,
                          void* stream) {
  if (!m || !x || !out || batch < 0 || ld_x < batch) return fail(KPP_SCHED_EINVAL, "bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  for (int r0 = 0; r0 < batch; r0 += kpp_sched_mlp::kInferRows) {
    const int rows = batch - r0 < kpp_sched_mlp::kInferRows ? batch - r0 : kpp_sched_mlp::kInferRows;
    Gemm last{};
    last.epi = kEpiBias;
    last.C = out + (long)r0 * m->nout;
    last.ldc = m->nout;
    // hidden activations ping-pong between the two inference buffers
    std::vector<bf16*> act(m->nhidden);
    for (int l = 0; l < m->nhidden; l++) act[l] = (l & 1) ? m->ib : m->ia;
    int rc = forward_layers(m, rows, (const bf16*)x + r0, ld_x, act.data(), nullptr, last, s);
    if (rc) return rc;
  }
  return KPP_SCHED_OK;
}

int kpp_sched_mlp_loss_grad(kpp_sched_mlp* m, int batch, const void* xv, long ld_x,
                            const float* y, float* loss, void* stream) {
  if (!m || !xv || !y || !loss || batch < 1 || batch > m->max_batch || ld_x < batch)
    return fail(KPP_SCHED_EINVAL, "bad argument (batch must be 1..max_batch)");
  cudaStream_t s = (cudaStream_t)stream;
  const bf16* x = (const bf16*)xv;
  const int L = m->nlayers, W = m->width;
  Gemm last{};
  last.epi = kEpiBias;
  last.C = m->out;
  last.ldc = m->nout;
  int rc = forward_layers(m, batch, x, ld_x, m->act.data(), m->pre.data(), last, s);
  if (rc) return rc;
  mse_kernel<<<1, 1024, 0, s>>>(m->out, y, (long)batch * m->nout, m->dout32, m->dout16, loss);
  if ((rc = launch_check("mse_kernel"))) return rc;

  const int splits = (batch + 511) / 512;
  for (int l = L - 1; l >= 0; l--) {
    const bool top = l == L - 1;
    const bf16* dz16 = top ? m->dout16 : m->dpb[l];
    const float* dz32 = top ? m->dout32 : m->dpf[l];
    const long ldz = top ? m->nout : W;
    const int fo = m->fout[l], fi = m->fin[l];
    // dW_l[o][i] = sum_b dZ[b][o] In[b][i], split over b, reduced in order
    Gemm gw{};
    gw.M = fo;
    gw.N = fi;
    gw.K = batch;
    gw.A = dz16;
    gw.a_sm = 1;
    gw.a_sk = ldz;
    if (l == 0) {
      gw.B = x;
      gw.b_sn = ld_x;
      gw.b_sk = 1;
    } else {
      gw.B = m->act[l - 1];
      gw.b_sn = 1;
      gw.b_sk = W;
    }
    gw.epi = kEpiF32;
    gw.C = m->split;
    gw.ldc = fi;
    gw.ksplit = 512;
    gw.split_stride = (long)fo * fi;
    if ((rc = run_gemm(gw, splits, s))) return rc;
    reduce_splits_kernel<<<blocks_for((long)fo * fi, 256), 256, 0, s>>>(
        m->split, splits, (long)fo * fi, m->g32 + m->w_off[l]);
    if ((rc = launch_check("reduce_splits_kernel"))) return rc;
    colsum_kernel<<<blocks_for(fo, 128), 128, 0, s>>>(dz32, batch, fo, ldz, m->g32 + m->b_off[l]);
    if ((rc = launch_check("colsum_kernel"))) return rc;
    if (l == 0) break;
    // dIn[b][i] = sum_o dZ[b][o] W[o][i], times GELU'(pre of layer l-1)
    Gemm gx{};
    gx.M = batch;
    gx.N = fi;
    gx.K = fo;
    gx.A = dz16;
    gx.a_sm = ldz;
    gx.a_sk = 1;
    gx.B = m->w16 + m->w_off[l];
    gx.b_sn = 1;
    gx.b_sk = fi;
    gx.epi = kEpiGeluGrad;
    gx.pre = m->pre[l - 1];
    gx.ldpre = W;
    gx.C = m->dpf[l - 1];
    gx.ldc = W;
    gx.Cb = m->dpb[l - 1];
    gx.ldcb = W;
    if ((rc = run_gemm(gx, 1, s))) return rc;
  }
  return KPP_SCHED_OK;
}

int kpp_sched_mlp_adam(kpp_sched_mlp* m, float lr, float b1, float b2, float eps, void* stream) {
  if (!m) return fail(KPP_SCHED_EINVAL, "null argument");
  m->adam_t++;
  const float bc1 = 1.0f - powf(b1, (float)m->adam_t), bc2 = 1.0f - powf(b2, (float)m->adam_t);
  adam_kernel<<<blocks_for(m->nparam, 256), 256, 0, (cudaStream_t)stream>>>(
      m->w32, m->g32, m->m32, m->v32, m->w16, m->nparam, lr, b1, b2, eps, bc1, bc2);
  return launch_check("adam_kernel");
}

int kpp_sched_gather_columns(int nrows, int n, const int* idx, const void* src, long ld_src,
                             void* dst, long ld_dst, void* stream) {
  if (n <= 0) return KPP_SCHED_OK;
  if (!idx || !src || !dst || ld_dst < n) return fail(KPP_SCHED_EINVAL, "bad argument");
  gather_columns_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
      nrows, n, idx, (const bf16*)src, ld_src, (bf16*)dst, ld_dst);
  return launch_check("gather_columns_kernel");
}

int kpp_sched_features(const kpp_sched_mlp* m, int ncells, int ld, int nvar, const double* var,
                       const double* temp, const double* cfactor, const double* sun,
                       const double* tstart, const double* tend, double dt, void* x, long ld_x,
                       void* stream) {
  if (!m || nvar + 4 != m->nin) return fail(KPP_SCHED_EINVAL, "model inputs must be nvar + 4");
  if (ncells <= 0) return KPP_SCHED_OK;
  if (!var || !temp || !tstart || !x || ld < ncells || ld_x < ncells)
    return fail(KPP_SCHED_EINVAL, "bad argument");
  features_kernel<<<blocks_for(ncells, 128), 128, 0, (cudaStream_t)stream>>>(
      ncells, ld, nvar, var, temp, cfactor, sun, tstart, tend, dt, m->in_mu, m->in_isd,
      (bf16*)x, ld_x);
  return launch_check("features_kernel");
}

int kpp_sched_plan(kpp_sched_mlp* m, int ncells, int ld, int nvar, const double* var,
                   const double* temp, const double* cfactor, const double* sun,
                   const double* tstart, const double* tend, double dt, double hmin,
                   double hmax, int nbins, float lnn_lo, float lnn_hi, double* hstart,
                   int* order, float* pred, void* stream) {
  if (!m || m->nout != 2) return fail(KPP_SCHED_EINVAL, "plan needs a network with 2 outputs");
  if (nbins < 1 || nbins > kpp_sched_mlp::kMaxBins || !(lnn_hi > lnn_lo) || !(hmax >= hmin))
    return fail(KPP_SCHED_EINVAL, "bad binning or Hstart bounds");
  if (ncells <= 0) return KPP_SCHED_OK;
  if (!var || !temp || !tstart || !hstart || !order || ld < ncells)
    return fail(KPP_SCHED_EINVAL, "bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  int rc;
  if (m->bins_cap < ncells) {
    int* nb = nullptr;
    if ((rc = cuda_check(cudaMalloc(&nb, (size_t)ncells * sizeof(int)), "cudaMalloc(bins)")))
      return rc;
    m->allocs.push_back(nb);
    m->bins = nb;
    m->bins_cap = ncells;
  }
  if ((rc = cuda_check(cudaMemsetAsync(m->hist, 0, nbins * sizeof(int), s), "memset(hist)")))
    return rc;
  std::vector<bf16*> act(m->nhidden);
  for (int l = 0; l < m->nhidden; l++) act[l] = (l & 1) ? m->ib : m->ia;
  for (int c0 = 0; c0 < ncells; c0 += kpp_sched_mlp::kInferRows) {
    const int rows = ncells - c0 < kpp_sched_mlp::kInferRows ? ncells - c0 : kpp_sched_mlp::kInferRows;
    rc = kpp_sched_features(m, rows, ld, nvar, var + c0, temp + c0, cfactor ? cfactor + c0 : nullptr,
                            sun ? sun + c0 : nullptr, tstart + c0, tend ? tend + c0 : nullptr, dt,
                            m->ix, rows, s);
    if (rc) return rc;
    Gemm last{};
    last.epi = kEpiPlan;
    last.C = pred ? pred + (long)c0 * 2 : nullptr;
    last.ldc = 2;
    last.plan.out_mu0 = m->out_mu[0];
    last.plan.out_sd0 = m->out_sd[0];
    last.plan.out_mu1 = m->out_mu[1];
    last.plan.out_sd1 = m->out_sd[1];
    last.plan.hmin = hmin;
    last.plan.hmax = hmax;
    last.plan.hstart = hstart + c0;
    last.plan.bin = m->bins + c0;
    last.plan.hist = m->hist;
    last.plan.nbins = nbins;
    last.plan.lnn_lo = lnn_lo;
    last.plan.lnn_hi = lnn_hi;
    if ((rc = forward_layers(m, rows, m->ix, rows, act.data(), nullptr, last, s))) return rc;
  }
  scan_bins_kernel<<<1, 32, 0, s>>>(m->hist, nbins, m->cursor);
  if ((rc = launch_check("scan_bins_kernel"))) return rc;
  scatter_bins_kernel<<<blocks_for(ncells, 256), 256, 0, s>>>(ncells, m->bins, m->cursor, order);
  return launch_check("scatter_bins_kernel");
}

}  // extern "C"
