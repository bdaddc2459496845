// wt_reduce.cu -- FP64 reductions (energy, weighted norms, power-iteration
// norm) and streaming vector updates (RK4 stage update, axpy, fills).
// Reductions write one partial sum per block; the host adds the partials in
// a fixed order, so results are deterministic run to run.
#include "wt_common.cuh"

#include <algorithm>

namespace wt {

static constexpr int RB = 256;

int reduce_blocks() { return 1184; }  // 8 x 148 SMs

__device__ inline double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;
}

// wave3d_energy: sum 1/2 [Pi^2/sqrtg + sqrtg gu^{ij} D_i D_j] H; lapse = 1: the
// integrand times alpha (the norm the system conserves for a static background
// without shift)
template <typename real>
__global__ void k_energy(long long nn, const double* __restrict__ c11, const real* __restrict__ Pi,
                         const real* __restrict__ g, const double* __restrict__ H, double* __restrict__ partial,
                         int lapse) {
  __shared__ double red[32];
  double acc = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const double sg = c11[nn + n];
    const double d1 = g[n], d2 = g[nn + n], d3 = g[2 * nn + n];
    const double p = Pi[n];
    const double w = lapse ? c11[n] : 1.0;
    acc += w *
           (p * p / sg + sg * (c11[5 * nn + n] * d1 * d1 + c11[8 * nn + n] * d2 * d2 + c11[10 * nn + n] * d3 * d3 +
                               2 * c11[6 * nn + n] * d1 * d2 + 2 * c11[7 * nn + n] * d1 * d3 +
                               2 * c11[9 * nn + n] * d2 * d3)) *
           H[n] / 2;
  }
  double s = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// mode 0: sum a b H; mode 1: sum (a - b)^2 H (b may be null); mode 2: sum a^2 (no weight)
template <typename real>
__global__ void k_wdot(long long nn, int mode, const real* __restrict__ a, const real* __restrict__ b,
                       const double* __restrict__ H, double* __restrict__ partial) {
  __shared__ double red[32];
  double acc = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const double av = a[n];
    if (mode == 0) acc += av * (double)b[n] * H[n];
    else if (mode == 1) { const double d = av - (b ? (double)b[n] : 0.0); acc += d * d * H[n]; }
    else acc += av * av;
  }
  double s = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

template <typename real>
__global__ void k_scale(long long n, real* __restrict__ a, real s) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = a[i] / s;
}
template <typename real>
__global__ void k_fill(long long n, real* __restrict__ a, real v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = v;
}
template <typename real>
__global__ void k_copy(long long n, real* __restrict__ d, const real* __restrict__ s) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    d[i] = s[i];
}
template <typename real>
__global__ void k_axpy(long long n, real* __restrict__ y, real a, const real* __restrict__ x) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = y[i] + a * x[i];
}
// low-storage classic RK4 stage update (same arithmetic as the fused epilogue)
// Explicit RK stage/step combination: out = y + dt * sum_j a_j k_j (j < nk),
// summed in j order.
struct ErkSum {
  const void* k[WT_ERK_MAX_STAGES];
  double a[WT_ERK_MAX_STAGES];
  int nk;
};
template <typename real>
__global__ void k_erk_combine(long long n, double dt, const real* __restrict__ y, real* __restrict__ out, ErkSum S) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    real acc = 0;
    for (int j = 0; j < S.nk; ++j) acc += (real)S.a[j] * ((const real*)S.k[j])[i];
    out[i] = y[i] + (real)dt * acc;
  }
}

int launch_erk_combine(long long n, int precision, double dt, const void* y, void* out, int nk, const void* const* k,
                       const double* a, cudaStream_t s) {
  if (nk < 0 || nk > WT_ERK_MAX_STAGES) return -1;
  ErkSum S;
  S.nk = nk;
  for (int j = 0; j < WT_ERK_MAX_STAGES; ++j) {
    S.k[j] = j < nk ? k[j] : nullptr;
    S.a[j] = j < nk ? a[j] : 0.0;
  }
  const unsigned grid = (unsigned)std::min<long long>((n + 255) / 256, 4096);
  if (precision == 0)
    k_erk_combine<double><<<grid, 256, 0, s>>>(n, dt, (const double*)y, (double*)out, S);
  else
    k_erk_combine<float><<<grid, 256, 0, s>>>(n, dt, (const float*)y, (float*)out, S);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename real>
__global__ void k_rk_update(long long n, int stage, double dt, real* __restrict__ y, real* __restrict__ acc,
                            real* __restrict__ out, const real* __restrict__ k, real* __restrict__ comp) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const real kv = k[i];
    if (comp) {  // increment form with a Kahan-compensated final sum (see rk_epilogue)
      if (stage == 0) {
        out[i] = y[i] + (real)(0.5 * dt) * kv;
        acc[i] = (real)(dt / 6.0) * kv;
      } else if (stage == 1) {
        out[i] = y[i] + (real)(0.5 * dt) * kv;
        acc[i] = acc[i] + (real)(dt / 3.0) * kv;
      } else if (stage == 2) {
        out[i] = y[i] + (real)dt * kv;
        acc[i] = acc[i] + (real)(dt / 3.0) * kv;
      } else {
        const real inc = acc[i] + (real)(dt / 6.0) * kv;
        const real yv = y[i];
        const real t = inc + comp[i];
        const real v = yv + t;
        comp[i] = t - (v - yv);
        y[i] = v;
      }
      continue;
    }
    if (stage == 0) {
      const real yv = y[i];
      out[i] = yv + (real)(0.5 * dt) * kv;
      acc[i] = yv + (real)(dt / 6.0) * kv;
    } else if (stage == 1) {
      out[i] = y[i] + (real)(0.5 * dt) * kv;
      acc[i] = acc[i] + (real)(dt / 3.0) * kv;
    } else if (stage == 2) {
      out[i] = y[i] + (real)dt * kv;
      acc[i] = acc[i] + (real)(dt / 3.0) * kv;
    } else {
      y[i] = acc[i] + (real)(dt / 6.0) * kv;
    }
  }
}
// the reference's power-iteration start: isodd(i+j+k+m) ? 1 : -1 (1-based)
template <typename real>
__global__ void k_alt_sign(int N, long long nn, real* __restrict__ v) {
  const long long N3 = (long long)N * N * N;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const long long e = n / N3;
    const int t = (int)(n - e * N3);
    const int i = t % N, j = (t / N) % N, k = t / (N * N);
    v[n] = ((i + j + k + e + 4) & 1) ? (real)1 : (real)-1;
  }
}
template <typename real>
__global__ void k_finite(long long n, const real* __restrict__ a, unsigned int* flag) {
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    bad |= !isfinite((double)a[i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1u);
}

static inline unsigned gblocks(long long n) {
  long long b = (n + RB - 1) / RB;
  return (unsigned)(b < 4736 ? (b > 0 ? b : 1) : 4736);
}

int launch_energy(const DevMesh& m, const DevCoef& c, const void* Pi, const void* grad, int use_metric,
                  double* partial, int nblocks, cudaStream_t s, int lapse) {
  const double* H = use_metric ? m.Hd : m.Hphys;
  if (m.precision == 0)
    k_energy<double><<<nblocks, RB, 0, s>>>(m.nn, c.c11, (const double*)Pi, (const double*)grad, H, partial, lapse);
  else
    k_energy<float><<<nblocks, RB, 0, s>>>(m.nn, c.c11, (const float*)Pi, (const float*)grad, H, partial, lapse);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_dot_weighted(const DevMesh& m, const void* a, const void* b, const void*, const void*, int weight_kind,
                        int mode, double* partial, int nblocks, cudaStream_t s) {
  const double* H = weight_kind ? m.Hd : m.Hphys;
  if (m.precision == 0)
    k_wdot<double><<<nblocks, RB, 0, s>>>(m.nn, mode, (const double*)a, (const double*)b, H, partial);
  else
    k_wdot<float><<<nblocks, RB, 0, s>>>(m.nn, mode, (const float*)a, (const float*)b, H, partial);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_sumsq(long long n, int precision, const void* a, double* partial, int nblocks, cudaStream_t s) {
  if (precision == 0)
    k_wdot<double><<<nblocks, RB, 0, s>>>(n, 2, (const double*)a, nullptr, nullptr, partial);
  else
    k_wdot<float><<<nblocks, RB, 0, s>>>(n, 2, (const float*)a, nullptr, nullptr, partial);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_scale(long long n, int precision, void* a, double sc, cudaStream_t st) {
  if (precision == 0) k_scale<double><<<gblocks(n), RB, 0, st>>>(n, (double*)a, sc);
  else k_scale<float><<<gblocks(n), RB, 0, st>>>(n, (float*)a, (float)sc);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
int launch_fill(long long n, int precision, void* a, double v, cudaStream_t st) {
  if (precision == 0) k_fill<double><<<gblocks(n), RB, 0, st>>>(n, (double*)a, v);
  else k_fill<float><<<gblocks(n), RB, 0, st>>>(n, (float*)a, (float)v);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
int launch_copy(long long n, int precision, void* d, const void* s, cudaStream_t st) {
  if (precision == 0) k_copy<double><<<gblocks(n), RB, 0, st>>>(n, (double*)d, (const double*)s);
  else k_copy<float><<<gblocks(n), RB, 0, st>>>(n, (float*)d, (const float*)s);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
// FP64 values -> FP32 high part + FP32 low part (hi + lo carries ~48 bits)
__global__ void k_split_f64(long long n, const double* __restrict__ a, float* __restrict__ hi, float* __restrict__ lo) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = a[i];
    const float h = (float)v;
    hi[i] = h;
    lo[i] = (float)(v - (double)h);
  }
}

int launch_split_f64(long long n, const double* a, float* hi, float* lo, cudaStream_t st) {
  k_split_f64<<<gblocks(n), RB, 0, st>>>(n, a, hi, lo);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_rk_update(long long n, int precision, int stage, double dt, void* y, void* acc, void* out, const void* k,
                     cudaStream_t st, void* comp) {
  if (precision == 0)
    k_rk_update<double><<<gblocks(n), RB, 0, st>>>(n, stage, dt, (double*)y, (double*)acc, (double*)out,
                                                  (const double*)k, (double*)comp);
  else
    k_rk_update<float><<<gblocks(n), RB, 0, st>>>(n, stage, dt, (float*)y, (float*)acc, (float*)out,
                                                 (const float*)k, (float*)comp);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
int launch_axpy(long long n, int precision, void* y, double a, const void* x, cudaStream_t st) {
  if (precision == 0) k_axpy<double><<<gblocks(n), RB, 0, st>>>(n, (double*)y, a, (const double*)x);
  else k_axpy<float><<<gblocks(n), RB, 0, st>>>(n, (float*)y, (float)a, (const float*)x);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
int launch_alt_sign(const DevMesh& m, void* v, cudaStream_t st) {
  if (m.precision == 0) k_alt_sign<double><<<gblocks(m.nn), RB, 0, st>>>(m.N, m.nn, (double*)v);
  else k_alt_sign<float><<<gblocks(m.nn), RB, 0, st>>>(m.N, m.nn, (float*)v);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
int launch_finite_check(long long n, int precision, const void* a, unsigned int* flag, cudaStream_t st) {
  if (precision == 0) k_finite<double><<<gblocks(n), RB, 0, st>>>(n, (const double*)a, flag);
  else k_finite<float><<<gblocks(n), RB, 0, st>>>(n, (const float*)a, flag);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// out[q] = field[nodes[q]] in FP64 (device-side diagnostics: slices, probes)
template <typename real>
__global__ void k_gather(int count, const real* __restrict__ field, const int64_t* __restrict__ nodes,
                         double* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x)
    out[q] = (double)field[nodes[q]];
}

int launch_gather(int precision, int count, const void* field, const int64_t* nodes, double* out, cudaStream_t s) {
  const unsigned blocks = (unsigned)((count + 255) / 256 < 4096 ? (count + 255) / 256 : 4096);
  if (blocks == 0) return 0;
  if (precision == 0) k_gather<double><<<blocks, 256, 0, s>>>(count, (const double*)field, nodes, out);
  else k_gather<float><<<blocks, 256, 0, s>>>(count, (const float*)field, nodes, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace wt
