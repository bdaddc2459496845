// wt_second.cu -- second-order-in-space forms u_tt = L u on the device:
//   * rhs_wave3d! (src/wave.jl:573-611): the SIPG Laplacian of HexSBPSAT's
//     apply_laplacian! (restated from README.md:57-80) on axis-aligned affine
//     meshes, plus the tag-7 Sommerfeld pass (src/wave.jl:453-542).  Two
//     passes: a face-trace kernel (each element's physical normal derivative
//     at its six faces) and the volume + SAT kernel that reads the
//     neighbour's trace (the reference's pass-1/pass-2 structure,
//     src/wave.jl:594-597).
//   * wave_strong_rhs_mesh! (src/wave_strong_rhs.jl:95-341): chain-rule
//     curvilinear Laplacian with Mattsson-Nordstrom SAT and BGT Sommerfeld.
//   * wave_lap_strong_conservative_mesh! (src/wave_lap_strong.jl:183-308).
#include "wt_common.cuh"

namespace wt {

template <int N>
struct Sp {
  static constexpr int N3 = N * N * N;
  static constexpr int N2 = N * N;
  static constexpr int EPB = N3 >= 100 ? 1 : (128 / N3);
  static constexpr int T = N3 * EPB;
};

template <int N, typename real>
__device__ __forceinline__ real ctr(const real* __restrict__ f, const real* __restrict__ GT, int i, int j, int k, int d) {
  real s = 0;
  if (d == 0) {
#pragma unroll
    for (int p = 0; p < N; ++p) s += GT[p * N + i] * f[p + N * (j + N * k)];
  } else if (d == 1) {
#pragma unroll
    for (int p = 0; p < N; ++p) s += GT[p * N + j] * f[i + N * (p + N * k)];
  } else {
#pragma unroll
    for (int p = 0; p < N; ++p) s += GT[p * N + k] * f[i + N * (j + N * p)];
  }
  return s;
}

// pass 1: trace[(6e + f) N^2 + pq] = s_ax * (G_ax u)(face node)
template <int N, typename real>
__global__ void __launch_bounds__(Sp<N>::T) k_sipg_trace(long long Ne, const real* __restrict__ u,
                                                        real* __restrict__ trace, const real* __restrict__ sdiag,
                                                        const double* __restrict__ G) {
  constexpr int N3 = Sp<N>::N3, N2 = Sp<N>::N2, EPB = Sp<N>::EPB;
  __shared__ real GT[N2];
  __shared__ real su[EPB][N3];
  const int tid = threadIdx.x;
  const int le = tid / N3, t = tid - le * N3;
  const long long e = (long long)blockIdx.x * EPB + le;
  const bool valid = e < Ne;
  const long long ec = valid ? e : 0;
  if (tid < N2) GT[(tid % N) * N + tid / N] = (real)G[tid];
  su[le][t] = valid ? u[ec * N3 + t] : (real)0;
  __syncthreads();
  if (!valid) return;
  for (int idx = t; idx < 6 * N2; idx += N3) {
    const int f = idx / N2, pq = idx - f * N2;
    const int ax = f >> 1, r = frow(f, N), p = pq % N, q = pq / N;
    const int fnode = face_node(ax, r, p, q, N);
    const int i = fnode % N, j = (fnode / N) % N, k = fnode / N2;
    trace[(6 * ec + f) * N2 + pq] = sdiag[3 * ec + ax] * ctr<N>(su[le], GT, i, j, k, ax);
  }
}

template <typename real>
struct SipgP {
  long long Ne;
  const real* u;
  const real* ut;
  real* utt;
  const real* trace;
  const real* sdiag;
  const int32_t* nbr;
  const int32_t* nbrf;
  const int32_t* bdry;
  const int32_t* bslot;
  int nbf;
  const real* bnorm;
  const double* G;
  const double* H;
  real bv[6];
  real tau, inv_R;
};

template <int N, typename real>
__global__ void __launch_bounds__(Sp<N>::T) k_sipg_rhs(const SipgP<real> P) {
  constexpr int N3 = Sp<N>::N3, N2 = Sp<N>::N2, EPB = Sp<N>::EPB;
  __shared__ real GT[N2];
  __shared__ real Hs[N];
  __shared__ real su[EPB][N3];
  __shared__ real sD[EPB][3][N3];
  __shared__ real sdu[EPB][6][N2];
  const int tid = threadIdx.x;
  const int le = tid / N3, t = tid - le * N3;
  const int i = t % N, j = (t / N) % N, k = t / N2;
  const long long e = (long long)blockIdx.x * EPB + le;
  const bool valid = e < P.Ne;
  const long long ec = valid ? e : 0;
  const long long n = ec * N3 + t;
  if (tid < N2) GT[(tid % N) * N + tid / N] = (real)P.G[tid];
  if (tid < N) Hs[tid] = (real)P.H[tid];
  const real uv = valid ? P.u[n] : (real)0;
  su[le][t] = uv;
  real sd[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) sd[d] = P.sdiag[3 * ec + d];
  __syncthreads();
  real D[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    D[d] = sd[d] * ctr<N>(su[le], GT, i, j, k, d);
    sD[le][d][t] = D[d];
  }
  // face jumps du (0 on inactive faces)
  for (int idx = t; idx < 6 * N2; idx += N3) {
    const int f = idx / N2, pq = idx - f * N2;
    real du = 0;
    if (valid) {
      const int tag = P.bdry[f + 6 * ec];
      const int en = P.nbr[f + 6 * ec];
      const int ax = f >> 1;
      const int fl = face_node(ax, frow(f, N), pq % N, pq / N, N);
      if (tag == 0 && en >= 0) {
        const int fn = P.nbrf[f + 6 * ec];
        du = su[le][fl] - P.u[(long long)en * N3 + face_node(faxis(fn), frow(fn, N), pq % N, pq / N, N)];
      } else if (tag >= 1 && tag <= 6) {
        du = su[le][fl] - P.bv[tag - 1];
      }
    }
    sdu[le][f][pq] = du;
  }
  __syncthreads();
  if (!valid) return;
  real acc = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) acc += sd[d] * ctr<N>(sD[le][d], GT, i, j, k, d);
  const int idx3[3] = {i, j, k};
  for (int f = 0; f < 6; ++f) {
    const int tag = P.bdry[f + 6 * ec];
    const int en = P.nbr[f + 6 * ec];
    const bool interior = tag == 0 && en >= 0;
    const bool dir = tag >= 1 && tag <= 6;
    if (!interior && !dir) continue;
    const int ax = f >> 1, r = frow(f, N);
    const real nh = (f & 1) ? (real)1 : (real)-1;
    const real s = sd[ax];
    const real al = interior ? (real)0.5 : (real)1;
    const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
    const real du = sdu[le][f][p + N * q];
    const int l = idx3[ax];
    // alpha G^T B du, lifted
    acc += al * nh * s * s * GT[l * N + r] / Hs[l] * du;
    if (l == r) {
      real dGu = 0;
      if (interior) {
        const int fn = P.nbrf[f + 6 * ec];
        dGu = D[ax] - P.trace[((long long)6 * en + fn) * N2 + p + N * q];
      }
      acc += -P.tau * s * s / Hs[r] * du;
      acc += (real)-0.5 * nh * s / Hs[r] * dGu;
    }
  }
  // Sommerfeld pass on tag-7 outer faces
  for (int f = 0; f < 6; ++f) {
    if (P.nbr[f + 6 * ec] >= 0 || P.bdry[f + 6 * ec] != 7) continue;
    const int ax = f >> 1;
    if (idx3[ax] != frow(f, N)) continue;
    const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
    const long long nb = (long long)P.nbf * N2;
    const long long bi = (long long)P.bslot[f + 6 * ec] * N2 + p + N * q;
    const real nx = P.bnorm[bi], ny = P.bnorm[nb + bi], nz = P.bnorm[2 * nb + bi], wFH = P.bnorm[4 * nb + bi];
    const real Gn = nx * D[0] + ny * D[1] + nz * D[2];
    acc -= wFH * (P.ut[n] + Gn + P.inv_R * uv);
  }
  P.utt[n] = acc;
}

// ---------------------------------------------------------------------------
// wave_strong_rhs_element! restated on the device (orientation 0).
template <typename real>
struct StrongP {
  long long Ne;
  const real* u;
  const real* ut;
  real* utt;
  const double* invjac;
  const double* dinvjac;
  const double* detjac;
  const double* Hphys;
  const int32_t* nbr;
  const int32_t* nbrf;
  const int32_t* bdry;
  const double* G;
  const double* H;
  double tau, inv_R;
};

template <int N, typename real>
__global__ void __launch_bounds__(Sp<N>::T) k_strong(const StrongP<real> P) {
  constexpr int N3 = Sp<N>::N3, N2 = Sp<N>::N2, EPB = Sp<N>::EPB;
  __shared__ double GT[N2];
  __shared__ double Hs[N];
  __shared__ double su[EPB][N3];
  __shared__ double sdu[EPB][3][N3];
  __shared__ double suf[EPB][6][N2];
  const int tid = threadIdx.x;
  const int le = tid / N3, t = tid - le * N3;
  const int i = t % N, j = (t / N) % N, k = t / N2;
  const long long e = (long long)blockIdx.x * EPB + le;
  const bool valid = e < P.Ne;
  const long long ec = valid ? e : 0;
  const long long n = ec * N3 + t;
  if (tid < N2) GT[(tid % N) * N + tid / N] = P.G[tid];
  if (tid < N) Hs[tid] = P.H[tid];
  const double uv = valid ? (double)P.u[n] : 0.0;
  su[le][t] = uv;
  for (int idx = t; idx < 6 * N2; idx += N3) {
    const int f = idx / N2, pq = idx - f * N2;
    double v = 0.0;
    if (valid) {
      const int en = P.nbr[f + 6 * ec];
      if (en >= 0) {
        const int fn = P.nbrf[f + 6 * ec];
        v = (double)P.u[(long long)en * N3 + face_node(faxis(fn), frow(fn, N), pq % N, pq / N, N)];
      }
    }
    suf[le][f][pq] = v;
  }
  __syncthreads();
  double du[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    du[c] = ctr<N>(su[le], GT, i, j, k, c);
    sdu[le][c][t] = du[c];
  }
  __syncthreads();
  if (!valid) return;
  double dd[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = c; d < 3; ++d) dd[c][d] = ctr<N>(sdu[le][c], GT, i, j, k, d);
  const double* ij = P.invjac + 9 * n;
  const double* dij = P.dinvjac + 27 * n;
  double I[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) I[c] = ij[c];
  double dphys[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) dphys[a] = I[0 + 3 * a] * du[0] + I[1 + 3 * a] * du[1] + I[2 + 3 * a] * du[2];
  double s = 0.0;
#pragma unroll
  for (int al = 0; al < 3; ++al) {
    double Gaa = I[al] * I[al] + I[al + 3] * I[al + 3] + I[al + 6] * I[al + 6];
    s += Gaa * dd[al][al];
#pragma unroll
    for (int be = al + 1; be < 3; ++be) {
      double Gab = I[al] * I[be] + I[al + 3] * I[be + 3] + I[al + 6] * I[be + 6];
      s += 2.0 * Gab * dd[al][be];
    }
  }
#pragma unroll
  for (int be = 0; be < 3; ++be) {
    double Wb = 0.0;
#pragma unroll
    for (int al = 0; al < 3; ++al)
#pragma unroll
      for (int ii = 0; ii < 3; ++ii) Wb += I[al + 3 * ii] * dij[be + 3 * ii + 9 * al];
    s += Wb * du[be];
  }
  const int idx3[3] = {i, j, k};
  for (int f = 0; f < 6; ++f) {
    const int al = f >> 1, fr = frow(f, N);
    if (idx3[al] != fr) continue;
    const int tag = P.bdry[f + 6 * ec];
    if (tag == 8) continue;
    const bool somm = tag == 7;
    const bool intdir = tag == 0 || (tag >= 1 && tag <= 6);
    const int p = al == 0 ? j : i, q = al == 2 ? j : k;
    const double fs = (f & 1) ? 1.0 : -1.0;
    const double nux = I[al], nuy = I[al + 3], nuz = I[al + 6];
    const double nrm = sqrt(nux * nux + nuy * nuy + nuz * nuz);
    const double dnu = (fs * nux / nrm) * dphys[0] + (fs * nuy / nrm) * dphys[1] + (fs * nuz / nrm) * dphys[2];
    if (intdir) {
      const double w = nrm / Hs[fr];
      s += -w * dnu;
      s += -P.tau * w * (uv - suf[le][f][p + N * q]);
    } else if (somm) {
      const double wF = nrm * P.detjac[n] * Hs[p] * Hs[q];
      s -= wF * ((double)P.ut[n] + dnu + P.inv_R * uv) / P.Hphys[n];
    }
  }
  P.utt[n] = (real)s;
}

// wave_lap_strong_conservative_element! on every element (uniform h).
template <int N, typename real>
__global__ void __launch_bounds__(Sp<N>::T) k_lap_strong_cons(long long Ne, const real* __restrict__ u,
                                                             real* __restrict__ Lu, double inv_h, double tau,
                                                             const int32_t* __restrict__ nbr,
                                                             const int32_t* __restrict__ nbrf,
                                                             const double* __restrict__ G,
                                                             const double* __restrict__ H) {
  constexpr int N3 = Sp<N>::N3, N2 = Sp<N>::N2, EPB = Sp<N>::EPB;
  __shared__ double GT[N2];
  __shared__ double su[EPB][N3];
  __shared__ double sdu[EPB][3][N3];
  const int tid = threadIdx.x;
  const int le = tid / N3, t = tid - le * N3;
  const int i = t % N, j = (t / N) % N, k = t / N2;
  const long long e = (long long)blockIdx.x * EPB + le;
  const bool valid = e < Ne;
  const long long ec = valid ? e : 0;
  const long long n = ec * N3 + t;
  if (tid < N2) GT[(tid % N) * N + tid / N] = G[tid];
  const double uv = valid ? (double)u[n] : 0.0;
  su[le][t] = uv;
  __syncthreads();
  double du[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    du[c] = ctr<N>(su[le], GT, i, j, k, c) * inv_h;
    sdu[le][c][t] = du[c];
  }
  __syncthreads();
  if (!valid) return;
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) s += ctr<N>(sdu[le][c], GT, i, j, k, c);
  s *= inv_h;
  const int idx3[3] = {i, j, k};
  for (int f = 0; f < 6; ++f) {
    const int al = f >> 1, fr = frow(f, N);
    if (idx3[al] != fr) continue;
    const double fs = (f & 1) ? 1.0 : -1.0;
    const double coef_neu = -fs * inv_h / H[fr];
    const double coef_dir = -tau * inv_h / H[fr];
    const int p = al == 0 ? j : i, q = al == 2 ? j : k;
    double uf = 0.0;
    const int en = nbr[f + 6 * ec];
    if (en >= 0) {
      const int fn = nbrf[f + 6 * ec];
      uf = (double)u[(long long)en * N3 + face_node(faxis(fn), frow(fn, N), p, q, N)];
    }
    s += coef_neu * du[al];
    s += coef_dir * (uv - uf);
  }
  Lu[n] = (real)s;
}

// ---------------------------------------------------------------------------
#define WT_DISPATCH_N2(N_, CALL)  \
  switch (N_) {                   \
    case 2: { constexpr int NN = 2; return CALL; } \
    case 3: { constexpr int NN = 3; return CALL; } \
    case 4: { constexpr int NN = 4; return CALL; } \
    case 5: { constexpr int NN = 5; return CALL; } \
    case 6: { constexpr int NN = 6; return CALL; } \
    case 7: { constexpr int NN = 7; return CALL; } \
    case 8: { constexpr int NN = 8; return CALL; } \
    default: return -4;           \
  }

template <int N, typename real>
static int sipg_dispatch(const DevMesh& m, const void* u, const void* ut, void* utt, void* trace,
                         const double bvals[6], double tau, double inv_R, cudaStream_t s) {
  const unsigned blocks = (unsigned)((m.Ne + Sp<N>::EPB - 1) / Sp<N>::EPB);
  k_sipg_trace<N, real><<<blocks, Sp<N>::T, 0, s>>>(m.Ne, (const real*)u, (real*)trace, (const real*)m.sdiag, m.G);
  SipgP<real> P;
  P.Ne = m.Ne; P.u = (const real*)u; P.ut = (const real*)ut; P.utt = (real*)utt; P.trace = (const real*)trace;
  P.sdiag = (const real*)m.sdiag; P.nbr = m.nbr; P.nbrf = m.nbrf; P.bdry = m.bdry; P.bslot = m.bslot;
  P.nbf = m.nbf; P.bnorm = (const real*)m.bnorm; P.G = m.G; P.H = m.H;
  for (int f = 0; f < 6; ++f) P.bv[f] = (real)bvals[f];
  P.tau = (real)tau; P.inv_R = (real)inv_R;
  k_sipg_rhs<N, real><<<blocks, Sp<N>::T, 0, s>>>(P);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_sipg(const DevMesh& m, const void* u, const void* ut, void* utt, void* trace, const double bvals[6],
                double tau, double inv_R, cudaStream_t s) {
  if (m.precision == 0) {
    WT_DISPATCH_N2(m.N, (sipg_dispatch<NN, double>(m, u, ut, utt, trace, bvals, tau, inv_R, s)));
  } else {
    WT_DISPATCH_N2(m.N, (sipg_dispatch<NN, float>(m, u, ut, utt, trace, bvals, tau, inv_R, s)));
  }
}

template <int N, typename real>
static int strong_dispatch(const DevMesh& m, const void* u, const void* ut, void* utt, double tau, double inv_R,
                           cudaStream_t s) {
  StrongP<real> P;
  P.Ne = m.Ne; P.u = (const real*)u; P.ut = (const real*)ut; P.utt = (real*)utt;
  P.invjac = m.invjac; P.dinvjac = m.dinvjac; P.detjac = m.detjac; P.Hphys = m.Hphys;
  P.nbr = m.nbr; P.nbrf = m.nbrf; P.bdry = m.bdry; P.G = m.G; P.H = m.H; P.tau = tau; P.inv_R = inv_R;
  const unsigned blocks = (unsigned)((m.Ne + Sp<N>::EPB - 1) / Sp<N>::EPB);
  k_strong<N, real><<<blocks, Sp<N>::T, 0, s>>>(P);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_strong(const DevMesh& m, const void* u, const void* ut, void* utt, double tau, double inv_R,
                  cudaStream_t s) {
  if (m.precision == 0) {
    WT_DISPATCH_N2(m.N, (strong_dispatch<NN, double>(m, u, ut, utt, tau, inv_R, s)));
  } else {
    WT_DISPATCH_N2(m.N, (strong_dispatch<NN, float>(m, u, ut, utt, tau, inv_R, s)));
  }
}

template <int N, typename real>
static int lsc_dispatch(const DevMesh& m, const void* u, void* Lu, double h, double tau, cudaStream_t s) {
  const unsigned blocks = (unsigned)((m.Ne + Sp<N>::EPB - 1) / Sp<N>::EPB);
  k_lap_strong_cons<N, real><<<blocks, Sp<N>::T, 0, s>>>(m.Ne, (const real*)u, (real*)Lu, 1.0 / h, tau, m.nbr,
                                                         m.nbrf, m.G, m.H);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_lap_strong_cons(const DevMesh& m, const void* u, void* Lu, double h, double tau, cudaStream_t s) {
  if (m.precision == 0) {
    WT_DISPATCH_N2(m.N, (lsc_dispatch<NN, double>(m, u, Lu, h, tau, s)));
  } else {
    WT_DISPATCH_N2(m.N, (lsc_dispatch<NN, float>(m, u, Lu, h, tau, s)));
  }
}

}  // namespace wt
