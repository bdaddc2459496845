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

#include <algorithm>

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
      const int en = ::wt::bc_elem(P.nbr[f + 6 * ec], P.Ne);
      const int ax = f >> 1;
      const int fl = face_node(ax, frow(f, N), pq % N, pq / N, N);
      if (tag == 0 && en >= 0) {
        const int fs = P.nbrf[f + 6 * ec];  // fn | ori << 3
        du = su[le][fl] - P.u[(long long)en * N3 + nbr_face_node(fs, pq % N, pq / N, N)];
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
    const int en = ::wt::bc_elem(P.nbr[f + 6 * ec], P.Ne);
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
        const int fs = P.nbrf[f + 6 * ec];  // fn | ori << 3
        int pn, qn;
        face_perm((fs >> 3) & 7, p, q, N, pn, qn);
        dGu = D[ax] - P.trace[((long long)6 * en + (fs & 7)) * N2 + pn + N * qn];
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
    const long long bi = (long long)::wt::bc_slot(P.bslot[f + 6 * ec], P.nbf) * N2 + p + N * q;
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
      const int en = ::wt::bc_elem(P.nbr[f + 6 * ec], P.Ne);
      if (en >= 0) {
        const int fs = P.nbrf[f + 6 * ec];  // fn | ori << 3
        v = (double)P.u[(long long)en * N3 + nbr_face_node(fs, pq % N, pq / N, N)];
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
    const int en = ::wt::bc_elem(nbr[f + 6 * ec], Ne);
    if (en >= 0) {
      const int fs = nbrf[f + 6 * ec];  // fn | ori << 3
      uf = (double)u[(long long)en * N3 + nbr_face_node(fs, p, q, N)];
    }
    s += coef_neu * du[al];
    s += coef_dir * (uv - uf);
  }
  Lu[n] = (real)s;
}

// Scalar wave on a prescribed 4-metric (wave_curved_rhs_element! /
// wave_curved_rhs_conservative_element!, src/wave_curved_rhs.jl:45-136 and
// 217-348) on every element of a uniform Cartesian mesh: the gradients of phi
// and phidot (centred-flux SAT on the perpendicular component of each face
// unless CONS), the six Hessian components as a second G sweep of the gradient
// of phi, the pointwise solve
//   phidd = (Gam.(phidot, dphi) - 2 g^{ti} d_i phidot - g^{ij} d_ij phi) / g^{tt}
// and, when CONS, the Mattsson-Nordstrom SAT pair on the faces.  ginv holds
// (tt,tx,ty,tz,xx,xy,xz,yy,yz,zz) and gam (t,x,y,z) per node, component
// fastest; faces without a neighbour see zero traces.  FP64 arithmetic.
template <int N, typename real, bool CONS>
__global__ void __launch_bounds__(Sp<N>::T) k_curved4(long long Ne, const real* __restrict__ u,
                                                     const real* __restrict__ ud, real* __restrict__ udd,
                                                     const real* __restrict__ ginv, const real* __restrict__ gam,
                                                     double inv_h, double tau, const int32_t* __restrict__ nbr,
                                                     const int32_t* __restrict__ nbrf, const double* __restrict__ G,
                                                     const double* __restrict__ H) {
  constexpr int N3 = Sp<N>::N3, N2 = Sp<N>::N2, EPB = Sp<N>::EPB;
  __shared__ double GT[N2];
  __shared__ double su[EPB][N3];
  __shared__ double sv[EPB][N3];
  __shared__ double sdu[EPB][3][N3];
  const int tid = threadIdx.x;
  const int le = tid / N3, t = tid - le * N3;
  const int i = t % N, j = (t / N) % N, k = t / N2;
  const long long e = (long long)blockIdx.x * EPB + le;
  const bool valid = e < Ne;
  const long long ec = valid ? e : 0;
  const long long n = ec * N3 + t;
  if (tid < N2) GT[(tid % N) * N + tid / N] = G[tid];
  const double uv = valid ? (double)u[n] : 0.0, vv = valid ? (double)ud[n] : 0.0;
  su[le][t] = uv;
  sv[le][t] = vv;
  // neighbour traces of phi and phidot at this node's faces (zero without one)
  const int idx3[3] = {i, j, k};
  double uf[6], vf[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    uf[f] = 0.0;
    vf[f] = 0.0;
    const int al = f >> 1;
    if (!valid || idx3[al] != frow(f, N)) continue;
    const int en = ::wt::bc_elem(nbr[f + 6 * ec], Ne);
    if (en < 0) continue;
    const int fs = nbrf[f + 6 * ec];  // fn | ori << 3
    const int p = al == 0 ? j : i, q = al == 2 ? j : k;
    const long long src = (long long)en * N3 + nbr_face_node(fs, p, q, N);
    uf[f] = (double)u[src];
    vf[f] = (double)ud[src];
  }
  __syncthreads();
  double du[3], dv[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    du[c] = ctr<N>(su[le], GT, i, j, k, c) * inv_h;
    dv[c] = ctr<N>(sv[le], GT, i, j, k, c) * inv_h;
  }
  if (!CONS) {
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int al = f >> 1, fr = frow(f, N);
      if (idx3[al] != fr) continue;
      const double coef = ((f & 1) ? 1.0 : -1.0) * 0.5 * (1.0 / H[fr]) * inv_h;
      du[al] += coef * (uf[f] - uv);
      dv[al] += coef * (vf[f] - vv);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) sdu[le][c][t] = du[c];
  __syncthreads();
  if (!valid) return;
  // Hessian: xx, xy, xz of d_x phi; yy, yz of d_y phi; zz of d_z phi
  const double dxx = ctr<N>(sdu[le][0], GT, i, j, k, 0) * inv_h;
  const double dxy = ctr<N>(sdu[le][0], GT, i, j, k, 1) * inv_h;
  const double dxz = ctr<N>(sdu[le][0], GT, i, j, k, 2) * inv_h;
  const double dyy = ctr<N>(sdu[le][1], GT, i, j, k, 1) * inv_h;
  const double dyz = ctr<N>(sdu[le][1], GT, i, j, k, 2) * inv_h;
  const double dzz = ctr<N>(sdu[le][2], GT, i, j, k, 2) * inv_h;
  double g[10], gm[4];
#pragma unroll
  for (int c = 0; c < 10; ++c) g[c] = (double)ginv[10 * n + c];
#pragma unroll
  for (int c = 0; c < 4; ++c) gm[c] = (double)gam[4 * n + c];
  const double gdd = gm[0] * vv + gm[1] * du[0] + gm[2] * du[1] + gm[3] * du[2];
  const double gti = g[1] * dv[0] + g[2] * dv[1] + g[3] * dv[2];
  const double gij = g[4] * dxx + g[7] * dyy + g[9] * dzz + 2 * g[5] * dxy + 2 * g[6] * dxz + 2 * g[8] * dyz;
  double s = (gdd - 2 * gti - gij) / g[0];
  if (CONS) {
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int al = f >> 1, fr = frow(f, N);
      if (idx3[al] != fr) continue;
      const double coef_neu = -((f & 1) ? 1.0 : -1.0) * inv_h * (1.0 / H[fr]);
      const double coef_dir = -(tau * inv_h) * (1.0 / H[fr]);
      s += coef_neu * du[al];
      s += coef_dir * (uv - uf[f]);
    }
  }
  udd[n] = (real)s;
}

// Prescribed 4-metrics at the nodes (eval_curved_background!,
// src/wave_curved_rhs.jl:373-418): kind 0 Minkowski, kind 1 the gauge wave
// ds^2 = (1 - H)(-dt^2 + dx^2) + dy^2 + dz^2, H = A sin(2 pi (x - t)/d)
// (Alcubierre et al. 2004), p = (A, d).  Its inverse is diag(-1/(1-H),
// 1/(1-H), 1, 1) and its contracted Christoffels vanish (harmonic gauge).
template <typename real>
__global__ void k_curved4_bg(long long nn, const double* __restrict__ coords, int kind, double A, double d, double t,
                             real* __restrict__ ginv, real* __restrict__ gam) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    double f = 1.0;
    if (kind == 1) f = 1.0 - A * sin(2.0 * M_PI * (coords[3 * n] - t) / d);
    real* g = ginv + 10 * n;
#pragma unroll
    for (int c = 0; c < 10; ++c) g[c] = (real)0;
    g[0] = (real)(-1.0 / f);
    g[4] = (real)(1.0 / f);
    g[7] = (real)1;
    g[9] = (real)1;
#pragma unroll
    for (int c = 0; c < 4; ++c) gam[4 * n + c] = (real)0;
  }
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

template <int N, typename real>
static int c4_dispatch(const DevMesh& m, const void* u, const void* ud, void* udd, const void* ginv, const void* gam,
                       double h, int cons, double tau, cudaStream_t s) {
  const unsigned blocks = (unsigned)((m.Ne + Sp<N>::EPB - 1) / Sp<N>::EPB);
  if (cons)
    k_curved4<N, real, true><<<blocks, Sp<N>::T, 0, s>>>(m.Ne, (const real*)u, (const real*)ud, (real*)udd,
                                                          (const real*)ginv, (const real*)gam, 1.0 / h, tau, m.nbr,
                                                          m.nbrf, m.G, m.H);
  else
    k_curved4<N, real, false><<<blocks, Sp<N>::T, 0, s>>>(m.Ne, (const real*)u, (const real*)ud, (real*)udd,
                                                           (const real*)ginv, (const real*)gam, 1.0 / h, tau, m.nbr,
                                                           m.nbrf, m.G, m.H);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_curved4(const DevMesh& m, const void* u, const void* ud, void* udd, const void* ginv, const void* gam,
                   double h, int conservative, double tau, cudaStream_t s) {
  if (m.precision == 0) {
    WT_DISPATCH_N2(m.N, (c4_dispatch<NN, double>(m, u, ud, udd, ginv, gam, h, conservative, tau, s)));
  } else {
    WT_DISPATCH_N2(m.N, (c4_dispatch<NN, float>(m, u, ud, udd, ginv, gam, h, conservative, tau, s)));
  }
}

int launch_curved4_background(const DevMesh& m, int kind, const double* p, double t, void* ginv, void* gam,
                              cudaStream_t s) {
  const unsigned blocks = (unsigned)std::min<long long>((m.nn + 255) / 256, 8192);
  if (m.precision == 0)
    k_curved4_bg<double><<<blocks, 256, 0, s>>>(m.nn, m.coords, kind, p[0], p[1], t, (double*)ginv, (double*)gam);
  else
    k_curved4_bg<float><<<blocks, 256, 0, s>>>(m.nn, m.coords, kind, p[0], p[1], t, (float*)ginv, (float*)gam);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// this file's bounds word (bounds-check build; 0 otherwise)
WT_BOUNDS_TAKE(bounds_take_second)

}  // namespace wt
