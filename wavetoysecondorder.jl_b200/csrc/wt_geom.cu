// wt_geom.cu -- one-time set-up on the device, all in FP64: GLL operators,
// analytic hex geometry, curl-form metric terms, metric derivatives, boundary
// normals, ADM background sampling and the combined streamed coefficients.
//
// Reference counterparts (arithmetic in the unvendored HexSBPSAT/HexMeshes is
// restated from its documentation): make_element/make_operators,
// make_uniform_hex / make_warped_uniform_hex + make_geometry
// (src/evolve.jl:1174-1191), make_metric_terms3d (METHODS.md:156-166),
// make_metric_derivs (src/wave_strong_rhs.jl:376-391), _sample_bg3d_kernel!
// (src/wave3d_curved.jl:75-96), _min_node_spacing_3d (src/evolve.jl:60-69).
#include "wt_common.cuh"

#include <cmath>
#include <cfloat>

namespace wt {

// ---------------------------------------------------------------------------
// GLL nodes/weights/differentiation on [0,1].  Interior nodes are the roots of
// P'_p (p = N-1), found by Newton's method on P'_p using the Legendre
// recurrence for P_p, P'_p, P''_p; weights 2/(p(p+1) P_p^2); the
// differentiation matrix is the closed form D_ij = P_p(x_i)/(P_p(x_j)(x_i-x_j))
// with D_ii = -sum_{j!=i} D_ij (Canuto et al., "Spectral Methods", 2.3.2).
static void legendre3(int p, long double x, long double& P, long double& dP, long double& d2P) {
  long double p0 = 1.0L, p1 = x;
  if (p == 0) { P = 1; dP = 0; d2P = 0; return; }
  for (int k = 2; k <= p; ++k) {
    long double pk = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
    p0 = p1; p1 = pk;
  }
  P = p1;
  // (1-x^2) P' = p (P_{p-1} - x P_p)
  dP = p * (p0 - x * p1) / (1.0L - x * x);
  // Legendre ODE: (1-x^2) P'' - 2x P' + p(p+1) P = 0
  d2P = (2.0L * x * dP - p * (p + 1.0L) * P) / (1.0L - x * x);
}

// Evaluated in extended precision (long double) and rounded once to double,
// so the operators are correctly rounded independently of the algorithm.
HostOps gll_operators(int N) {
  HostOps o; o.N = N;
  const int p = N - 1;
  std::vector<long double> xs(N), ws(N), Pv(N);
  xs[0] = -1.0L; xs[p] = 1.0L;
  for (int j = 1; j < p; ++j) {
    if (2 * j > p) break;
    long double x = -cosl(3.14159265358979323846264338327950288L * j / p);  // Chebyshev-Gauss-Lobatto start
    if (2 * j == p) x = 0.0L;
    for (int it = 0; it < 80 && 2 * j != p; ++it) {
      long double P, dP, d2P;
      legendre3(p, x, P, dP, d2P);
      long double dx = dP / d2P;
      x -= dx;
      if (fabsl(dx) < 1e-20L) break;
    }
    xs[j] = x; xs[p - j] = -x;
  }
  for (int j = 0; j < N; ++j) {
    long double P;
    if (j == 0) P = (p % 2 == 0) ? 1.0L : -1.0L;
    else if (j == p) P = 1.0L;
    else { long double dP, d2P; legendre3(p, xs[j], P, dP, d2P); }
    Pv[j] = P;
    ws[j] = 2.0L / (p * (p + 1.0L) * P * P);
  }
  o.x.resize(N); o.H.resize(N); o.G.assign(N * N, 0.0);
  for (int i = 0; i < N; ++i) {
    long double sacc = 0.0L;
    std::vector<long double> row(N, 0.0L);
    for (int j = 0; j < N; ++j) {
      if (i == j) continue;
      row[j] = Pv[i] / (Pv[j] * (xs[i] - xs[j]));
      sacc += row[j];
    }
    (void)sacc;
    // exact GLL diagonal: 0 inside, -p(p+1)/4 and +p(p+1)/4 at the ends
    row[i] = i == 0 ? -p * (p + 1.0L) / 4.0L : (i == p ? p * (p + 1.0L) / 4.0L : 0.0L);
    for (int j = 0; j < N; ++j) o.G[i * N + j] = (double)(2.0L * row[j]);
    o.x[i] = (double)(0.5L * (1.0L + xs[i]));
    o.H[i] = (double)(0.5L * ws[i]);
  }
  o.x[0] = 0.0; o.x[p] = 1.0;
  return o;
}

// ---------------------------------------------------------------------------
// coords + analytic Jacobian of x = x0 + L (s + A P(s)), s the uniform
// reference position, element numbering e = ex + Mx (ey + My ez).
// Mz is the element count of the whole mesh along z; element layer ez of this
// mesh is layer ez + z0 of the whole mesh (taken modulo Mz: a z-slab of a
// periodic mesh may wrap around).
__global__ void k_geom_analytic(int N, int Mx, int My, int Mz, int z0, double x0, double L, double A,
                                const double* __restrict__ xg, long long nn, double* __restrict__ coords,
                                double* __restrict__ jac) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= nn) return;
  int N3 = N * N * N;
  long long e = n / N3;
  int t = (int)(n - e * N3);
  int i = t % N, j = (t / N) % N, k = t / (N * N);
  int ex = (int)(e % Mx), ey = (int)((e / Mx) % My), ez = (int)(e / ((long long)Mx * My)) + z0;
  if (ez < 0) ez += Mz;
  if (ez >= Mz) ez -= Mz;
  double s[3] = {(ex + xg[i]) / Mx, (ey + xg[j]) / My, (ez + xg[k]) / Mz};
  const double tp = 2.0 * M_PI;
  double sn[3], cs[3];
  for (int a = 0; a < 3; ++a) sincos(tp * s[a], &sn[a], &cs[a]);
  double P = sn[0] * sn[1] * sn[2];
  double dP[3] = {tp * cs[0] * sn[1] * sn[2], tp * sn[0] * cs[1] * sn[2], tp * sn[0] * sn[1] * cs[2]};
  double Ms[3] = {(double)Mx, (double)My, (double)Mz};
  for (int a = 0; a < 3; ++a) {
    coords[a + 3 * n] = x0 + L * (s[a] + A * P);
    for (int b = 0; b < 3; ++b) jac[a + 3 * b + 9 * n] = L * ((a == b ? 1.0 : 0.0) + A * dP[b]) / Ms[b];
  }
}

// invjac (cofactor / det), detjac, Hphys = H_i H_j H_k |det|.
__global__ void k_geom_derived(int N, long long nn, const double* __restrict__ Hq, const double* __restrict__ jac,
                               double* __restrict__ invjac, double* __restrict__ detjac, double* __restrict__ Hphys) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= nn) return;
  int N3 = N * N * N;
  int t = (int)(n % N3);
  int i = t % N, j = (t / N) % N, k = t / (N * N);
  const double* J = jac + 9 * n;
#define JJ(a, b) J[(a) + 3 * (b)]
  double c00 = JJ(1, 1) * JJ(2, 2) - JJ(1, 2) * JJ(2, 1);
  double c01 = JJ(1, 2) * JJ(2, 0) - JJ(1, 0) * JJ(2, 2);
  double c02 = JJ(1, 0) * JJ(2, 1) - JJ(1, 1) * JJ(2, 0);
  double det = JJ(0, 0) * c00 + JJ(0, 1) * c01 + JJ(0, 2) * c02;
  double* I = invjac + 9 * n;
  I[0 + 3 * 0] = c00 / det;
  I[1 + 3 * 0] = c01 / det;
  I[2 + 3 * 0] = c02 / det;
  I[0 + 3 * 1] = (JJ(0, 2) * JJ(2, 1) - JJ(0, 1) * JJ(2, 2)) / det;
  I[1 + 3 * 1] = (JJ(0, 0) * JJ(2, 2) - JJ(0, 2) * JJ(2, 0)) / det;
  I[2 + 3 * 1] = (JJ(0, 1) * JJ(2, 0) - JJ(0, 0) * JJ(2, 1)) / det;
  I[0 + 3 * 2] = (JJ(0, 1) * JJ(1, 2) - JJ(0, 2) * JJ(1, 1)) / det;
  I[1 + 3 * 2] = (JJ(0, 2) * JJ(1, 0) - JJ(0, 0) * JJ(1, 2)) / det;
  I[2 + 3 * 2] = (JJ(0, 0) * JJ(1, 1) - JJ(0, 1) * JJ(1, 0)) / det;
#undef JJ
  detjac[n] = det;
  Hphys[n] = Hq[i] * Hq[j] * Hq[k] * fabs(det);
}

__global__ void k_handed(int N, long long Ne, const double* __restrict__ detjac, int32_t* __restrict__ handed) {
  long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= Ne) return;
  handed[e] = detjac[e * N * N * N] < 0 ? -1 : 1;
}

// Element-local reference derivative along axis d of a smem field (N^3).
__device__ inline double sm_deriv(const double* __restrict__ f, const double* __restrict__ G, int N, int i, int j,
                                  int k, int d) {
  double s = 0.0;
  int id = d == 0 ? i : d == 1 ? j : k;
  for (int p = 0; p < N; ++p) {
    int src = d == 0 ? p + N * (j + N * k) : d == 1 ? i + N * (p + N * k) : i + N * (j + N * p);
    s += G[id * N + p] * f[src];
  }
  return s;
}

// Double-double arithmetic (Dekker 1971; Shewchuk 1997): error-free products
// via FMA and two-sums, so the strongly cancelling curl form is evaluated to
// ~2^-104 and rounded once to double.
struct dd { double hi, lo; };
__device__ __forceinline__ dd two_sum(double a, double b) {
  double s = a + b, bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  double lo = s.lo + a.lo + b.lo;
  double hi = s.hi + lo;
  return {hi, lo - (hi - s.hi)};
}
__device__ __forceinline__ dd dd_mul_d(dd a, double b) {  // (hi + lo) * b
  double p = a.hi * b, e = fma(a.hi, b, -p);
  e = fma(a.lo, b, e);
  double hi = p + e;
  return {hi, e - (hi - p)};
}
__device__ __forceinline__ dd dd_neg(dd a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ double dd_round(dd a) { return a.hi + a.lo; }

// reference derivative along axis d of a double-double smem field (hi/lo arrays)
__device__ inline dd dd_deriv(const double* __restrict__ fh, const double* __restrict__ fl,
                              const double* __restrict__ G, int N, int i, int j, int k, int d) {
  dd s = {0.0, 0.0};
  const int id = d == 0 ? i : d == 1 ? j : k;
  for (int p = 0; p < N; ++p) {
    const int src = d == 0 ? p + N * (j + N * k) : d == 1 ? i + N * (p + N * k) : i + N * (j + N * p);
    s = dd_add(s, dd_mul_d({fh[src], fl ? fl[src] : 0.0}, G[id * N + p]));
  }
  return s;
}

// Curl-form metric terms, one element per CTA, N^3 threads, in double-double.
// smem: X[3], dX[9] (hi, lo), C[3] (hi, lo), G -> (3 + 18 + 6) N^3 + N^2 doubles.
__global__ void k_metric(int N, long long Ne, const double* __restrict__ Gg, const double* __restrict__ Hq,
                         const double* __restrict__ coords, const double* __restrict__ detjac,
                         double* __restrict__ Ja, double* __restrict__ invdetJ, double* __restrict__ Hd) {
  extern __shared__ double sm[];
  const int N3 = N * N * N;
  double* X = sm;                 // 3 N3
  double* dXh = X + 3 * N3;       // 9 N3
  double* dXl = dXh + 9 * N3;     // 9 N3
  double* Ch = dXl + 9 * N3;      // 3 N3
  double* Cl = Ch + 3 * N3;       // 3 N3
  double* G = Cl + 3 * N3;
  const long long e = blockIdx.x;
  const long long nn = Ne * N3;
  const int t = threadIdx.x;
  const int i = t % N, j = (t / N) % N, k = t / (N * N);
  if (t < N * N) G[t] = Gg[t];
  const long long n = e * N3 + t;
  for (int a = 0; a < 3; ++a) X[a * N3 + t] = coords[a + 3 * n];
  __syncthreads();
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      dd v = dd_deriv(X + a * N3, nullptr, G, N, i, j, k, b);
      dXh[(a * 3 + b) * N3 + t] = v.hi;
      dXl[(a * 3 + b) * N3 + t] = v.lo;
    }
  __syncthreads();
  for (int c = 0; c < 3; ++c) {
    const int l = (c + 1) % 3, m = (c + 2) % 3;
    for (int b = 0; b < 3; ++b) {
      dd p1 = dd_mul_d({dXh[(m * 3 + b) * N3 + t], dXl[(m * 3 + b) * N3 + t]}, X[l * N3 + t]);
      dd p2 = dd_mul_d({dXh[(l * 3 + b) * N3 + t], dXl[(l * 3 + b) * N3 + t]}, X[m * N3 + t]);
      dd v = dd_add(p1, dd_neg(p2));
      Ch[b * N3 + t] = 0.5 * v.hi;
      Cl[b * N3 + t] = 0.5 * v.lo;
    }
    __syncthreads();
    for (int al = 0; al < 3; ++al) {
      const int b1 = (al + 1) % 3, b2 = (al + 2) % 3;
      dd v = dd_add(dd_deriv(Ch + b2 * N3, Cl + b2 * N3, G, N, i, j, k, b1),
                    dd_neg(dd_deriv(Ch + b1 * N3, Cl + b1 * N3, G, N, i, j, k, b2)));
      Ja[(al * 3 + c) * nn + n] = dd_round(v);
    }
    __syncthreads();
  }
  invdetJ[n] = 1.0 / detjac[n];
  Hd[n] = Hq[i] * Hq[j] * Hq[k] * fabs(detjac[n]);
}

// dinvjac[a,c,d] = Dhat_d invjac[a,c] (make_metric_derivs).
__global__ void k_dinvjac(int N, long long Ne, const double* __restrict__ Gg, const double* __restrict__ invjac,
                          double* __restrict__ dinvjac) {
  extern __shared__ double sm[];
  const int N3 = N * N * N;
  double* f = sm;
  double* G = f + N3;
  const long long e = blockIdx.x;
  const int t = threadIdx.x;
  const int i = t % N, j = (t / N) % N, k = t / (N * N);
  if (t < N * N) G[t] = Gg[t];
  const long long n = e * N3 + t;
  for (int ac = 0; ac < 9; ++ac) {
    __syncthreads();
    f[t] = invjac[ac + 9 * n];
    __syncthreads();
    for (int d = 0; d < 3; ++d) dinvjac[ac + 9 * d + 27 * n] = sm_deriv(f, G, N, i, j, k, d);
  }
}

// Per boundary-face node: physical outward normal from the analytic Jacobian
// columns x handedness (src/boundaries3d.jl:186-207, src/wave.jl:471-492):
// (nx, ny, nz, JF/(H[row] detJ), JF H_p H_q / Hphys).
template <typename real>
__global__ void k_bnorm(int N, long long Ne, const int32_t* __restrict__ bslot, const int32_t* __restrict__ handed,
                        const double* __restrict__ Hq, const double* __restrict__ jac,
                        const double* __restrict__ detjac, const double* __restrict__ Hphys, int nbf,
                        real* __restrict__ bnorm) {
  long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long total = 6 * Ne * (long long)(N * N);
  if (gid >= total) return;
  const int pq = (int)(gid % (N * N));
  const long long fe = gid / (N * N);
  const int f = (int)(fe % 6);
  const long long e = fe / 6;
  const int slot = bslot[f + 6 * e] < 0 ? -1 : ::wt::bc_slot(bslot[f + 6 * e], nbf);
  if (slot < 0) return;
  const int p = pq % N, q = pq / N;
  const int ai = faxis(f), row = frow(f, N);
  const int ap = ai == 0 ? 1 : 0, aq = ai == 2 ? 1 : 2;
  const double so = fsign(f) * (ai == 1 ? -1.0 : 1.0) * (double)handed[e];
  const long long n = e * N * N * N + face_node(ai, row, p, q, N);
  const double* J = jac + 9 * n;
  double tpx = J[0 + 3 * ap], tpy = J[1 + 3 * ap], tpz = J[2 + 3 * ap];
  double tqx = J[0 + 3 * aq], tqy = J[1 + 3 * aq], tqz = J[2 + 3 * aq];
  double nfx = so * (tpy * tqz - tpz * tqy);
  double nfy = so * (tpz * tqx - tpx * tqz);
  double nfz = so * (tpx * tqy - tpy * tqx);
  double JF = sqrt(nfx * nfx + nfy * nfy + nfz * nfz);
  const long long b = (long long)slot * N * N + pq;
  const long long nb = (long long)nbf * N * N;
  bnorm[0 * nb + b] = (real)(nfx / JF);
  bnorm[1 * nb + b] = (real)(nfy / JF);
  bnorm[2 * nb + b] = (real)(nfz / JF);
  bnorm[3 * nb + b] = (real)(JF / (Hq[row] * detjac[n]));
  bnorm[4 * nb + b] = (real)(JF * Hq[p] * Hq[q] / Hphys[n]);
}

template <typename real>
__global__ void k_streamed_geom(int N, long long Ne, const double* __restrict__ Ja, const double* __restrict__ invdetJ,
                                const double* __restrict__ invjac, real* __restrict__ Ja_r, real* __restrict__ invdetJ_r,
                                real* __restrict__ sdiag) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nn = Ne * N * N * N;
  if (n >= nn) return;
  for (int c = 0; c < 9; ++c) Ja_r[c * nn + n] = (real)Ja[c * nn + n];
  invdetJ_r[n] = (real)invdetJ[n];
  if (n % (N * N * N) == 0) {
    long long e = n / (N * N * N);
    for (int d = 0; d < 3; ++d) sdiag[3 * e + d] = (real)invjac[d + 3 * d + 9 * n];
  }
}

// Background sampling: alpha, sqrt(det gamma), beta, gamma^{ij} (symmetric
// cofactor inverse) exactly as _sample_bg3d_kernel!.
// Kinds 4 and 5 are the spacetime-metric backgrounds at time *d_t + toff (the
// time lives on the device so that a captured RK4 step stays valid).
__global__ void k_background(long long nn, int kind, const double* __restrict__ coords, double p0, double p1,
                             double p2, double p3, double p4, double p5, double p6, double s11, double s12,
                             double s13, double s22, double s23, double s33, const double* __restrict__ d_t,
                             double toff, double* __restrict__ c11) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= nn) return;
  const double x = coords[3 * n], y = coords[3 * n + 1], z = coords[3 * n + 2];
  double al = 1, b1 = 0, b2 = 0, b3 = 0, g11 = 1, g12 = 0, g13 = 0, g22 = 1, g23 = 0, g33 = 1;
  if (kind == 4 || kind == 5) {
    const double t = d_t[0] + toff, ph = 2.0 * M_PI * (x - t) / p1;
    if (kind == 4) {  // gauge wave
      const double H = 1.0 - p0 * sin(ph);
      al = sqrt(H);
      g11 = H;
    } else {          // sine shift
      const double ac = p0 * cos(ph);
      b1 = -ac / (1.0 + ac);
      g11 = (1.0 + ac) * (1.0 + ac);
    }
  } else if (kind == 1) {
    b1 = p0; b2 = p1; b3 = p2;
  } else if (kind == 2) {
    const double tp = 2.0 * M_PI;
    al = 1.0 + p0 * sin(tp * x);
    b1 = p1 * cos(tp * x); b2 = p1 * cos(tp * y); b3 = p1 * cos(tp * z);
    double dx = x - p4, dy = y - p5, dz = z - p6;
    double g = p2 * exp(-(dx * dx + dy * dy + dz * dz) / p3);
    g11 = 1.0 + g * (1.0 + 0.5 * s11);
    g12 = g * (0.5 * s12);
    g13 = g * (0.5 * s13);
    g22 = 1.0 + g * (1.0 + 0.5 * s22);
    g23 = g * (0.5 * s23);
    g33 = 1.0 + g * (1.0 + 0.5 * s33);
  } else if (kind == 3) {
    double r = sqrt(x * x + y * y + z * z);
    double br = p0 + (p1 - p0) * (r - p2) / (p3 - p2);
    if (r > 0) { b1 = br * x / r; b2 = br * y / r; b3 = br * z / r; }
  }
  double det = g11 * (g22 * g33 - g23 * g23) - g12 * (g12 * g33 - g23 * g13) + g13 * (g12 * g23 - g22 * g13);
  c11[0 * nn + n] = al;
  c11[1 * nn + n] = sqrt(det);
  c11[2 * nn + n] = b1; c11[3 * nn + n] = b2; c11[4 * nn + n] = b3;
  c11[5 * nn + n] = (g22 * g33 - g23 * g23) / det;
  c11[6 * nn + n] = (g13 * g23 - g12 * g33) / det;
  c11[7 * nn + n] = (g12 * g23 - g13 * g22) / det;
  c11[8 * nn + n] = (g11 * g33 - g13 * g13) / det;
  c11[9 * nn + n] = (g12 * g13 - g11 * g23) / det;
  c11[10 * nn + n] = (g11 * g22 - g12 * g12) / det;
}

// Streamed coefficients: a = alpha/sqrtg, beta^i, K^{ij} = alpha sqrtg gamma^{ij}.
template <typename real>
__global__ void k_coef_combine(long long nn, const double* __restrict__ c11, real* __restrict__ c10) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= nn) return;
  const double al = c11[n], sg = c11[nn + n];
  const double as = al * sg;
  c10[0 * nn + n] = (real)(al / sg);
  c10[1 * nn + n] = (real)c11[2 * nn + n];
  c10[2 * nn + n] = (real)c11[3 * nn + n];
  c10[3 * nn + n] = (real)c11[4 * nn + n];
  for (int c = 0; c < 6; ++c) c10[(4 + c) * nn + n] = (real)(as * c11[(5 + c) * nn + n]);
}

__global__ void k_min_spacing(int N, long long nn, const double* __restrict__ coords, double* __restrict__ partial) {
  __shared__ double red[256];
  double h = DBL_MAX;
  const int N3 = N * N * N;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    int t = (int)(n % N3);
    int i = t % N, j = (t / N) % N, k = t / (N * N);
    const double* c = coords + 3 * n;
    if (i > 0) { const double* o = coords + 3 * (n - 1); h = fmin(h, sqrt((c[0]-o[0])*(c[0]-o[0]) + (c[1]-o[1])*(c[1]-o[1]) + (c[2]-o[2])*(c[2]-o[2]))); }
    if (j > 0) { const double* o = coords + 3 * (n - N); h = fmin(h, sqrt((c[0]-o[0])*(c[0]-o[0]) + (c[1]-o[1])*(c[1]-o[1]) + (c[2]-o[2])*(c[2]-o[2]))); }
    if (k > 0) { const double* o = coords + 3 * (n - N * N); h = fmin(h, sqrt((c[0]-o[0])*(c[0]-o[0]) + (c[1]-o[1])*(c[1]-o[1]) + (c[2]-o[2])*(c[2]-o[2]))); }
  }
  red[threadIdx.x] = h;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// ---------------------------------------------------------------------------
static inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

int launch_geom_analytic(DevMesh& m, double x0, double x1, double A, cudaStream_t s, int z0, int Mz) {
  k_geom_analytic<<<nblk(m.nn, 256), 256, 0, s>>>(m.N, m.M[0], m.M[1], Mz > 0 ? Mz : m.M[2], z0, x0, x1 - x0, A, m.x,
                                                  m.nn, m.coords, m.jac);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_geom_derived(DevMesh& m, cudaStream_t s) {
  k_geom_derived<<<nblk(m.nn, 256), 256, 0, s>>>(m.N, m.nn, m.H, m.jac, m.invjac, m.detjac, m.Hphys);
  k_handed<<<nblk(m.Ne, 256), 256, 0, s>>>(m.N, m.Ne, m.detjac, m.handed);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_metric(DevMesh& m, cudaStream_t s) {
  const int N3 = m.N * m.N * m.N;
  size_t smem = (27 * (size_t)N3 + m.N * m.N) * sizeof(double);
  cudaFuncSetAttribute(k_metric, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_metric<<<(unsigned)m.Ne, N3, smem, s>>>(m.N, m.Ne, m.G, m.H, m.coords, m.detjac, m.Ja, m.invdetJ, m.Hd);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_dinvjac(DevMesh& m, cudaStream_t s) {
  const int N3 = m.N * m.N * m.N;
  size_t smem = ((size_t)N3 + m.N * m.N) * sizeof(double);
  k_dinvjac<<<(unsigned)m.Ne, N3, smem, s>>>(m.N, m.Ne, m.G, m.invjac, m.dinvjac);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_boundary_normals(DevMesh& m, cudaStream_t s) {
  if (m.nbf == 0) return 0;
  long long total = 6 * m.Ne * (long long)(m.N * m.N);
  if (m.precision == 0)
    k_bnorm<double><<<nblk(total, 256), 256, 0, s>>>(m.N, m.Ne, m.bslot, m.handed, m.H, m.jac, m.detjac, m.Hphys,
                                                     m.nbf, (double*)m.bnorm);
  else
    k_bnorm<float><<<nblk(total, 256), 256, 0, s>>>(m.N, m.Ne, m.bslot, m.handed, m.H, m.jac, m.detjac, m.Hphys,
                                                    m.nbf, (float*)m.bnorm);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_streamed_geometry(DevMesh& m, cudaStream_t s) {
  if (m.precision == 0)
    k_streamed_geom<double><<<nblk(m.nn, 256), 256, 0, s>>>(m.N, m.Ne, m.Ja, m.invdetJ, m.invjac, (double*)m.Ja_r,
                                                            (double*)m.invdetJ_r, (double*)m.sdiag);
  else
    k_streamed_geom<float><<<nblk(m.nn, 256), 256, 0, s>>>(m.N, m.Ne, m.Ja, m.invdetJ, m.invjac, (float*)m.Ja_r,
                                                           (float*)m.invdetJ_r, (float*)m.sdiag);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_background(const DevMesh& m, DevCoef& c, int kind, const double* p, cudaStream_t s, const double* d_t,
                      double toff) {
  if ((kind == 4 || kind == 5) && !d_t) return -1;
  k_background<<<nblk(m.nn, 256), 256, 0, s>>>(m.nn, kind, m.coords, p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7],
                                               p[8], p[9], p[10], p[11], p[12], d_t, toff, c.c11);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

__global__ void k_advance_time(double* __restrict__ d_t, double dt) { d_t[0] += dt; }

int launch_advance_time(double* d_t, double dt, cudaStream_t s) {
  k_advance_time<<<1, 1, 0, s>>>(d_t, dt);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_coef_combine(const DevMesh& m, DevCoef& c, cudaStream_t s) {
  if (c.precision == 0)
    k_coef_combine<double><<<nblk(m.nn, 256), 256, 0, s>>>(m.nn, c.c11, (double*)c.c10);
  else
    k_coef_combine<float><<<nblk(m.nn, 256), 256, 0, s>>>(m.nn, c.c11, (float*)c.c10);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_min_spacing(const DevMesh& m, double* out, cudaStream_t s) {
  const int nb = 1024;
  double* partial = nullptr;
  if (cudaMallocAsync(&partial, nb * sizeof(double), s) != cudaSuccess) return -3;
  k_min_spacing<<<nb, 256, 0, s>>>(m.N, m.nn, m.coords, partial);
  std::vector<double> h(nb);
  cudaMemcpyAsync(h.data(), partial, nb * sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(partial, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
  double r = DBL_MAX;
  for (double v : h) r = std::fmin(r, v);
  *out = r;
  return 0;
}

}  // namespace wt

namespace wt {

// ---------------------------------------------------------------------------
// Initial data on the device (src/wave.jl:100-323, src/evolve.jl:1115-1118,
// 1257-1263).  kind: 0 eigenmode_cartesian! (A, kx, ky, kz, omega, x0, x1),
// 1 sum of Gaussians (count; then cx, cy, cz, A, w per pulse),
// 2 outgoing_pulse! (A, s0, sigma, cx, cy, cz), 3 plane wave of the
// constant-shift background (k, omega, s = bx+by+bz): Phi = sin(k(x+y+z) - omega t),
// Pi = (-omega - k s) cos(...), 4 eigenmode_radial! (A, R, n, cx, cy, cz).
__device__ inline double sinhc_dev(double x) {
  const double x2 = x * x;
  if (x2 < 1.0 / 1000.0) return 1.0 + x2 * (1.0 / 6.0 + x2 * (1.0 / 120.0 + x2 * (1.0 / 5040.0)));
  return sinh(x) / x;
}

template <typename real>
__global__ void k_initial(long long nn, int kind, const double* __restrict__ coords, const double* __restrict__ p,
                          int np, double t, real* __restrict__ u, real* __restrict__ ut) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= nn) return;
  const double x = coords[3 * n], y = coords[3 * n + 1], z = coords[3 * n + 2];
  double uv = 0.0, vv = 0.0;
  if (kind == 0) {
    const double A = p[0], kx = p[1], ky = p[2], kz = p[3], om = p[4], x0 = p[5], L = p[6] - p[5];
    const double s = sin(kx * (x - x0) / L) * sin(ky * (y - x0) / L) * sin(kz * (z - x0) / L);
    uv = A * s * cos(om * t);
    vv = -A * om * s * sin(om * t);
  } else if (kind == 1) {
    const int cnt = (int)p[0];
    for (int q = 0; q < cnt && 1 + 5 * q + 4 < np; ++q) {
      const double* g = p + 1 + 5 * q;
      const double d2 = (x - g[0]) * (x - g[0]) + (y - g[1]) * (y - g[1]) + (z - g[2]) * (z - g[2]);
      uv += g[3] * exp(-d2 / (2.0 * g[4] * g[4]));
    }
  } else if (kind == 2) {
    const double A = p[0], s0 = p[1], sg = p[2];
    const double isg2 = 1.0 / (sg * sg);
    const double be = t + s0, be2 = be * be;
    const double r2 = (x - p[3]) * (x - p[3]) + (y - p[4]) * (y - p[4]) + (z - p[5]) * (z - p[5]);
    const double r = sqrt(r2);
    const double ex = exp(-0.5 * (be2 + r2) * isg2);
    uv = 2.0 * A * be * isg2 * sinhc_dev(be * r * isg2) * ex;
    vv = -2.0 * A * isg2 * ex * (be2 * isg2 * sinhc_dev(be * r * isg2) - cosh(be * r * isg2));
  } else if (kind == 3) {
    const double k = p[0], om = p[1], s = p[2];
    uv = sin(k * (x + y + z) - om * t);
    vv = (-om - k * s) * cos(k * (x + y + z) - om * t);
  } else if (kind == 4) {
    const double A = p[0], R = p[1], nr = p[2];
    const double om = nr * M_PI / R;
    const double r = sqrt((x - p[3]) * (x - p[3]) + (y - p[4]) * (y - p[4]) + (z - p[5]) * (z - p[5]));
    const double arg = nr * r / R;
    const double sc = arg == 0.0 ? 1.0 : sin(M_PI * arg) / (M_PI * arg);
    uv = A * sc * cos(om * t);
    vv = -A * om * sc * sin(om * t);
  }
  u[n] = (real)uv;
  if (ut) ut[n] = (real)vv;
}

int launch_initial(const DevMesh& m, int kind, const double* dparams, int np, double t, void* u, void* ut,
                   cudaStream_t s, bool f64) {
  const unsigned b = (unsigned)((m.nn + 255) / 256);
  if (m.precision == 0 || f64)
    k_initial<double><<<b, 256, 0, s>>>(m.nn, kind, m.coords, dparams, np, t, (double*)u, (double*)ut);
  else
    k_initial<float><<<b, 256, 0, s>>>(m.nn, kind, m.coords, dparams, np, t, (float*)u, (float*)ut);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// this file's bounds word (bounds-check build; 0 otherwise)
WT_BOUNDS_TAKE(bounds_take_geom)

}  // namespace wt
