// wavetoy_oracle.cpp -- CPU Float64 restatement of WaveToySecondOrder.jl's 3D
// hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
// baseline.  Nothing in the shipped library (wavetoysecondorder.jl_b200/) links,
// loads or calls it; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg may load it, and then only as the checker.
//
// Parity status: PARTLY UNPINNED.  The reference is pure Julia and its core
// arithmetic lives in two unvendored, unpinned packages (HexSBPSAT: apply_D!,
// apply_gradient3d!/apply_divergence3d!, apply_laplacian!, make_operators,
// make_geometry, make_metric_terms3d; HexMeshes: mesh builders).  There is no
// Julia toolchain here and the reference ships no golden vectors.  Those pieces
// are restated from the reference's own documentation of them (README.md:14-80,
// METHODS.md:151-170 and 256-264) and from the published methods named beside
// each function; they are pinned by the reference's property tests (spectrum,
// free-stream, convergence, energy, symmetry), which tests/ port.  The in-repo
// Julia (src/wave3d_curved.jl, src/boundaries3d.jl, src/boundaries1d.jl,
// src/wave.jl:453-611, src/wave_strong_rhs.jl, src/wave_lap_strong.jl,
// RK4 of test/wave3d_tests.jl:32-44) is restated line by line.
//
// Conventions (shared with the CUDA library, chosen to match the reference's
// Julia column-major arrays): a field is (N,N,N,Ne) with node index
//   n = i + N*(j + N*(k + N*e))          (0-based here, i fastest)
// jac[a,b,node] = dx_a/dxi_b at jac[a + 3*b + 9*node]; invjac[al,be,node] =
// dxi_al/dx_be at invjac[al + 3*be + 9*node].  Faces f = 0..5 are
// (-x,+x,-y,+y,-z,+z): axis f/2, row 0 or N-1, outward sign -1/+1.  Face node
// (p,q) = (j,k) | (i,k) | (i,j) for axis 0 | 1 | 2 (src/wave_lap_strong.jl:72-74).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <limits>
#include <string>
#include <omp.h>

namespace {

// ---------------------------------------------------------------------------
// Gauss-Lobatto-Legendre SBP operators on the reference interval [0,1].
// Nodes: +-1 and the roots of P'_{N-1} (Newton on q = P_N - P_{N-2}, as in
// Kopriva 2009, "Implementing Spectral Methods for PDEs", Alg. 25).  Weights
// 2/(p(p+1)P_p(x)^2).  Differentiation matrix from barycentric weights
// (Berrut & Trefethen 2004) with the negative-sum diagonal.  Mapped to [0,1]:
// x -> (x+1)/2, H -> w/2, G -> 2D.  For GLL collocation HG + (HG)^T = B with
// B = diag(-1,0,...,0,1) (README.md:14-19), so D = G and L = G*G.
struct Ops {
  int N = 0;
  std::vector<double> x, H, G;  // G[i*N + p] = d/dx of Lagrange basis p at node i
};

void legendre_q(int p, long double x, long double& q, long double& dq, long double& Lp) {
  // q(x) = L_{p+1}(x) - L_{p-1}(x), derivative dq, and L_p(x).
  long double L[64], dL[64];
  L[0] = 1.0L; dL[0] = 0.0L;
  L[1] = x; dL[1] = 1.0L;
  for (int k = 2; k <= p + 1; ++k) {
    L[k] = ((2.0L * k - 1.0L) * x * L[k - 1] - (k - 1.0L) * L[k - 2]) / k;
    dL[k] = dL[k - 2] + (2.0L * k - 1.0L) * L[k - 1];
  }
  q = L[p + 1] - L[p - 1];
  dq = dL[p + 1] - dL[p - 1];
  Lp = L[p];
}

// Computed in extended precision (x87 long double) and rounded once to
// double, so the operators are correctly rounded (to within the extended
// format's own round-off) independently of the algorithm.
Ops make_ops(int N) {
  Ops o; o.N = N;
  int p = N - 1;
  std::vector<long double> xs(N), ws(N);
  xs[0] = -1.0L; xs[p] = 1.0L;
  long double Lp;
  ws[0] = ws[p] = 2.0L / (p * (p + 1.0L));
  for (int j = 1; j < N / 2; ++j) {
    // initial guess: Chebyshev-Gauss-Lobatto node
    long double x = -cosl(3.14159265358979323846264338327950288L * j / p);
    for (int it = 0; it < 100; ++it) {
      long double q, dq;
      legendre_q(p, x, q, dq, Lp);
      long double dx = -q / dq;
      x += dx;
      if (fabsl(dx) <= 1e-19L * (1.0L + fabsl(x))) break;
    }
    long double q, dq; legendre_q(p, x, q, dq, Lp);
    xs[j] = x; xs[p - j] = -x;
    ws[j] = ws[p - j] = 2.0L / (p * (p + 1.0L) * Lp * Lp);
  }
  if (N % 2 == 1) {  // centre node
    int c = N / 2; long double q, dq; legendre_q(p, 0.0L, q, dq, Lp);
    xs[c] = 0.0L; ws[c] = 2.0L / (p * (p + 1.0L) * Lp * Lp);
  }
  // barycentric weights
  std::vector<long double> lam(N, 1.0L);
  for (int j = 0; j < N; ++j)
    for (int k = 0; k < N; ++k)
      if (k != j) lam[j] /= (xs[j] - xs[k]);
  std::vector<long double> D(N * N, 0.0L);
  for (int i = 0; i < N; ++i) {
    long double sacc = 0.0L;
    for (int j = 0; j < N; ++j) {
      if (j == i) continue;
      D[i * N + j] = (lam[j] / lam[i]) / (xs[i] - xs[j]);
      sacc += D[i * N + j];
    }
    (void)sacc;
    // exact GLL diagonal: 0 inside, -p(p+1)/4 and +p(p+1)/4 at the ends
    D[i * N + i] = i == 0 ? -p * (p + 1.0L) / 4.0L : (i == p ? p * (p + 1.0L) / 4.0L : 0.0L);
  }
  o.x.resize(N); o.H.resize(N); o.G.resize(N * N);
  for (int i = 0; i < N; ++i) { o.x[i] = (double)(0.5L * (xs[i] + 1.0L)); o.H[i] = (double)(0.5L * ws[i]); }
  o.x[0] = 0.0; o.x[p] = 1.0;
  for (int i = 0; i < N * N; ++i) o.G[i] = (double)(2.0L * D[i]);
  return o;
}

inline int faxis(int f) { return f >> 1; }
inline int frow(int f, int N) { return (f & 1) ? N - 1 : 0; }
inline double fsign(int f) { return (f & 1) ? 1.0 : -1.0; }

// node index helpers
inline long nid(int N, int i, int j, int k, long e) { return i + (long)N * (j + (long)N * (k + (long)N * e)); }
inline void face_ijk(int ax, int r, int p, int q, int& i, int& j, int& k) {
  if (ax == 0) { i = r; j = p; k = q; }
  else if (ax == 1) { i = p; j = r; k = q; }
  else { i = p; j = q; k = r; }
}

// Bookkeeping for one mesh plus its geometry and metric terms.
struct Mesh {
  int N = 0; long Ne = 0; int M[3] = {0, 0, 0};
  int periodic = 0; double x0 = 0, x1 = 1, A = 0;
  Ops ops;
  std::vector<int32_t> nbr, nbrf, orient, bdry;   // [f + 6e]; nbr -1 = none
  std::vector<double> coords, jac, invjac, detjac, Hphys;
  std::vector<int32_t> handed;
  std::vector<double> Ja;        // 9 fields: Ja[(al*3 + i)*nn + node] = J dxi_al/dx_i (curl form)
  std::vector<double> invdetJ, Hd;
  std::vector<double> dinvjac;   // 27 per node, lazily: [a + 3c + 9d + 27 node] = Dhat_d invjac[a,c]
  double mu = -1.0, inv_mu5 = 0.0;
  long nn() const { return (long)N * N * N * Ne; }
};

// Neighbour element's node (a,b,c) coinciding with node (p,q) of face f of
// element e.  Face orientation orient[f + 6e] is the D4 map of the library's
// convention (include/wavetoy_b200.h, "orientation"): swap p and q if bit 2,
// then reverse the first index if bit 0 and the second if bit 1.  This is
// the role of _neigh_pq in _extract_face_oriented! (src/wave_strong_rhs.jl:41-73).
inline void nbr_face_ijk(const Mesh& m, long e, int f, int p, int q, int& a, int& b, int& c) {
  const int N = m.N, fn = m.nbrf[f + 6 * e], ori = m.orient[f + 6 * e];
  int u = (ori & 4) ? q : p, v = (ori & 4) ? p : q;
  if (ori & 1) u = N - 1 - u;
  if (ori & 2) v = N - 1 - v;
  face_ijk(faxis(fn), frow(fn, N), u, v, a, b, c);
}

// Reference derivative along axis d of field u (element-local, no scaling):
// out[node] = sum_p G[idx_d(node), p] * u[node with idx_d = p].
void ref_deriv(const Mesh& m, const double* u, double* out, int d, long e) {
  const int N = m.N; const double* G = m.ops.G.data();
  for (int k = 0; k < N; ++k)
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) {
        double s = 0.0;
        int id = d == 0 ? i : d == 1 ? j : k;
        for (int p = 0; p < N; ++p) {
          long src = d == 0 ? nid(N, p, j, k, e) : d == 1 ? nid(N, i, p, k, e) : nid(N, i, j, p, e);
          s += G[id * N + p] * u[src];
        }
        out[nid(N, i, j, k, e)] = s;
      }
}

// ---------------------------------------------------------------------------
// Mesh builder: uniform hex on [x0,x1]^3 with Mx*My*Mz elements, optionally
// warped by the smooth map of the reference's warped-cube tests
// (make_warped_uniform_hex, test/dirichlet_warped_tests.jl:23-40):
//   X = s + A*P(s),  P = sin(2 pi s1) sin(2 pi s2) sin(2 pi s3)  (same P for
//   all three components: the map "cyclically permuted for y and z"),
// s in [0,1]^3 the uniform reference position, x = x0 + (x1-x0)*X.
// Element numbering e = ex + Mx*(ey + My*ez).  Outer-face tags: outer_tag = 0
// gives side tags 1..6 (the reference's Dirichlet convention,
// src/wave.jl:567-571); otherwise every outer face gets outer_tag (7 =
// Sommerfeld).  Jacobians are analytic (the reference's make_geometry
// Jacobians are analytic, METHODS.md:88-90).
void build_mesh(Mesh& m, int N, int Mx, int My, int Mz, double x0, double x1, double A,
                int periodic, int outer_tag) {
  m.N = N; m.M[0] = Mx; m.M[1] = My; m.M[2] = Mz; m.Ne = (long)Mx * My * Mz;
  m.periodic = periodic; m.x0 = x0; m.x1 = x1; m.A = A;
  m.ops = make_ops(N);
  const long Ne = m.Ne, nn = m.nn();
  m.nbr.assign(6 * Ne, -1); m.nbrf.assign(6 * Ne, 0); m.orient.assign(6 * Ne, 0); m.bdry.assign(6 * Ne, 0);
  for (int ez = 0; ez < Mz; ++ez)
    for (int ey = 0; ey < My; ++ey)
      for (int ex = 0; ex < Mx; ++ex) {
        long e = ex + (long)Mx * (ey + (long)My * ez);
        int c[3] = {ex, ey, ez};
        for (int f = 0; f < 6; ++f) {
          int ax = faxis(f); int dir = (f & 1) ? 1 : -1;
          int cc[3] = {c[0], c[1], c[2]};
          cc[ax] += dir;
          bool outside = cc[ax] < 0 || cc[ax] >= m.M[ax];
          if (outside && !periodic) {
            m.nbr[f + 6 * e] = -1;
            m.bdry[f + 6 * e] = outer_tag == 0 ? f + 1 : outer_tag;
            continue;
          }
          cc[ax] = (cc[ax] + m.M[ax]) % m.M[ax];
          long en = cc[0] + (long)Mx * (cc[1] + (long)My * cc[2]);
          m.nbr[f + 6 * e] = (int32_t)en;
          m.nbrf[f + 6 * e] = f ^ 1;
        }
      }
  m.coords.assign(3 * nn, 0); m.jac.assign(9 * nn, 0); m.invjac.assign(9 * nn, 0);
  m.detjac.assign(nn, 0); m.Hphys.assign(nn, 0); m.handed.assign(Ne, 1);
  const double L = x1 - x0, tp = 2.0 * M_PI;
#pragma omp parallel for schedule(static)
  for (long e = 0; e < Ne; ++e) {
    int ex = (int)(e % Mx), ey = (int)((e / Mx) % My), ez = (int)(e / ((long)Mx * My));
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          long n = nid(N, i, j, k, e);
          double s[3] = {(ex + m.ops.x[i]) / Mx, (ey + m.ops.x[j]) / My, (ez + m.ops.x[k]) / Mz};
          double sn[3] = {std::sin(tp * s[0]), std::sin(tp * s[1]), std::sin(tp * s[2])};
          double cs[3] = {std::cos(tp * s[0]), std::cos(tp * s[1]), std::cos(tp * s[2])};
          double P = sn[0] * sn[1] * sn[2];
          double dP[3] = {tp * cs[0] * sn[1] * sn[2], tp * sn[0] * cs[1] * sn[2], tp * sn[0] * sn[1] * cs[2]};
          double Ms[3] = {(double)Mx, (double)My, (double)Mz};
          double J[3][3];
          for (int a = 0; a < 3; ++a) {
            m.coords[a + 3 * n] = x0 + L * (s[a] + A * P);
            for (int b = 0; b < 3; ++b) J[a][b] = L * ((a == b ? 1.0 : 0.0) + A * dP[b]) / Ms[b];
          }
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) m.jac[a + 3 * b + 9 * n] = J[a][b];
          double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
          double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
          double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
          double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
          // inverse: invjac[al][be] = cof(J)[be][al] / det
          double inv[3][3];
          inv[0][0] = c00 / det;
          inv[1][0] = c01 / det;
          inv[2][0] = c02 / det;
          inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
          inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
          inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
          inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
          inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
          inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) m.invjac[a + 3 * b + 9 * n] = inv[a][b];
          m.detjac[n] = det;
          m.Hphys[n] = m.ops.H[i] * m.ops.H[j] * m.ops.H[k] * std::fabs(det);
        }
    m.handed[e] = m.detjac[nid(N, 0, 0, 0, e)] < 0 ? -1 : 1;
  }
}

// Mesh from arrays (coords (3,N,N,N,Ne), jac = dx_a/dxi_b, 0-based topology with
// face orientations): invjac, detjac, Hphys and handedness from the Jacobian as
// in build_mesh.
void build_mesh_arrays(Mesh& m, int N, long Ne, const double* coords, const double* jac, const int32_t* nbr,
                       const int32_t* nbrf, const int32_t* orient, const int32_t* bdry) {
  m.N = N; m.Ne = Ne; m.M[0] = m.M[1] = m.M[2] = 0;
  m.ops = make_ops(N);
  const long nn = m.nn();
  m.nbr.assign(nbr, nbr + 6 * Ne); m.nbrf.assign(nbrf, nbrf + 6 * Ne);
  m.orient.assign(orient, orient + 6 * Ne); m.bdry.assign(bdry, bdry + 6 * Ne);
  m.coords.assign(coords, coords + 3 * nn); m.jac.assign(jac, jac + 9 * nn);
  m.invjac.assign(9 * nn, 0); m.detjac.assign(nn, 0); m.Hphys.assign(nn, 0); m.handed.assign(Ne, 1);
#pragma omp parallel for schedule(static)
  for (long e = 0; e < Ne; ++e) {
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          long n = nid(N, i, j, k, e);
          double J[3][3];
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) J[a][b] = m.jac[a + 3 * b + 9 * n];
          double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
          double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
          double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
          double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
          double inv[3][3];
          inv[0][0] = c00 / det;
          inv[1][0] = c01 / det;
          inv[2][0] = c02 / det;
          inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
          inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
          inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
          inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
          inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
          inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) m.invjac[a + 3 * b + 9 * n] = inv[a][b];
          m.detjac[n] = det;
          m.Hphys[n] = m.ops.H[i] * m.ops.H[j] * m.ops.H[k] * std::fabs(det);
        }
    m.handed[e] = m.detjac[nid(N, 0, 0, 0, e)] < 0 ? -1 : 1;
  }
}

// Discrete curl-form metric terms J a^al_i (Kopriva 2006, J. Sci. Comput.
// 26:301; Thomas & Lombard 1979), as HexSBPSAT.make_metric_terms3d is
// documented (METHODS.md:156-166): J a^n = curl_xi C^n,
// C^n = 1/2 (X_l grad_xi X_m - X_m grad_xi X_l), (n,l,m) cyclic.  The
// discrete metric identity sum_al Dhat_al(J a^al_i) = 0 then holds to
// round-off because tensor-product derivatives commute.  Hd = H_ref*detJ is
// the energy mass of the split-form operators, invdetJ = 1/detJ.
void build_metric(Mesh& m) {
  // Evaluated in extended precision (long double) and rounded once: the curl
  // form cancels strongly (terms ~ h sum|G| for a result ~ h^2), and a plain
  // double evaluation carries ~5e-12 relative error.
  const int N = m.N; const long Ne = m.Ne, nn = m.nn(); const long ne3 = (long)N * N * N;
  m.Ja.assign(9 * nn, 0); m.invdetJ.assign(nn, 0); m.Hd.assign(nn, 0);
  std::vector<long double> GL(m.ops.G.begin(), m.ops.G.end());
  auto derL = [&](const long double* f, long double* o, int d) {
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          int id = d == 0 ? i : d == 1 ? j : k;
          long double acc = 0.0L;
          for (int p = 0; p < N; ++p) {
            long src = d == 0 ? nid(N, p, j, k, 0) : d == 1 ? nid(N, i, p, k, 0) : nid(N, i, j, p, 0);
            acc += GL[id * N + p] * f[src];
          }
          o[nid(N, i, j, k, 0)] = acc;
        }
  };
#pragma omp parallel
  {
    std::vector<long double> X(3 * ne3), dX(9 * ne3), C(3 * ne3), t1(ne3), t2(ne3);
#pragma omp for schedule(static)
    for (long e = 0; e < Ne; ++e) {
      for (long t = 0; t < ne3; ++t)
        for (int a = 0; a < 3; ++a) X[a * ne3 + t] = m.coords[a + 3 * (t + ne3 * e)];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) derL(&X[a * ne3], &dX[(a * 3 + b) * ne3], b);
      for (int n = 0; n < 3; ++n) {
        int l = (n + 1) % 3, mm = (n + 2) % 3;
        for (int b = 0; b < 3; ++b)
          for (long t = 0; t < ne3; ++t)
            C[b * ne3 + t] = 0.5L * (X[l * ne3 + t] * dX[(mm * 3 + b) * ne3 + t] - X[mm * ne3 + t] * dX[(l * 3 + b) * ne3 + t]);
        // (curl C)_al = Dhat_{al+1} C_{al+2} - Dhat_{al+2} C_{al+1}
        for (int al = 0; al < 3; ++al) {
          int b1 = (al + 1) % 3, b2 = (al + 2) % 3;
          derL(&C[b2 * ne3], t1.data(), b1);
          derL(&C[b1 * ne3], t2.data(), b2);
          for (long t = 0; t < ne3; ++t) m.Ja[(al * 3 + n) * nn + t + ne3 * e] = (double)(t1[t] - t2[t]);
        }
      }
      for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i) {
            long t = nid(N, i, j, k, e);
            m.invdetJ[t] = 1.0 / m.detjac[t];
            m.Hd[t] = m.ops.H[i] * m.ops.H[j] * m.ops.H[k] * std::fabs(m.detjac[t]);
          }
    }
  }
}

// ---------------------------------------------------------------------------
// apply_D!(Du, u, d): per-axis first derivative, reference SBP G along
// reference axis d scaled to physical by s = invjac[d,d] taken at the
// element's first node, plus the centred-flux SAT n*s*(u_nbr - u)/(2 H[row])
// = n*(u_nbr - u)/(2 Hphys_face) on interior d-faces (METHODS.md:256-264,
// 151-155); faces with bdry != 0 get no SAT (one-sided).  On axis-aligned
// affine meshes s = 1/h_d and H*D is exactly skew (D_1d (x) I).  On curved
// meshes the element-constant s keeps D skew in the weighted norm
// H_i H_j H_k / s_e, so the Kreiss-Oliger term mu^-5 D^6 stays dissipative.
void apply_D(const Mesh& m, const double* u, double* out, int d) {
  const int N = m.N; const long Ne = m.Ne;
  const double* G = m.ops.G.data(); const double* H = m.ops.H.data();
#pragma omp parallel for schedule(static)
  for (long e = 0; e < Ne; ++e) {
    const double sc = m.invjac[d + 3 * d + 9 * nid(N, 0, 0, 0, e)];
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          int id = d == 0 ? i : d == 1 ? j : k;
          double s = 0.0;
          for (int p = 0; p < N; ++p) {
            long src = d == 0 ? nid(N, p, j, k, e) : d == 1 ? nid(N, i, p, k, e) : nid(N, i, j, p, e);
            s += G[id * N + p] * u[src];
          }
          long n = nid(N, i, j, k, e);
          out[n] = sc * s;
        }
    for (int f = 2 * d; f < 2 * d + 2; ++f) {
      if (m.bdry[f + 6 * e] != 0) continue;
      long en = m.nbr[f + 6 * e]; if (en < 0) continue;
      int fn = m.nbrf[f + 6 * e];
      int r = frow(f, N), rn = frow(fn, N); double nh = fsign(f);
      for (int q = 0; q < N; ++q)
        for (int p = 0; p < N; ++p) {
          int i, j, k, a, b, c;
          face_ijk(d, r, p, q, i, j, k);
          nbr_face_ijk(m, e, f, p, q, a, b, c);
          long n = nid(N, i, j, k, e), nb = nid(N, a, b, c, en);
          out[n] += nh * sc / (2.0 * H[r]) * (u[nb] - u[n]);
        }
    }
  }
}

// Split-form (1/2 conservative + 1/2 advective) curvilinear gradient with
// curl-form metric terms and centred-flux SAT, as HexSBPSAT's
// apply_gradient3d! is documented (METHODS.md:156-170, 124-135):
//   d_i u = (1/J) sum_al [1/2 Dhat_al(Ja^al_i u) + 1/2 Ja^al_i Dhat_al u]
//   + on interior al-faces: n * Ja^al_i (u_nbr - u) / (2 H[row] J).
// With the matching divergence below, Hd*grad and Hd*div are adjoint up to
// outer-boundary terms (skew-adjoint pair).
void grad3d(const Mesh& m, const double* u, double* g1, double* g2, double* g3) {
  const int N = m.N; const long Ne = m.Ne, nn = m.nn(); const long ne3 = (long)N * N * N;
  const double* H = m.ops.H.data();
  double* g[3] = {g1, g2, g3};
#pragma omp parallel
  {
    Mesh loc; loc.N = N; loc.ops = m.ops; loc.Ne = 1;
    std::vector<double> ue(ne3), du(ne3), w(ne3), dw(ne3), acc(3 * ne3);
#pragma omp for schedule(static)
    for (long e = 0; e < Ne; ++e) {
      std::copy(u + ne3 * e, u + ne3 * (e + 1), ue.begin());
      std::fill(acc.begin(), acc.end(), 0.0);
      for (int al = 0; al < 3; ++al) {
        ref_deriv(loc, ue.data(), du.data(), al, 0);
        for (int i = 0; i < 3; ++i) {
          const double* mJ = &m.Ja[(al * 3 + i) * nn + ne3 * e];
          for (long t = 0; t < ne3; ++t) w[t] = mJ[t] * ue[t];
          ref_deriv(loc, w.data(), dw.data(), al, 0);
          for (long t = 0; t < ne3; ++t) acc[i * ne3 + t] += 0.5 * dw[t] + 0.5 * mJ[t] * du[t];
        }
      }
      for (int f = 0; f < 6; ++f) {
        if (m.bdry[f + 6 * e] != 0) continue;
        long en = m.nbr[f + 6 * e]; if (en < 0) continue;
        int fn = m.nbrf[f + 6 * e], al = faxis(f);
        int r = frow(f, N), rn = frow(fn, N); double nh = fsign(f);
        for (int q = 0; q < N; ++q)
          for (int p = 0; p < N; ++p) {
            int i, j, k, a, b, c;
            face_ijk(al, r, p, q, i, j, k);
            nbr_face_ijk(m, e, f, p, q, a, b, c);
            long t = nid(N, i, j, k, 0), nb = nid(N, a, b, c, en);
            double jump = u[nb] - ue[t];
            for (int ii = 0; ii < 3; ++ii)
              acc[ii * ne3 + t] += nh * m.Ja[(al * 3 + ii) * nn + ne3 * e + t] * jump / (2.0 * H[r]);
          }
      }
      for (int i = 0; i < 3; ++i)
        for (long t = 0; t < ne3; ++t) g[i][ne3 * e + t] = acc[i * ne3 + t] * m.invdetJ[ne3 * e + t];
    }
  }
}

// Split-form curvilinear divergence (apply_divergence3d!, METHODS.md:156-170):
//   div F = (1/J) sum_al [1/2 Dhat_al(sum_i Ja^al_i F_i) + 1/2 sum_i Ja^al_i Dhat_al F_i]
//   + on interior al-faces: n * sum_i Ja^al_i (F_i,nbr - F_i) / (2 H[row] J).
void div3d(const Mesh& m, const double* F1, const double* F2, const double* F3, double* out) {
  const int N = m.N; const long Ne = m.Ne, nn = m.nn(); const long ne3 = (long)N * N * N;
  const double* H = m.ops.H.data();
  const double* F[3] = {F1, F2, F3};
#pragma omp parallel
  {
    Mesh loc; loc.N = N; loc.ops = m.ops; loc.Ne = 1;
    std::vector<double> Fe(3 * ne3), dF(ne3), w(ne3), dw(ne3), acc(ne3);
#pragma omp for schedule(static)
    for (long e = 0; e < Ne; ++e) {
      for (int i = 0; i < 3; ++i) std::copy(F[i] + ne3 * e, F[i] + ne3 * (e + 1), Fe.begin() + i * ne3);
      std::fill(acc.begin(), acc.end(), 0.0);
      for (int al = 0; al < 3; ++al) {
        const double* mJ[3] = {&m.Ja[(al * 3 + 0) * nn + ne3 * e], &m.Ja[(al * 3 + 1) * nn + ne3 * e],
                               &m.Ja[(al * 3 + 2) * nn + ne3 * e]};
        for (long t = 0; t < ne3; ++t)
          w[t] = mJ[0][t] * Fe[t] + mJ[1][t] * Fe[ne3 + t] + mJ[2][t] * Fe[2 * ne3 + t];
        ref_deriv(loc, w.data(), dw.data(), al, 0);
        for (long t = 0; t < ne3; ++t) acc[t] += 0.5 * dw[t];
        for (int i = 0; i < 3; ++i) {
          ref_deriv(loc, &Fe[i * ne3], dF.data(), al, 0);
          for (long t = 0; t < ne3; ++t) acc[t] += 0.5 * mJ[i][t] * dF[t];
        }
      }
      for (int f = 0; f < 6; ++f) {
        if (m.bdry[f + 6 * e] != 0) continue;
        long en = m.nbr[f + 6 * e]; if (en < 0) continue;
        int fn = m.nbrf[f + 6 * e], al = faxis(f);
        int r = frow(f, N), rn = frow(fn, N); double nh = fsign(f);
        for (int q = 0; q < N; ++q)
          for (int p = 0; p < N; ++p) {
            int i, j, k, a, b, c;
            face_ijk(al, r, p, q, i, j, k);
            nbr_face_ijk(m, e, f, p, q, a, b, c);
            long t = nid(N, i, j, k, 0), nb = nid(N, a, b, c, en);
            double s = 0.0;
            for (int ii = 0; ii < 3; ++ii)
              s += m.Ja[(al * 3 + ii) * nn + ne3 * e + t] * (F[ii][nb] - Fe[ii * ne3 + t]);
            acc[t] += nh * s / (2.0 * H[r]);
          }
      }
      for (long t = 0; t < ne3; ++t) out[ne3 * e + t] = acc[t] * m.invdetJ[ne3 * e + t];
    }
  }
}

// ---------------------------------------------------------------------------
// Background sampling (src/wave3d_curved.jl:75-96): per node
// (alpha, beta^i, gamma_ij) -> coef = (alpha, sqrt(det gamma), b1, b2, b3,
// gu11, gu12, gu13, gu22, gu23, gu33) with the symmetric cofactor inverse.
// Analytic backgrounds:
//   kind 0  Minkowski: alpha = 1, beta = 0, gamma = I
//   kind 1  constant shift (p[0..2] = beta)
//   kind 2  perturbed ADM background of the warped-cube workloads:
//           alpha = 1 + p0 sin(2 pi x), beta^i = p1 cos(2 pi x_i),
//           gamma_ij = d_ij + p2 exp(-|x-c|^2/p3) (d_ij + 0.5 s_ij),
//           c = (p4,p5,p6), s = (p7..p12) = (s11,s12,s13,s22,s23,s33)
//   kind 3  radial shift (src/evolve.jl:1128-1145): alpha = 1, gamma = I,
//           beta = beta_r(r) x/r with beta_r linear from p0 at r=p2 to p1 at r=p3.
// adm_decompose of a 4-metric g (lower indices, g[mu][nu], mu = 0 time):
// gamma_ij = g_ij, beta_i = g_0i, beta^i = gamma^ij beta_j,
// alpha = sqrt(beta_i beta^i - g_00) (the standard 3+1 split; SpacetimeMetrics'
// adm_decompose, called at src/wave3d_curved.jl:68, is unvendored).
void adm_from_metric(const double g[4][4], double out[10]) {
  const double g11 = g[1][1], g12 = g[1][2], g13 = g[1][3], g22 = g[2][2], g23 = g[2][3], g33 = g[3][3];
  const double det = g11 * (g22 * g33 - g23 * g23) - g12 * (g12 * g33 - g23 * g13) + g13 * (g12 * g23 - g22 * g13);
  const double u[3][3] = {{(g22 * g33 - g23 * g23) / det, (g13 * g23 - g12 * g33) / det, (g12 * g23 - g13 * g22) / det},
                          {(g13 * g23 - g12 * g33) / det, (g11 * g33 - g13 * g13) / det, (g12 * g13 - g11 * g23) / det},
                          {(g12 * g23 - g13 * g22) / det, (g12 * g13 - g11 * g23) / det, (g11 * g22 - g12 * g12) / det}};
  const double bl[3] = {g[0][1], g[0][2], g[0][3]};
  double bu[3], bb = 0.0;
  for (int i = 0; i < 3; ++i) {
    bu[i] = u[i][0] * bl[0] + u[i][1] * bl[1] + u[i][2] * bl[2];
    bb += bl[i] * bu[i];
  }
  out[0] = std::sqrt(bb - g[0][0]);
  out[1] = bu[0]; out[2] = bu[1]; out[3] = bu[2];
  out[4] = g11; out[5] = g12; out[6] = g13; out[7] = g22; out[8] = g23; out[9] = g33;
}

// The spacetime metrics of the time-dependent backgrounds at (t, x) (flat in y, z):
//   gauge wave  ds^2 = -H dt^2 + H dx^2 + dy^2 + dz^2, H = 1 - A sin(2 pi (x - t)/d)
//   sine shift  the metric whose 3+1 split is alpha = 1, beta^x = -A c/(1 + A c),
//               gamma_xx = (1 + A c)^2, c = cos(2 pi (x - t)/d)  (src/evolve.jl:171-195)
void spacetime_metric(int kind, double A, double d, double t, double x, double g[4][4]) {
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) g[a][b] = a == b ? (a == 0 ? -1.0 : 1.0) : 0.0;
  const double ph = 2.0 * M_PI * (x - t) / d;
  if (kind == 4) {
    const double H = 1.0 - A * std::sin(ph);
    g[0][0] = -H; g[1][1] = H;
  } else if (kind == 5) {
    const double ac = A * std::cos(ph), gxx = (1.0 + ac) * (1.0 + ac), bx = -ac / (1.0 + ac);
    g[1][1] = gxx;
    g[0][1] = g[1][0] = gxx * bx;            // beta_x = gamma_xx beta^x
    g[0][0] = -1.0 + gxx * bx * bx;          // -alpha^2 + beta_i beta^i
  }
}

void bg_point(int kind, const double* p, double x, double y, double z, double out[10]) {
  double al = 1, b1 = 0, b2 = 0, b3 = 0, g11 = 1, g12 = 0, g13 = 0, g22 = 1, g23 = 0, g33 = 1;
  if (kind == 4 || kind == 5) {  // MetricBackground3D at time p[2]: A = p[0], d = p[1]
    double g[4][4];
    spacetime_metric(kind, p[0], p[1], p[2], x, g);
    adm_from_metric(g, out);
    return;
  }
  if (kind == 1) { b1 = p[0]; b2 = p[1]; b3 = p[2]; }
  else if (kind == 2) {
    const double tp = 2.0 * M_PI;
    al = 1.0 + p[0] * std::sin(tp * x);
    b1 = p[1] * std::cos(tp * x); b2 = p[1] * std::cos(tp * y); b3 = p[1] * std::cos(tp * z);
    double dx = x - p[4], dy = y - p[5], dz = z - p[6];
    double g = p[2] * std::exp(-(dx * dx + dy * dy + dz * dz) / p[3]);
    g11 = 1.0 + g * (1.0 + 0.5 * p[7]);
    g12 = g * (0.5 * p[8]);
    g13 = g * (0.5 * p[9]);
    g22 = 1.0 + g * (1.0 + 0.5 * p[10]);
    g23 = g * (0.5 * p[11]);
    g33 = 1.0 + g * (1.0 + 0.5 * p[12]);
  } else if (kind == 3) {
    double r = std::sqrt(x * x + y * y + z * z);
    double br = p[0] + (p[1] - p[0]) * (r - p[2]) / (p[3] - p[2]);
    if (r > 0) { b1 = br * x / r; b2 = br * y / r; b3 = br * z / r; }
  }
  out[0] = al; out[1] = b1; out[2] = b2; out[3] = b3;
  out[4] = g11; out[5] = g12; out[6] = g13; out[7] = g22; out[8] = g23; out[9] = g33;
}

void sample_background(const Mesh& m, int kind, const double* p, double* coef) {
  const long nn = m.nn();
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nn; ++n) {
    double v[10];
    bg_point(kind, p, m.coords[3 * n], m.coords[3 * n + 1], m.coords[3 * n + 2], v);
    double g11 = v[4], g12 = v[5], g13 = v[6], g22 = v[7], g23 = v[8], g33 = v[9];
    double det = g11 * (g22 * g33 - g23 * g23) - g12 * (g12 * g33 - g23 * g13) + g13 * (g12 * g23 - g22 * g13);
    coef[0 * nn + n] = v[0];
    coef[1 * nn + n] = std::sqrt(det);
    coef[2 * nn + n] = v[1]; coef[3 * nn + n] = v[2]; coef[4 * nn + n] = v[3];
    coef[5 * nn + n] = (g22 * g33 - g23 * g23) / det;
    coef[6 * nn + n] = (g13 * g23 - g12 * g33) / det;
    coef[7 * nn + n] = (g12 * g23 - g13 * g22) / det;
    coef[8 * nn + n] = (g11 * g33 - g13 * g13) / det;
    coef[9 * nn + n] = (g12 * g13 - g11 * g23) / det;
    coef[10 * nn + n] = (g11 * g22 - g12 * g12) / det;
  }
}

// mu of make_wave3d_workspace (src/wave3d_curved.jl:158-178): 30 steps of
// power iteration v <- D_1^2 v / ||D_1^2 v|| from the alternating-sign start
// isodd(i+j+k+m) ? 1 : -1 (1-based indices), mu = sqrt(||D_1^2 v||).
void compute_mu(Mesh& m) {
  const int N = m.N; const long Ne = m.Ne, nn = m.nn();
  std::vector<double> v(nn), w(nn);
  for (long e = 0; e < Ne; ++e)
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
          v[nid(N, i, j, k, e)] = ((i + j + k + e + 4) & 1) ? 1.0 : -1.0;
  double mu2 = 0.0;
  for (int it = 0; it < 30; ++it) {
    apply_D(m, v.data(), w.data(), 0);
    apply_D(m, w.data(), v.data(), 0);
    double s = 0.0;
    for (long n = 0; n < nn; ++n) s += v[n] * v[n];
    mu2 = std::sqrt(s);
    if (!(mu2 > 0)) break;
    for (long n = 0; n < nn; ++n) v[n] /= mu2;
  }
  m.mu = std::sqrt(mu2);
  m.inv_mu5 = m.mu > 0 ? std::pow(1.0 / m.mu, 5) : 0.0;
}

// _ko_axis3! (src/wave3d_curved.jl:182-192): dst += koT * D_d^6 field.
void ko_axis(const Mesh& m, double* dst, const double* field, int d, double koT,
             std::vector<double>& s1, std::vector<double>& s2) {
  const long nn = m.nn();
  apply_D(m, field, s1.data(), d);
  apply_D(m, s1.data(), s2.data(), d);
  apply_D(m, s2.data(), s1.data(), d);
  apply_D(m, s1.data(), s2.data(), d);
  apply_D(m, s2.data(), s1.data(), d);
  apply_D(m, s1.data(), s2.data(), d);
  for (long n = 0; n < nn; ++n) dst[n] += koT * s2[n];
}

}  // namespace

// ===========================================================================
// extern "C" interface (loaded by tests/ and bench.py with ctypes).
extern "C" {

struct or_bc {
  int32_t kinds[6];        // BC_DIRICHLET=1, SOMMERFELD=2, EXCISION=3, FULL_DIRICHLET=4
  double sigma;
  int32_t excision_tag;
  const double* gPhi;      // NULL = nothing
  const double* gPi;
  const double* gDx;
  const double* gDy;
  const double* gDz;
};

void* or_mesh_create(int N, int Mx, int My, int Mz, double x0, double x1, double A,
                     int periodic, int outer_tag) {
  Mesh* m = new Mesh();
  build_mesh(*m, N, Mx, My, Mz, x0, x1, A, periodic, outer_tag);
  build_metric(*m);
  return m;
}
void* or_mesh_create_arrays(int N, long Ne, const double* coords, const double* jac, const int32_t* nbr,
                            const int32_t* nbrf, const int32_t* orient, const int32_t* bdry) {
  Mesh* m = new Mesh();
  build_mesh_arrays(*m, N, Ne, coords, jac, nbr, nbrf, orient, bdry);
  build_metric(*m);
  return m;
}
void or_mesh_destroy(void* h) { delete static_cast<Mesh*>(h); }
long or_mesh_ne(void* h) { return static_cast<Mesh*>(h)->Ne; }

void or_ops(int N, double* x, double* H, double* G) {
  Ops o = make_ops(N);
  std::memcpy(x, o.x.data(), N * sizeof(double));
  std::memcpy(H, o.H.data(), N * sizeof(double));
  std::memcpy(G, o.G.data(), N * N * sizeof(double));
}

// copy out a mesh array by name
int or_get(void* h, const char* name, void* out) {
  Mesh& m = *static_cast<Mesh*>(h);
  auto cpd = [&](const std::vector<double>& v) { std::memcpy(out, v.data(), v.size() * sizeof(double)); return 0; };
  auto cpi = [&](const std::vector<int32_t>& v) { std::memcpy(out, v.data(), v.size() * sizeof(int32_t)); return 0; };
  std::string s(name);
  if (s == "coords") return cpd(m.coords);
  if (s == "jac") return cpd(m.jac);
  if (s == "invjac") return cpd(m.invjac);
  if (s == "detjac") return cpd(m.detjac);
  if (s == "Hphys") return cpd(m.Hphys);
  if (s == "Ja") return cpd(m.Ja);
  if (s == "invdetJ") return cpd(m.invdetJ);
  if (s == "Hd") return cpd(m.Hd);
  if (s == "nbr") return cpi(m.nbr);
  if (s == "nbrf") return cpi(m.nbrf);
  if (s == "orient") return cpi(m.orient);
  if (s == "bdry") return cpi(m.bdry);
  if (s == "handed") return cpi(m.handed);
  return -1;
}

// overwrite a geometry array (tests use it to run the oracle on the device's
// geometry, separating input round-off from arithmetic differences)
int or_set(void* h, const char* name, const double* in) {
  Mesh& m = *static_cast<Mesh*>(h);
  auto cp = [&](std::vector<double>& v) { std::memcpy(v.data(), in, v.size() * sizeof(double)); return 0; };
  std::string s(name);
  if (s == "coords") return cp(m.coords);
  if (s == "jac") return cp(m.jac);
  if (s == "invjac") return cp(m.invjac);
  if (s == "detjac") return cp(m.detjac);
  if (s == "Hphys") return cp(m.Hphys);
  if (s == "Ja") return cp(m.Ja);
  if (s == "invdetJ") return cp(m.invdetJ);
  if (s == "Hd") return cp(m.Hd);
  return -1;
}

// overwrite bdry tags (tests use it to mark faces as excision etc.)
void or_set_bdry(void* h, const int32_t* bdry) {
  Mesh& m = *static_cast<Mesh*>(h);
  std::memcpy(m.bdry.data(), bdry, m.bdry.size() * sizeof(int32_t));
}

void or_sample_background(void* h, int kind, const double* p, double* coef) {
  sample_background(*static_cast<Mesh*>(h), kind, p, coef);
}

double or_mu(void* h) {
  Mesh& m = *static_cast<Mesh*>(h);
  if (m.mu < 0) compute_mu(m);
  return m.mu;
}

void or_apply_D(void* h, const double* u, double* out, int d) { apply_D(*static_cast<Mesh*>(h), u, out, d); }
void or_grad3d(void* h, const double* u, double* g1, double* g2, double* g3) {
  grad3d(*static_cast<Mesh*>(h), u, g1, g2, g3);
}
void or_div3d(void* h, const double* F1, const double* F2, const double* F3, double* out) {
  div3d(*static_cast<Mesh*>(h), F1, F2, F3, out);
}
void or_ko_add(void* h, double* dst, const double* field, double koT) {
  Mesh& m = *static_cast<Mesh*>(h);
  std::vector<double> s1(m.nn()), s2(m.nn());
  for (int d = 0; d < 3; ++d) ko_axis(m, dst, field, d, koT, s1, s2);
}

// wave3d_curved_rhs! (src/wave3d_curved.jl:205-258) including the affine
// boundary pass _apply_bc3d! (src/boundaries3d.jl:58-124) and the curvilinear
// pass _apply_bc3d_curv! (src/boundaries3d.jl:131-232).  coef is the 11-field
// bundle of sample_background3d!.  DPhi (3*nn, may be NULL) receives ws.DPhi.
void or_rhs_curved(void* h, const double* coef, const double* Phi, const double* Pi,
                   double* Phid, double* Pid, double eps_ko, const or_bc* bc, int use_metric,
                   double* DPhi_out) {
  Mesh& m = *static_cast<Mesh*>(h);
  const int N = m.N; const long nn = m.nn(), Ne = m.Ne;
  const double* alpha = coef + 0 * nn; const double* sg = coef + 1 * nn;
  const double* b1 = coef + 2 * nn; const double* b2 = coef + 3 * nn; const double* b3 = coef + 4 * nn;
  const double* gu11 = coef + 5 * nn; const double* gu12 = coef + 6 * nn; const double* gu13 = coef + 7 * nn;
  const double* gu22 = coef + 8 * nn; const double* gu23 = coef + 9 * nn; const double* gu33 = coef + 10 * nn;
  std::vector<double> D1(nn), D2(nn), D3(nn), F1(nn), F2(nn), F3(nn), s1(nn), s2(nn), s3(nn);
  if (!use_metric) {
    apply_D(m, Phi, D1.data(), 0); apply_D(m, Phi, D2.data(), 1); apply_D(m, Phi, D3.data(), 2);
  } else {
    grad3d(m, Phi, D1.data(), D2.data(), D3.data());
  }
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nn; ++n) {
    F1[n] = b1[n] * Pi[n] + alpha[n] * sg[n] * (gu11[n] * D1[n] + gu12[n] * D2[n] + gu13[n] * D3[n]);
    F2[n] = b2[n] * Pi[n] + alpha[n] * sg[n] * (gu12[n] * D1[n] + gu22[n] * D2[n] + gu23[n] * D3[n]);
    F3[n] = b3[n] * Pi[n] + alpha[n] * sg[n] * (gu13[n] * D1[n] + gu23[n] * D2[n] + gu33[n] * D3[n]);
  }
  if (!use_metric) {
    apply_D(m, F1.data(), s1.data(), 0); apply_D(m, F2.data(), s2.data(), 1); apply_D(m, F3.data(), s3.data(), 2);
    for (long n = 0; n < nn; ++n) Pid[n] = s1[n] + s2[n] + s3[n];
  } else {
    div3d(m, F1.data(), F2.data(), F3.data(), Pid);
  }
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nn; ++n)
    Phid[n] = b1[n] * D1[n] + b2[n] * D2[n] + b3[n] * D3[n] + (alpha[n] / sg[n]) * Pi[n];
  if (eps_ko != 0.0) {
    if (m.mu < 0) compute_mu(m);
    double koT = eps_ko * m.inv_mu5;
    for (int d = 0; d < 3; ++d) ko_axis(m, Phid, Phi, d, koT, s1, s2);
    for (int d = 0; d < 3; ++d) ko_axis(m, Pid, Pi, d, koT, s1, s2);
  }
  if (bc) {
    const double* H = m.ops.H.data();
    const double sigma = bc->sigma;
    if (!use_metric) {
#pragma omp parallel for schedule(static)
      for (long e = 0; e < Ne; ++e)
        for (int k = 0; k < N; ++k)
          for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
              long n = nid(N, i, j, k, e);
              double dF = 0.0, dP = 0.0;
              for (int f = 0; f < 6; ++f) {
                if (m.bdry[f + 6 * e] == 0) continue;
                int kind = bc->kinds[f];
                if (kind == 3) continue;
                int dn = f / 2, fn = (f & 1) ? N - 1 : 0;
                bool on = dn == 0 ? (i == fn) : dn == 1 ? (j == fn) : (k == fn);
                if (!on) continue;
                double nh = fsign(f);
                double a0 = alpha[n], sgv = sg[n];
                double gunn = dn == 0 ? gu11[n] : dn == 1 ? gu22[n] : gu33[n];
                double bax = dn == 0 ? b1[n] : dn == 1 ? b2[n] : b3[n];
                double ij = m.invjac[dn + 3 * dn + 9 * n];
                double a = a0 / sgv, a_n = a0 * std::sqrt(gunn), bn = nh * bax, wt = ij / H[fn];
                if (kind == 4) {
                  double tau = sigma * (std::fabs(a_n - bax) + std::fabs(a_n + bax)) * wt;
                  double gp = bc->gPhi ? bc->gPhi[n] : 0.0, gq = bc->gPi ? bc->gPi[n] : 0.0;
                  dF += -tau * (Phi[n] - gp);
                  dP += -tau * (Pi[n] - gq);
                } else {
                  double Dn = dn == 0 ? D1[n] : dn == 1 ? D2[n] : D3[n];
                  double qv = nh * Dn;
                  double r = Pi[n] + ((bn + a_n) / a) * qv;
                  double g = kind == 2 ? 0.0 : (bc->gPhi ? bc->gPhi[n] : 0.0);
                  double s_in = a_n + bn;
                  dP += -sigma * std::fabs(s_in) * wt * (r - g);
                }
              }
              Phid[n] += dF; Pid[n] += dP;
            }
    } else {
      int kind = bc->kinds[0];
      int exc = bc->excision_tag;
      if (!(kind == 3 && exc == 0)) {
#pragma omp parallel for schedule(static)
        for (long e = 0; e < Ne; ++e)
          for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
              for (int i = 0; i < N; ++i) {
                long n = nid(N, i, j, k, e);
                double dF = 0.0, dP = 0.0;
                for (int f = 0; f < 6; ++f) {
                  int tag = m.bdry[f + 6 * e];
                  if (tag == 0 || tag == exc) continue;
                  int ai = f / 2, row = (f & 1) ? N - 1 : 0;
                  bool on = ai == 0 ? (i == row) : ai == 1 ? (j == row) : (k == row);
                  if (!on) continue;
                  int ap = ai == 0 ? 1 : 0, aq = ai == 2 ? 1 : 2;
                  double sgn_f = fsign(f), sgn_c = ai == 1 ? -1.0 : 1.0;
                  double so = sgn_f * sgn_c * (double)m.handed[e];
                  const double* J = &m.jac[9 * n];
                  double tpx = J[0 + 3 * ap], tpy = J[1 + 3 * ap], tpz = J[2 + 3 * ap];
                  double tqx = J[0 + 3 * aq], tqy = J[1 + 3 * aq], tqz = J[2 + 3 * aq];
                  double nfx = so * (tpy * tqz - tpz * tqy);
                  double nfy = so * (tpz * tqx - tpx * tqz);
                  double nfz = so * (tpx * tqy - tpy * tqx);
                  double JF = std::sqrt(nfx * nfx + nfy * nfy + nfz * nfz);
                  double nx = nfx / JF, ny = nfy / JF, nz = nfz / JF;
                  double av = alpha[n], sgv = sg[n];
                  double a = av / sgv;
                  double a_n = av * std::sqrt(gu11[n] * nx * nx + gu22[n] * ny * ny + gu33[n] * nz * nz +
                                              2 * gu12[n] * nx * ny + 2 * gu13[n] * nx * nz + 2 * gu23[n] * ny * nz);
                  double bn = b1[n] * nx + b2[n] * ny + b3[n] * nz;
                  double wt = JF / (H[row] * m.detjac[n]);
                  if (kind == 4) {
                    double tau = sigma * (std::fabs(a_n - bn) + std::fabs(a_n + bn)) * wt;
                    double gp = bc->gPhi ? bc->gPhi[n] : 0.0, gq = bc->gPi ? bc->gPi[n] : 0.0;
                    dF += -tau * (Phi[n] - gp);
                    dP += -tau * (Pi[n] - gq);
                  } else {
                    double qv = nx * D1[n] + ny * D2[n] + nz * D3[n];
                    double r = Pi[n] + ((bn + a_n) / a) * qv;
                    double g = 0.0;
                    if (kind != 2) {
                      double gq = bc->gPi ? bc->gPi[n] : 0.0;
                      double gx = bc->gDx ? bc->gDx[n] : 0.0, gy = bc->gDy ? bc->gDy[n] : 0.0,
                             gz = bc->gDz ? bc->gDz[n] : 0.0;
                      g = gq + ((bn + a_n) / a) * (nx * gx + ny * gy + nz * gz);
                    }
                    double s_in = a_n + bn;
                    dP += -sigma * std::fabs(s_in) * wt * (r - g);
                  }
                }
                Phid[n] += dF; Pid[n] += dP;
              }
      }
    }
  }
  if (DPhi_out) {
    std::memcpy(DPhi_out, D1.data(), nn * sizeof(double));
    std::memcpy(DPhi_out + nn, D2.data(), nn * sizeof(double));
    std::memcpy(DPhi_out + 2 * nn, D3.data(), nn * sizeof(double));
  }
}

// wave3d_energy (src/wave3d_curved.jl:268-287):
// E = sum 1/2 [Pi^2/sqrtg + sqrtg gu^{ij} dPhi_i dPhi_j] H.
// lapse = 1: the same integrand times alpha (coef field 0),
// E_alpha = sum 1/2 [(alpha/sqrtg) Pi^2 + alpha sqrtg gu^{ij} dPhi_i dPhi_j] H -- the
// norm the first-order system conserves for a static background with zero
// shift (the reference's wave3d_energy is exactly conserved only for alpha = 1,
// src/wave3d_curved.jl:263-266).
double or_energy_w(void* h, const double* coef, const double* Phi, const double* Pi, int use_metric, int lapse) {
  Mesh& m = *static_cast<Mesh*>(h);
  const long nn = m.nn();
  std::vector<double> D1(nn), D2(nn), D3(nn);
  if (!use_metric) { apply_D(m, Phi, D1.data(), 0); apply_D(m, Phi, D2.data(), 1); apply_D(m, Phi, D3.data(), 2); }
  else grad3d(m, Phi, D1.data(), D2.data(), D3.data());
  const double* H = use_metric ? m.Hd.data() : m.Hphys.data();
  const double* sg = coef + 1 * nn;
  const double *g11 = coef + 5 * nn, *g12 = coef + 6 * nn, *g13 = coef + 7 * nn, *g22 = coef + 8 * nn,
               *g23 = coef + 9 * nn, *g33 = coef + 10 * nn;
  double E = 0.0;
  for (long n = 0; n < nn; ++n) {
    double d1 = D1[n], d2 = D2[n], d3 = D3[n];
    const double w = lapse ? coef[n] : 1.0;
    E += w * (Pi[n] * Pi[n] / sg[n] +
              sg[n] * (g11[n] * d1 * d1 + g22[n] * d2 * d2 + g33[n] * d3 * d3 + 2 * g12[n] * d1 * d2 +
                       2 * g13[n] * d1 * d3 + 2 * g23[n] * d2 * d3)) * H[n] / 2;
  }
  return E;
}
double or_energy(void* h, const double* coef, const double* Phi, const double* Pi, int use_metric) {
  return or_energy_w(h, coef, Phi, Pi, use_metric, 0);
}

// ---------------------------------------------------------------------------
// SIPG second-order RHS (rhs_wave3d!, src/wave.jl:573-611) on axis-aligned
// affine meshes.  apply_laplacian! (HexSBPSAT) restated from its documented
// formula (README.md:57-80), per axis d and element with s = 1/h_d:
//   u_tt = sum_d s^2 G_d G_d u
//        + H^-1 [ alpha G^T B du - 1/2 B dGu - tau |B| du ]   (per d-face)
// du = u - u_nbr (interior, alpha = 1/2), du = u - g_tag with dGu = 0 (outer
// Dirichlet faces tag 1..6, alpha = 1, mirror convention); tag-7 (Sommerfeld)
// and tag-8 faces are free.  Then the Sommerfeld pass (src/wave.jl:453-542):
// at tag-7 face nodes u_tt -= wF (u_t + d_n u + u/R)/Hphys, wF = JF H_p H_q.
void or_rhs_sipg(void* h, const double* u, const double* ut, double* utt, const double* bdry_values,
                 double tau, double inv_R) {
  Mesh& m = *static_cast<Mesh*>(h);
  const int N = m.N; const long Ne = m.Ne; const long ne3 = (long)N * N * N;
  const double* G = m.ops.G.data(); const double* H = m.ops.H.data();
  // per-element physical derivatives along each axis (needed for neighbour traces)
  const long nn = m.nn();
  std::vector<double> Du(3 * nn);
#pragma omp parallel
  {
    Mesh loc; loc.N = N; loc.ops = m.ops; loc.Ne = 1;
#pragma omp for schedule(static)
    for (long e = 0; e < Ne; ++e)
      for (int d = 0; d < 3; ++d) {
        ref_deriv(loc, u + ne3 * e, &Du[d * nn + ne3 * e], d, 0);
        for (long t = 0; t < ne3; ++t) Du[d * nn + ne3 * e + t] *= m.invjac[d + 3 * d + 9 * (ne3 * e + t)];
      }
  }
#pragma omp parallel
  {
    Mesh loc; loc.N = N; loc.ops = m.ops; loc.Ne = 1;
    std::vector<double> tmp(ne3), acc(ne3);
#pragma omp for schedule(static)
    for (long e = 0; e < Ne; ++e) {
      std::fill(acc.begin(), acc.end(), 0.0);
      for (int d = 0; d < 3; ++d) {
        // second sweep on the (physical) first derivative: s * G_d (Du_d)
        ref_deriv(loc, &Du[d * nn + ne3 * e], tmp.data(), d, 0);
        for (long t = 0; t < ne3; ++t) acc[t] += m.invjac[d + 3 * d + 9 * (ne3 * e + t)] * tmp[t];
      }
      for (int f = 0; f < 6; ++f) {
        int tag = m.bdry[f + 6 * e];
        if (tag == 7 || tag == 8) continue;
        long en = m.nbr[f + 6 * e];
        if (tag == 0 && en < 0) continue;
        int d = faxis(f), r = frow(f, N); double nh = fsign(f);
        double al = tag == 0 ? 0.5 : 1.0;
        int fn = m.nbrf[f + 6 * e], rn = frow(fn, N);
        for (int q = 0; q < N; ++q)
          for (int p = 0; p < N; ++p) {
            int i, j, k; face_ijk(d, r, p, q, i, j, k);
            long t = nid(N, i, j, k, 0), n = t + ne3 * e;
            double s = m.invjac[d + 3 * d + 9 * n];
            double du, dGu;
            if (tag == 0) {
              int a, b, c; nbr_face_ijk(m, e, f, p, q, a, b, c);
              long nb = nid(N, a, b, c, en);
              du = u[n] - u[nb];
              dGu = Du[d * nn + n] - Du[d * nn + nb];
            } else {
              du = u[n] - bdry_values[tag - 1];
              dGu = 0.0;
            }
            acc[t] += -tau * s * s / H[r] * du;
            acc[t] += -0.5 * nh * s / H[r] * dGu;
            for (int l = 0; l < N; ++l) {
              int ii = d == 0 ? l : i, jj = d == 1 ? l : j, kk = d == 2 ? l : k;
              long tl = nid(N, ii, jj, kk, 0);
              acc[tl] += al * nh * s * s * G[r * N + l] / H[l] * du;
            }
          }
      }
      // Sommerfeld pass
      for (int f = 0; f < 6; ++f) {
        if (m.nbr[f + 6 * e] >= 0 || m.bdry[f + 6 * e] != 7) continue;
        int ai = faxis(f), row = frow(f, N);
        int ap = ai == 0 ? 1 : 0, aq = ai == 2 ? 1 : 2;
        double sgn_f = fsign(f), sgn_c = ai == 1 ? -1.0 : 1.0;
        for (int q = 0; q < N; ++q)
          for (int p = 0; p < N; ++p) {
            int i, j, k; face_ijk(ai, row, p, q, i, j, k);
            long t = nid(N, i, j, k, 0), n = t + ne3 * e;
            const double* J = &m.jac[9 * n];
            double so = sgn_f * sgn_c * (double)m.handed[e];
            double tpx = J[0 + 3 * ap], tpy = J[1 + 3 * ap], tpz = J[2 + 3 * ap];
            double tqx = J[0 + 3 * aq], tqy = J[1 + 3 * aq], tqz = J[2 + 3 * aq];
            double nx_ = so * (tpy * tqz - tpz * tqy), ny_ = so * (tpz * tqx - tpx * tqz), nz_ = so * (tpx * tqy - tpy * tqx);
            double JF = std::sqrt(nx_ * nx_ + ny_ * ny_ + nz_ * nz_);
            double nx = nx_ / JF, ny = ny_ / JF, nz = nz_ / JF;
            double wF = JF * H[p] * H[q];
            // physical gradient: d_{x_a} u = sum_al invjac[al,a] Dhat_al u
            double dref[3];
            for (int al = 0; al < 3; ++al) dref[al] = Du[al * nn + n] / m.invjac[al + 3 * al + 9 * n];
            double g[3];
            for (int a = 0; a < 3; ++a) {
              g[a] = 0.0;
              for (int al = 0; al < 3; ++al) g[a] += m.invjac[al + 3 * a + 9 * n] * dref[al];
            }
            double Gn = nx * g[0] + ny * g[1] + nz * g[2];
            acc[t] -= wF * (ut[n] + Gn + inv_R * u[n]) / m.Hphys[n];
          }
      }
      std::copy(acc.begin(), acc.end(), utt + ne3 * e);
    }
  }
}

// ---------------------------------------------------------------------------
// Strong-form curvilinear RHS (wave_strong_rhs_element!/_mesh!,
// src/wave_strong_rhs.jl:95-341, make_metric_derivs :376-391), restated
// line by line.  Orientation 0 only (uniform / warped meshes).
void or_rhs_strong(void* h, const double* u, const double* ut, double* utt, double tau, double inv_R) {
  Mesh& m = *static_cast<Mesh*>(h);
  const int N = m.N; const long Ne = m.Ne; const long ne3 = (long)N * N * N;
  const double* H = m.ops.H.data();
  if (m.dinvjac.empty()) {
    m.dinvjac.assign(27 * m.nn(), 0.0);
#pragma omp parallel
    {
      Mesh loc; loc.N = N; loc.ops = m.ops; loc.Ne = 1;
      std::vector<double> src(ne3), dst(ne3);
#pragma omp for schedule(static)
      for (long e = 0; e < Ne; ++e)
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) {
            for (long t = 0; t < ne3; ++t) src[t] = m.invjac[a + 3 * c + 9 * (ne3 * e + t)];
            for (int d = 0; d < 3; ++d) {
              ref_deriv(loc, src.data(), dst.data(), d, 0);
              for (long t = 0; t < ne3; ++t) m.dinvjac[a + 3 * c + 9 * d + 27 * (ne3 * e + t)] = dst[t];
            }
          }
    }
  }
#pragma omp parallel
  {
    Mesh loc; loc.N = N; loc.ops = m.ops; loc.Ne = 1;
    std::vector<double> ue(ne3), du(3 * ne3), ddu(9 * ne3), dphys(3 * ne3), out(ne3), uface(6 * N * N);
#pragma omp for schedule(static)
    for (long e = 0; e < Ne; ++e) {
      std::copy(u + ne3 * e, u + ne3 * (e + 1), ue.begin());
      for (int f = 0; f < 6; ++f) {
        long en = m.nbr[f + 6 * e];
        int fn = m.nbrf[f + 6 * e], rn = frow(fn, N);
        for (int q = 0; q < N; ++q)
          for (int p = 0; p < N; ++p) {
            double v = 0.0;
            if (en >= 0) { int a, b, c; nbr_face_ijk(m, e, f, p, q, a, b, c); v = u[nid(N, a, b, c, en)]; }
            uface[f * N * N + p + N * q] = v;
          }
      }
      for (int c = 0; c < 3; ++c) ref_deriv(loc, ue.data(), &du[c * ne3], c, 0);
      // ddu[(c*3+d)] = Dhat_d Dhat_c u for c <= d
      for (int c = 0; c < 3; ++c)
        for (int d = c; d < 3; ++d) ref_deriv(loc, &du[c * ne3], &ddu[(c * 3 + d) * ne3], d, 0);
      for (long t = 0; t < ne3; ++t) {
        const double* ij = &m.invjac[9 * (ne3 * e + t)];
        for (int a = 0; a < 3; ++a) {
          double s = 0.0;
          for (int al = 0; al < 3; ++al) s += ij[al + 3 * a] * du[al * ne3 + t];
          dphys[a * ne3 + t] = s;
        }
      }
      for (long t = 0; t < ne3; ++t) {
        const double* ij = &m.invjac[9 * (ne3 * e + t)];
        const double* dij = &m.dinvjac[27 * (ne3 * e + t)];
        double s = 0.0;
        for (int al = 0; al < 3; ++al) {
          double Gaa = 0.0;
          for (int ii = 0; ii < 3; ++ii) Gaa += ij[al + 3 * ii] * ij[al + 3 * ii];
          s += Gaa * ddu[(al * 3 + al) * ne3 + t];
          for (int be = al + 1; be < 3; ++be) {
            double Gab = 0.0;
            for (int ii = 0; ii < 3; ++ii) Gab += ij[al + 3 * ii] * ij[be + 3 * ii];
            s += 2.0 * Gab * ddu[(al * 3 + be) * ne3 + t];
          }
        }
        for (int be = 0; be < 3; ++be) {
          double Wb = 0.0;
          for (int al = 0; al < 3; ++al)
            for (int ii = 0; ii < 3; ++ii) Wb += ij[al + 3 * ii] * dij[be + 3 * ii + 9 * al];
          s += Wb * du[be * ne3 + t];
        }
        out[t] = s;
      }
      for (int f = 0; f < 6; ++f) {
        int al = f / 2; double fs = fsign(f); int fr = frow(f, N);
        int tag = m.bdry[f + 6 * e];
        if (tag == 8) continue;
        bool somm = tag == 7, dir = tag >= 1 && tag <= 6;
        bool intdir = tag == 0 || dir;
        for (int q = 0; q < N; ++q)
          for (int p = 0; p < N; ++p) {
            int i, j, k; face_ijk(al, fr, p, q, i, j, k);
            long t = nid(N, i, j, k, 0), n = t + ne3 * e;
            const double* ij = &m.invjac[9 * n];
            double nux = ij[al + 0], nuy = ij[al + 3], nuz = ij[al + 6];
            double nn_ = std::sqrt(nux * nux + nuy * nuy + nuz * nuz);
            double nx = fs * nux / nn_, ny = fs * nuy / nn_, nz = fs * nuz / nn_;
            double dnu = nx * dphys[t] + ny * dphys[ne3 + t] + nz * dphys[2 * ne3 + t];
            double Hp = m.Hphys[n];
            if (intdir) {
              double w = nn_ / H[fr];
              out[t] += -w * dnu;
              out[t] += -tau * w * (ue[t] - uface[f * N * N + p + N * q]);
            } else if (somm) {
              double wF = nn_ * m.detjac[n] * H[p] * H[q];
              out[t] -= wF * (ut[n] + dnu + inv_R * ue[t]) / Hp;
            }
          }
      }
      std::copy(out.begin(), out.end(), utt + ne3 * e);
    }
  }
}

// Strong-form Cartesian conservative Laplacian (wave_lap_strong_conservative_
// element!/_mesh!, src/wave_lap_strong.jl:183-308), uniform h, orientation 0.
void or_lap_strong_cons(void* h, const double* u, double* Lu, double hel, double tau) {
  Mesh& m = *static_cast<Mesh*>(h);
  const int N = m.N; const long Ne = m.Ne; const long ne3 = (long)N * N * N;
  const double* G = m.ops.G.data(); const double* H = m.ops.H.data();
  const double inv_h = 1.0 / hel;
#pragma omp parallel
  {
    Mesh loc; loc.N = N; loc.ops = m.ops; loc.Ne = 1;
    std::vector<double> ue(ne3), du(3 * ne3), out(ne3);
#pragma omp for schedule(static)
    for (long e = 0; e < Ne; ++e) {
      std::copy(u + ne3 * e, u + ne3 * (e + 1), ue.begin());
      for (int c = 0; c < 3; ++c) {
        ref_deriv(loc, ue.data(), &du[c * ne3], c, 0);
        for (long t = 0; t < ne3; ++t) du[c * ne3 + t] *= inv_h;
      }
      for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
          for (int i = 0; i < N; ++i) {
            double s = 0.0;
            for (int p = 0; p < N; ++p) s += G[i * N + p] * du[0 * ne3 + nid(N, p, j, k, 0)];
            for (int p = 0; p < N; ++p) s += G[j * N + p] * du[1 * ne3 + nid(N, i, p, k, 0)];
            for (int p = 0; p < N; ++p) s += G[k * N + p] * du[2 * ne3 + nid(N, i, j, p, 0)];
            out[nid(N, i, j, k, 0)] = s * inv_h;
          }
      for (int f = 0; f < 6; ++f) {
        int al = f / 2; double fs = fsign(f); int fr = frow(f, N);
        double coef_neu = -fs * inv_h / H[fr];
        double coef_dir = -tau * inv_h / H[fr];
        long en = m.nbr[f + 6 * e]; int fn = m.nbrf[f + 6 * e], rn = frow(fn, N);
        for (int q = 0; q < N; ++q)
          for (int p = 0; p < N; ++p) {
            int i, j, k; face_ijk(al, fr, p, q, i, j, k);
            long t = nid(N, i, j, k, 0);
            double uf = 0.0;
            if (en >= 0) { int a, b, c; nbr_face_ijk(m, e, f, p, q, a, b, c); uf = u[nid(N, a, b, c, en)]; }
            out[t] += coef_neu * du[al * ne3 + t];
            out[t] += coef_dir * (ue[t] - uf);
          }
      }
      std::copy(out.begin(), out.end(), Lu + ne3 * e);
    }
  }
}

// ---------------------------------------------------------------------------
// Scalar wave on a prescribed 4-metric, fully second order (wave_curved_rhs_*,
// src/wave_curved_rhs.jl:45-362): per element, the SBP gradients of phi and
// phidot (centred-flux SAT on the perpendicular component of each face, or no
// SAT in the conservative variant), the six Hessian components as a second G
// sweep of the (SAT-corrected) gradient, the pointwise solve
//   phidd = (Gam.dphi - 2 g^{ti} d_i phidot - g^{ij} d_ij phi) / g^{tt}
// and, conservative variant, the Mattsson-Nordstrom SAT pair per face
// (src/wave_curved_rhs.jl:332-345).  ginv is (10,N,N,N,Ne) (tt,tx,ty,tz,xx,xy,
// xz,yy,yz,zz), gam is (4,N,N,N,Ne); faces without a neighbour get zero traces
// (src/wave_curved_rhs.jl:168-184).  Uniform Cartesian elements of edge hel.
void or_rhs_curved4(void* h, const double* phi, const double* phid, double* phidd, const double* ginv,
                    const double* gam, double hel, int conservative, double tau) {
  Mesh& m = *static_cast<Mesh*>(h);
  const int N = m.N; const long Ne = m.Ne; const long ne3 = (long)N * N * N;
  const double* H = m.ops.H.data();
  const double inv_h = 1.0 / hel;
#pragma omp parallel
  {
    Mesh loc; loc.N = N; loc.ops = m.ops; loc.Ne = 1;
    std::vector<double> ue(ne3), ve(ne3), du(3 * ne3), dv(3 * ne3), dd(6 * ne3), out(ne3);
    std::vector<double> uf(6 * N * N), vf(6 * N * N);
#pragma omp for schedule(static)
    for (long e = 0; e < Ne; ++e) {
      std::copy(phi + ne3 * e, phi + ne3 * (e + 1), ue.begin());
      std::copy(phid + ne3 * e, phid + ne3 * (e + 1), ve.begin());
      for (int f = 0; f < 6; ++f) {  // neighbour face traces (zero without a neighbour)
        long en = m.nbr[f + 6 * e]; int fn = m.nbrf[f + 6 * e], rn = frow(fn, N);
        for (int q = 0; q < N; ++q)
          for (int p = 0; p < N; ++p) {
            double a_ = 0.0, b_ = 0.0;
            if (en >= 0) {
              int a, b, c; nbr_face_ijk(m, e, f, p, q, a, b, c);
              a_ = phi[nid(N, a, b, c, en)]; b_ = phid[nid(N, a, b, c, en)];
            }
            uf[f * N * N + p + N * q] = a_; vf[f * N * N + p + N * q] = b_;
          }
      }
      for (int c = 0; c < 3; ++c) {
        ref_deriv(loc, ue.data(), &du[c * ne3], c, 0);
        ref_deriv(loc, ve.data(), &dv[c * ne3], c, 0);
        for (long t = 0; t < ne3; ++t) { du[c * ne3 + t] *= inv_h; dv[c * ne3 + t] *= inv_h; }
      }
      if (!conservative) {
        for (int f = 0; f < 6; ++f) {
          int al = f / 2, fr = frow(f, N);
          double coef = fsign(f) * 0.5 * (1.0 / H[fr]) * inv_h;
          for (int q = 0; q < N; ++q)
            for (int p = 0; p < N; ++p) {
              int i, j, k; face_ijk(al, fr, p, q, i, j, k);
              long t = nid(N, i, j, k, 0);
              du[al * ne3 + t] += coef * (uf[f * N * N + p + N * q] - ue[t]);
              dv[al * ne3 + t] += coef * (vf[f * N * N + p + N * q] - ve[t]);
            }
        }
      }
      // Hessian: xx, xy, xz from d_x phi; yy, yz from d_y phi; zz from d_z phi
      const int src[6] = {0, 0, 0, 1, 1, 2}, axis[6] = {0, 1, 2, 1, 2, 2};
      for (int c = 0; c < 6; ++c) {
        ref_deriv(loc, &du[src[c] * ne3], &dd[c * ne3], axis[c], 0);
        for (long t = 0; t < ne3; ++t) dd[c * ne3 + t] *= inv_h;
      }
      for (long t = 0; t < ne3; ++t) {
        const double* g = ginv + 10 * (t + ne3 * e);
        const double* G4 = gam + 4 * (t + ne3 * e);
        double gdd = G4[0] * ve[t] + G4[1] * du[t] + G4[2] * du[ne3 + t] + G4[3] * du[2 * ne3 + t];
        double gti = g[1] * dv[t] + g[2] * dv[ne3 + t] + g[3] * dv[2 * ne3 + t];
        double gij = g[4] * dd[t] + g[7] * dd[3 * ne3 + t] + g[9] * dd[5 * ne3 + t] + 2 * g[5] * dd[ne3 + t] +
                     2 * g[6] * dd[2 * ne3 + t] + 2 * g[8] * dd[4 * ne3 + t];
        out[t] = (gdd - 2 * gti - gij) / g[0];
      }
      if (conservative) {
        for (int f = 0; f < 6; ++f) {
          int al = f / 2, fr = frow(f, N);
          double coef_neu = -fsign(f) * inv_h * (1.0 / H[fr]);
          double coef_dir = -(tau * inv_h) * (1.0 / H[fr]);
          for (int q = 0; q < N; ++q)
            for (int p = 0; p < N; ++p) {
              int i, j, k; face_ijk(al, fr, p, q, i, j, k);
              long t = nid(N, i, j, k, 0);
              out[t] += coef_neu * du[al * ne3 + t];
              out[t] += coef_dir * (ue[t] - uf[f * N * N + p + N * q]);
            }
        }
      }
      std::copy(out.begin(), out.end(), phidd + ne3 * e);
    }
  }
}

// Prescribed 4-metrics at the mesh nodes (eval_curved_background!,
// src/wave_curved_rhs.jl:373-418): kind 0 Minkowski; kind 1 the gauge wave of
// the Apples-with-Apples tests (Alcubierre et al. 2004), ds^2 = (1 - H)(-dt^2 +
// dx^2) + dy^2 + dz^2, H = A sin(2 pi (x - t)/d), p = (A, d).  Its inverse is
// diag(-1/(1-H), 1/(1-H), 1, 1), and the contracted Christoffels
// g^{ab} Gam^c_ab = -(1/sqrt(-g)) d_a(sqrt(-g) g^{ac}) vanish (sqrt(-g) g^{tt}
// = -1, sqrt(-g) g^{xx} = 1 are constant: the metric is in harmonic gauge).
void or_curved4_background(void* h, int kind, const double* p, double t, double* ginv, double* gam) {
  Mesh& m = *static_cast<Mesh*>(h);
  const long nn = m.nn();
  for (long n = 0; n < nn; ++n) {
    double* g = ginv + 10 * n;
    for (int c = 0; c < 10; ++c) g[c] = 0.0;
    for (int c = 0; c < 4; ++c) gam[4 * n + c] = 0.0;
    double f = 1.0;
    if (kind == 1) f = 1.0 - p[0] * std::sin(2.0 * M_PI * (m.coords[3 * n] - t) / p[1]);
    g[0] = -1.0 / f;
    g[4] = 1.0 / f;
    g[7] = 1.0;
    g[9] = 1.0;
  }
}

// ---------------------------------------------------------------------------
// Classic RK4 (the reference's _rk4_3d!, test/wave3d_tests.jl:32-44; also
// OrdinaryDiffEq RK4() with a fixed step): k1..k4 and
// u += dt/6 (k1 + 2 k2 + 2 k3 + k4).  energy (nsteps+1, may be NULL) records
// wave3d_energy after every step (index 0 = initial).
void or_evolve_curved(void* h, const double* coef, double* Phi, double* Pi, double dt, int nsteps,
                      double eps_ko, const or_bc* bc, int use_metric, double* energy) {
  Mesh& m = *static_cast<Mesh*>(h);
  const long nn = m.nn();
  std::vector<double> k1(nn), k2(nn), k3(nn), k4(nn), k5(nn), k6(nn), k7(nn), k8(nn), Ps(nn), Qs(nn);
  if (energy) energy[0] = or_energy(h, coef, Phi, Pi, use_metric);
  for (int s = 0; s < nsteps; ++s) {
    or_rhs_curved(h, coef, Phi, Pi, k1.data(), k2.data(), eps_ko, bc, use_metric, nullptr);
    for (long n = 0; n < nn; ++n) { Ps[n] = Phi[n] + dt / 2 * k1[n]; Qs[n] = Pi[n] + dt / 2 * k2[n]; }
    or_rhs_curved(h, coef, Ps.data(), Qs.data(), k3.data(), k4.data(), eps_ko, bc, use_metric, nullptr);
    for (long n = 0; n < nn; ++n) { Ps[n] = Phi[n] + dt / 2 * k3[n]; Qs[n] = Pi[n] + dt / 2 * k4[n]; }
    or_rhs_curved(h, coef, Ps.data(), Qs.data(), k5.data(), k6.data(), eps_ko, bc, use_metric, nullptr);
    for (long n = 0; n < nn; ++n) { Ps[n] = Phi[n] + dt * k5[n]; Qs[n] = Pi[n] + dt * k6[n]; }
    or_rhs_curved(h, coef, Ps.data(), Qs.data(), k7.data(), k8.data(), eps_ko, bc, use_metric, nullptr);
    for (long n = 0; n < nn; ++n) {
      Phi[n] += dt / 6 * (k1[n] + 2 * k3[n] + 2 * k5[n] + k7[n]);
      Pi[n] += dt / 6 * (k2[n] + 2 * k4[n] + 2 * k6[n] + k8[n]);
    }
    if (energy) energy[s + 1] = or_energy(h, coef, Phi, Pi, use_metric);
  }
}

// RK4 with a time-dependent background re-sampled at every stage time, as
// evolve3d's rhs! closure calls sample_background3d!(coef, bg, t)
// (src/evolve.jl:1287-1307); p[2] is the start time t0.
void or_evolve_curved_td(void* h, int kind, const double* p0, double* Phi, double* Pi, double dt, int nsteps,
                         double eps_ko, const or_bc* bc, int use_metric) {
  Mesh& m = *static_cast<Mesh*>(h);
  const long nn = m.nn();
  std::vector<double> k1(nn), k2(nn), k3(nn), k4(nn), k5(nn), k6(nn), k7(nn), k8(nn), Ps(nn), Qs(nn), coef(11 * nn);
  double p[16];
  std::memcpy(p, p0, sizeof(p));
  const double t0 = p0[2];
  auto at = [&](double t) { p[2] = t; sample_background(m, kind, p, coef.data()); };
  for (int s = 0; s < nsteps; ++s) {
    const double t = t0 + s * dt;
    at(t);
    or_rhs_curved(h, coef.data(), Phi, Pi, k1.data(), k2.data(), eps_ko, bc, use_metric, nullptr);
    for (long n = 0; n < nn; ++n) { Ps[n] = Phi[n] + dt / 2 * k1[n]; Qs[n] = Pi[n] + dt / 2 * k2[n]; }
    at(t + dt / 2);
    or_rhs_curved(h, coef.data(), Ps.data(), Qs.data(), k3.data(), k4.data(), eps_ko, bc, use_metric, nullptr);
    for (long n = 0; n < nn; ++n) { Ps[n] = Phi[n] + dt / 2 * k3[n]; Qs[n] = Pi[n] + dt / 2 * k4[n]; }
    or_rhs_curved(h, coef.data(), Ps.data(), Qs.data(), k5.data(), k6.data(), eps_ko, bc, use_metric, nullptr);
    for (long n = 0; n < nn; ++n) { Ps[n] = Phi[n] + dt * k5[n]; Qs[n] = Pi[n] + dt * k6[n]; }
    at(t + dt);
    or_rhs_curved(h, coef.data(), Ps.data(), Qs.data(), k7.data(), k8.data(), eps_ko, bc, use_metric, nullptr);
    for (long n = 0; n < nn; ++n) {
      Phi[n] += dt / 6 * (k1[n] + 2 * k3[n] + 2 * k5[n] + k7[n]);
      Pi[n] += dt / 6 * (k2[n] + 2 * k4[n] + 2 * k6[n] + k8[n]);
    }
  }
}

// Fixed-step explicit RK with a Butcher tableau (pick_integrator_first_order,
// src/evolve.jl:43-48, run with adaptive = false): method 1 = Tsit5 (Ch. Tsitouras,
// Comput. Math. Appl. 62 (2011) 770-775; fifth-order weights), method 0 = classic
// RK4.  kind >= 0: the time-dependent background of that kind (params p, start
// time p[2]) re-sampled at every stage time; kind < 0: the static coef.
struct OrTableau { int s; double c[7]; double a[7][7]; double b[7]; };
OrTableau or_tableau(int method) {
  OrTableau T{};
  if (method == 0) {
    T.s = 4;
    T.c[1] = T.c[2] = 0.5; T.c[3] = 1.0;
    T.a[1][0] = 0.5; T.a[2][1] = 0.5; T.a[3][2] = 1.0;
    T.b[0] = T.b[3] = 1.0 / 6.0; T.b[1] = T.b[2] = 1.0 / 3.0;
    return T;
  }
  T.s = 7;
  const double c[7] = {0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0, 1.0};
  const double a[7][6] = {
      {0, 0, 0, 0, 0, 0},
      {0.161, 0, 0, 0, 0, 0},
      {-0.008480655492356989, 0.335480655492357, 0, 0, 0, 0},
      {2.897153057105493, -6.359448489975075, 4.3622954328695815, 0, 0, 0},
      {5.325864828439257, -11.748883564062828, 7.4955393428898365, -0.09249506636175525, 0, 0},
      {5.86145544294642, -12.92096931784711, 8.159367898576159, -0.071584973281401, -0.028269050394068383, 0},
      {0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081, 2.324710524099774}};
  for (int i = 0; i < 7; ++i) {
    T.c[i] = c[i];
    for (int j = 0; j < 6; ++j) T.a[i][j] = a[i][j];
  }
  for (int j = 0; j < 6; ++j) T.b[j] = a[6][j];
  return T;
}

int or_erk_tableau(int method, double* c, double* A, double* b) {
  OrTableau T = or_tableau(method);
  for (int i = 0; i < T.s; ++i) {
    c[i] = T.c[i]; b[i] = T.b[i];
    for (int j = 0; j < T.s; ++j) A[i * T.s + j] = T.a[i][j];
  }
  return T.s;
}

void or_evolve_curved_erk(void* h, const double* coef0, int kind, const double* p0, double* Phi, double* Pi, double dt,
                          int nsteps, int method, double eps_ko, const or_bc* bc, int use_metric) {
  Mesh& m = *static_cast<Mesh*>(h);
  const long nn = m.nn();
  const OrTableau T = or_tableau(method);
  std::vector<std::vector<double>> kP(T.s, std::vector<double>(nn)), kQ(T.s, std::vector<double>(nn));
  std::vector<double> Ps(nn), Qs(nn), coef(coef0 ? coef0 : nullptr, coef0 ? coef0 + 11 * nn : nullptr);
  double p[16] = {};
  if (kind >= 0) { std::memcpy(p, p0, sizeof(p)); coef.assign(11 * nn, 0.0); }
  const double t0 = kind >= 0 ? p0[2] : 0.0;
  for (int n = 0; n < nsteps; ++n) {
    for (int st = 0; st < T.s; ++st) {
      bool used = false;  // a stage that no later stage and no weight uses is skipped
      for (int i = st + 1; i < T.s; ++i) used |= T.a[i][st] != 0.0;
      if (!used && T.b[st] == 0.0) continue;
      for (long q = 0; q < nn; ++q) {
        double sp = 0.0, sq = 0.0;
        for (int j = 0; j < st; ++j) { sp += T.a[st][j] * kP[j][q]; sq += T.a[st][j] * kQ[j][q]; }
        Ps[q] = Phi[q] + dt * sp; Qs[q] = Pi[q] + dt * sq;
      }
      if (kind >= 0) { p[2] = t0 + n * dt + T.c[st] * dt; sample_background(m, kind, p, coef.data()); }
      or_rhs_curved(h, coef.data(), Ps.data(), Qs.data(), kP[st].data(), kQ[st].data(), eps_ko, bc, use_metric,
                    nullptr);
    }
    for (long q = 0; q < nn; ++q) {
      double sp = 0.0, sq = 0.0;
      for (int j = 0; j < T.s; ++j) { sp += T.b[j] * kP[j][q]; sq += T.b[j] * kQ[j][q]; }
      Phi[q] += dt * sp; Pi[q] += dt * sq;
    }
  }
}

// RK4 on the second-order SIPG system written first order: (u, v = u_t) with
//   u' = v + eps mu^-5 sum_d D_d^6 u,   v' = L_SAT u (+ Sommerfeld) + eps mu^-5 sum_d D_d^6 v.
void or_sipg_f(void* h, const double* u, const double* v, double* du, double* dv, const double* bvals,
               double tau, double inv_R, double eps_ko) {
  Mesh& m = *static_cast<Mesh*>(h);
  const long nn = m.nn();
  or_rhs_sipg(h, u, v, dv, bvals, tau, inv_R);
  for (long n = 0; n < nn; ++n) du[n] = v[n];
  if (eps_ko != 0.0) {
    if (m.mu < 0) compute_mu(m);
    double koT = eps_ko * m.inv_mu5;
    std::vector<double> s1(nn), s2(nn);
    for (int d = 0; d < 3; ++d) ko_axis(m, du, u, d, koT, s1, s2);
    for (int d = 0; d < 3; ++d) ko_axis(m, dv, v, d, koT, s1, s2);
  }
}

// discrete H-norm energy of the SIPG system: 1/2 <v,v>_H - 1/2 <u, L_SAT u>_H
// (test/kernels3d_tests.jl:39-47; homogeneous boundary values, no Sommerfeld u_t term)
double or_energy_sipg(void* h, const double* u, const double* v, double tau) {
  Mesh& m = *static_cast<Mesh*>(h);
  const long nn = m.nn();
  std::vector<double> Lu(nn), zero(nn, 0.0);
  double bz[6] = {0, 0, 0, 0, 0, 0};
  or_rhs_sipg(h, u, zero.data(), Lu.data(), bz, tau, 0.0);
  double K = 0.0, V = 0.0;
  for (long n = 0; n < nn; ++n) { K += v[n] * v[n] * m.Hphys[n]; V += u[n] * Lu[n] * m.Hphys[n]; }
  return K / 2 - V / 2;
}

void or_evolve_sipg(void* h, double* u, double* v, double dt, int nsteps, const double* bvals, double tau,
                    double inv_R, double eps_ko, double* energy) {
  Mesh& m = *static_cast<Mesh*>(h);
  const long nn = m.nn();
  std::vector<double> k1(nn), k2(nn), k3(nn), k4(nn), k5(nn), k6(nn), k7(nn), k8(nn), us(nn), vs(nn);
  if (energy) energy[0] = or_energy_sipg(h, u, v, tau);
  for (int s = 0; s < nsteps; ++s) {
    or_sipg_f(h, u, v, k1.data(), k2.data(), bvals, tau, inv_R, eps_ko);
    for (long n = 0; n < nn; ++n) { us[n] = u[n] + dt / 2 * k1[n]; vs[n] = v[n] + dt / 2 * k2[n]; }
    or_sipg_f(h, us.data(), vs.data(), k3.data(), k4.data(), bvals, tau, inv_R, eps_ko);
    for (long n = 0; n < nn; ++n) { us[n] = u[n] + dt / 2 * k3[n]; vs[n] = v[n] + dt / 2 * k4[n]; }
    or_sipg_f(h, us.data(), vs.data(), k5.data(), k6.data(), bvals, tau, inv_R, eps_ko);
    for (long n = 0; n < nn; ++n) { us[n] = u[n] + dt * k5[n]; vs[n] = v[n] + dt * k6[n]; }
    or_sipg_f(h, us.data(), vs.data(), k7.data(), k8.data(), bvals, tau, inv_R, eps_ko);
    for (long n = 0; n < nn; ++n) {
      u[n] += dt / 6 * (k1[n] + 2 * k3[n] + 2 * k5[n] + k7[n]);
      v[n] += dt / 6 * (k2[n] + 2 * k4[n] + 2 * k6[n] + k8[n]);
    }
    if (energy) energy[s + 1] = or_energy_sipg(h, u, v, tau);
  }
}

// _min_node_spacing_3d (src/evolve.jl:60-69)
double or_min_spacing(void* h) {
  Mesh& m = *static_cast<Mesh*>(h);
  const int N = m.N; double hm = std::numeric_limits<double>::max();
  auto dist = [&](long a, long b) {
    double dx = m.coords[3 * a] - m.coords[3 * b], dy = m.coords[3 * a + 1] - m.coords[3 * b + 1],
           dz = m.coords[3 * a + 2] - m.coords[3 * b + 2];
    return std::sqrt(dx * dx + dy * dy + dz * dz);
  };
  for (long e = 0; e < m.Ne; ++e)
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          long n = nid(N, i, j, k, e);
          if (i > 0) hm = std::min(hm, dist(n, nid(N, i - 1, j, k, e)));
          if (j > 0) hm = std::min(hm, dist(n, nid(N, i, j - 1, k, e)));
          if (k > 0) hm = std::min(hm, dist(n, nid(N, i, j, k - 1, e)));
        }
  return hm;
}

int or_num_threads() {
  int n = 1;
#pragma omp parallel
  {
#pragma omp single
    n = omp_get_num_threads();
  }
  return n;
}

}  // extern "C"
