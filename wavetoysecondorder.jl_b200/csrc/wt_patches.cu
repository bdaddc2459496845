// wt_patches.cu -- meshes built from node coordinates: the multi-patch
// curvilinear meshes of evolve3d's mesh kinds (src/evolve.jl:1176-1184:
// cubed cube, inflated cube, radial shell) and the face matching and
// orientation inference that every coordinate-built mesh goes through.
//
// The reference builds these meshes in HexMeshes (unvendored); the maps here
// are this library's own:
//   cubed cube (M, R): the cube [-1,1]^3 as a centre cube [-R,R]^3 and six
//     frustum patches, each blending the centre cube's face (w = 0) linearly
//     into the outer cube face (w = 1); outer faces flat.
//   inflated cube (L, R1, R2, M): a centre cube [-L,L]^3, six patches blending
//     its faces into the sphere of radius R1, and six spherical-shell patches
//     from R1 to R2 (13 M^3 elements); outer faces on the sphere R2.
//   radial shell (R1, R2, M): six spherical-shell patches between R1 (inner
//     faces, the excision tag) and R2 (outer faces).
// Sphere points use the equiangular cubed-sphere direction of patch (A, s):
// d = s e_A + tan(pi/4 (2u-1)) e_B + tan(pi/4 (2v-1)) e_C, normalised.  Every
// patch is right-handed (e_B x e_C = s e_A), M^3 elements, element (a, b, c)
// covering (u, v, w) in [a/M, (a+1)/M] x ..., numbered patch by patch with a
// fastest.  The Jacobian is the SBP derivative of the node coordinates.
#include "wt_common.cuh"
#include "../../include/wavetoy_b200.h"

#include <cmath>
#include <unordered_map>
#include <vector>

namespace wt {

namespace {

struct PatchGeo {
  int kind;        // 0 centre cube, 1 cube-face blend to a cube (cubed cube), 2 cube-face blend to a sphere, 3 shell
  int A = 0, s = 1;  // radial axis and sign (patches 1..3)
  double r0 = 0, r1 = 0;  // inner / outer half-width or radius
};

void frame(int A, int s, int& B, int& C) {
  B = (A + 1) % 3;
  C = (A + 2) % 3;
  if (s < 0) std::swap(B, C);
}

double tan_edge(double t) {  // tan(pi/4 t) for t in [-1, 1], exact at the ends
  if (t == -1.0) return -1.0;
  if (t == 1.0) return 1.0;
  return std::tan(0.25 * M_PI * t);
}

void point(const PatchGeo& g, double u, double v, double w, double X[3]) {
  if (g.kind == 0) {
    X[0] = g.r1 * (2.0 * u - 1.0);
    X[1] = g.r1 * (2.0 * v - 1.0);
    X[2] = g.r1 * (2.0 * w - 1.0);
    return;
  }
  int B, C;
  frame(g.A, g.s, B, C);
  const double su = 2.0 * u - 1.0, sv = 2.0 * v - 1.0;
  double Pin[3];
  Pin[g.A] = g.s * g.r0; Pin[B] = g.r0 * su; Pin[C] = g.r0 * sv;
  if (g.kind == 1) {
    double Pout[3];
    Pout[g.A] = g.s * g.r1; Pout[B] = g.r1 * su; Pout[C] = g.r1 * sv;
    for (int a = 0; a < 3; ++a) X[a] = (1.0 - w) * Pin[a] + w * Pout[a];
    return;
  }
  double d[3];
  d[g.A] = g.s; d[B] = tan_edge(su); d[C] = tan_edge(sv);
  const double nd = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  for (int a = 0; a < 3; ++a) d[a] /= nd;
  if (g.kind == 2) {
    for (int a = 0; a < 3; ++a) X[a] = (1.0 - w) * Pin[a] + w * (g.r1 * d[a]);
  } else {
    const double r = w == 0.0 ? g.r0 : w == 1.0 ? g.r1 : g.r0 + (g.r1 - g.r0) * w;
    for (int a = 0; a < 3; ++a) X[a] = r * d[a];
  }
}

// spatial hash of face centroids (cell size h; a query looks at the 27 cells around it)
struct Key {
  long long x, y, z;
  bool operator==(const Key& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct KeyHash {
  size_t operator()(const Key& k) const {
    return (size_t)(k.x * 73856093LL) ^ (size_t)(k.y * 19349663LL) ^ (size_t)(k.z * 83492791LL);
  }
};

}  // namespace

int infer_orientation(int N, const double* X, long long e, int f, long long en, int fn, double tol, bool shift) {
  const long long N3 = (long long)N * N * N;
  for (int ori = 0; ori < 8; ++ori) {
    double d0[3] = {0, 0, 0};
    bool ok = true;
    for (int q = 0; q < N && ok; ++q)
      for (int p = 0; p < N && ok; ++p) {
        int pn, qn;
        face_perm(ori, p, q, N, pn, qn);
        const long long a = e * N3 + face_node(faxis(f), frow(f, N), p, q, N);
        const long long b = en * N3 + face_node(faxis(fn), frow(fn, N), pn, qn, N);
        for (int c = 0; c < 3; ++c) {
          const double d = X[c + 3 * a] - X[c + 3 * b];
          if (shift && p == 0 && q == 0) d0[c] = d;
          if (std::fabs(d - d0[c]) > tol) ok = false;
        }
      }
    if (ok) return ori;
  }
  return -1;
}

int match_faces(int N, long long Ne, const double* X, double tol, std::vector<int32_t>& nbr,
                std::vector<int32_t>& nbrf) {
  const long long N3 = (long long)N * N * N;
  nbr.assign(6 * Ne, -1);
  nbrf.assign(6 * Ne, 0);
  std::vector<double> cen(3 * 6 * Ne);
  for (long long e = 0; e < Ne; ++e)
    for (int f = 0; f < 6; ++f)
      for (int c = 0; c < 3; ++c) {
        double sacc = 0.0;
        for (int q = 0; q < 2; ++q)
          for (int p = 0; p < 2; ++p)
            sacc += X[c + 3 * (e * N3 + face_node(faxis(f), frow(f, N), p * (N - 1), q * (N - 1), N))];
        cen[c + 3 * (f + 6 * e)] = 0.25 * sacc;
      }
  const double h = 1e3 * tol;
  auto key = [&](long long i, int dx, int dy, int dz) {
    return Key{(long long)std::floor(cen[3 * i] / h) + dx, (long long)std::floor(cen[3 * i + 1] / h) + dy,
               (long long)std::floor(cen[3 * i + 2] / h) + dz};
  };
  std::unordered_map<Key, std::vector<long long>, KeyHash> cells;
  cells.reserve(12 * Ne);
  for (long long i = 0; i < 6 * Ne; ++i) cells[key(i, 0, 0, 0)].push_back(i);
  for (long long i = 0; i < 6 * Ne; ++i) {
    if (nbr[i] >= 0) continue;
    const long long e = i / 6;
    const int f = (int)(i % 6);
    for (int dz = -1; dz <= 1 && nbr[i] < 0; ++dz)
      for (int dy = -1; dy <= 1 && nbr[i] < 0; ++dy)
        for (int dx = -1; dx <= 1 && nbr[i] < 0; ++dx) {
          auto it = cells.find(key(i, dx, dy, dz));
          if (it == cells.end()) continue;
          for (long long j : it->second) {
            if (j == i || j / 6 == e || nbr[j] >= 0) continue;
            double d2 = 0.0;
            for (int c = 0; c < 3; ++c) d2 += (cen[3 * i + c] - cen[3 * j + c]) * (cen[3 * i + c] - cen[3 * j + c]);
            if (d2 > tol * tol) continue;
            const long long en = j / 6;
            const int fn = (int)(j % 6);
            const int ori = infer_orientation(N, X, e, f, en, fn, tol, false);
            if (ori < 0) continue;
            int rori = -1;  // the neighbour's view of the same face pair
            rori = infer_orientation(N, X, en, fn, e, f, tol, false);
            if (rori < 0) return -1;
            nbr[i] = (int32_t)en; nbrf[i] = fn | (ori << 3);
            nbr[j] = (int32_t)e;  nbrf[j] = f | (rori << 3);
            break;
          }
        }
  }
  return 0;
}

// SBP derivative of the node coordinates: jac[a + 3 b + 9 n] = dX_a / dxi_b
void coords_jacobian(int N, long long Ne, const double* X, const std::vector<double>& G, double* jac) {
  const long long N3 = (long long)N * N * N;
  for (long long e = 0; e < Ne; ++e)
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          const long long n = e * N3 + i + N * (j + N * k);
          const int idx[3] = {i, j, k};
          for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) {
              double sacc = 0.0;
              for (int m = 0; m < N; ++m) {
                int ii = i, jj = j, kk = k;
                (b == 0 ? ii : b == 1 ? jj : kk) = m;
                sacc += G[idx[b] * N + m] * X[a + 3 * (e * N3 + ii + N * (jj + N * kk))];
              }
              jac[a + 3 * b + 9 * n] = sacc;
            }
        }
}

int build_patch_mesh(int kind, int N, int M, const double p[3], const std::vector<double>& xg,
                     std::vector<double>& X, double& scale) {
  std::vector<PatchGeo> patches;
  auto ring = [&](int k, double r0, double r1) {
    for (int A = 0; A < 3; ++A)
      for (int s = -1; s <= 1; s += 2) {
        PatchGeo g;
        g.kind = k; g.A = A; g.s = s; g.r0 = r0; g.r1 = r1;
        patches.push_back(g);
      }
  };
  if (kind == WT_MESH_CUBED_CUBE) {
    const double R = p[0];
    if (!(R > 0.0 && R < 1.0)) return -1;
    PatchGeo c; c.kind = 0; c.r1 = R;
    patches.push_back(c);
    ring(1, R, 1.0);
    scale = 1.0;
  } else if (kind == WT_MESH_INFLATED_CUBE) {
    const double L = p[0], R1 = p[1], R2 = p[2];
    if (!(L > 0.0 && L * std::sqrt(3.0) < R1 && R1 < R2)) return -1;
    PatchGeo c; c.kind = 0; c.r1 = L;
    patches.push_back(c);
    ring(2, L, R1);
    ring(3, R1, R2);
    scale = R2;
  } else if (kind == WT_MESH_RADIAL_SHELL) {
    const double R1 = p[0], R2 = p[1];
    if (!(R1 > 0.0 && R1 < R2)) return -1;
    ring(3, R1, R2);
    scale = R2;
  } else {
    return -2;
  }
  const long long E = (long long)M * M * M, N3 = (long long)N * N * N;
  X.assign(3 * N3 * E * patches.size(), 0.0);
  for (size_t pi = 0; pi < patches.size(); ++pi)
    for (int c = 0; c < M; ++c)
      for (int b = 0; b < M; ++b)
        for (int a = 0; a < M; ++a) {
          const long long e = (long long)pi * E + a + M * (b + (long long)M * c);
          for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
              for (int i = 0; i < N; ++i) {
                const double u = (a + xg[i]) / M, v = (b + xg[j]) / M, w = (c + xg[k]) / M;
                point(patches[pi], u, v, w, &X[3 * (e * N3 + i + N * (j + N * k))]);
              }
        }
  return 0;
}

}  // namespace wt
