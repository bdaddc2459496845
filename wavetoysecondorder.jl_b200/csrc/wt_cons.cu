// wt_cons.cu -- the hot path: the conservative first-order (Phi, Pi) ADM wave
// right-hand side of wave3d_curved_rhs! (src/wave3d_curved.jl:205-258) with
// its boundary passes (src/boundaries3d.jl:58-232), Kreiss-Oliger
// dissipation (src/wave3d_curved.jl:182-192) and the RK4 stage update.
//
// One RHS evaluation is two element-parallel kernels (the two-pass structure
// HexSBPSAT uses, GOALS.md:138-151, because the divergence SAT needs the
// neighbour's flux, which needs the neighbour's gradient):
//   K1  per element: Phi -> smem, neighbour Phi face traces -> smem; split-form
//       (or affine per-axis) gradient with centred-flux SAT; flux
//       F^i = beta^i Pi + K^{ij} d_j Phi; Phidot = beta.grad + a Pi; boundary
//       increments; writes F (3 fields) and either Phidot or the fused RK4
//       stage update of Phi.
//   K2  per element: F -> smem, neighbour F face traces -> smem; split-form
//       divergence with centred-flux SAT; adds the boundary increments; writes
//       Pidot or the fused RK4 stage update of Pi.
// One CTA owns EPB elements with one thread per node; every element block is a
// contiguous N^3 run, so all global loads are fully coalesced; the reference
// derivative matrix is held transposed in smem so the N-term contractions read
// conflict-free.  Streamed coefficients: a, beta (3), K (6) and, curvilinear,
// Ja (9) and 1/J.
#include "wt_common.cuh"

#include <initializer_list>
#include <type_traits>

namespace wt {

template <int N>
struct Ep {
  static constexpr int N3 = N * N * N;
  static constexpr int N2 = N * N;
  static constexpr int EPB = N3 >= 100 ? 1 : (128 / N3);
  static constexpr int T = N3 * EPB;
};

template <typename real>
struct K1P {
  long long Ne, nn;
  long long e0, e1;  // single-solve launches: the elements [e0, e1) the launch covers
  const real* Phi;
  const real* Pi;
  const real* c10;  // a, b1, b2, b3, K11, K12, K13, K22, K23, K33 (nullptr: gradient only)
  const real* Ja;
  const real* invdetJ;
  const real* sdiag;
  const int32_t* nbr;
  const int32_t* nbrf;
  const int32_t* bdry;
  const int32_t* bslot;
  const int32_t* emask;  // per element: SAT face mask (bits 0-5), outer face (bit 6)
  const int32_t* fsrc;   // per (f,e): 8 * neighbour + neighbour face, -1 without SAT
  const double* G;
  const double* H;
  real* F;
  real* Phidot;
  real* bbuf;
  real* grad_out;
  int bc_on, bc_curv, exc_tag, nbf;
  int kinds[6];
  real sigma;
  const real* bnorm;
  const real* gPhi;
  const real* gPi;
  const real* gDx;
  const real* gDy;
  const real* gDz;
  int epi, stage;
  double dt;
  real* y;
  real* acc;
  real* out;
  real* comp;
  unsigned int* nonfinite;
  // compensated FP32 form (CP instantiation): the Phi the stage reads is Phi +
  // Phit (Phit: the state's low part at stage 0, the previous stage's small
  // output after it; NULL = zero); Ja = Ja0 [9e + c] (FP64, element constant)
  // + dJa (FP32, node order); stage 2 copies Phi into hcopy for stage 3
  const real* Phit;
  const real* dJa;
  const double* Ja0;
  real* hcopy;
};

// Low-storage classic RK4 stage update.  Without compensation acc holds
// y + partial increments.  With compensation (FP32 state) acc holds the
// increment of the step alone and the final y + increment is a Kahan sum; comp
// holds the low part the FP32 y lost (the state is y + comp), so that small
// increments are not lost to the rounding of y over many steps.
template <typename real>
__device__ __forceinline__ void rk_epilogue(int stage, double dt, real k, real yin, real* y, real* acc, real* out,
                                            real* comp, long long n, unsigned int* nonfinite) {
  if (comp) {
    if (stage == 0) {
      out[n] = yin + (real)(0.5 * dt) * k;
      acc[n] = (real)(dt / 6.0) * k;
    } else if (stage == 1) {
      out[n] = y[n] + (real)(0.5 * dt) * k;
      acc[n] = acc[n] + (real)(dt / 3.0) * k;
    } else if (stage == 2) {
      out[n] = y[n] + (real)dt * k;
      acc[n] = acc[n] + (real)(dt / 3.0) * k;
    } else {
      const real inc = acc[n] + (real)(dt / 6.0) * k;
      const real yv = y[n];
      const real t = inc + comp[n];
      const real v = yv + t;
      comp[n] = t - (v - yv);
      y[n] = v;
      if (nonfinite && !isfinite((double)v)) atomicOr(nonfinite, 1u);
    }
    return;
  }
  if (stage == 0) {
    out[n] = yin + (real)(0.5 * dt) * k;
    acc[n] = yin + (real)(dt / 6.0) * k;
  } else if (stage == 1) {
    out[n] = y[n] + (real)(0.5 * dt) * k;
    acc[n] = acc[n] + (real)(dt / 3.0) * k;
  } else if (stage == 2) {
    out[n] = y[n] + (real)dt * k;
    acc[n] = acc[n] + (real)(dt / 3.0) * k;
  } else {
    real v = acc[n] + (real)(dt / 6.0) * k;
    y[n] = v;
    if (nonfinite && !isfinite((double)v)) atomicOr(nonfinite, 1u);
  }
}

// RK4 stage update of the compensated FP32 form (the Phi side, K1): the state
// is (y, comp) = (high, low part) and the stage the next K1 reads is its high
// part plus out = low part + c dt k; the step's final sum is formed in FP64 and
// split again.  hi: this node's high part of the state (the K1 input).
__device__ __forceinline__ void rk_epilogue_cp(int stage, double dt, float k, float hi, float* y, float* acc,
                                               float* out, float* comp, float* hcopy, long long n,
                                               unsigned int* nonfinite) {
  const float lo = comp[n];
  if (stage == 0) {
    out[n] = lo + (float)(0.5 * dt) * k;
    acc[n] = (float)(dt / 6.0) * k;
  } else if (stage == 1) {
    out[n] = lo + (float)(0.5 * dt) * k;
    acc[n] = acc[n] + (float)(dt / 3.0) * k;
  } else if (stage == 2) {
    out[n] = lo + (float)dt * k;
    acc[n] = acc[n] + (float)(dt / 3.0) * k;
    hcopy[n] = hi;
  } else {
    const float inc = acc[n] + (float)(dt / 6.0) * k;
    const double v = (double)hi + ((double)lo + (double)inc);
    const float h = (float)v;
    y[n] = h;
    comp[n] = (float)(v - (double)h);
    if (nonfinite && !isfinite(h)) atomicOr(nonfinite, 1u);
  }
}

// Per-thread asynchronous copy of one word (4 or 8 bytes) global -> shared,
// and the wait for all of this thread's copies.  The generic kernels copy the
// words their node pass reads at their own node (coefficients, Pi, RK state)
// at kernel start, so that those loads run under the contraction; each thread
// reads back only its own words, so the wait needs no CTA barrier.
template <typename T>
__device__ __forceinline__ void cp_async_word(T* dst, const T* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_own() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The RK4 stage updates above with the words they read at node n passed in
// (yv = y[n], accv = acc[n], compv = comp[n]; only those the stage reads need
// to be valid): the same arithmetic in the same order.
template <typename real>
__device__ __forceinline__ void rk_epilogue_v(int stage, double dt, real k, real yin, real yv, real accv, real compv,
                                              real* y, real* acc, real* out, real* comp, long long n,
                                              unsigned int* nonfinite) {
  if (comp) {
    if (stage == 0) {
      out[n] = yin + (real)(0.5 * dt) * k;
      acc[n] = (real)(dt / 6.0) * k;
    } else if (stage == 1) {
      out[n] = yv + (real)(0.5 * dt) * k;
      acc[n] = accv + (real)(dt / 3.0) * k;
    } else if (stage == 2) {
      out[n] = yv + (real)dt * k;
      acc[n] = accv + (real)(dt / 3.0) * k;
    } else {
      const real inc = accv + (real)(dt / 6.0) * k;
      const real t = inc + compv;
      const real v = yv + t;
      comp[n] = t - (v - yv);
      y[n] = v;
      if (nonfinite && !isfinite((double)v)) atomicOr(nonfinite, 1u);
    }
    return;
  }
  if (stage == 0) {
    out[n] = yin + (real)(0.5 * dt) * k;
    acc[n] = yin + (real)(dt / 6.0) * k;
  } else if (stage == 1) {
    out[n] = yv + (real)(0.5 * dt) * k;
    acc[n] = accv + (real)(dt / 3.0) * k;
  } else if (stage == 2) {
    out[n] = yv + (real)dt * k;
    acc[n] = accv + (real)(dt / 3.0) * k;
  } else {
    real v = accv + (real)(dt / 6.0) * k;
    y[n] = v;
    if (nonfinite && !isfinite((double)v)) atomicOr(nonfinite, 1u);
  }
}

// rk_epilogue_cp with lov = comp[n] and accv = acc[n] passed in
__device__ __forceinline__ void rk_epilogue_cp_v(int stage, double dt, float k, float hi, float lov, float accv,
                                                 float* y, float* acc, float* out, float* comp, float* hcopy,
                                                 long long n, unsigned int* nonfinite) {
  const float lo = lov;
  if (stage == 0) {
    out[n] = lo + (float)(0.5 * dt) * k;
    acc[n] = (float)(dt / 6.0) * k;
  } else if (stage == 1) {
    out[n] = lo + (float)(0.5 * dt) * k;
    acc[n] = accv + (float)(dt / 3.0) * k;
  } else if (stage == 2) {
    out[n] = lo + (float)dt * k;
    acc[n] = accv + (float)(dt / 3.0) * k;
    hcopy[n] = hi;
  } else {
    const float inc = accv + (float)(dt / 6.0) * k;
    const double v = (double)hi + ((double)lo + (double)inc);
    const float h = (float)v;
    y[n] = h;
    comp[n] = (float)(v - (double)h);
    if (nonfinite && !isfinite(h)) atomicOr(nonfinite, 1u);
  }
}

// contraction along axis d of a smem field f (N^3) with transposed G (GT[p*N+i] = G[i][p])
template <int N, typename real>
__device__ __forceinline__ real contract(const real* __restrict__ f, const real* __restrict__ GT, int i, int j, int k,
                                         int d) {
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

// resident CTAs per SM the generic kernels are compiled for: about 1024 threads
template <int T>
struct GenOcc {
  static constexpr int value = T >= 1024 ? 1 : 1024 / T;
};

// The node pass of K1 at node n (element ec, node (i, j, k)): flux, Phidot,
// boundary terms (into bbuf) and the RK4 stage update or Phidot.  g: the
// gradient; u: the stage input (CP: its high part), ug: the value the gradient
// differentiated; sd: the affine axis scales; a, b, K, Pi: the node's
// coefficients and Pi.  PRE: the RK words the update reads (yv, accv, compv)
// were loaded by the caller; otherwise the update reads them itself.
template <int N, typename real, bool CP, bool PRE, typename gt>
__device__ __forceinline__ void k1_finish(const K1P<real>& P, long long ec, long long n, int i, int j, int k,
                                          int emask, const real g[3], real u, gt ug, const real sd[3], real Hend,
                                          real a, const real b[3], const real K[6], real Pi, real yv, real accv,
                                          real compv) {
  constexpr int N2 = Ep<N>::N2;
  const long long nn = P.nn;
  // flux and Phidot
  const real F0 = b[0] * Pi + (K[0] * g[0] + K[1] * g[1] + K[2] * g[2]);
  const real F1 = b[1] * Pi + (K[1] * g[0] + K[3] * g[1] + K[4] * g[2]);
  const real F2 = b[2] * Pi + (K[2] * g[0] + K[4] * g[1] + K[5] * g[2]);
  real phid = b[0] * g[0] + b[1] * g[1] + b[2] * g[2] + a * Pi;
  // boundary increments (per boundary face of the node; Pi parts go to the face slot)
  if (P.bc_on && (emask >> 6)) {
    const int idx3[3] = {i, j, k};
    for (int f = 0; f < 6; ++f) {
      const int tag = P.bdry[f + 6 * ec];
      if (tag == 0) continue;
      const int ax = f >> 1;
      if (idx3[ax] != frow(f, N)) continue;
      const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
      const int slot = ::wt::bc_slot(P.bslot[f + 6 * ec], P.nbf);
      real dF = 0, dP = 0;
      if (!P.bc_curv) {
        const int kind = P.kinds[f];
        if (kind != 3) {
          const real nh = (f & 1) ? (real)1 : (real)-1;
          const real Kdd = ax == 0 ? K[0] : ax == 1 ? K[3] : K[5];
          const real a_n = sqrt(a * Kdd);
          const real bax = b[ax];
          const real bn = nh * bax;
          const real wt = sd[ax] / Hend;
          if (kind == 4) {
            const real tau = P.sigma * (fabs(a_n - bax) + fabs(a_n + bax)) * wt;
            const real gp = P.gPhi ? P.gPhi[n] : (real)0, gq = P.gPi ? P.gPi[n] : (real)0;
            dF = -tau * ((real)ug - gp);
            dP = -tau * (Pi - gq);
          } else {
            const real qv = nh * g[ax];
            const real r = Pi + ((bn + a_n) / a) * qv;
            const real gv = kind == 2 ? (real)0 : (P.gPhi ? P.gPhi[n] : (real)0);
            dP = -P.sigma * fabs(a_n + bn) * wt * (r - gv);
          }
        }
      } else if (tag != P.exc_tag) {
        const int kind = P.kinds[0];
        const long long nb = (long long)P.nbf * N2;
        const long long bi = (long long)slot * N2 + p + N * q;
        const real nx = P.bnorm[bi], ny = P.bnorm[nb + bi], nz = P.bnorm[2 * nb + bi], wt = P.bnorm[3 * nb + bi];
        const real Kn = K[0] * nx * nx + K[3] * ny * ny + K[5] * nz * nz +
                        (real)2 * (K[1] * nx * ny + K[2] * nx * nz + K[4] * ny * nz);
        const real a_n = sqrt(a * Kn);
        const real bn = b[0] * nx + b[1] * ny + b[2] * nz;
        if (kind == 4) {
          const real tau = P.sigma * (fabs(a_n - bn) + fabs(a_n + bn)) * wt;
          const real gp = P.gPhi ? P.gPhi[n] : (real)0, gq = P.gPi ? P.gPi[n] : (real)0;
          dF = -tau * ((real)ug - gp);
          dP = -tau * (Pi - gq);
        } else {
          const real qv = nx * g[0] + ny * g[1] + nz * g[2];
          const real r = Pi + ((bn + a_n) / a) * qv;
          real gv = 0;
          if (kind != 2) {
            const real gq = P.gPi ? P.gPi[n] : (real)0;
            const real gx = P.gDx ? P.gDx[n] : (real)0, gy = P.gDy ? P.gDy[n] : (real)0,
                       gz = P.gDz ? P.gDz[n] : (real)0;
            gv = gq + ((bn + a_n) / a) * (nx * gx + ny * gy + nz * gz);
          }
          dP = -P.sigma * fabs(a_n + bn) * wt * (r - gv);
        }
      }
      phid += dF;
      P.bbuf[(long long)slot * N2 + p + N * q] = dP;
    }
  }
  P.F[n] = F0;
  P.F[nn + n] = F1;
  P.F[2 * nn + n] = F2;
  if constexpr (PRE) {
    if constexpr (CP) {
      if (P.epi)
        rk_epilogue_cp_v(P.stage, P.dt, phid, u, compv, accv, P.y, P.acc, P.out, P.comp, P.hcopy, n, P.nonfinite);
      else
        P.Phidot[n] = phid;
    } else {
      if (P.epi)
        rk_epilogue_v<real>(P.stage, P.dt, phid, u, yv, accv, compv, P.y, P.acc, P.out, P.comp, n, P.nonfinite);
      else
        P.Phidot[n] = phid;
    }
  } else if constexpr (CP) {
    if (P.epi)
      rk_epilogue_cp(P.stage, P.dt, phid, u, P.y, P.acc, P.out, P.comp, P.hcopy, n, P.nonfinite);
    else
      P.Phidot[n] = phid;
  } else {
    if (P.epi)
      rk_epilogue<real>(P.stage, P.dt, phid, u, P.y, P.acc, P.out, P.comp, n, P.nonfinite);
    else
      P.Phidot[n] = phid;
  }
}

// BATCH: the CTA's elements come from a work list of (solve, element) tiles
// and each tile reads the parameter block of its solve (plist); otherwise
// element blockIdx.x * EPB + le of the single solve P0.  EPB_: elements per CTA.
// CP (real = float): the compensated form -- the Phi the stage reads (high
// plus small part) and the split-form gradient of it in FP64.
template <int N, typename real, bool CURV, bool BATCH, int EPB_, bool CP = false>
__global__ void __launch_bounds__(Ep<N>::N3 * EPB_, GenOcc<Ep<N>::N3 * EPB_>::value) k_cons_k1(const K1P<real> P0, const K1P<real>* __restrict__ plist,
                                                            const int2* __restrict__ tiles, long long ntiles) {
  constexpr int N3 = Ep<N>::N3, N2 = Ep<N>::N2, EPB = EPB_;
  // CP: u = Phi + Phit and its derivative D u in FP64; with Ja = Ja0 + dJa
  // (Ja0 element-constant, FP64) the split form is
  //   0.5 D(Ja u) + 0.5 Ja D u = (Ja0 + 0.5 dJa) D u + 0.5 D(dJa u),
  // and only the last contraction, of the small dJa u, runs in FP32
  using gt = typename std::conditional<CP, double, real>::type;  // precision of u and D u
  __shared__ gt GT[N2];
  __shared__ real GTr[CP ? N2 : 1];  // CP: the operator in FP32 for D(dJa u)
  __shared__ gt su[EPB][N3];
  __shared__ gt sun[EPB][6][N2];
  __shared__ real sw[CURV ? EPB : 1][CURV ? 9 : 1][CURV ? N3 : 1];
  const int tid = threadIdx.x;
  const int le = tid / N3, t = tid - le * N3;
  const int i = t % N, j = (t / N) % N, k = t / N2;
  long long e = (BATCH ? 0 : P0.e0) + (long long)blockIdx.x * EPB + le;
  int sid = 0;
  bool valid;
  if constexpr (BATCH) {
    valid = e < ntiles;
    if (valid) {
      const int2 tl = tiles[e];
      sid = tl.x;
      e = tl.y;
    }
  } else {
    valid = e < P0.e1;
  }
  const K1P<real>& P = BATCH ? plist[sid] : P0;
  const long long ec = valid ? e : 0;  // clamp for address arithmetic
  const long long n = ec * N3 + t;
  const long long nn = P.nn;
  if (tid < N2) GT[(tid % N) * N + tid / N] = (gt)P.G[tid];
  if constexpr (CP) {
    if (tid < N2) GTr[(tid % N) * N + tid / N] = (real)P.G[tid];
  }
  // the node pass's own-node words, copied now (cp.async) so that their loads run
  // under the contraction: c10 [0..9], Pi [10], RK state y [11], acc [12],
  // comp [13] (only the words this stage's update reads)
  constexpr bool PF = 14 * N3 * EPB * sizeof(real) <= 24576;
  __shared__ real spf[PF ? EPB : 1][PF ? 14 : 1][PF ? N3 : 1];
  const bool grad_only = P.c10 == nullptr;
  const bool pf_y = P.epi && (P.stage == 1 || P.stage == 2 || (!CP && P.comp && P.stage == 3));
  const bool pf_acc = P.epi && P.stage >= 1;
  const bool pf_comp = P.epi && (CP || (P.comp && P.stage == 3));
  if constexpr (PF) {
    if (valid && !grad_only) {
#pragma unroll
      for (int c = 0; c < 10; ++c) cp_async_word(&spf[le][c][t], P.c10 + c * nn + n);
      cp_async_word(&spf[le][10][t], P.Pi + n);
      if (pf_y) cp_async_word(&spf[le][11][t], P.y + n);
      if (pf_acc) cp_async_word(&spf[le][12][t], P.acc + n);
      if (pf_comp) cp_async_word(&spf[le][13][t], P.comp + n);
    }
  }
  const real u = valid ? P.Phi[n] : (real)0;  // CP: the high part
  gt ug = u;                                   // the value the gradient differentiates
  if constexpr (CP) {
    if (valid && P.Phit) ug += (gt)P.Phit[n];
  }
  su[le][t] = ug;
  // element tables: SAT mask / outer-face flag, and the neighbour face sources
  const int emask = valid ? P.emask[ec] : 0;
  // neighbour Phi face traces (fsrc is -1 exactly where the SAT mask bit is 0,
  // so the trace loads need not wait for the mask)
  for (int idx = t; idx < 6 * N2; idx += N3) {
    const int f = idx / N2, pq = idx - f * N2;
    gt v = 0;
    const int src = valid ? ::wt::bc_src(P.fsrc[f + 6 * ec], P.Ne) : -1;
    if (src >= 0) {
      const long long nb = (long long)(src >> 6) * N3 + nbr_face_node(src, pq % N, pq / N, N);
      v = P.Phi[nb];
      if constexpr (CP) {
        if (P.Phit) v += (gt)P.Phit[nb];
      }
    }
    sun[le][f][pq] = v;
  }
  real m[CURV ? 9 : 1];   // Ja (CP: its deviation dJa)
  real m0[CP && CURV ? 9 : 1];  // CP: the element-constant part Ja0
  real invJ = 0, sd[3];
  if (CURV) {
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      if constexpr (CP) {
        m[c] = valid ? P.dJa[c * nn + n] : (real)0;
        m0[c] = valid ? (real)P.Ja0[9 * ec + c] : (real)0;
      } else {
        m[c] = valid ? P.Ja[c * nn + n] : (real)0;
      }
    }
    invJ = valid ? P.invdetJ[n] : (real)0;
  } else {
#pragma unroll
    for (int d = 0; d < 3; ++d) sd[d] = P.sdiag[3 * ec + d];
  }
  const real Hend = (real)P.H[0];
  if (CURV) {
#pragma unroll
    for (int c = 0; c < 9; ++c) sw[le][c][t] = m[c] * (real)ug;  // CP: dJa u
  }
  __syncthreads();
  real du[3];  // D u (CP: formed in FP64, then a gradient-sized value)
#pragma unroll
  for (int d = 0; d < 3; ++d) du[d] = (real)contract<N>(su[le], GT, i, j, k, d);
  real g[3];
  if (CURV) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      real acc = 0;
#pragma unroll
      for (int al = 0; al < 3; ++al) {
        if constexpr (CP)
          acc += (real)0.5 * contract<N>(sw[le][al * 3 + c], GTr, i, j, k, al) +
                 (m0[al * 3 + c] + (real)0.5 * m[al * 3 + c]) * du[al];
        else
          acc += (real)0.5 * contract<N>(sw[le][al * 3 + c], GT, i, j, k, al) + (real)0.5 * m[al * 3 + c] * du[al];
      }
      g[c] = acc;
    }
  } else {
#pragma unroll
    for (int d = 0; d < 3; ++d) g[d] = sd[d] * du[d];
  }
  // centred-flux SAT on interior faces through this node (CP: the jump formed in FP64)
  if (valid) {
    const int idx3[3] = {i, j, k};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int ax = f >> 1;
      if (idx3[ax] != frow(f, N)) continue;
      if (!((emask >> f) & 1)) continue;
      const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
      const real jump = (real)(sun[le][f][p + N * q] - ug);
      const real nh = (f & 1) ? (real)1 : (real)-1;
      if (CURV) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          real mc = m[ax * 3 + c];
          if constexpr (CP) mc += m0[ax * 3 + c];
          g[c] += nh * mc * jump / ((real)2 * Hend);
        }
      } else {
        g[ax] += nh * sd[ax] / ((real)2 * Hend) * jump;
      }
    }
  }
  if (CURV) {
#pragma unroll
    for (int c = 0; c < 3; ++c) g[c] *= invJ;
  }
  if (!valid) return;
  // the node's coefficients and Pi: from the words copied at kernel start, or
  // (no room for them) loaded only now -- held in registers across the
  // contraction they would cost the registers that keep more CTAs resident
  real a = 0, b[3] = {0, 0, 0}, K[6] = {0, 0, 0, 0, 0, 0}, Pi = 0;
  if (!grad_only) {
    if constexpr (PF) {
      cp_async_wait_own();
      a = spf[le][0][t];
#pragma unroll
      for (int c = 0; c < 3; ++c) b[c] = spf[le][1 + c][t];
#pragma unroll
      for (int c = 0; c < 6; ++c) K[c] = spf[le][4 + c][t];
      Pi = spf[le][10][t];
    } else {
      a = P.c10[n];
#pragma unroll
      for (int c = 0; c < 3; ++c) b[c] = P.c10[(1 + c) * nn + n];
#pragma unroll
      for (int c = 0; c < 6; ++c) K[c] = P.c10[(4 + c) * nn + n];
      Pi = P.Pi[n];
    }
  }
  if (P.grad_out) {
#pragma unroll
    for (int c = 0; c < 3; ++c) P.grad_out[c * nn + n] = g[c];
  }
  if (grad_only) return;
  k1_finish<N, real, CP, PF>(P, ec, n, i, j, k, emask, g, u, ug, sd, Hend, a, b, K, Pi,
                             PF && pf_y ? spf[le][11][t] : (real)0, PF && pf_acc ? spf[le][12][t] : (real)0,
                             PF && pf_comp ? spf[le][13][t] : (real)0);
}

// ---------------------------------------------------------------------------
// Persistent, cp.async-pipelined K1 for work lists of n < 8 solves (the batch's
// and the server's n = 4 and n = 6 groups).  The generic K1 above loads its
// inputs when its one element starts (the face traces behind two dependent
// loads), so it waits on global memory: about 0.2 of DRAM throughput, long-
// scoreboard stalls.  Here a CTA loops over groups of EPB tiles and copies
// everything group g + 1 reads at its own nodes -- Phi (and Phit), the metric
// terms, 1/J, the ten coefficients, Pi, the RK words, the neighbour face
// traces (sources loaded one group earlier) and Ja0 -- into the second of two
// shared buffers while it computes group g.  The arithmetic is the generic
// K1's (same contractions, same order, k1_finish for the node pass), so both
// give the same bits.
template <int N, typename real, bool CP>
struct PipeK1 {
  static constexpr int N3 = Ep<N>::N3, N2 = Ep<N>::N2, EPB = Ep<N>::EPB, T = N3 * EPB;
  // own-node word planes of an element block in a buffer
  static constexpr int PHI = 0, PHIT = 1, JA = CP ? 2 : 1, INVJ = JA + 9, C10 = INVJ + 1, PI = C10 + 10,
                       Y = PI + 1, ACC = Y + 1, COMP = ACC + 1, NW = COMP + 1;
  static constexpr int NF = CP ? 12 : 6;               // face-trace planes: Phi [+ Phit] on the 6 faces
  static constexpr int NFR = (6 * N2 + N3 - 1) / N3;  // face entries per thread
  // words of one element block (padded to 16 bytes) and of one buffer
  static constexpr size_t EW = ((NW * N3 + NF * N2) * sizeof(real) + (CP ? 9 * sizeof(double) : 0) + 15) / 16 * 16;
  static constexpr size_t BUF = EPB * EW;
  using gt = typename std::conditional<CP, double, real>::type;
  static constexpr size_t SU = ((size_t)EPB * N3 * sizeof(gt) + 15) / 16 * 16;
  static constexpr size_t SW = ((size_t)EPB * 9 * N3 * sizeof(real) + 15) / 16 * 16;
  static constexpr size_t SMEM = 2 * BUF + SU + SW + N2 * sizeof(gt) + N2 * sizeof(real) + 16;
  // resident CTAs per SM the registers are sized for: as many as the shared memory
  // allows, up to 1024 threads
  static constexpr int OCC_SM = (int)(220000 / SMEM) > 0 ? (int)(220000 / SMEM) : 1;
  static constexpr int OCC = OCC_SM < 1024 / T ? OCC_SM : 1024 / T;
  static_assert(!CP || ((NW * N3 + NF * N2) * sizeof(real)) % 8 == 0, "Ja0 must be 8-byte aligned in a block");
};

// 4- or 8-byte cp.async, zero-filled (src not read) when !valid
template <typename T>
__device__ __forceinline__ void cp_async_word_z(T* dst, const T* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}

template <int N, typename real, bool CP>
__global__ void __launch_bounds__(PipeK1<N, real, CP>::T, PipeK1<N, real, CP>::OCC)
    k_cons_k1_pipe(const K1P<real>* __restrict__ plist, const int2* __restrict__ tiles, long long ntiles) {
  using L = PipeK1<N, real, CP>;
  using gt = typename L::gt;
  constexpr int N3 = L::N3, N2 = L::N2, EPB = L::EPB, NFR = L::NFR;
  extern __shared__ __align__(16) unsigned char smraw[];
  gt* su = reinterpret_cast<gt*>(smraw + 2 * L::BUF);                   // [EPB][N3]
  real* sw = reinterpret_cast<real*>(smraw + 2 * L::BUF + L::SU);       // [EPB][9][N3]
  gt* GT = reinterpret_cast<gt*>(smraw + 2 * L::BUF + L::SU + L::SW);   // transposed G
  real* GTr = reinterpret_cast<real*>(GT + N2);                         // CP: G in FP32
  const int tid = threadIdx.x;
  const int le = tid / N3, t = tid - le * N3;
  const int i = t % N, j = (t / N) % N, k = t / N2;
  const long long ngroups = (ntiles + EPB - 1) / EPB;
  const long long GS = gridDim.x;
  auto blk = [&](int bb) -> real* { return reinterpret_cast<real*>(smraw + bb * L::BUF + le * L::EW); };
  // this thread's tile in group gg (x = -1: none)
  auto tile_of = [&](long long gg) -> int2 {
    const long long ti = gg * EPB + le;
    return (gg < ngroups && ti < ntiles) ? tiles[ti] : make_int2(-1, -1);
  };
  auto src_load = [&](int2 tl, int src[NFR]) {
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = t + r * N3;
      src[r] = (tl.x >= 0 && idx < 6 * N2) ? ::wt::bc_src(plist[tl.x].fsrc[idx / N2 + 6 * tl.y], plist[tl.x].Ne) : -1;
    }
  };
  // copy what tile tl reads at this thread's node, and this thread's face-trace
  // entries, into buffer bb
  auto issue = [&](int2 tl, const int src[NFR], int bb) {
    if (tl.x < 0) return;
    const K1P<real>& P = plist[tl.x];
    const long long e = tl.y, n = e * N3 + t, nn = P.nn;
    real* w = blk(bb);
    cp_async_word(w + L::PHI * N3 + t, P.Phi + n);
    if constexpr (CP) cp_async_word_z(w + L::PHIT * N3 + t, P.Phit ? P.Phit + n : P.Phi + n, P.Phit != nullptr);
    const real* ja = CP ? P.dJa : P.Ja;
#pragma unroll
    for (int c = 0; c < 9; ++c) cp_async_word(w + (L::JA + c) * N3 + t, ja + c * nn + n);
    cp_async_word(w + L::INVJ * N3 + t, P.invdetJ + n);
    if (P.c10) {
#pragma unroll
      for (int c = 0; c < 10; ++c) cp_async_word(w + (L::C10 + c) * N3 + t, P.c10 + c * nn + n);
      cp_async_word(w + L::PI * N3 + t, P.Pi + n);
    }
    if (P.epi && (P.stage == 1 || P.stage == 2 || (!CP && P.comp && P.stage == 3)))
      cp_async_word(w + L::Y * N3 + t, P.y + n);
    if (P.epi && P.stage >= 1) cp_async_word(w + L::ACC * N3 + t, P.acc + n);
    if (P.epi && (CP || (P.comp && P.stage == 3))) cp_async_word(w + L::COMP * N3 + t, P.comp + n);
    real* fc = w + L::NW * N3;
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = t + r * N3;
      if (idx < 6 * N2) {
        const int f = idx / N2, pq = idx - f * N2, sr = src[r];
        const long long nb = sr >= 0 ? (long long)(sr >> 6) * N3 + nbr_face_node(sr, pq % N, pq / N, N) : 0;
        cp_async_word_z(fc + f * N2 + pq, P.Phi + nb, sr >= 0);
        if constexpr (CP) cp_async_word_z(fc + (6 + f) * N2 + pq, (P.Phit ? P.Phit : P.Phi) + nb, sr >= 0 && P.Phit);
      }
    }
    if constexpr (CP) {
      if (t < 9) cp_async_word(reinterpret_cast<double*>(fc + L::NF * N2) + t, P.Ja0 + 9 * e + t);
    }
  };

  if (tid < N2) {
    GT[(tid % N) * N + tid / N] = (gt)plist[0].G[tid];  // every solve of a group has the same N, hence G
    if constexpr (CP) GTr[(tid % N) * N + tid / N] = (real)plist[0].G[tid];
  }
  long long g = blockIdx.x;
  int2 tcur = tile_of(g), tnext = tile_of(g + GS);
  int src[NFR];
  src_load(tcur, src);
  issue(tcur, src, 0);
  src_load(tnext, src);
  int emcur = tcur.x >= 0 ? plist[tcur.x].emask[tcur.y] : 0;
  for (int it = 0; g < ngroups; g += GS, ++it) {
    const int bb = it & 1;
    const int2 tn2 = tile_of(g + 2 * GS);
    const int emnext = tnext.x >= 0 ? plist[tnext.x].emask[tnext.y] : 0;
    cp_async_wait_own();
    // this group's words are visible to every thread, and every thread is done
    // with the previous group: the other buffer, su and sw are free
    __syncthreads();
    issue(tnext, src, bb ^ 1);
    src_load(tn2, src);
    const bool valid = tcur.x >= 0;
    const K1P<real>& P = plist[valid ? tcur.x : 0];
    const long long ec = valid ? tcur.y : 0, n = ec * N3 + t;
    const real* w = blk(bb);
    const real* fc = w + L::NW * N3;
    const int emask = emcur;
    const real u = valid ? w[L::PHI * N3 + t] : (real)0;  // CP: the high part
    gt ug = u;
    if constexpr (CP) {
      if (valid && P.Phit) ug += (gt)w[L::PHIT * N3 + t];
    }
    su[le * N3 + t] = ug;
    real m[9], m0[CP ? 9 : 1];
    const double* ja0 = reinterpret_cast<const double*>(fc + L::NF * N2);
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      m[c] = valid ? w[(L::JA + c) * N3 + t] : (real)0;
      if constexpr (CP) m0[c] = valid ? (real)ja0[c] : (real)0;
    }
    const real invJ = valid ? w[L::INVJ * N3 + t] : (real)0;
    const real Hend = (real)P.H[0];
#pragma unroll
    for (int c = 0; c < 9; ++c) sw[(le * 9 + c) * N3 + t] = m[c] * (real)ug;
    __syncthreads();
    real du[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) du[d] = (real)contract<N>(su + le * N3, GT, i, j, k, d);
    real g3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      real acc = 0;
#pragma unroll
      for (int al = 0; al < 3; ++al) {
        if constexpr (CP)
          acc += (real)0.5 * contract<N>(sw + (le * 9 + al * 3 + c) * N3, GTr, i, j, k, al) +
                 (m0[al * 3 + c] + (real)0.5 * m[al * 3 + c]) * du[al];
        else
          acc += (real)0.5 * contract<N>(sw + (le * 9 + al * 3 + c) * N3, GT, i, j, k, al) +
                 (real)0.5 * m[al * 3 + c] * du[al];
      }
      g3[c] = acc;
    }
    if (valid) {
      const int idx3[3] = {i, j, k};
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int ax = f >> 1;
        if (idx3[ax] != frow(f, N)) continue;
        if (!((emask >> f) & 1)) continue;
        const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
        gt sv = fc[f * N2 + p + N * q];
        if constexpr (CP) {
          if (P.Phit) sv += (gt)fc[(6 + f) * N2 + p + N * q];
        }
        const real jump = (real)(sv - ug);
        const real nh = (f & 1) ? (real)1 : (real)-1;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          real mc = m[ax * 3 + c];
          if constexpr (CP) mc += m0[ax * 3 + c];
          g3[c] += nh * mc * jump / ((real)2 * Hend);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) g3[c] *= invJ;
    if (valid) {
      if (P.grad_out) {
#pragma unroll
        for (int c = 0; c < 3; ++c) P.grad_out[c * P.nn + n] = g3[c];
      }
      if (P.c10) {
        const real a = w[L::C10 * N3 + t];
        real b[3], K[6];
#pragma unroll
        for (int c = 0; c < 3; ++c) b[c] = w[(L::C10 + 1 + c) * N3 + t];
#pragma unroll
        for (int c = 0; c < 6; ++c) K[c] = w[(L::C10 + 4 + c) * N3 + t];
        const real Pi = w[L::PI * N3 + t];
        const bool pf_y = P.epi && (P.stage == 1 || P.stage == 2 || (!CP && P.comp && P.stage == 3));
        const bool pf_acc = P.epi && P.stage >= 1;
        const bool pf_comp = P.epi && (CP || (P.comp && P.stage == 3));
        const real sd[3] = {0, 0, 0};
        k1_finish<N, real, CP, true>(P, ec, n, i, j, k, emask, g3, u, ug, sd, Hend, a, b, K, Pi,
                                     pf_y ? w[L::Y * N3 + t] : (real)0, pf_acc ? w[L::ACC * N3 + t] : (real)0,
                                     pf_comp ? w[L::COMP * N3 + t] : (real)0);
      }
    }
    tcur = tnext;
    tnext = tn2;
    emcur = emnext;
  }
  cp_async_wait_own();
}

template <typename real>
struct K2P {
  long long Ne, nn;
  long long e0, e1;  // single-solve launches: the elements [e0, e1) the launch covers
  const real* F0;
  const real* F1;
  const real* F2;
  const real* Ja;
  const real* invdetJ;
  const real* sdiag;
  const int32_t* nbr;
  const int32_t* nbrf;
  const int32_t* bdry;
  const int32_t* bslot;
  const int32_t* emask;
  const int32_t* fsrc;
  const double* G;
  const double* H;
  const real* bbuf;
  int bc_on, nbf;
  real* Pidot;
  int epi, stage;
  double dt;
  real* y;
  real* acc;
  real* out;
  real* comp;
  unsigned int* nonfinite;
};

template <int N, typename real, bool CURV, bool BATCH, int EPB_>
__global__ void __launch_bounds__(Ep<N>::N3 * EPB_) k_cons_k2(const K2P<real> P0, const K2P<real>* __restrict__ plist,
                                                            const int2* __restrict__ tiles, long long ntiles) {
  constexpr int N3 = Ep<N>::N3, N2 = Ep<N>::N2, EPB = EPB_;
  __shared__ real GT[N2];
  __shared__ real sF[EPB][3][N3];
  __shared__ real sFn[EPB][6][CURV ? 3 : 1][N2];
  __shared__ real sw[CURV ? EPB : 1][CURV ? 3 : 1][CURV ? N3 : 1];
  const int tid = threadIdx.x;
  const int le = tid / N3, t = tid - le * N3;
  const int i = t % N, j = (t / N) % N, k = t / N2;
  long long e = (BATCH ? 0 : P0.e0) + (long long)blockIdx.x * EPB + le;
  int sid = 0;
  bool valid;
  if constexpr (BATCH) {
    valid = e < ntiles;
    if (valid) {
      const int2 tl = tiles[e];
      sid = tl.x;
      e = tl.y;
    }
  } else {
    valid = e < P0.e1;
  }
  const K2P<real>& P = BATCH ? plist[sid] : P0;
  const long long ec = valid ? e : 0;
  const long long n = ec * N3 + t;
  const long long nn = P.nn;
  if (tid < N2) GT[(tid % N) * N + tid / N] = (real)P.G[tid];
  // the RK state words the stage update reads at this node, copied now (see K1):
  // y [0], acc [1], comp [2]
  constexpr bool PF = 3 * N3 * EPB * sizeof(real) <= 12288;
  __shared__ real spf[PF ? EPB : 1][PF ? 3 : 1][PF ? N3 : 1];
  const bool pf_y = P.epi && (P.stage <= 2 || (P.comp && P.stage == 3));
  const bool pf_acc = P.epi && P.stage >= 1;
  const bool pf_comp = P.epi && P.comp && P.stage == 3;
  if constexpr (PF) {
    if (valid) {
      if (pf_y) cp_async_word(&spf[le][0][t], P.y + n);
      if (pf_acc) cp_async_word(&spf[le][1][t], P.acc + n);
      if (pf_comp) cp_async_word(&spf[le][2][t], P.comp + n);
    }
  }
  const real* Fp[3] = {P.F0, P.F1, P.F2};
  real Fv[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Fv[c] = valid ? Fp[c][n] : (real)0;
    sF[le][c][t] = Fv[c];
  }
  const int emask = valid ? P.emask[ec] : 0;
  for (int idx = t; idx < 6 * N2; idx += N3) {
    const int f = idx / N2, pq = idx - f * N2;
    long long src = -1;
    const int fs = valid ? ::wt::bc_src(P.fsrc[f + 6 * ec], P.Ne) : -1;  // -1 exactly where the SAT mask bit is 0
    if (fs >= 0) src = (long long)(fs >> 6) * N3 + nbr_face_node(fs, pq % N, pq / N, N);
    if (CURV) {
#pragma unroll
      for (int c = 0; c < 3; ++c) sFn[le][f][c][pq] = src >= 0 ? Fp[c][src] : (real)0;
    } else {
      sFn[le][f][0][pq] = src >= 0 ? Fp[f >> 1][src] : (real)0;
    }
  }
  real m[CURV ? 9 : 1];
  real invJ = 0, sd[3];
  if (CURV) {
#pragma unroll
    for (int c = 0; c < 9; ++c) m[c] = valid ? P.Ja[c * nn + n] : (real)0;
    invJ = valid ? P.invdetJ[n] : (real)0;
#pragma unroll
    for (int al = 0; al < 3; ++al) sw[le][al][t] = m[al * 3] * Fv[0] + m[al * 3 + 1] * Fv[1] + m[al * 3 + 2] * Fv[2];
  } else {
#pragma unroll
    for (int d = 0; d < 3; ++d) sd[d] = P.sdiag[3 * ec + d];
  }
  const real Hend = (real)P.H[0];
  __syncthreads();
  real dv = 0;
  if (CURV) {
#pragma unroll
    for (int al = 0; al < 3; ++al) {
      dv += (real)0.5 * contract<N>(sw[le][al], GT, i, j, k, al);
#pragma unroll
      for (int c = 0; c < 3; ++c) dv += (real)0.5 * m[al * 3 + c] * contract<N>(sF[le][c], GT, i, j, k, al);
    }
  } else {
#pragma unroll
    for (int d = 0; d < 3; ++d) dv += sd[d] * contract<N>(sF[le][d], GT, i, j, k, d);
  }
  if (!valid) return;
  const int idx3[3] = {i, j, k};
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const int ax = f >> 1;
    if (idx3[ax] != frow(f, N)) continue;
    if (!((emask >> f) & 1)) continue;
    const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
    const real nh = (f & 1) ? (real)1 : (real)-1;
    if (CURV) {
      real s = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) s += m[ax * 3 + c] * (sFn[le][f][c][p + N * q] - Fv[c]);
      dv += nh * s / ((real)2 * Hend);
    } else {
      dv += nh * sd[ax] / ((real)2 * Hend) * (sFn[le][f][0][p + N * q] - Fv[ax]);
    }
  }
  if (CURV) dv *= invJ;
  if (P.bc_on && (emask >> 6)) {
    for (int f = 0; f < 6; ++f) {
      if (P.bdry[f + 6 * ec] == 0) continue;
      const int ax = f >> 1;
      if (idx3[ax] != frow(f, N)) continue;
      const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
      dv += P.bbuf[(long long)::wt::bc_slot(P.bslot[f + 6 * ec], P.nbf) * N2 + p + N * q];
    }
  }
  if (P.epi) {
    if constexpr (PF) {
      cp_async_wait_own();
      const real yv = pf_y ? spf[le][0][t] : (real)0, accv = pf_acc ? spf[le][1][t] : (real)0,
                 compv = pf_comp ? spf[le][2][t] : (real)0;
      rk_epilogue_v<real>(P.stage, P.dt, dv, P.stage == 0 ? yv : (real)0, yv, accv, compv, P.y, P.acc, P.out, P.comp,
                          n, P.nonfinite);
    } else {
      const real yin = P.stage == 0 ? P.y[n] : (real)0;
      rk_epilogue<real>(P.stage, P.dt, dv, yin, P.y, P.acc, P.out, P.comp, n, P.nonfinite);
    }
  } else {
    P.Pidot[n] = dv;
  }
}

// Persistent, cp.async-pipelined K2 for work lists of n < 8 solves (see
// k_cons_k1_pipe): group g + 1's F, metric terms, 1/J, RK words and neighbour
// flux face traces are copied into the second shared buffer while group g is
// computed with the generic K2's arithmetic.
template <int N, typename real>
struct PipeK2 {
  static constexpr int N3 = Ep<N>::N3, N2 = Ep<N>::N2, EPB = Ep<N>::EPB, T = N3 * EPB;
  static constexpr int F = 0, JA = 3, INVJ = 12, Y = 13, ACC = 14, COMP = 15, NW = 16;
  static constexpr int NF = 18;                        // face-trace planes: F_c on the 6 faces
  static constexpr int NFR = (6 * N2 + N3 - 1) / N3;  // face points per thread (3 components each)
  static constexpr size_t EW = ((NW * N3 + NF * N2) * sizeof(real) + 15) / 16 * 16;
  static constexpr size_t BUF = EPB * EW;
  static constexpr size_t SW = ((size_t)EPB * 3 * N3 * sizeof(real) + 15) / 16 * 16;
  static constexpr size_t SMEM = 2 * BUF + SW + N2 * sizeof(real) + 16;
  static constexpr int OCC_SM = (int)(220000 / SMEM) > 0 ? (int)(220000 / SMEM) : 1;
  static constexpr int OCC = OCC_SM < 1024 / T ? OCC_SM : 1024 / T;
};

template <int N, typename real>
__global__ void __launch_bounds__(PipeK2<N, real>::T, PipeK2<N, real>::OCC)
    k_cons_k2_pipe(const K2P<real>* __restrict__ plist, const int2* __restrict__ tiles, long long ntiles) {
  using L = PipeK2<N, real>;
  constexpr int N3 = L::N3, N2 = L::N2, EPB = L::EPB, NFR = L::NFR;
  extern __shared__ __align__(16) unsigned char smraw[];
  real* sw = reinterpret_cast<real*>(smraw + 2 * L::BUF);              // [EPB][3][N3]
  real* GT = reinterpret_cast<real*>(smraw + 2 * L::BUF + L::SW);      // transposed G
  const int tid = threadIdx.x;
  const int le = tid / N3, t = tid - le * N3;
  const int i = t % N, j = (t / N) % N, k = t / N2;
  const long long ngroups = (ntiles + EPB - 1) / EPB;
  const long long GS = gridDim.x;
  auto blk = [&](int bb) -> real* { return reinterpret_cast<real*>(smraw + bb * L::BUF + le * L::EW); };
  auto tile_of = [&](long long gg) -> int2 {
    const long long ti = gg * EPB + le;
    return (gg < ngroups && ti < ntiles) ? tiles[ti] : make_int2(-1, -1);
  };
  auto src_load = [&](int2 tl, int src[NFR]) {
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = t + r * N3;
      src[r] = (tl.x >= 0 && idx < 6 * N2) ? ::wt::bc_src(plist[tl.x].fsrc[idx / N2 + 6 * tl.y], plist[tl.x].Ne) : -1;
    }
  };
  auto issue = [&](int2 tl, const int src[NFR], int bb) {
    if (tl.x < 0) return;
    const K2P<real>& P = plist[tl.x];
    const long long e = tl.y, n = e * N3 + t, nn = P.nn;
    const real* Fp[3] = {P.F0, P.F1, P.F2};
    real* w = blk(bb);
#pragma unroll
    for (int c = 0; c < 3; ++c) cp_async_word(w + (L::F + c) * N3 + t, Fp[c] + n);
#pragma unroll
    for (int c = 0; c < 9; ++c) cp_async_word(w + (L::JA + c) * N3 + t, P.Ja + c * nn + n);
    cp_async_word(w + L::INVJ * N3 + t, P.invdetJ + n);
    if (P.epi && (P.stage <= 2 || (P.comp && P.stage == 3))) cp_async_word(w + L::Y * N3 + t, P.y + n);
    if (P.epi && P.stage >= 1) cp_async_word(w + L::ACC * N3 + t, P.acc + n);
    if (P.epi && P.comp && P.stage == 3) cp_async_word(w + L::COMP * N3 + t, P.comp + n);
    real* fc = w + L::NW * N3;
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = t + r * N3;
      if (idx < 6 * N2) {
        const int f = idx / N2, pq = idx - f * N2, sr = src[r];
        const long long nb = sr >= 0 ? (long long)(sr >> 6) * N3 + nbr_face_node(sr, pq % N, pq / N, N) : 0;
#pragma unroll
        for (int c = 0; c < 3; ++c) cp_async_word_z(fc + (f * 3 + c) * N2 + pq, Fp[c] + nb, sr >= 0);
      }
    }
  };
  if (tid < N2) GT[(tid % N) * N + tid / N] = (real)plist[0].G[tid];
  long long g = blockIdx.x;
  int2 tcur = tile_of(g), tnext = tile_of(g + GS);
  int src[NFR];
  src_load(tcur, src);
  issue(tcur, src, 0);
  src_load(tnext, src);
  int emcur = tcur.x >= 0 ? plist[tcur.x].emask[tcur.y] : 0;
  for (int it = 0; g < ngroups; g += GS, ++it) {
    const int bb = it & 1;
    const int2 tn2 = tile_of(g + 2 * GS);
    const int emnext = tnext.x >= 0 ? plist[tnext.x].emask[tnext.y] : 0;
    cp_async_wait_own();
    __syncthreads();  // see k_cons_k1_pipe
    issue(tnext, src, bb ^ 1);
    src_load(tn2, src);
    const bool valid = tcur.x >= 0;
    const K2P<real>& P = plist[valid ? tcur.x : 0];
    const long long ec = valid ? tcur.y : 0, n = ec * N3 + t;
    const real* w = blk(bb);
    const real* fc = w + L::NW * N3;
    const int emask = emcur;
    real Fv[3], m[9];
#pragma unroll
    for (int c = 0; c < 3; ++c) Fv[c] = valid ? w[(L::F + c) * N3 + t] : (real)0;
#pragma unroll
    for (int c = 0; c < 9; ++c) m[c] = valid ? w[(L::JA + c) * N3 + t] : (real)0;
    const real invJ = valid ? w[L::INVJ * N3 + t] : (real)0;
#pragma unroll
    for (int al = 0; al < 3; ++al)
      sw[(le * 3 + al) * N3 + t] = m[al * 3] * Fv[0] + m[al * 3 + 1] * Fv[1] + m[al * 3 + 2] * Fv[2];
    const real Hend = (real)P.H[0];
    __syncthreads();
    real dv = 0;
#pragma unroll
    for (int al = 0; al < 3; ++al) {
      dv += (real)0.5 * contract<N>(sw + (le * 3 + al) * N3, GT, i, j, k, al);
#pragma unroll
      for (int c = 0; c < 3; ++c) dv += (real)0.5 * m[al * 3 + c] * contract<N>(w + (L::F + c) * N3, GT, i, j, k, al);
    }
    if (valid) {
      const int idx3[3] = {i, j, k};
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int ax = f >> 1;
        if (idx3[ax] != frow(f, N)) continue;
        if (!((emask >> f) & 1)) continue;
        const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
        const real nh = (f & 1) ? (real)1 : (real)-1;
        real sacc = 0;
#pragma unroll
        for (int c = 0; c < 3; ++c) sacc += m[ax * 3 + c] * (fc[(f * 3 + c) * N2 + p + N * q] - Fv[c]);
        dv += nh * sacc / ((real)2 * Hend);
      }
      dv *= invJ;
      if (P.bc_on && (emask >> 6)) {
        for (int f = 0; f < 6; ++f) {
          if (P.bdry[f + 6 * ec] == 0) continue;
          const int ax = f >> 1;
          if (idx3[ax] != frow(f, N)) continue;
          const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
          dv += P.bbuf[(long long)::wt::bc_slot(P.bslot[f + 6 * ec], P.nbf) * N2 + p + N * q];
        }
      }
      if (P.epi) {
        const bool pf_y = P.stage <= 2 || (P.comp && P.stage == 3);
        const real yv = pf_y ? w[L::Y * N3 + t] : (real)0;
        const real accv = P.stage >= 1 ? w[L::ACC * N3 + t] : (real)0;
        const real compv = P.comp && P.stage == 3 ? w[L::COMP * N3 + t] : (real)0;
        rk_epilogue_v<real>(P.stage, P.dt, dv, P.stage == 0 ? yv : (real)0, yv, accv, compv, P.y, P.acc, P.out,
                            P.comp, n, P.nonfinite);
      } else {
        P.Pidot[n] = dv;
      }
    }
    tcur = tnext;
    tnext = tn2;
    emcur = emnext;
  }
  cp_async_wait_own();
}

// ---------------------------------------------------------------------------
// apply_D!(Du, u, d): s_{d,e} G_d u + centred-flux SAT on interior d-faces,
// s_{d,e} = invjac[d,d] at the element's first node.
template <int N, typename real>
__global__ void __launch_bounds__(Ep<N>::T) k_apply_D(long long Ne, const real* __restrict__ u, real* __restrict__ out,
                                                     int d, const real* __restrict__ sdiag,
                                                     const int32_t* __restrict__ nbr, const int32_t* __restrict__ nbrf,
                                                     const int32_t* __restrict__ bdry, const double* __restrict__ G,
                                                     const double* __restrict__ H) {
  constexpr int N3 = Ep<N>::N3, N2 = Ep<N>::N2, EPB = Ep<N>::EPB;
  __shared__ real GT[N2];
  __shared__ real su[EPB][N3];
  const int tid = threadIdx.x;
  const int le = tid / N3, t = tid - le * N3;
  const int i = t % N, j = (t / N) % N, k = t / N2;
  const long long e = (long long)blockIdx.x * EPB + le;
  const bool valid = e < Ne;
  const long long ec = valid ? e : 0;
  const long long n = ec * N3 + t;
  if (tid < N2) GT[(tid % N) * N + tid / N] = (real)G[tid];
  const real uv = valid ? u[n] : (real)0;
  su[le][t] = uv;
  __syncthreads();
  if (!valid) return;
  const real s = sdiag[3 * ec + d];
  real r = s * contract<N>(su[le], GT, i, j, k, d);
  const int idx3[3] = {i, j, k};
  for (int f = 2 * d; f < 2 * d + 2; ++f) {
    if (idx3[d] != frow(f, N)) continue;
    if (bdry[f + 6 * ec] != 0) continue;
    const int en = ::wt::bc_elem(nbr[f + 6 * ec], Ne);
    if (en < 0) continue;
    const int p = d == 0 ? j : i, q = d == 2 ? j : k;
    const real un = u[(long long)en * N3 + nbr_face_node(nbrf[f + 6 * ec], p, q, N)];
    const real nh = (f & 1) ? (real)1 : (real)-1;
    r += nh * s / ((real)2 * (real)H[0]) * (un - uv);
  }
  out[n] = r;
}

// ---------------------------------------------------------------------------
// Line-local Kreiss-Oliger: dst += koT * D_d^6 field.  D_d couples only nodes
// on the same axis-d grid line (METHODS.md:151-155), so a CTA loads N pencils
// of one whole element line (N * len * N values) into smem and applies D_d six
// times there; one thread per (pencil, element segment) keeps its N values in
// registers.  The line's values come in and go out by cooperative loads and
// stores in node order (consecutive threads, consecutive addresses), staged
// through the same shared buffer; a thread loading its own pencil directly
// would read N consecutive words with a stride of N words between threads (the
// kernel then ran at 0.14 of DRAM bandwidth).  Arithmetic is that of six
// apply_D! calls.
template <int N, typename real>
__global__ void k_ko_line(int d, int len, int closed, const int32_t* __restrict__ lines, real* __restrict__ dst,
                          const real* __restrict__ field, real koT, const real* __restrict__ sdiag,
                          const double* __restrict__ G, const double* __restrict__ H) {
  extern __shared__ unsigned char smraw[];
  // [N pencils][len*N], pencil stride len*N + 1: the N pencils a warp touches at
  // once fall into different banks (with stride len*N they all share one)
  const int PS = len * N + 1;
  real* buf = reinterpret_cast<real*>(smraw);
  int* se = reinterpret_cast<int*>(buf + N * PS);  // the line's elements
  __shared__ real Gs[N * N];
  constexpr int N2 = N * N, N3 = N * N * N;
  const int line = blockIdx.x;
  const int g = blockIdx.y;       // pencil group (second tangential index)
  const int tid = threadIdx.x;
  const int pb = tid % N;         // pencil within group (fastest tangential index)
  const int sg = tid / N;         // element segment along the line
  for (int idx = tid; idx < N * N; idx += blockDim.x) Gs[idx] = (real)G[idx];
  for (int q = tid; q < len; q += blockDim.x) se[q] = lines[(long long)line * len + q];
  const bool act = sg < len;
  // node of position l along axis d of pencil p in the element of segment sq
  auto node = [&](int sq, int p, int l) -> long long {
    int ii, jj, kk;
    if (d == 0) { ii = l; jj = p; kk = g; }
    else if (d == 1) { ii = p; jj = l; kk = g; }
    else { ii = p; jj = g; kk = l; }
    return (long long)se[sq] * N3 + ii + N * (jj + N * kk);
  };
  // (pencil, position) of the w-th of an element's N^2 nodes in this group, w in
  // increasing node order: the cooperative loads and stores below run over
  // (segment, w), so that consecutive threads touch consecutive addresses
  auto split = [&](int w, int& p, int& l) {
    if (d == 0) { l = w % N; p = w / N; }
    else { p = w % N; l = w / N; }
  };
  __syncthreads();
  for (int q = tid; q < len * N2; q += blockDim.x) {
    const int sq = q / N2;
    int p, l;
    split(q - sq * N2, p, l);
    buf[p * PS + sq * N + l] = field[node(sq, p, l)];
  }
  __syncthreads();
  real v[N];
  if (act) {
#pragma unroll
    for (int l = 0; l < N; ++l) v[l] = buf[pb * PS + sg * N + l];
  }
  const real s = act ? sdiag[3 * se[sg] + d] : (real)0;
  const real Hend = (real)H[0];
  const bool has_prev = closed || sg > 0;
  const bool has_next = closed || sg < len - 1;
  const int sp = sg == 0 ? len - 1 : sg - 1;
  const int sn = sg == len - 1 ? 0 : sg + 1;
  for (int it = 0; it < 6; ++it) {
    if (act) {
#pragma unroll
      for (int l = 0; l < N; ++l) buf[pb * PS + sg * N + l] = v[l];
    }
    __syncthreads();
    if (act) {
      real w[N];
#pragma unroll
      for (int l = 0; l < N; ++l) {
        real acc = 0;
#pragma unroll
        for (int p = 0; p < N; ++p) acc += Gs[l * N + p] * v[p];
        w[l] = s * acc;
      }
      if (has_prev) w[0] += -s / ((real)2 * Hend) * (buf[pb * PS + sp * N + (N - 1)] - v[0]);
      if (has_next) w[N - 1] += s / ((real)2 * Hend) * (buf[pb * PS + sn * N + 0] - v[N - 1]);
#pragma unroll
      for (int l = 0; l < N; ++l) v[l] = w[l];
    }
    __syncthreads();
  }
  if (act) {
#pragma unroll
    for (int l = 0; l < N; ++l) buf[pb * PS + sg * N + l] = v[l];
  }
  __syncthreads();
  for (int q = tid; q < len * N2; q += blockDim.x) {
    const int sq = q / N2;
    int p, l;
    split(q - sq * N2, p, l);
    const long long nd = node(sq, p, l);
    dst[nd] = dst[nd] + koT * buf[p * PS + sq * N + l];
  }
}

// ---------------------------------------------------------------------------
// launchers
template <typename real>
static K1P<real> k1p_params(const DevMesh& m, const DevCoef& c, const void* Phi, const void* Pi, void* F, void* Phidot,
                            void* bbuf, void* grad_out, const ConsBC& bc, const RKStage& rk) {
  K1P<real> P;
  P.Ne = m.Ne; P.nn = m.nn; P.e0 = 0; P.e1 = m.Ne;
  P.Phi = (const real*)Phi; P.Pi = (const real*)Pi;
  P.c10 = (const real*)c.c10;
  P.Ja = (const real*)m.Ja_r; P.invdetJ = (const real*)m.invdetJ_r; P.sdiag = (const real*)m.sdiag;
  P.nbr = m.nbr; P.nbrf = m.nbrf; P.bdry = m.bdry; P.bslot = m.bslot;
  P.emask = m.emask; P.fsrc = m.fsrc;
  P.G = m.G; P.H = m.H;
  P.F = (real*)F; P.Phidot = (real*)Phidot; P.bbuf = (real*)bbuf; P.grad_out = (real*)grad_out;
  P.bc_on = bc.on; P.bc_curv = bc.curv; P.exc_tag = bc.exc_tag; P.nbf = m.nbf;
  for (int f = 0; f < 6; ++f) P.kinds[f] = bc.kinds[f];
  P.sigma = (real)bc.sigma; P.bnorm = (const real*)m.bnorm;
  P.gPhi = (const real*)bc.gPhi; P.gPi = (const real*)bc.gPi;
  P.gDx = (const real*)bc.gDx; P.gDy = (const real*)bc.gDy; P.gDz = (const real*)bc.gDz;
  P.epi = rk.on; P.stage = rk.stage; P.dt = rk.dt;
  P.y = (real*)rk.y; P.acc = (real*)rk.acc; P.out = (real*)rk.out; P.comp = (real*)rk.comp; P.nonfinite = rk.nonfinite;
  P.Phit = (const real*)rk.phit; P.dJa = (const real*)m.dJa; P.Ja0 = m.Ja0; P.hcopy = (real*)rk.hcopy;
  return P;
}

// the generic K1 runs the compensated instantiation for the default FP32 form
// (not for the gradient-only launches of the energy)
static bool gen_cp(const DevMesh& m, const void* grad_out) {
  return m.precision == WT_F32 && m.fp32_form == WT_FP32_COMPENSATED && grad_out == nullptr && m.Ja0 && m.dJa;
}

template <typename real>
static K2P<real> k2p_params(const DevMesh& m, const void* F, void* Pidot, const void* bbuf, const ConsBC& bc,
                            const RKStage& rk, unsigned int* nonfinite, const void* F1, const void* F2) {
  K2P<real> P;
  P.Ne = m.Ne; P.nn = m.nn; P.e0 = 0; P.e1 = m.Ne;
  P.F0 = (const real*)F;
  P.F1 = F1 ? (const real*)F1 : (const real*)F + m.nn;
  P.F2 = F2 ? (const real*)F2 : (const real*)F + 2 * m.nn;
  P.Ja = (const real*)m.Ja_r; P.invdetJ = (const real*)m.invdetJ_r; P.sdiag = (const real*)m.sdiag;
  P.nbr = m.nbr; P.nbrf = m.nbrf; P.bdry = m.bdry; P.bslot = m.bslot;
  P.emask = m.emask; P.fsrc = m.fsrc;
  P.G = m.G; P.H = m.H;
  P.bbuf = (const real*)bbuf; P.bc_on = bc.on; P.nbf = m.nbf;
  P.Pidot = (real*)Pidot;
  P.epi = rk.on; P.stage = rk.stage; P.dt = rk.dt;
  P.y = (real*)rk.y; P.acc = (real*)rk.acc; P.out = (real*)rk.out; P.comp = (real*)rk.comp; P.nonfinite = nonfinite;
  return P;
}

template <int N, typename real>
static int k1_dispatch(const DevMesh& m, const DevCoef& c, const void* Phi, const void* Pi, void* F, void* Phidot,
                       void* bbuf, void* grad_out, int use_metric, const ConsBC& bc, const RKStage& rk,
                       cudaStream_t s, long long e0 = 0, long long e1 = -1) {
  K1P<real> P = k1p_params<real>(m, c, Phi, Pi, F, Phidot, bbuf, grad_out, bc, rk);
  P.e0 = e0;
  P.e1 = e1 < 0 ? m.Ne : e1;
  const unsigned blocks = (unsigned)((P.e1 - P.e0 + Ep<N>::EPB - 1) / Ep<N>::EPB);
  if (blocks == 0) return 0;
  constexpr bool F32 = std::is_same<real, float>::value;
  if (F32 && gen_cp(m, grad_out)) {
    if (use_metric)
      k_cons_k1<N, real, true, false, Ep<N>::EPB, F32><<<blocks, Ep<N>::T, 0, s>>>(P, nullptr, nullptr, 0);
    else
      k_cons_k1<N, real, false, false, Ep<N>::EPB, F32><<<blocks, Ep<N>::T, 0, s>>>(P, nullptr, nullptr, 0);
  } else if (use_metric) {
    k_cons_k1<N, real, true, false, Ep<N>::EPB><<<blocks, Ep<N>::T, 0, s>>>(P, nullptr, nullptr, 0);
  } else {
    k_cons_k1<N, real, false, false, Ep<N>::EPB><<<blocks, Ep<N>::T, 0, s>>>(P, nullptr, nullptr, 0);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <int N, typename real>
static int k2_dispatch(const DevMesh& m, const void* F, void* Pidot, const void* bbuf, int use_metric,
                       const ConsBC& bc, const RKStage& rk, unsigned int* nonfinite, cudaStream_t s,
                       const void* F1 = nullptr, const void* F2 = nullptr, long long e0 = 0, long long e1 = -1) {
  K2P<real> P = k2p_params<real>(m, F, Pidot, bbuf, bc, rk, nonfinite, F1, F2);
  P.e0 = e0;
  P.e1 = e1 < 0 ? m.Ne : e1;
  const unsigned blocks = (unsigned)((P.e1 - P.e0 + Ep<N>::EPB - 1) / Ep<N>::EPB);
  if (blocks == 0) return 0;
  if (use_metric)
    k_cons_k2<N, real, true, false, Ep<N>::EPB><<<blocks, Ep<N>::T, 0, s>>>(P, nullptr, nullptr, 0);
  else
    k_cons_k2<N, real, false, false, Ep<N>::EPB><<<blocks, Ep<N>::T, 0, s>>>(P, nullptr, nullptr, 0);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// elements per CTA of the work-list (batched) generic kernels: the default or twice it
template <int N>
struct EpAlt {
  // the alternative must fit 1024 threads and the 48 KB of static shared memory
  // of the curvilinear K1 (Phi, 6 face traces, 9 products per element, FP64)
  static constexpr bool fits = Ep<N>::N3 * 2 * Ep<N>::EPB <= 1024 &&
                               (10 * Ep<N>::N3 + 6 * Ep<N>::N2) * 2 * Ep<N>::EPB * 8 + 8 * Ep<N>::N2 <= 48 * 1024;
  static constexpr int V1 = fits ? 2 * Ep<N>::EPB : Ep<N>::EPB;
};

template <int N, typename real, int EPB>
static int gen_batch(int which, bool cp, const void* plist, const int2* tiles, long long ntiles, cudaStream_t s) {
  const unsigned blocks = (unsigned)((ntiles + EPB - 1) / EPB);
  if (blocks == 0) return 0;
  constexpr bool F32 = std::is_same<real, float>::value;
  if (which == 1 && F32 && cp)
    k_cons_k1<N, real, true, true, EPB, F32><<<blocks, Ep<N>::N3 * EPB, 0, s>>>(K1P<real>(), (const K1P<real>*)plist,
                                                                               tiles, ntiles);
  else if (which == 1)
    k_cons_k1<N, real, true, true, EPB><<<blocks, Ep<N>::N3 * EPB, 0, s>>>(K1P<real>(), (const K1P<real>*)plist, tiles,
                                                                          ntiles);
  else
    k_cons_k2<N, real, true, true, EPB><<<blocks, Ep<N>::N3 * EPB, 0, s>>>(K2P<real>(), (const K2P<real>*)plist, tiles,
                                                                          ntiles);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

static int gen_sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// the pipelined kernels: a persistent grid of up to OCC CTAs per SM
template <int N, typename real, bool CP>
static int pipe_batch(int which, const void* plist, const int2* tiles, long long ntiles, cudaStream_t s) {
  static bool attr1 = false, attr2 = false;
  if (which == 1) {
    using L = PipeK1<N, real, CP>;
    if (!attr1) {
      if (cudaFuncSetAttribute(k_cons_k1_pipe<N, real, CP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)L::SMEM) != cudaSuccess)
        return -2;
      attr1 = true;
    }
    const long long ng = (ntiles + L::EPB - 1) / L::EPB, cap = (long long)gen_sm_count() * L::OCC;
    const long long grid = ng < cap ? ng : cap;
    if (grid <= 0) return 0;
    k_cons_k1_pipe<N, real, CP><<<(unsigned)grid, L::T, L::SMEM, s>>>((const K1P<real>*)plist, tiles, ntiles);
  } else {
    using L = PipeK2<N, real>;
    if (!attr2) {
      if (cudaFuncSetAttribute(k_cons_k2_pipe<N, real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::SMEM) !=
          cudaSuccess)
        return -2;
      attr2 = true;
    }
    const long long ng = (ntiles + L::EPB - 1) / L::EPB, cap = (long long)gen_sm_count() * L::OCC;
    const long long grid = ng < cap ? ng : cap;
    if (grid <= 0) return 0;
    k_cons_k2_pipe<N, real><<<(unsigned)grid, L::T, L::SMEM, s>>>((const K2P<real>*)plist, tiles, ntiles);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// variant: 0 the generic kernels at Ep<N>::EPB elements per CTA, 1 at the
// alternative EPB, 2 the pipelined kernels (n = 4 and 6; otherwise as 0)
template <int N>
static int gen_batch_n(int which, int precision, int variant, bool cp, const void* plist, const int2* tiles,
                       long long ntiles, cudaStream_t s) {
  if constexpr (N == 4 || N == 6) {
    if (variant == 2) {
      if (precision == 0) return pipe_batch<N, double, false>(which, plist, tiles, ntiles, s);
      return cp ? pipe_batch<N, float, true>(which, plist, tiles, ntiles, s)
                : pipe_batch<N, float, false>(which, plist, tiles, ntiles, s);
    }
  }
  if (precision == 0)
    return variant == 1 ? gen_batch<N, double, EpAlt<N>::V1>(which, false, plist, tiles, ntiles, s)
                        : gen_batch<N, double, Ep<N>::EPB>(which, false, plist, tiles, ntiles, s);
  return variant == 1 ? gen_batch<N, float, EpAlt<N>::V1>(which, cp, plist, tiles, ntiles, s)
                      : gen_batch<N, float, Ep<N>::EPB>(which, cp, plist, tiles, ntiles, s);
}

bool cons_gen_pipe_available(int N) { return N == 4 || N == 6; }

size_t cons_gen_param_size(int precision, int which) {
  if (precision == 0) return which == 1 ? sizeof(K1P<double>) : sizeof(K2P<double>);
  return which == 1 ? sizeof(K1P<float>) : sizeof(K2P<float>);
}

void cons_gen_fill_params(int which, const SolveStage& ss, unsigned* flag, void* dst) {
  const DevMesh& m = *ss.m;
  if (m.precision == 0) {
    if (which == 1)
      *(K1P<double>*)dst = k1p_params<double>(m, *ss.c, ss.Phi, ss.Pi, ss.F, nullptr, ss.bbuf, nullptr, ss.bc, ss.rkP);
    else
      *(K2P<double>*)dst = k2p_params<double>(m, ss.F, nullptr, ss.bbuf, ss.bc, ss.rkQ, flag, nullptr, nullptr);
  } else {
    if (which == 1)
      *(K1P<float>*)dst = k1p_params<float>(m, *ss.c, ss.Phi, ss.Pi, ss.F, nullptr, ss.bbuf, nullptr, ss.bc, ss.rkP);
    else
      *(K2P<float>*)dst = k2p_params<float>(m, ss.F, nullptr, ss.bbuf, ss.bc, ss.rkQ, flag, nullptr, nullptr);
  }
}

#define WT_DISPATCH_N(N_, CALL)   \
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

static inline bool a16(const void* p) { return p == nullptr || ((uintptr_t)p & 15u) == 0; }

// The pipelined n = 8 kernels stage element blocks with bulk copies, which
// need 16-byte aligned global addresses; anything else takes the generic path.
bool cons_n8_path(const DevMesh& m, const DevCoef& c, int use_metric, const ConsBC& bc, const RKStage& rkP,
                  const RKStage& rkQ, std::initializer_list<const void*> ptrs) {
  if (m.N != 8 || !use_metric || m.Ja_n8 == nullptr) return false;
  if (c.c10 == nullptr) return false;
  if (bc.on && !bc.curv) return false;
  for (const RKStage* rk : {&rkP, &rkQ})
    if (!a16(rk->y) || !a16(rk->acc) || !a16(rk->out)) return false;
  for (const void* p : ptrs)
    if (!a16(p)) return false;
  return a16(c.c10) && a16(m.invdetJ_r);
}

bool cons_gen_cp_supported(const DevMesh& m) { return gen_cp(m, nullptr); }

int launch_cons_k1(const DevMesh& m, const DevCoef& c, const void* Phi, const void* Pi, void* F, void* Phidot,
                   void* bbuf, void* grad_out, int use_metric, const ConsBC& bc, const RKStage& rk,
                   cudaStream_t s, bool n8, long long e0, long long e1) {
  if (n8 && grad_out == nullptr)
    return launch_cons_k1_n8(m, c, Phi, Pi, F, Phidot, bbuf, bc, rk, m.errflag, s, e0, e1);
  if (m.precision == 0) {
    WT_DISPATCH_N(m.N, (k1_dispatch<NN, double>(m, c, Phi, Pi, F, Phidot, bbuf, grad_out, use_metric, bc, rk, s, e0,
                                                e1)));
  } else {
    WT_DISPATCH_N(m.N, (k1_dispatch<NN, float>(m, c, Phi, Pi, F, Phidot, bbuf, grad_out, use_metric, bc, rk, s, e0,
                                               e1)));
  }
}

int launch_cons_k2(const DevMesh& m, const void* F, void* Pidot, const void* bbuf, int use_metric,
                   const ConsBC& bc, const RKStage& rk, unsigned int* nonfinite, cudaStream_t s, bool n8,
                   long long e0, long long e1) {
  if (n8) return launch_cons_k2_n8(m, F, Pidot, bbuf, bc, rk, m.errflag, s, e0, e1);
  if (m.precision == 0) {
    WT_DISPATCH_N(m.N, (k2_dispatch<NN, double>(m, F, Pidot, bbuf, use_metric, bc, rk, nonfinite, s, nullptr,
                                                nullptr, e0, e1)));
  } else {
    WT_DISPATCH_N(m.N, (k2_dispatch<NN, float>(m, F, Pidot, bbuf, use_metric, bc, rk, nonfinite, s, nullptr,
                                               nullptr, e0, e1)));
  }
}

int launch_div3d(const DevMesh& m, const void* F, void* out, cudaStream_t s) {
  // F: 3 consecutive fields
  ConsBC bc;
  RKStage rk;
  if (m.precision == 0) {
    WT_DISPATCH_N(m.N, (k2_dispatch<NN, double>(m, F, out, nullptr, 1, bc, rk, nullptr, s)));
  } else {
    WT_DISPATCH_N(m.N, (k2_dispatch<NN, float>(m, F, out, nullptr, 1, bc, rk, nullptr, s)));
  }
}

template <int N, typename real>
static int applyD_dispatch(const DevMesh& m, const void* u, void* out, int d, cudaStream_t s) {
  const unsigned blocks = (unsigned)((m.Ne + Ep<N>::EPB - 1) / Ep<N>::EPB);
  k_apply_D<N, real><<<blocks, Ep<N>::T, 0, s>>>(m.Ne, (const real*)u, (real*)out, d, (const real*)m.sdiag, m.nbr,
                                                 m.nbrf, m.bdry, m.G, m.H);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_apply_D(const DevMesh& m, const void* u, void* out, int d, cudaStream_t s) {
  if (m.precision == 0) {
    WT_DISPATCH_N(m.N, (applyD_dispatch<NN, double>(m, u, out, d, s)));
  } else {
    WT_DISPATCH_N(m.N, (applyD_dispatch<NN, float>(m, u, out, d, s)));
  }
}

template <typename real>
__global__ void k_axpy(long long n, real a, const real* __restrict__ x, real* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

// Kreiss-Oliger along axis d: on whole grid lines in shared memory where the
// elements form straight lines along d (k_ko_line), otherwise as the
// reference's _ko_axis3! does it (src/wave3d_curved.jl:182-192): six apply_D!
// calls ping-ponging through scratch (2 nn words), then dst += koT * result.
// The second form serves multi-patch meshes, whose axis-d neighbours may meet
// at another face or orientation.
template <int N, typename real>
static int ko_dispatch(const DevMesh& m, void* dst, const void* field, double koT, cudaStream_t s, void* scratch) {
  for (int d = 0; d < 3; ++d) {
    const int len = m.line_len[d];
    if (!m.line_ok[d] || len * N > 1024) {
      if (!scratch) return -4;
      real* buf[2] = {(real*)scratch, (real*)scratch + m.nn};
      const real* src = (const real*)field;
      for (int r = 0; r < 6; ++r) {
        if (applyD_dispatch<N, real>(m, src, buf[r & 1], d, s)) return -2;
        src = buf[r & 1];
      }
      k_axpy<real><<<4096, 256, 0, s>>>(m.nn, (real)koT, src, (real*)dst);
      if (cudaGetLastError() != cudaSuccess) return -2;
      continue;
    }
    dim3 grid((unsigned)m.nlines[d], N);
    size_t smem = (size_t)N * (len * N + 1) * sizeof(real) + (size_t)len * sizeof(int);
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_ko_line<N, real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_ko_line<N, real><<<grid, len * N, smem, s>>>(d, len, m.line_closed[d], m.lines[d], (real*)dst,
                                                   (const real*)field, (real)koT, (const real*)m.sdiag, m.G, m.H);
    if (cudaGetLastError() != cudaSuccess) return -2;
  }
  return 0;
}

int launch_ko_add(const DevMesh& m, void* dst, const void* field, double koT, cudaStream_t s, void* scratch) {
  if (m.precision == 0) {
    WT_DISPATCH_N(m.N, (ko_dispatch<NN, double>(m, dst, field, koT, s, scratch)));
  } else {
    WT_DISPATCH_N(m.N, (ko_dispatch<NN, float>(m, dst, field, koT, s, scratch)));
  }
}

int launch_cons_gen_batch(int which, int N, int precision, int epb_variant, int cp, const void* plist, const int2* tiles,
                          long long ntiles, cudaStream_t s) {
  WT_DISPATCH_N(N, (gen_batch_n<NN>(which, precision, epb_variant, cp != 0, plist, tiles, ntiles, s)));
}

// this file's bounds word (bounds-check build; 0 otherwise)
WT_BOUNDS_TAKE(bounds_take_cons)

}  // namespace wt
