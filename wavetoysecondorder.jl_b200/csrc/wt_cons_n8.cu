// wt_cons_n8.cu -- the n = 8 FP64 curvilinear hot path as persistent,
// TMA-pipelined, tensor-core kernels.
//
// Same arithmetic as k_cons_k1 / k_cons_k2 in wt_cons.cu (the split-form
// gradient / flux / Phidot and the split-form divergence of
// wave3d_curved_rhs!, src/wave3d_curved.jl:205-258, with the curvilinear
// Sommerfeld/Dirichlet pass of src/boundaries3d.jl:131-232 and the fused RK4
// stage update), organised for B200:
//   * one CTA of 8 warps per SM loops over elements (persistent grid);
//   * every per-node field of the next element (a contiguous 4 KB block per
//     field) is staged into shared memory by one elected thread with 1D bulk
//     copies (cp.async.bulk ... mbarrier::complete_tx) while the current
//     element computes -- a two-stage pipeline on two mbarriers, with bounded
//     waits that raise an error flag instead of spinning forever;
//   * the 8x8 reference-derivative contractions run on the FP64 tensor cores
//     (mma.sync.m8n8k4.f64): for axis al the element's 64 pencils are the N
//     dimension, G the A operand (held in registers for the whole kernel),
//     the staged field -- or the split-form product Ja*u / Ja.F formed while
//     loading the B fragment -- the B operand; warp w owns pencils 8w..8w+7;
//   * the three axes accumulate into a per-node smem array, then a node phase
//     (2 nodes per thread) adds the SATs, flux, boundary terms and the RK4
//     stage update and writes coalesced results.
// Neighbour face traces of the next element are prefetched into registers
// during the current element and parked in smem at the end of the iteration.
#include "wt_common.cuh"

namespace wt {

namespace n8 {

constexpr int N = 8, N2 = 64, N3 = 512, THREADS = 256;
constexpr unsigned FIELD_BYTES = N3 * sizeof(double);  // 4096
constexpr long long WAIT_LIMIT = 1LL << 24;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D (8x8) += A (8x4, row) * B (4x8, col), FP64 tensor core
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// node index of position p along axis al of pencil q (q = j+8k | i+8k | i+8j)
__device__ __forceinline__ int pnode(int al, int p, int q) {
  return al == 0 ? p + 8 * q : al == 1 ? (q & 7) + 8 * p + 64 * (q >> 3) : q + 64 * p;
}

// bounded wait on an mbarrier phase; returns false (and sets *err) on timeout
__device__ __forceinline__ bool wait_phase(uint64_t* bar, unsigned parity, unsigned* err) {
  for (long long it = 0; it < WAIT_LIMIT; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicOr(err, 2u);
  return false;
}

}  // namespace n8

// ---------------------------------------------------------------------------
// K1: staged fields per element: 0 Phi, 1 Pi, 2..11 c10, 12..20 Ja, 21 invJ,
// 22 y (stages 1, 2), 23 acc (stages 1..3).
struct K1N8 {
  long long Ne, nn;
  const double* Phi;
  const double* Pi;
  const double* c10;
  const double* Ja;
  const double* invdetJ;
  const int32_t* nbr;
  const int32_t* nbrf;
  const int32_t* bdry;
  const int32_t* bslot;
  const double* G;
  const double* H;
  double* F;
  double* Phidot;
  double* bbuf;
  int bc_on, exc_tag, nbf, kind;
  double sigma;
  const double* bnorm;
  const double* gPhi;
  const double* gPi;
  const double* gDx;
  const double* gDy;
  const double* gDz;
  int epi, stage;
  double dt;
  double* y;
  double* acc;
  double* out;
  unsigned* flag;
};

constexpr int K1_FIELDS = 24;
constexpr size_t K1_STAGE = (size_t)K1_FIELDS * n8::N3;  // doubles
constexpr size_t K1_SMEM = (2 * K1_STAGE + 3 * n8::N3 + 2 * 6 * n8::N2 + n8::N2) * sizeof(double) + 64;

__global__ void __launch_bounds__(n8::THREADS, 1) k_cons_k1_n8(const K1N8 P) {
  using namespace n8;
  extern __shared__ __align__(128) unsigned char smraw[];
  double* stg = reinterpret_cast<double*>(smraw);       // 2 stages
  double* sg = stg + 2 * K1_STAGE;                      // 3 x 512 gradient accumulators
  double* sface = sg + 3 * N3;                          // 2 x 6 x 64
  double* sG = sface + 2 * 6 * N2;                      // 64
  uint64_t* bar = reinterpret_cast<uint64_t*>(sG + N2);  // 2
  __shared__ int abort_flag;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tig = lane & 3;
  const long long nn = P.nn;
  const double Hend = P.H[0];
  const bool need_y = P.epi && (P.stage == 1 || P.stage == 2);
  const bool need_acc = P.epi && P.stage >= 1;
  const unsigned tx_bytes = (22u + (need_y ? 1u : 0u) + (need_acc ? 1u : 0u)) * FIELD_BYTES;

  if (tid < N2) sG[tid] = P.G[tid];
  if (tid == 0) {
    abort_flag = 0;
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();

  auto issue = [&](long long e, int s) {
    double* d = stg + s * K1_STAGE;
    const long long o = e * N3;
    fence_proxy_async();
    mbar_expect_tx(&bar[s], tx_bytes);
    bulk_g2s(d + 0 * N3, P.Phi + o, FIELD_BYTES, &bar[s]);
    bulk_g2s(d + 1 * N3, P.Pi + o, FIELD_BYTES, &bar[s]);
    for (int c = 0; c < 10; ++c) bulk_g2s(d + (2 + c) * N3, P.c10 + c * nn + o, FIELD_BYTES, &bar[s]);
    for (int c = 0; c < 9; ++c) bulk_g2s(d + (12 + c) * N3, P.Ja + c * nn + o, FIELD_BYTES, &bar[s]);
    bulk_g2s(d + 21 * N3, P.invdetJ + o, FIELD_BYTES, &bar[s]);
    if (need_y) bulk_g2s(d + 22 * N3, P.y + o, FIELD_BYTES, &bar[s]);
    if (need_acc) bulk_g2s(d + 23 * N3, P.acc + o, FIELD_BYTES, &bar[s]);
  };
  // neighbour Phi face traces of element e: 384 values, <= 2 per thread
  auto face_load = [&](long long e, double fr[2]) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int idx = tid + r * THREADS;
      double v = 0.0;
      if (e >= 0 && idx < 6 * N2) {
        const int f = idx >> 6, pq = idx & 63;
        const int en = P.nbr[f + 6 * e];
        if (en >= 0 && P.bdry[f + 6 * e] == 0) {
          const int fn = P.nbrf[f + 6 * e];
          v = P.Phi[(long long)en * N3 + face_node(faxis(fn), frow(fn, N), pq & 7, pq >> 3, N)];
        }
      }
      fr[r] = v;
    }
  };
  auto face_store = [&](int s, const double fr[2]) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int idx = tid + r * THREADS;
      if (idx < 6 * N2) sface[s * 6 * N2 + idx] = fr[r];
    }
  };

  long long e = blockIdx.x;
  if (e < P.Ne) {
    if (tid == 0) issue(e, 0);
    double fr[2];
    face_load(e, fr);
    face_store(0, fr);
  }
  __syncthreads();
  // A fragments of G: row g, columns 4 kc + tig
  const double aG0 = sG[gq * 8 + tig], aG1 = sG[gq * 8 + 4 + tig];

  for (int it = 0; e < P.Ne; ++it, e += gridDim.x) {
    const int s = it & 1;
    const unsigned parity = (it >> 1) & 1;
    const long long en = e + gridDim.x;
    if (tid == 0 && en < P.Ne) issue(en, s ^ 1);
    double fr[2];
    face_load(en < P.Ne ? en : -1, fr);
    if (!wait_phase(&bar[s], parity, P.flag)) abort_flag = 1;
    __syncthreads();
    if (abort_flag) {
      if (tid == 0 && en < P.Ne) wait_phase(&bar[s ^ 1], ((it + 1) >> 1) & 1, nullptr);
      return;
    }
    const double* d = stg + s * K1_STAGE;
    const double* sPhi = d;
    const double* sJa = d + 12 * N3;
    // ---- tensor-core contractions, one axis per phase ----
#pragma unroll 1
    for (int al = 0; al < 3; ++al) {
      double c[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
      const double* m0 = sJa + (al * 3 + 0) * N3;
      const double* m1 = sJa + (al * 3 + 1) * N3;
      const double* m2 = sJa + (al * 3 + 2) * N3;
#pragma unroll
      for (int kc = 0; kc < 2; ++kc) {
        const int nd = pnode(al, 4 * kc + tig, 8 * warp + gq);
        const double u = sPhi[nd];
        const double a = kc ? aG1 : aG0;
        dmma(c[0][0], c[0][1], a, u);
        dmma(c[1][0], c[1][1], a, m0[nd] * u);
        dmma(c[2][0], c[2][1], a, m1[nd] * u);
        dmma(c[3][0], c[3][1], a, m2[nd] * u);
      }
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int no = pnode(al, gq, 8 * warp + 2 * tig + b);
        const double du = c[0][b];
        const double r0 = 0.5 * c[1][b] + 0.5 * m0[no] * du;
        const double r1 = 0.5 * c[2][b] + 0.5 * m1[no] * du;
        const double r2 = 0.5 * c[3][b] + 0.5 * m2[no] * du;
        if (al == 0) {
          sg[no] = r0; sg[N3 + no] = r1; sg[2 * N3 + no] = r2;
        } else {
          sg[no] += r0; sg[N3 + no] += r1; sg[2 * N3 + no] += r2;
        }
      }
      __syncthreads();
    }
    // ---- node phase ----
    const double* sface_s = sface + s * 6 * N2;
#pragma unroll 1
    for (int r = 0; r < 2; ++r) {
      const int t = tid + r * THREADS;
      const int i = t & 7, j = (t >> 3) & 7, k = t >> 6;
      const long long n = e * N3 + t;
      const double u = sPhi[t];
      double g[3] = {sg[t], sg[N3 + t], sg[2 * N3 + t]};
      const int idx3[3] = {i, j, k};
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int ax = f >> 1;
        if (idx3[ax] != ((f & 1) ? 7 : 0)) continue;
        if (P.bdry[f + 6 * e] != 0 || P.nbr[f + 6 * e] < 0) continue;
        const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
        const double jump = sface_s[f * N2 + p + 8 * q] - u;
        const double nh = (f & 1) ? 1.0 : -1.0;
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) g[cc] += nh * sJa[(ax * 3 + cc) * N3 + t] * jump / (2.0 * Hend);
      }
      const double invJ = d[21 * N3 + t];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) g[cc] *= invJ;
      const double a = d[2 * N3 + t];
      const double b0 = d[3 * N3 + t], b1 = d[4 * N3 + t], b2 = d[5 * N3 + t];
      const double K0 = d[6 * N3 + t], K1v = d[7 * N3 + t], K2 = d[8 * N3 + t];
      const double K3 = d[9 * N3 + t], K4 = d[10 * N3 + t], K5 = d[11 * N3 + t];
      const double Pi = d[1 * N3 + t];
      const double F0 = b0 * Pi + (K0 * g[0] + K1v * g[1] + K2 * g[2]);
      const double F1 = b1 * Pi + (K1v * g[0] + K3 * g[1] + K4 * g[2]);
      const double F2 = b2 * Pi + (K2 * g[0] + K4 * g[1] + K5 * g[2]);
      double phid = b0 * g[0] + b1 * g[1] + b2 * g[2] + a * Pi;
      if (P.bc_on) {
        for (int f = 0; f < 6; ++f) {
          const int tag = P.bdry[f + 6 * e];
          if (tag == 0) continue;
          const int ax = f >> 1;
          if (idx3[ax] != ((f & 1) ? 7 : 0)) continue;
          const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
          const int slot = P.bslot[f + 6 * e];
          double dF = 0.0, dP = 0.0;
          if (tag != P.exc_tag) {
            const long long nb = (long long)P.nbf * N2;
            const long long bi = (long long)slot * N2 + p + 8 * q;
            const double nx = P.bnorm[bi], ny = P.bnorm[nb + bi], nz = P.bnorm[2 * nb + bi],
                         wt = P.bnorm[3 * nb + bi];
            const double Kn = K0 * nx * nx + K3 * ny * ny + K5 * nz * nz + 2.0 * (K1v * nx * ny + K2 * nx * nz + K4 * ny * nz);
            const double a_n = sqrt(a * Kn);
            const double bn = b0 * nx + b1 * ny + b2 * nz;
            if (P.kind == 4) {
              const double tau = P.sigma * (fabs(a_n - bn) + fabs(a_n + bn)) * wt;
              const double gp = P.gPhi ? P.gPhi[n] : 0.0, gqv = P.gPi ? P.gPi[n] : 0.0;
              dF = -tau * (u - gp);
              dP = -tau * (Pi - gqv);
            } else {
              const double qv = nx * g[0] + ny * g[1] + nz * g[2];
              const double rr = Pi + ((bn + a_n) / a) * qv;
              double gv = 0.0;
              if (P.kind != 2) {
                const double gqv = P.gPi ? P.gPi[n] : 0.0;
                const double gx = P.gDx ? P.gDx[n] : 0.0, gy = P.gDy ? P.gDy[n] : 0.0, gz = P.gDz ? P.gDz[n] : 0.0;
                gv = gqv + ((bn + a_n) / a) * (nx * gx + ny * gy + nz * gz);
              }
              dP = -P.sigma * fabs(a_n + bn) * wt * (rr - gv);
            }
          }
          phid += dF;
          P.bbuf[(long long)slot * N2 + p + 8 * q] = dP;
        }
      }
      P.F[n] = F0;
      P.F[nn + n] = F1;
      P.F[2 * nn + n] = F2;
      if (P.epi) {
        const double dt = P.dt;
        if (P.stage == 0) {
          P.out[n] = u + (0.5 * dt) * phid;
          P.acc[n] = u + (dt / 6.0) * phid;
        } else if (P.stage == 1) {
          P.out[n] = d[22 * N3 + t] + (0.5 * dt) * phid;
          P.acc[n] = d[23 * N3 + t] + (dt / 3.0) * phid;
        } else if (P.stage == 2) {
          P.out[n] = d[22 * N3 + t] + dt * phid;
          P.acc[n] = d[23 * N3 + t] + (dt / 3.0) * phid;
        } else {
          const double v = d[23 * N3 + t] + (dt / 6.0) * phid;
          P.y[n] = v;
          if (P.flag && !isfinite(v)) atomicOr(P.flag, 1u);
        }
      } else {
        P.Phidot[n] = phid;
      }
    }
    face_store(s ^ 1, fr);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// K2: staged fields per element: 0..2 F, 3..11 Ja, 12 invJ, 13 y (stages 0..2),
// 14 acc (stages 1..3).
struct K2N8 {
  long long Ne, nn;
  const double* F0;
  const double* F1;
  const double* F2;
  const double* Ja;
  const double* invdetJ;
  const int32_t* nbr;
  const int32_t* nbrf;
  const int32_t* bdry;
  const int32_t* bslot;
  const double* G;
  const double* H;
  const double* bbuf;
  int bc_on;
  double* Pidot;
  int epi, stage;
  double dt;
  double* y;
  double* acc;
  double* out;
  unsigned* flag;
};

constexpr int K2_FIELDS = 15;
constexpr size_t K2_STAGE = (size_t)K2_FIELDS * n8::N3;
constexpr size_t K2_SMEM = (2 * K2_STAGE + n8::N3 + 2 * 6 * 3 * n8::N2 + n8::N2) * sizeof(double) + 64;

__global__ void __launch_bounds__(n8::THREADS, 1) k_cons_k2_n8(const K2N8 P) {
  using namespace n8;
  extern __shared__ __align__(128) unsigned char smraw[];
  double* stg = reinterpret_cast<double*>(smraw);
  double* sdiv = stg + 2 * K2_STAGE;                     // 512
  double* sface = sdiv + N3;                             // 2 x 6 x 3 x 64
  double* sG = sface + 2 * 6 * 3 * N2;                   // 64
  uint64_t* bar = reinterpret_cast<uint64_t*>(sG + N2);
  __shared__ int abort_flag;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tig = lane & 3;
  const long long nn = P.nn;
  const double Hend = P.H[0];
  const bool need_y = P.epi && P.stage <= 2;
  const bool need_acc = P.epi && P.stage >= 1;
  const unsigned tx_bytes = (13u + (need_y ? 1u : 0u) + (need_acc ? 1u : 0u)) * FIELD_BYTES;
  const double* Fp[3] = {P.F0, P.F1, P.F2};

  if (tid < N2) sG[tid] = P.G[tid];
  if (tid == 0) {
    abort_flag = 0;
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();

  auto issue = [&](long long e, int s) {
    double* d = stg + s * K2_STAGE;
    const long long o = e * N3;
    fence_proxy_async();
    mbar_expect_tx(&bar[s], tx_bytes);
    for (int c = 0; c < 3; ++c) bulk_g2s(d + c * N3, Fp[c] + o, FIELD_BYTES, &bar[s]);
    for (int c = 0; c < 9; ++c) bulk_g2s(d + (3 + c) * N3, P.Ja + c * nn + o, FIELD_BYTES, &bar[s]);
    bulk_g2s(d + 12 * N3, P.invdetJ + o, FIELD_BYTES, &bar[s]);
    if (need_y) bulk_g2s(d + 13 * N3, P.y + o, FIELD_BYTES, &bar[s]);
    if (need_acc) bulk_g2s(d + 14 * N3, P.acc + o, FIELD_BYTES, &bar[s]);
  };
  // neighbour flux face traces: 6 faces x 3 components x 64 = 1152 values
  constexpr int NF = 6 * 3 * N2;
  constexpr int PER = (NF + THREADS - 1) / THREADS;  // 5
  auto face_load = [&](long long e, double fr[PER]) {
#pragma unroll
    for (int r = 0; r < PER; ++r) {
      const int idx = tid + r * THREADS;
      double v = 0.0;
      if (e >= 0 && idx < NF) {
        const int f = idx / (3 * N2), rem = idx - f * 3 * N2, c = rem >> 6, pq = rem & 63;
        const int en = P.nbr[f + 6 * e];
        if (en >= 0 && P.bdry[f + 6 * e] == 0) {
          const int fn = P.nbrf[f + 6 * e];
          v = Fp[c][(long long)en * N3 + face_node(faxis(fn), frow(fn, N), pq & 7, pq >> 3, N)];
        }
      }
      fr[r] = v;
    }
  };
  auto face_store = [&](int s, const double fr[PER]) {
#pragma unroll
    for (int r = 0; r < PER; ++r) {
      const int idx = tid + r * THREADS;
      if (idx < NF) sface[s * NF + idx] = fr[r];
    }
  };

  long long e = blockIdx.x;
  if (e < P.Ne) {
    if (tid == 0) issue(e, 0);
    double fr[PER];
    face_load(e, fr);
    face_store(0, fr);
  }
  __syncthreads();
  const double aG0 = sG[gq * 8 + tig], aG1 = sG[gq * 8 + 4 + tig];

  for (int it = 0; e < P.Ne; ++it, e += gridDim.x) {
    const int s = it & 1;
    const unsigned parity = (it >> 1) & 1;
    const long long en = e + gridDim.x;
    if (tid == 0 && en < P.Ne) issue(en, s ^ 1);
    double fr[PER];
    face_load(en < P.Ne ? en : -1, fr);
    if (!wait_phase(&bar[s], parity, P.flag)) abort_flag = 1;
    __syncthreads();
    if (abort_flag) {
      if (tid == 0 && en < P.Ne) wait_phase(&bar[s ^ 1], ((it + 1) >> 1) & 1, nullptr);
      return;
    }
    const double* d = stg + s * K2_STAGE;
    const double* sF = d;
    const double* sJa = d + 3 * N3;
#pragma unroll 1
    for (int al = 0; al < 3; ++al) {
      double c[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
      const double* m0 = sJa + (al * 3 + 0) * N3;
      const double* m1 = sJa + (al * 3 + 1) * N3;
      const double* m2 = sJa + (al * 3 + 2) * N3;
#pragma unroll
      for (int kc = 0; kc < 2; ++kc) {
        const int nd = pnode(al, 4 * kc + tig, 8 * warp + gq);
        const double f0 = sF[nd], f1 = sF[N3 + nd], f2 = sF[2 * N3 + nd];
        const double ft = m0[nd] * f0 + m1[nd] * f1 + m2[nd] * f2;
        const double a = kc ? aG1 : aG0;
        dmma(c[0][0], c[0][1], a, ft);
        dmma(c[1][0], c[1][1], a, f0);
        dmma(c[2][0], c[2][1], a, f1);
        dmma(c[3][0], c[3][1], a, f2);
      }
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int no = pnode(al, gq, 8 * warp + 2 * tig + b);
        const double r = 0.5 * c[0][b] + (0.5 * m0[no] * c[1][b] + 0.5 * m1[no] * c[2][b] + 0.5 * m2[no] * c[3][b]);
        if (al == 0) sdiv[no] = r;
        else sdiv[no] += r;
      }
      __syncthreads();
    }
    const double* sface_s = sface + s * NF;
#pragma unroll 1
    for (int r = 0; r < 2; ++r) {
      const int t = tid + r * THREADS;
      const int i = t & 7, j = (t >> 3) & 7, k = t >> 6;
      const long long n = e * N3 + t;
      double dv = sdiv[t];
      const int idx3[3] = {i, j, k};
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int ax = f >> 1;
        if (idx3[ax] != ((f & 1) ? 7 : 0)) continue;
        if (P.bdry[f + 6 * e] != 0 || P.nbr[f + 6 * e] < 0) continue;
        const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
        const double nh = (f & 1) ? 1.0 : -1.0;
        double sacc = 0.0;
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
          sacc += sJa[(ax * 3 + cc) * N3 + t] * (sface_s[(f * 3 + cc) * N2 + p + 8 * q] - sF[cc * N3 + t]);
        dv += nh * sacc / (2.0 * Hend);
      }
      dv *= d[12 * N3 + t];
      if (P.bc_on) {
        for (int f = 0; f < 6; ++f) {
          if (P.bdry[f + 6 * e] == 0) continue;
          const int ax = f >> 1;
          if (idx3[ax] != ((f & 1) ? 7 : 0)) continue;
          const int p = ax == 0 ? j : i, q = ax == 2 ? j : k;
          dv += P.bbuf[(long long)P.bslot[f + 6 * e] * N2 + p + 8 * q];
        }
      }
      if (P.epi) {
        const double dt = P.dt;
        if (P.stage == 0) {
          const double yv = d[13 * N3 + t];
          P.out[n] = yv + (0.5 * dt) * dv;
          P.acc[n] = yv + (dt / 6.0) * dv;
        } else if (P.stage == 1) {
          P.out[n] = d[13 * N3 + t] + (0.5 * dt) * dv;
          P.acc[n] = d[14 * N3 + t] + (dt / 3.0) * dv;
        } else if (P.stage == 2) {
          P.out[n] = d[13 * N3 + t] + dt * dv;
          P.acc[n] = d[14 * N3 + t] + (dt / 3.0) * dv;
        } else {
          const double v = d[14 * N3 + t] + (dt / 6.0) * dv;
          P.y[n] = v;
          if (P.flag && !isfinite(v)) atomicOr(P.flag, 1u);
        }
      } else {
        P.Pidot[n] = dv;
      }
    }
    face_store(s ^ 1, fr);
    __syncthreads();
  }
}

static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

int launch_cons_k1_n8(const DevMesh& m, const DevCoef& c, const void* Phi, const void* Pi, void* F, void* Phidot,
                      void* bbuf, const ConsBC& bc, const RKStage& rk, unsigned* flag, cudaStream_t s) {
  K1N8 P;
  P.Ne = m.Ne; P.nn = m.nn;
  P.Phi = (const double*)Phi; P.Pi = (const double*)Pi; P.c10 = (const double*)c.c10;
  P.Ja = (const double*)m.Ja_r; P.invdetJ = (const double*)m.invdetJ_r;
  P.nbr = m.nbr; P.nbrf = m.nbrf; P.bdry = m.bdry; P.bslot = m.bslot; P.G = m.G; P.H = m.H;
  P.F = (double*)F; P.Phidot = (double*)Phidot; P.bbuf = (double*)bbuf;
  P.bc_on = bc.on; P.exc_tag = bc.exc_tag; P.nbf = m.nbf; P.kind = bc.kinds[0]; P.sigma = bc.sigma;
  P.bnorm = (const double*)m.bnorm;
  P.gPhi = (const double*)bc.gPhi; P.gPi = (const double*)bc.gPi;
  P.gDx = (const double*)bc.gDx; P.gDy = (const double*)bc.gDy; P.gDz = (const double*)bc.gDz;
  P.epi = rk.on; P.stage = rk.stage; P.dt = rk.dt;
  P.y = (double*)rk.y; P.acc = (double*)rk.acc; P.out = (double*)rk.out; P.flag = flag;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_cons_k1_n8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K1_SMEM);
    attr = true;
  }
  const long long grid = m.Ne < sm_count() ? m.Ne : sm_count();
  k_cons_k1_n8<<<(unsigned)grid, n8::THREADS, K1_SMEM, s>>>(P);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_cons_k2_n8(const DevMesh& m, const void* F, void* Pidot, const void* bbuf, const ConsBC& bc,
                      const RKStage& rk, unsigned* flag, cudaStream_t s) {
  K2N8 P;
  P.Ne = m.Ne; P.nn = m.nn;
  P.F0 = (const double*)F; P.F1 = (const double*)F + m.nn; P.F2 = (const double*)F + 2 * m.nn;
  P.Ja = (const double*)m.Ja_r; P.invdetJ = (const double*)m.invdetJ_r;
  P.nbr = m.nbr; P.nbrf = m.nbrf; P.bdry = m.bdry; P.bslot = m.bslot; P.G = m.G; P.H = m.H;
  P.bbuf = (const double*)bbuf; P.bc_on = bc.on;
  P.Pidot = (double*)Pidot;
  P.epi = rk.on; P.stage = rk.stage; P.dt = rk.dt;
  P.y = (double*)rk.y; P.acc = (double*)rk.acc; P.out = (double*)rk.out; P.flag = flag;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_cons_k2_n8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K2_SMEM);
    attr = true;
  }
  const long long grid = m.Ne < sm_count() ? m.Ne : sm_count();
  k_cons_k2_n8<<<(unsigned)grid, n8::THREADS, K2_SMEM, s>>>(P);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace wt
