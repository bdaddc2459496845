// wt_cons_n8.cu -- the n = 8 FP64 curvilinear hot path as persistent,
// TMA-pipelined, tensor-core kernels.
//
// Same arithmetic as k_cons_k1 / k_cons_k2 in wt_cons.cu (the split-form
// gradient / flux / Phidot and the split-form divergence of
// wave3d_curved_rhs!, src/wave3d_curved.jl:205-258, with the curvilinear
// boundary pass of src/boundaries3d.jl:131-232 and the fused RK4 stage
// update), organised for B200:
//   * one CTA of 16 warps per SM loops over elements (persistent grid);
//   * the fields the derivative contractions read at other nodes of an
//     element (Phi and the nine metric terms in K1; the three flux components
//     and the metric terms in K2) are staged into shared memory with 1D bulk
//     copies (cp.async.bulk ... mbarrier::complete_tx), one copy per field
//     block; the metric terms and the flux live in global memory in a
//     plane-padded element layout (k-plane stride 68 doubles) that makes the
//     tensor-core operand loads (nearly) bank-conflict-free.  A ring of
//     NSTAGE stages keeps NSTAGE - 1 elements in flight; every wait is
//     bounded and raises an error flag instead of spinning forever;
//   * the fields used only at their own node (background coefficients, Pi,
//     1/J, the RK4 state) are prefetched into registers one element ahead;
//   * the 8x8 reference-derivative contractions run on the FP64 tensor cores
//     (mma.sync.m8n8k4.f64): for axis al an element's 64 pencils are the N
//     dimension, G the A operand (in registers), the staged field -- or the
//     split-form product Ja*u / Ja.F formed while loading -- the B operand.
//     Warp w owns pencil tile w&7; warps w and w+8 split the fields of a tile,
//     and every axis writes its own partial sums, so one barrier separates
//     the contraction pass from the node pass.  The centred-flux SATs are
//     added in the same pass: an output row l = 0 or 7 of the MMA is the node
//     row on face 2al or 2al+1;
//   * a node phase (one node per thread) forms flux, Phidot / divergence,
//     boundary terms (boundary elements only) and the RK4 stage update and
//     writes coalesced results;
//   * per-element tables (SAT face mask, neighbour face sources) are loaded
//     one element before the neighbour traces they address, so no load in
//     the loop waits on another load.
#include "wt_common.cuh"

namespace wt {

namespace n8 {

constexpr int N = 8, N2 = 64, N3 = 512, THREADS = 512;
constexpr int PS = 68;             // padded k-plane stride (doubles)
constexpr int FS = 8 * PS;         // padded field size (544 doubles = 4352 B)
constexpr long long WAIT_LIMIT = 1LL << 24;
// staged elements in flight: element e + (NSTAGE - 1) * grid is copied while e
// is processed
constexpr int NSTAGE = 2;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
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
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
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

__device__ __forceinline__ int pad(int i, int j, int k) { return i + 8 * j + PS * k; }
// padded index -> unpadded node index (i + 8 j + 64 k)
__device__ __forceinline__ int unpad(int d) { return d - (PS - 64) * (d / PS); }

// Per-lane operand / output node offsets (padded) for axis al, tile w:
//   B operand: position p = 4 kc + tig along al, pencil slot g;
//   outputs:   row l = g along al, pencil slot 2 tig + b.
// Pencil orders: al=0 (j = w, k = slot); al=1 (i = slot, k = w); al=2 (i = slot, j = w).
__device__ __forceinline__ int bnode(int al, int w, int kc, int g, int tig) {
  const int p = 4 * kc + tig;
  return al == 0 ? pad(p, w, g) : al == 1 ? pad(g, p, w) : pad(g, w, p);
}
__device__ __forceinline__ int onode(int al, int w, int b, int g, int tig) {
  const int sl = 2 * tig + b;
  return al == 0 ? pad(g, w, sl) : al == 1 ? pad(sl, g, w) : pad(sl, w, g);
}
// face-trace index (p + 8 q) of an output node on the al-face
__device__ __forceinline__ int opq(int al, int w, int b, int tig) {
  const int sl = 2 * tig + b;
  return al == 0 ? w + 8 * sl : al == 1 ? sl + 8 * w : sl + 8 * w;
}

__device__ __forceinline__ bool wait_phase(uint64_t* bar, unsigned parity, unsigned* err) {
  for (long long it = 0; it < WAIT_LIMIT; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicOr(err, 2u);
  return false;
}

}  // namespace n8

// ---------------------------------------------------------------------------
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
  const int32_t* emask;
  const int32_t* fsrc;
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

// K1 staged fields: Phi (unpadded, 512) and Ja (9 padded fields, one 4352-byte
// block each from the padded global copy).  Register prefetch: c10 (10), Pi,
// invJ, y, acc.
constexpr size_t K1_STAGE = (size_t)n8::N3 + 9 * (size_t)n8::FS;
constexpr size_t K1_SMEM = (n8::NSTAGE * K1_STAGE + 9 * n8::FS + 2 * 6 * n8::N2 + n8::N2) * sizeof(double) + 64;

__global__ void __launch_bounds__(n8::THREADS, 1) k_cons_k1_n8(const K1N8 P) {
  using namespace n8;
  extern __shared__ __align__(128) unsigned char smraw[];
  double* stg = reinterpret_cast<double*>(smraw);       // 2 stages x 10 padded fields
  double* sg = stg + NSTAGE * K1_STAGE;                      // 9 padded partial gradients [al*3 + c]
  double* sface = sg + 9 * FS;                          // 2 x 6 x 64
  double* sG = sface + 2 * 6 * N2;                      // 64
  uint64_t* bar = reinterpret_cast<uint64_t*>(sG + N2);  // NSTAGE
  __shared__ int abort_flag;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tig = lane & 3, wt8 = warp & 7, half = warp >> 3;
  const long long nn = P.nn;
  const double inv2H = 1.0 / (2.0 * P.H[0]);
  const bool need_y = P.epi && (P.stage == 1 || P.stage == 2);
  const bool need_acc = P.epi && P.stage >= 1;
  const unsigned tx_bytes = N3 * 8u + 9u * FS * 8u;
  // node-phase coordinates of this thread
  const int ti = tid & 7, tj = (tid >> 3) & 7, tk = tid >> 6;
  const int tpad = pad(ti, tj, tk);

  if (tid < N2) sG[tid] = P.G[tid];
  if (tid == 0) {
    abort_flag = 0;
    for (int k = 0; k < NSTAGE; ++k) mbar_init(&bar[k], 1);
    fence_barrier_init();
  }
  __syncthreads();

  // warp 0 stages element e into stage s: 10 whole-block copies
  auto issue = [&](long long e, int s) {
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[s], tx_bytes);
    }
    __syncwarp();
    double* d = stg + s * K1_STAGE;
    if (lane == 0) bulk_g2s(d, P.Phi + e * N3, N3 * 8u, &bar[s]);
    else if (lane <= 9)
      bulk_g2s(d + N3 + (lane - 1) * FS, P.Ja + ((long long)(lane - 1) * P.Ne + e) * FS, FS * 8u, &bar[s]);
  };
  // neighbour Phi face traces (384 values; threads 0..383).  The face source
  // (8 * neighbour + neighbour face) of an element is loaded one iteration
  // before the trace itself, so no load waits on another inside the loop.
  const int my_f = tid >> 6, my_pq = tid & 63;
  auto src_load = [&](long long e) -> int { return (e >= 0 && tid < 6 * N2) ? P.fsrc[my_f + 6 * e] : -1; };
  auto face_load = [&](int src) -> double {
    if (src < 0) return 0.0;
    const int fn = src & 7;
    return P.Phi[(long long)(src >> 3) * N3 + face_node(faxis(fn), frow(fn, N), my_pq & 7, my_pq >> 3, N)];
  };
  // pointwise fields of this thread's node
  struct PW {
    double c[10], Pi, invJ, y, acc;
  };
  auto pw_load = [&](long long e, PW& w) {
    if (e < 0) return;
    const long long n = e * N3 + tid;
#pragma unroll
    for (int c = 0; c < 10; ++c) w.c[c] = P.c10[c * nn + n];
    w.Pi = P.Pi[n];
    w.invJ = P.invdetJ[n];
    w.y = need_y ? P.y[n] : 0.0;
    w.acc = need_acc ? P.acc[n] : 0.0;
  };

  long long e = blockIdx.x;
  PW cur;
  int emcur = 0, src1 = -1;
  if (e < P.Ne) {
    if (warp == 0)
      for (int k = 0; k < NSTAGE - 1; ++k)
        if (e + k * (long long)gridDim.x < P.Ne) issue(e + k * (long long)gridDim.x, k);
    emcur = P.emask[e];
    const double fv = face_load(src_load(e));
    if (tid < 6 * N2) sface[tid] = fv;
    pw_load(e, cur);
    src1 = src_load(e + gridDim.x < P.Ne ? e + gridDim.x : -1);
  }
  __syncthreads();
  const double aG0 = sG[gq * 8 + tig], aG1 = sG[gq * 8 + 4 + tig];

  for (int it = 0; e < P.Ne; ++it, e += gridDim.x) {
    const int s = it % NSTAGE, fb = it & 1;
    const unsigned parity = (it / NSTAGE) & 1;
    const long long en = e + gridDim.x, enn = en + gridDim.x;
    const bool has_next = en < P.Ne;
    const int emnext = has_next ? P.emask[en] : 0;
    const int src2 = src_load(enn < P.Ne ? enn : -1);
    const double fnext = face_load(has_next ? src1 : -1);
    PW nxt;
    pw_load(has_next ? en : -1, nxt);
    if (!wait_phase(&bar[s], parity, P.flag)) abort_flag = 1;
    // After this barrier every thread has finished the previous element, so its
    // stage (reused for element e + (NSTAGE - 1) grid), the partial gradients
    // and face buffer fb^1 are free.
    __syncthreads();
    if (abort_flag) {  // wait (bounded) for the copies still in flight, then leave
      if (warp == 0 && lane == 0)
        for (int k = 1; k < NSTAGE - 1; ++k)
          if (e + k * (long long)gridDim.x < P.Ne) wait_phase(&bar[(it + k) % NSTAGE], ((it + k) / NSTAGE) & 1, nullptr);
      return;
    }
    {
      const long long ei = e + (NSTAGE - 1) * (long long)gridDim.x;
      if (warp == 0 && ei < P.Ne) issue(ei, (it + NSTAGE - 1) % NSTAGE);
    }
    const double* d = stg + s * K1_STAGE;
    const double* sPhi = d;      // unpadded
    const double* sJa = d + N3;  // 9 padded fields, index (al*3 + c)
    const double* sfc = sface + fb * 6 * N2;
    const int mask = emcur & 63;
    const int bnd = emcur >> 6;
    // ---- tensor-core contractions ----
    // Each axis writes its own partial gradients sg[al*3 + c], so the axes need
    // no barrier between them.  Per pencil tile, warp w (half 0) does axis 0
    // and components 0, 1 of axis 1; warp w + 8 (half 1) component 2 of axis 1
    // and axis 2: 7 and 6 contraction chains.
    // comps: bit c set = produce component c of axis al.  The centred-flux SAT
    // of an interior al-face is added to the output rows on that face (row 0:
    // face 2 al, row 7: face 2 al + 1).
    auto grad_axis = [&](int al, int comps) {
      double cu[2] = {0, 0}, cm[3][2] = {{0, 0}, {0, 0}, {0, 0}};
#pragma unroll
      for (int kc = 0; kc < 2; ++kc) {
        const int nd = bnode(al, wt8, kc, gq, tig);
        const double u = sPhi[unpad(nd)];
        const double a = kc ? aG1 : aG0;
        dmma(cu[0], cu[1], a, u);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if ((comps >> c) & 1) dmma(cm[c][0], cm[c][1], a, sJa[(al * 3 + c) * FS + nd] * u);
      }
      const int sface_f = gq == 0 ? 2 * al : gq == 7 ? 2 * al + 1 : -1;
      const bool sat = sface_f >= 0 && ((mask >> sface_f) & 1);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int no = onode(al, wt8, b, gq, tig);
        double jump = 0.0;
        if (sat) jump = (gq ? inv2H : -inv2H) * (sfc[sface_f * N2 + opq(al, wt8, b, tig)] - sPhi[unpad(no)]);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if ((comps >> c) & 1) {
            const double m = sJa[(al * 3 + c) * FS + no];
            double r = 0.5 * cm[c][b] + 0.5 * m * cu[b];
            if (sat) r += m * jump;
            sg[(al * 3 + c) * FS + no] = r;
          }
      }
    };
    if (half == 0) {
      grad_axis(0, 7);
      grad_axis(1, 3);
    } else {
      grad_axis(1, 4);
      grad_axis(2, 7);
    }
    __syncthreads();
    // ---- node phase: one node per thread ----
    {
      const long long n = e * N3 + tid;
      const double u = sPhi[tid];
      double g0 = (sg[tpad] + sg[3 * FS + tpad]) + sg[6 * FS + tpad];
      double g1 = (sg[FS + tpad] + sg[4 * FS + tpad]) + sg[7 * FS + tpad];
      double g2 = (sg[2 * FS + tpad] + sg[5 * FS + tpad]) + sg[8 * FS + tpad];
      g0 *= cur.invJ; g1 *= cur.invJ; g2 *= cur.invJ;
      const double a = cur.c[0];
      const double b0 = cur.c[1], b1 = cur.c[2], b2 = cur.c[3];
      const double K0 = cur.c[4], K1v = cur.c[5], K2 = cur.c[6], K3 = cur.c[7], K4 = cur.c[8], K5 = cur.c[9];
      const double Pi = cur.Pi;
      const double F0 = b0 * Pi + (K0 * g0 + K1v * g1 + K2 * g2);
      const double F1 = b1 * Pi + (K1v * g0 + K3 * g1 + K4 * g2);
      const double F2 = b2 * Pi + (K2 * g0 + K4 * g1 + K5 * g2);
      double phid = b0 * g0 + b1 * g1 + b2 * g2 + a * Pi;
      if (bnd && P.bc_on) {
        const int idx3[3] = {ti, tj, tk};
        for (int f = 0; f < 6; ++f) {
          const int tag = P.bdry[f + 6 * e];
          if (tag == 0) continue;
          const int ax = f >> 1;
          if (idx3[ax] != ((f & 1) ? 7 : 0)) continue;
          const int p = ax == 0 ? tj : ti, q = ax == 2 ? tj : tk;
          const int slot = P.bslot[f + 6 * e];
          double dF = 0.0, dP = 0.0;
          if (tag != P.exc_tag) {
            const long long nb = (long long)P.nbf * N2;
            const long long bi = (long long)slot * N2 + p + 8 * q;
            const double nx = P.bnorm[bi], ny = P.bnorm[nb + bi], nz = P.bnorm[2 * nb + bi], wt = P.bnorm[3 * nb + bi];
            const double Kn =
                K0 * nx * nx + K3 * ny * ny + K5 * nz * nz + 2.0 * (K1v * nx * ny + K2 * nx * nz + K4 * ny * nz);
            const double a_n = sqrt(a * Kn);
            const double bn = b0 * nx + b1 * ny + b2 * nz;
            if (P.kind == 4) {
              const double tau = P.sigma * (fabs(a_n - bn) + fabs(a_n + bn)) * wt;
              const double gp = P.gPhi ? P.gPhi[n] : 0.0, gqv = P.gPi ? P.gPi[n] : 0.0;
              dF = -tau * (u - gp);
              dP = -tau * (Pi - gqv);
            } else {
              const double qv = nx * g0 + ny * g1 + nz * g2;
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
      {  // flux in the padded element-block layout read by K2
        const long long fo = e * FS + tpad, fstr = P.Ne * FS;
        P.F[fo] = F0;
        P.F[fstr + fo] = F1;
        P.F[2 * fstr + fo] = F2;
      }
      if (P.epi) {
        const double dt = P.dt;
        if (P.stage == 0) {
          P.out[n] = u + (0.5 * dt) * phid;
          P.acc[n] = u + (dt / 6.0) * phid;
        } else if (P.stage == 1) {
          P.out[n] = cur.y + (0.5 * dt) * phid;
          P.acc[n] = cur.acc + (dt / 3.0) * phid;
        } else if (P.stage == 2) {
          P.out[n] = cur.y + dt * phid;
          P.acc[n] = cur.acc + (dt / 3.0) * phid;
        } else {
          const double v = cur.acc + (dt / 6.0) * phid;
          P.y[n] = v;
          if (P.flag && !isfinite(v)) atomicOr(P.flag, 1u);
        }
      } else {
        P.Phidot[n] = phid;
      }
    }
    if (has_next && tid < 6 * N2) sface[(fb ^ 1) * 6 * N2 + tid] = fnext;
    cur = nxt;
    emcur = emnext;
    src1 = src2;
  }
}

// ---------------------------------------------------------------------------
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
  const int32_t* emask;
  const int32_t* fsrc;
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

// K2 staged fields: 0..2 F, 3..11 Ja.  Register prefetch: invJ, y, acc.
constexpr int K2_NF = 12;
constexpr size_t K2_STAGE = (size_t)K2_NF * n8::FS;
constexpr size_t K2_SMEM = (n8::NSTAGE * K2_STAGE + 6 * n8::FS + 2 * 6 * 3 * n8::N2 + n8::N2) * sizeof(double) + 64;

__global__ void __launch_bounds__(n8::THREADS, 1) k_cons_k2_n8(const K2N8 P) {
  using namespace n8;
  extern __shared__ __align__(128) unsigned char smraw[];
  double* stg = reinterpret_cast<double*>(smraw);
  double* sdiv = stg + NSTAGE * K2_STAGE;                     // 6 padded partial divergences [al*2 + half]
  double* sface = sdiv + 6 * FS;                         // 2 x 6 x 3 x 64
  double* sG = sface + 2 * 6 * 3 * N2;                   // 64
  uint64_t* bar = reinterpret_cast<uint64_t*>(sG + N2);
  __shared__ int abort_flag;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tig = lane & 3, wt8 = warp & 7, half = warp >> 3;
  const double inv2H = 1.0 / (2.0 * P.H[0]);
  const bool need_y = P.epi && P.stage <= 2;
  const bool need_acc = P.epi && P.stage >= 1;
  const unsigned tx_bytes = K2_NF * FS * 8u;
  const int ti = tid & 7, tj = (tid >> 3) & 7, tk = tid >> 6;
  const int tpad = pad(ti, tj, tk);
  constexpr int NFACE = 6 * 3 * N2;  // 1152

  if (tid < N2) sG[tid] = P.G[tid];
  if (tid == 0) {
    abort_flag = 0;
    for (int k = 0; k < NSTAGE; ++k) mbar_init(&bar[k], 1);
    fence_barrier_init();
  }
  __syncthreads();

  auto issue = [&](long long e, int s) {
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[s], tx_bytes);
    }
    __syncwarp();
    double* d = stg + s * K2_STAGE;
    if (lane < K2_NF) {
      const double* src = lane < 3 ? (lane == 0 ? P.F0 : lane == 1 ? P.F1 : P.F2) + e * FS
                                   : P.Ja + ((long long)(lane - 3) * P.Ne + e) * FS;
      bulk_g2s(d + lane * FS, src, FS * 8u, &bar[s]);
    }
  };
  // neighbour flux face traces: [f][c][pq], 1152 values, <= 3 per thread; the
  // face sources are loaded one iteration ahead of the traces (see K1)
  auto src_load = [&](long long e, int src[3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int idx = tid + r * THREADS;
      src[r] = (e >= 0 && idx < NFACE) ? P.fsrc[idx / (3 * N2) + 6 * e] : -1;
    }
  };
  auto face_load = [&](const int src[3], double fv[3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int idx = tid + r * THREADS;
      double v = 0.0;
      if (src[r] >= 0) {
        const int rem = idx % (3 * N2), c = rem >> 6, pq = rem & 63;
        const int fn = src[r] & 7;
        const double* Fc = c == 0 ? P.F0 : c == 1 ? P.F1 : P.F2;
        const int fnode = face_node(faxis(fn), frow(fn, N), pq & 7, pq >> 3, N);
        v = Fc[(long long)(src[r] >> 3) * FS + pad(fnode & 7, (fnode >> 3) & 7, fnode >> 6)];
      }
      fv[r] = v;
    }
  };
  struct PW {
    double invJ, y, acc;
  };
  auto pw_load = [&](long long e, PW& w) {
    if (e < 0) return;
    const long long n = e * N3 + tid;
    w.invJ = P.invdetJ[n];
    w.y = need_y ? P.y[n] : 0.0;
    w.acc = need_acc ? P.acc[n] : 0.0;
  };

  long long e = blockIdx.x;
  PW cur;
  int emcur = 0, src1[3] = {-1, -1, -1};
  if (e < P.Ne) {
    if (warp == 0)
      for (int k = 0; k < NSTAGE - 1; ++k)
        if (e + k * (long long)gridDim.x < P.Ne) issue(e + k * (long long)gridDim.x, k);
    emcur = P.emask[e];
    int src0[3];
    src_load(e, src0);
    double fv[3];
    face_load(src0, fv);
#pragma unroll
    for (int r = 0; r < 3; ++r)
      if (tid + r * THREADS < NFACE) sface[tid + r * THREADS] = fv[r];
    pw_load(e, cur);
    src_load(e + gridDim.x < P.Ne ? e + gridDim.x : -1, src1);
  }
  __syncthreads();
  const double aG0 = sG[gq * 8 + tig], aG1 = sG[gq * 8 + 4 + tig];

  for (int it = 0; e < P.Ne; ++it, e += gridDim.x) {
    const int s = it % NSTAGE, fb = it & 1;
    const unsigned parity = (it / NSTAGE) & 1;
    const long long en = e + gridDim.x, enn = en + gridDim.x;
    const bool has_next = en < P.Ne;
    const int emnext = has_next ? P.emask[en] : 0;
    int src2[3];
    src_load(enn < P.Ne ? enn : -1, src2);
    double fnext[3];
    face_load(src1, fnext);
    PW nxt;
    pw_load(has_next ? en : -1, nxt);
    if (!wait_phase(&bar[s], parity, P.flag)) abort_flag = 1;
    __syncthreads();  // the previous element is finished: its stage and the buffers are free (see K1)
    if (abort_flag) {  // wait (bounded) for the copies still in flight, then leave
      if (warp == 0 && lane == 0)
        for (int k = 1; k < NSTAGE - 1; ++k)
          if (e + k * (long long)gridDim.x < P.Ne) wait_phase(&bar[(it + k) % NSTAGE], ((it + k) / NSTAGE) & 1, nullptr);
      return;
    }
    {
      const long long ei = e + (NSTAGE - 1) * (long long)gridDim.x;
      if (warp == 0 && ei < P.Ne) issue(ei, (it + NSTAGE - 1) % NSTAGE);
    }
    const double* d = stg + s * K2_STAGE;
    const double* sF = d;           // 3 fields
    const double* sJa = d + 3 * FS;  // 9 fields
    const double* sfc = sface + fb * NFACE;
    const int mask = emcur & 63;
    const int bnd = emcur >> 6;
    // per-axis partial divergences sg[al*2 + half]: no barrier between axes
#pragma unroll
    for (int al = 0; al < 3; ++al) {
      const double* m0 = sJa + (al * 3 + 0) * FS;
      const double* m1 = sJa + (al * 3 + 1) * FS;
      const double* m2 = sJa + (al * 3 + 2) * FS;
      double cx[2] = {0, 0}, cy[2] = {0, 0};
#pragma unroll
      for (int kc = 0; kc < 2; ++kc) {
        const int nd = bnode(al, wt8, kc, gq, tig);
        const double a = kc ? aG1 : aG0;
        if (half == 0) {
          // contravariant flux Ja^al . F and F_0
          const double f0 = sF[nd];
          const double ft = m0[nd] * f0 + m1[nd] * sF[FS + nd] + m2[nd] * sF[2 * FS + nd];
          dmma(cx[0], cx[1], a, ft);
          dmma(cy[0], cy[1], a, f0);
        } else {
          dmma(cx[0], cx[1], a, sF[FS + nd]);
          dmma(cy[0], cy[1], a, sF[2 * FS + nd]);
        }
      }
      // half 1 adds the centred-flux SAT of an interior al-face on its rows
      const int sface_f = gq == 0 ? 2 * al : gq == 7 ? 2 * al + 1 : -1;
      const bool sat = half == 1 && sface_f >= 0 && ((mask >> sface_f) & 1);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int no = onode(al, wt8, b, gq, tig);
        double r;
        if (half == 0) {
          r = 0.5 * cx[b] + 0.5 * m0[no] * cy[b];
        } else {
          r = 0.5 * m1[no] * cx[b] + 0.5 * m2[no] * cy[b];
        }
        if (sat) {
          const int pq = opq(al, wt8, b, tig);
          const double sacc = m0[no] * (sfc[(sface_f * 3 + 0) * N2 + pq] - sF[no]) +
                              m1[no] * (sfc[(sface_f * 3 + 1) * N2 + pq] - sF[FS + no]) +
                              m2[no] * (sfc[(sface_f * 3 + 2) * N2 + pq] - sF[2 * FS + no]);
          r += (gq ? inv2H : -inv2H) * sacc;
        }
        sdiv[(al * 2 + half) * FS + no] = r;
      }
    }
    __syncthreads();
    {
      const long long n = e * N3 + tid;
      double dv = ((sdiv[tpad] + sdiv[2 * FS + tpad]) + sdiv[4 * FS + tpad]) +
                  ((sdiv[FS + tpad] + sdiv[3 * FS + tpad]) + sdiv[5 * FS + tpad]);
      dv *= cur.invJ;
      if (bnd && P.bc_on) {
        const int idx3[3] = {ti, tj, tk};
        for (int f = 0; f < 6; ++f) {
          if (P.bdry[f + 6 * e] == 0) continue;
          const int ax = f >> 1;
          if (idx3[ax] != ((f & 1) ? 7 : 0)) continue;
          const int p = ax == 0 ? tj : ti, q = ax == 2 ? tj : tk;
          dv += P.bbuf[(long long)P.bslot[f + 6 * e] * N2 + p + 8 * q];
        }
      }
      if (P.epi) {
        const double dt = P.dt;
        if (P.stage == 0) {
          P.out[n] = cur.y + (0.5 * dt) * dv;
          P.acc[n] = cur.y + (dt / 6.0) * dv;
        } else if (P.stage == 1) {
          P.out[n] = cur.y + (0.5 * dt) * dv;
          P.acc[n] = cur.acc + (dt / 3.0) * dv;
        } else if (P.stage == 2) {
          P.out[n] = cur.y + dt * dv;
          P.acc[n] = cur.acc + (dt / 3.0) * dv;
        } else {
          const double v = cur.acc + (dt / 6.0) * dv;
          P.y[n] = v;
          if (P.flag && !isfinite(v)) atomicOr(P.flag, 1u);
        }
      } else {
        P.Pidot[n] = dv;
      }
    }
    if (has_next) {
#pragma unroll
      for (int r = 0; r < 3; ++r)
        if (tid + r * THREADS < NFACE) sface[(fb ^ 1) * NFACE + tid + r * THREADS] = fnext[r];
    }
    cur = nxt;
    emcur = emnext;
#pragma unroll
    for (int r = 0; r < 3; ++r) src1[r] = src2[r];
  }
}

// padded element-block copy of the nine metric-term fields for the n = 8 path
__global__ void k_pad_fields(long long Ne, int nf, const double* __restrict__ src, double* __restrict__ dst) {
  const long long total = (long long)nf * Ne * n8::N3;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
    const long long f = x / (Ne * n8::N3);
    const long long r = x - f * Ne * n8::N3;
    const long long e = r / n8::N3;
    const int t = (int)(r - e * n8::N3);
    dst[(f * Ne + e) * n8::FS + n8::pad(t & 7, (t >> 3) & 7, t >> 6)] = src[x];
  }
}

int launch_pad_metric_n8(DevMesh& m, cudaStream_t s) {
  k_pad_fields<<<4096, 256, 0, s>>>(m.Ne, 9, m.Ja, m.Ja_n8);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

long long n8_padded_field_size(long long Ne) { return Ne * n8::FS; }

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
  P.Ja = (const double*)m.Ja_n8; P.invdetJ = (const double*)m.invdetJ_r;
  P.nbr = m.nbr; P.nbrf = m.nbrf; P.bdry = m.bdry; P.bslot = m.bslot; P.G = m.G; P.H = m.H;
  P.emask = m.emask; P.fsrc = m.fsrc;
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
  P.F0 = (const double*)F; P.F1 = (const double*)F + m.Ne * n8::FS; P.F2 = (const double*)F + 2 * m.Ne * n8::FS;
  P.Ja = (const double*)m.Ja_n8; P.invdetJ = (const double*)m.invdetJ_r;
  P.nbr = m.nbr; P.nbrf = m.nbrf; P.bdry = m.bdry; P.bslot = m.bslot; P.G = m.G; P.H = m.H;
  P.emask = m.emask; P.fsrc = m.fsrc;
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
