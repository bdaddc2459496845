// wt_cons_n8.cu -- the n = 8 curvilinear hot path as persistent,
// bulk-copy-pipelined, tensor-core kernels, in two precision forms.
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
//     block; the metric terms and the flux live in global memory in an
//     element layout that makes the shared-memory accesses bank-conflict-free
//     (FP64: an XOR swizzle of the node index; FP32: k-planes padded to 68
//     words; see Lay below).  A ring of
//     NSTAGE stages keeps NSTAGE - 1 elements in flight; one thread polls
//     each stage's mbarrier, the rest wait at the CTA barrier; every wait is
//     bounded and raises an error flag instead of spinning forever;
//   * the fields used only at their own node (background coefficients, Pi,
//     1/J, the RK4 state) are prefetched into registers one element ahead;
//   * the 8x8 reference-derivative contractions run on tensor cores.  For
//     axis al an element's 64 pencils form 8 tiles of 8 (the MMA N
//     dimension); warp w owns tile w&7 and warps w and w+8 split the fields
//     of a tile.  Every axis writes its own partial sums, so one barrier
//     separates the contraction pass from the node pass.  The centred-flux
//     SATs are added in the same pass: output row l = 0 or 7 of the MMA is
//     the node row on face 2al or 2al+1.
//       FP64 form: mma.sync.m8n8k4.f64, G the A operand in registers, the
//       staged field -- or the split-form product Ja*u / Ja.F formed while
//       loading -- the B operand.
//       FP32 forms: split-precision BF16, mma.sync.m16n8k16 with FP32
//       accumulation.  Three-term split (default): G and the operand v are
//       split into bf16 terms hi + mid + lo (24 significant bits, as FP32);
//       MMA 1 with A = [[G_hi, G_hi], [G_mid, G_mid]], B = [v_hi; v_mid] and
//       MMA 2 with A = [[G_hi, G_lo], [G_mid, 0]], B = [v_lo; v_hi] sum every
//       product down to relative size 2^-16 (rows 0-7 and 8-15 added in
//       FP32).  Two-term split (hi + lo): one MMA with A = [[G_hi, G_hi],
//       [G_lo, G_lo]], B = [v_hi; v_lo]; it carries ~16 significant bits and
//       misses FP32 accuracy by a factor of ~30 on the n = 8 warped workload,
//       so it is kept only for the precision study; there, because every row
//       of G sums to zero, the operand is taken relative to its value at node
//       3 of the pencil (D(v - c) = D v), so the split error scales with the
//       variation of the field along the pencil, not with its size;
//   * a node phase (one node per thread) forms flux, Phidot / divergence,
//     boundary terms (boundary elements only) and the RK4 stage update and
//     writes coalesced results (FP32 form: Kahan-compensated final sum);
//   * per-element tables (SAT face mask, neighbour face sources) are loaded
//     one element before the neighbour traces they address, so no load in
//     the loop waits on another load.
#include "wt_common.cuh"
#include "../../include/wavetoy_b200.h"

#include <cuda_bf16.h>
#include <type_traits>

namespace wt {

namespace n8 {

constexpr int N = 8, N2 = 64, N3 = 512, THREADS = 512;
constexpr int PS = 68;             // padded k-plane stride (words)
constexpr int FS = 8 * PS;         // padded field size (544 words)
constexpr long long WAIT_LIMIT = 1LL << 24;
// staged elements in flight: element e + (NSTAGE - 1) * grid is copied while e
// is processed
constexpr int NSTAGE = 2;
constexpr int PREF = 3;            // two-term FP32 form: pencil node whose value is the operand offset

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

__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

// D (16x8, FP32) += A (16x16 bf16, row) * B (16x8 bf16, col); b0 holds rows
// k = 2 tig, 2 tig + 1 and b1 rows k = 8 + 2 tig, 9 + 2 tig of column n = group.
__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// Split-precision contraction of the two operand values this lane holds
// (positions 2 tig, 2 tig + 1 of pencil `group`): NT = 3 three-term split
// (two MMAs, a1/a2 from split_G), NT = 2 hi + lo (one MMA with a1).
template <int NT>
__device__ __forceinline__ void mma_split(float d[4], const uint32_t a1[4], const uint32_t a2[4], float v0, float v1) {
  const __nv_bfloat162 hi = __floats2bfloat162_rn(v0, v1);
  const float2 hf = __bfloat1622float2(hi);
  const float r0 = v0 - hf.x, r1 = v1 - hf.y;
  const __nv_bfloat162 mid = __floats2bfloat162_rn(r0, r1);
  if constexpr (NT == 2) {
    mma_bf16(d, a1, bf2_bits(hi), bf2_bits(mid));
  } else {
    const float2 mf = __bfloat1622float2(mid);
    const __nv_bfloat162 lo = __floats2bfloat162_rn(r0 - mf.x, r1 - mf.y);
    mma_bf16(d, a1, bf2_bits(hi), bf2_bits(mid));
    mma_bf16(d, a2, bf2_bits(lo), bf2_bits(hi));
  }
}

__device__ __forceinline__ int pad(int i, int j, int k) { return i + 8 * j + PS * k; }

// Element-block layouts of the staged fields (the same in global memory and in
// shared memory, since a bulk copy moves the block verbatim).  n = i + 8 j + 64 k.
//   FP64: 512 words, the node index with bits 0, 2, 3 XOR-ed by bits 4-8
//     (bit0 ^= b4 ^ b6, bit2 ^= b4 ^ b6 ^ b8, bit3 ^= b7).  Each half-warp of
//     every 64-bit access the kernels make -- tensor-core operands along any
//     axis (position 4 kc + tig, pencil slot gq), accumulator rows (position
//     gq, slot 2 tig + b) and node order -- then touches 16 distinct 8-byte
//     bank pairs, i.e. no bank conflicts, and no padding is needed.
//   FP32: 544 words, k-planes padded to a stride of 68 words.
template <typename real>
struct Lay;
template <>
struct Lay<double> {
  static constexpr int FS = 512;
  __device__ __forceinline__ static int at(int n) {
    const int b4 = (n >> 4) & 1, b6 = (n >> 6) & 1, b7 = (n >> 7) & 1, b8 = (n >> 8) & 1;
    return n ^ ((b4 ^ b6) | ((b4 ^ b6 ^ b8) << 2) | (b7 << 3));
  }
};
template <>
struct Lay<float> {
  static constexpr int FS = ::wt::n8::FS;
  __device__ __forceinline__ static int at(int n) { return pad(n & 7, (n >> 3) & 7, n >> 6); }
};
// K1's Phi (the caller's unpadded element block).  FP64: every thread loads
// its node one element ahead (coalesced) and stores it into a double buffer in
// the Lay<double> layout (REG = true, conflict-free like the other fields;
// copying it by rows instead needs many small bulk copies, which the copy
// engine serialises).  FP32: one bulk copy into the stage (unpadded).
template <typename real>
struct PhiLay;
template <>
struct PhiLay<double> {
  static constexpr bool REG = true;
  static constexpr int SZ = 0;  // words in the stage
  __device__ __forceinline__ static int at(int n) { return Lay<double>::at(n); }
};
template <>
struct PhiLay<float> {
  static constexpr bool REG = false;
  static constexpr int SZ = N3;
  __device__ __forceinline__ static int at(int n) { return n; }
};

// Node of tile w for axis al at position p along al, pencil slot g.
// Pencil orders: al=0 (j = w, k = slot); al=1 (i = slot, k = w); al=2 (i = slot, j = w).
__device__ __forceinline__ int bn(int al, int w, int p, int g) {
  return al == 0 ? p + 8 * w + 64 * g : al == 1 ? g + 8 * p + 64 * w : g + 8 * w + 64 * p;
}
// FP64 B operand: position p = 4 kc + tig along al, pencil slot g
__device__ __forceinline__ int bnode(int al, int w, int kc, int g, int tig) { return bn(al, w, 4 * kc + tig, g); }
// outputs (both forms): row l = g along al, pencil slot 2 tig + b
__device__ __forceinline__ int onode(int al, int w, int b, int g, int tig) { return bn(al, w, g, 2 * tig + b); }
// face-trace index (p + 8 q) of an output node on the al-face
__device__ __forceinline__ int opq(int al, int w, int b, int tig) {
  const int sl = 2 * tig + b;
  return al == 0 ? w + 8 * sl : sl + 8 * w;
}

__device__ __forceinline__ bool wait_phase(uint64_t* bar, unsigned parity, unsigned* err) {
  for (long long it = 0; it < WAIT_LIMIT; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicOr(err, 2u);
  return false;
}

// A operand fragments of the FP32 forms (register i: rows gq / gq + 8 for
// i = 0, 2 / 1, 3; columns k < 8 for i < 2, k >= 8 otherwise).
//   NT = 3: a1 = [[G_hi, G_hi], [G_mid, G_mid]], a2 = [[G_hi, G_lo], [G_mid, 0]]
//   NT = 2: a1 = [[G_hi, G_hi], [G_lo, G_lo]]   (G_lo = the second term)
__device__ __forceinline__ void split_G(const double* G, int gq, int tig, int nt, uint32_t a1[4], uint32_t a2[4]) {
  const double g0 = G[gq * 8 + 2 * tig], g1 = G[gq * 8 + 2 * tig + 1];
  const __nv_bfloat162 hi = __floats2bfloat162_rn((float)g0, (float)g1);
  const float2 hf = __bfloat1622float2(hi);
  const double r0 = g0 - (double)hf.x, r1 = g1 - (double)hf.y;
  const __nv_bfloat162 mid = __floats2bfloat162_rn((float)r0, (float)r1);
  const float2 mf = __bfloat1622float2(mid);
  const __nv_bfloat162 lo = __floats2bfloat162_rn((float)(r0 - (double)mf.x), (float)(r1 - (double)mf.y));
  a1[0] = bf2_bits(hi);
  a1[1] = bf2_bits(mid);
  a1[2] = bf2_bits(hi);
  a1[3] = bf2_bits(mid);
  a2[0] = bf2_bits(hi);
  a2[1] = bf2_bits(mid);
  a2[2] = nt == 3 ? bf2_bits(lo) : 0u;
  a2[3] = 0u;
}

// resident CTAs per SM
template <typename real>
struct Occ {
  static constexpr int k1 = 1, k2 = 1;
};
template <>
struct Occ<float> {
  static constexpr int k1 = 2, k2 = 2;
};
// K1 stages the ten background coefficients with the copies instead of
// prefetching them into registers (FP32: two CTAs then fit on an SM; FP64:
// the registers go to the contraction pass)
template <typename real>
struct StageCoef {
  static constexpr bool value = true;
};

}  // namespace n8

// RK4 stage update shared by both kernels (see rk_epilogue in wt_cons.cu):
// with comp (FP32 state) acc holds the step increment and the final sum is
// Kahan-compensated, comp holding the low part the FP32 state lost (the state
// is y + comp); yv, accv, compv are this node's prefetched values.
template <typename real>
__device__ __forceinline__ void n8_rk(int stage, double dt, real k, real yin, real yv, real accv, real compv,
                                      long long n, real* y, real* acc, real* out, real* comp, unsigned* flag) {
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
      if (flag && !isfinite(v)) atomicOr(flag, 1u);
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
    const real v = accv + (real)(dt / 6.0) * k;
    y[n] = v;
    if (flag && !isfinite(v)) atomicOr(flag, 1u);
  }
}

// RK4 stage update of the compensated FP32 form (Phi in K1, CP): the state is
// the pair (y, lo) = (high, low part); the stage the next K1 reads is y + out
// with out = lo + c dt k, so the stage value keeps the state's low part and
// rounds only the small increment; acc holds the step increment; the step's
// final sum is formed in FP64 and split again into y and lo.  Stage 2 also
// copies y into hcopy, which stage 3 reads in place of y.  hi, accv, lov:
// this node's y, acc and lo.
__device__ __forceinline__ void n8_rk_cp(int stage, double dt, float k, float hi, float accv, float lov, long long n,
                                         float* y, float* acc, float* out, float* lo, float* hcopy, unsigned* flag) {
  if (stage == 0) {
    out[n] = lov + (float)(0.5 * dt) * k;
    acc[n] = (float)(dt / 6.0) * k;
  } else if (stage == 1) {
    out[n] = lov + (float)(0.5 * dt) * k;
    acc[n] = accv + (float)(dt / 3.0) * k;
  } else if (stage == 2) {
    out[n] = lov + (float)dt * k;
    acc[n] = accv + (float)(dt / 3.0) * k;
    hcopy[n] = hi;
  } else {
    const float inc = accv + (float)(dt / 6.0) * k;
    const double v = (double)hi + ((double)lov + (double)inc);
    const float h = (float)v;
    y[n] = h;
    lo[n] = (float)(v - (double)h);
    if (flag && !isfinite(h)) atomicOr(flag, 1u);
  }
}

// ---------------------------------------------------------------------------
template <typename real>
struct K1N8 {
  long long Ne, nn;
  long long e0;  // single-solve launches: the first element (the launch covers ntiles elements from it)
  const real* Phi;
  const real* Pi;
  const real* c10;
  const real* Ja;
  const real* invdetJ;
  const int32_t* nbr;
  const int32_t* nbrf;
  const int32_t* bdry;
  const int32_t* bslot;
  const int32_t* emask;
  const int32_t* fsrc;
  const double* G;
  const double* H;
  real* F;
  real* Phidot;
  real* bbuf;
  int bc_on, exc_tag, nbf, kind;
  double sigma;
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
  unsigned* flag;
  float Gh[64];  // 0.5 G in FP32 (the CUDA-core form reads it from the constant bank)
  real* gout;    // gradient-only launches (GR): the three components of the split-form gradient
  // Compensated FP32 form (cp = 1, CUDA-core kernels): the Phi the stage reads is
  // Phi + Phit, with Phit the low part of the state at stage 0 and the previous
  // stage's small output after it (NULL: zero); the split-form gradient of it is
  // evaluated in FP64 with the metric terms split into an element-constant FP64
  // part Ja0 [9e + al*3 + c] and an FP32 deviation dJa (LayC blocks).
  // Stage 3 reads a copy of the state's high part that stage 2 writes (hcopy),
  // so that stage 3 may overwrite the state while neighbours still read it.
  int cp;
  const real* Phit;
  const real* dJa;
  const double* Ja0;
  real* hcopy;
  double Gd[64];  // 0.5 G in FP64
};

// Boundary terms of K1 at a node on an outer face (the curvilinear boundary
// pass of src/boundaries3d.jl:131-232): characteristic SAT into phid and the
// Pi boundary contribution into bbuf (read by K2).  cc: the ten coefficients.
template <typename real>
__device__ __forceinline__ void k1_boundary(const K1N8<real>& Q, long long e, int ti, int tj, int tk, long long n,
                                            real u, real Pi, real g0, real g1, real g2, const real cc[10],
                                            real& phid) {
  using n8::N2;
  const real a = cc[0];
  const real b0 = cc[1], b1 = cc[2], b2 = cc[3];
  const real K0 = cc[4], K1v = cc[5], K2 = cc[6], K3 = cc[7], K4 = cc[8], K5 = cc[9];
  const int idx3[3] = {ti, tj, tk};
  for (int f = 0; f < 6; ++f) {
    const int tag = Q.bdry[f + 6 * e];
    if (tag == 0) continue;
    const int ax = f >> 1;
    if (idx3[ax] != ((f & 1) ? 7 : 0)) continue;
    const int p = ax == 0 ? tj : ti, q = ax == 2 ? tj : tk;
    const int slot = ::wt::bc_slot(Q.bslot[f + 6 * e], Q.nbf);
    real dF = 0, dP = 0;
    if (tag != Q.exc_tag) {
      const long long nb = (long long)Q.nbf * N2;
      const long long bi = (long long)slot * N2 + p + 8 * q;
      const real nx = Q.bnorm[bi], ny = Q.bnorm[nb + bi], nz = Q.bnorm[2 * nb + bi], wt = Q.bnorm[3 * nb + bi];
      const real Kn =
          K0 * nx * nx + K3 * ny * ny + K5 * nz * nz + (real)2 * (K1v * nx * ny + K2 * nx * nz + K4 * ny * nz);
      const real a_n = sqrt(a * Kn);
      const real bn_ = b0 * nx + b1 * ny + b2 * nz;
      const real sigma = (real)Q.sigma;
      if (Q.kind == 4) {
        const real tau = sigma * (fabs(a_n - bn_) + fabs(a_n + bn_)) * wt;
        const real gp = Q.gPhi ? Q.gPhi[n] : (real)0, gqv = Q.gPi ? Q.gPi[n] : (real)0;
        dF = -tau * (u - gp);
        dP = -tau * (Pi - gqv);
      } else {
        const real qv = nx * g0 + ny * g1 + nz * g2;
        const real rr = Pi + ((bn_ + a_n) / a) * qv;
        real gv = 0;
        if (Q.kind != 2) {
          const real gqv = Q.gPi ? Q.gPi[n] : (real)0;
          const real gx = Q.gDx ? Q.gDx[n] : (real)0, gy = Q.gDy ? Q.gDy[n] : (real)0,
                     gz = Q.gDz ? Q.gDz[n] : (real)0;
          gv = gqv + ((bn_ + a_n) / a) * (nx * gx + ny * gy + nz * gz);
        }
        dP = -sigma * fabs(a_n + bn_) * wt * (rr - gv);
      }
    }
    phid += dF;
    Q.bbuf[(long long)slot * N2 + p + 8 * q] = dP;
  }
}

// K1 staged fields: Phi (PhiLay), Ja (9 fields in the Lay layout, one block
// each from the global copy) and the ten coefficient fields (unpadded, read in
// node order).  Register prefetch: Pi, invJ, y, acc, comp.
template <typename real>
__host__ __device__ constexpr size_t k1_stage() {
  return (size_t)n8::PhiLay<real>::SZ + 9 * (size_t)n8::Lay<real>::FS +
         (n8::StageCoef<real>::value ? 10 * (size_t)n8::N3 : 0);
}
template <typename real>
constexpr size_t k1_smem() {
  return (n8::NSTAGE * k1_stage<real>() + 9 * n8::Lay<real>::FS + 2 * 6 * n8::N2 +
          (n8::PhiLay<real>::REG ? 2 * n8::N3 : 0)) *
             sizeof(real) +
         n8::N2 * sizeof(double) + 64;
}

// NT: FP32 split terms (3 or 2); ignored by the FP64 form.  BATCH: the
// persistent loop runs over a work list of (solve, element) tiles and every
// tile reads the parameter block of its solve (plist); P then only supplies
// what is common to the launch (stage, operator, status word).
// GR: gradient-only instantiation (the energy's apply_gradient3d!, src/wave3d_curved.jl:275-280):
// no coefficients, Pi or RK state are read; the node phase writes the gradient to P.gout.
template <typename real, int NT, bool BATCH, bool GR = false>
__global__ void __launch_bounds__(n8::THREADS, n8::Occ<real>::k1)
    k_cons_k1_n8(const K1N8<real> P, const K1N8<real>* __restrict__ plist, const int2* __restrict__ tiles,
                 long long ntiles) {
  using namespace n8;
  constexpr bool F64 = std::is_same<real, double>::value;
  constexpr bool SC = StageCoef<real>::value;
  constexpr int NCOPY_C = SC && !GR ? 10 : 0;  // coefficient blocks copied per stage
  constexpr size_t K1_STAGE = k1_stage<real>();
  constexpr int FS = Lay<real>::FS, PSZ = PhiLay<real>::SZ;
  extern __shared__ __align__(128) unsigned char smraw[];
  double* sG = reinterpret_cast<double*>(smraw);                // 64 (FP64 operator)
  real* stg = reinterpret_cast<real*>(sG + N2);                 // NSTAGE stages x 10 fields
  real* sg = stg + NSTAGE * K1_STAGE;                           // 9 padded partial gradients [al*3 + c]
  real* sface = sg + 9 * FS;                                    // 2 x 6 x 64
  real* sphi = sface + 2 * 6 * N2;                              // PhiLay::REG: 2 x 512 (Lay)
  constexpr bool PHIR = PhiLay<real>::REG;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sphi + (PHIR ? 2 * N3 : 0));  // NSTAGE
  __shared__ int abort_flag;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tig = lane & 3, wt8 = warp & 7, half = warp >> 3;
  const real inv2H = (real)(1.0 / (2.0 * P.H[0]));
  const bool comp_on = !F64 && P.epi && P.comp != nullptr;  // FP32 state only
  const bool need_y = P.epi && (P.stage == 1 || P.stage == 2 || (comp_on && P.stage == 3));
  const bool need_acc = P.epi && P.stage >= 1;
  const bool need_comp = comp_on && P.stage == 3;
  const unsigned tx_bytes = (unsigned)((K1_STAGE - (SC ? 10 - NCOPY_C : 0) * (size_t)N3) * sizeof(real));
  // node-phase coordinates of this thread
  const int ti = tid & 7, tj = (tid >> 3) & 7, tk = tid >> 6;
  const int tpad = Lay<real>::at(tid), tphi = PhiLay<real>::at(tid);
  const long long T = ntiles;
  const long long GS = gridDim.x;
  // tile t = (solve, element); (-1, -1) past the end
  auto tile_at = [&](long long t) -> int2 {
    if (t >= T) return make_int2(-1, -1);
    if constexpr (BATCH) return tiles[t];
    else return make_int2(0, (int)(P.e0 + t));
  };
  auto prm = [&](int sidx) -> const K1N8<real>& {
    if constexpr (BATCH) return plist[sidx];
    else return P;
  };

  if (tid < N2) sG[tid] = P.G[tid];
  if (tid == 0) {
    abort_flag = 0;
    for (int k = 0; k < NSTAGE; ++k) mbar_init(&bar[k], 1);
    fence_barrier_init();
  }
  __syncthreads();

  // warp 0 stages tile tl into stage s: whole-block copies
  auto issue = [&](int2 tl, int s) {
    const K1N8<real>& Q = prm(tl.x);
    const long long e = tl.y;
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[s], tx_bytes);
    }
    __syncwarp();
    real* d = stg + s * K1_STAGE;
    // copies: Phi (unless it goes through registers), 9 Ja, 10 coefficients
    constexpr int NPHI = PHIR ? 0 : 1;
    for (int c = lane; c < NPHI + 9 + NCOPY_C; c += 32) {
      if (c < NPHI) {
        bulk_g2s(d, Q.Phi + e * N3, N3 * (unsigned)sizeof(real), &bar[s]);
      } else if (c < NPHI + 9) {
        const int f = c - NPHI;
        bulk_g2s(d + PSZ + f * FS, Q.Ja + ((long long)f * Q.Ne + e) * FS, FS * (unsigned)sizeof(real), &bar[s]);
      } else {
        const int f = c - NPHI - 9;
        bulk_g2s(d + PSZ + 9 * FS + f * N3, Q.c10 + f * Q.nn + e * N3, N3 * (unsigned)sizeof(real), &bar[s]);
      }
    }
  };
  // neighbour Phi face traces (384 values; threads 0..383).  The face source
  // (8 * neighbour + neighbour face) of a tile is loaded one iteration before
  // the trace itself, and the tile two iterations before, so no load waits on
  // another inside the loop.
  const int my_f = tid >> 6, my_pq = tid & 63;
  auto src_load = [&](int2 tl) -> int { return (tl.x >= 0 && tid < 6 * N2) ? ::wt::bc_src(prm(tl.x).fsrc[my_f + 6 * tl.y], prm(tl.x).Ne) : -1; };
  auto face_load = [&](int src, int sidx) -> real {
    if (src < 0) return (real)0;
    return prm(sidx).Phi[(long long)(src >> 6) * N3 + nbr_face_node(src, my_pq & 7, my_pq >> 3, N)];
  };
  auto emask_at = [&](int2 tl) -> int { return tl.x >= 0 ? prm(tl.x).emask[tl.y] : 0; };
  // pointwise fields of this thread's node
  struct PW {
    real c[10], Pi, invJ, y, acc, comp, phi;
  };
  auto pw_load = [&](int2 tl, PW& w) {
    if (tl.x < 0) return;
    const K1N8<real>& Q = prm(tl.x);
    const long long n = (long long)tl.y * N3 + tid;
    if constexpr (PHIR) w.phi = Q.Phi[n];
    w.invJ = Q.invdetJ[n];
    if constexpr (GR) return;
    if constexpr (!SC) {
#pragma unroll
      for (int c = 0; c < 10; ++c) w.c[c] = Q.c10[c * Q.nn + n];
    }
    w.Pi = Q.Pi[n];
    w.y = need_y ? Q.y[n] : (real)0;
    w.acc = need_acc ? Q.acc[n] : (real)0;
    w.comp = need_comp ? Q.comp[n] : (real)0;
  };

  int2 t0 = tile_at(blockIdx.x), t1 = tile_at(blockIdx.x + GS), t2 = tile_at(blockIdx.x + 2 * GS);
  PW cur;
  int emcur = 0, src1 = -1;
  if (t0.x >= 0) {
    if (warp == 0)
      for (int k = 0; k < NSTAGE - 1; ++k) {
        const int2 tk_ = tile_at(blockIdx.x + k * GS);
        if (tk_.x >= 0) issue(tk_, k);
      }
    emcur = emask_at(t0);
    const real fv = face_load(src_load(t0), t0.x);
    if (tid < 6 * N2) sface[tid] = fv;
    pw_load(t0, cur);
    if constexpr (PHIR) sphi[tphi] = cur.phi;
    src1 = src_load(t1);
  }
  __syncthreads();
  // A operand: FP64 G entries (rows gq, columns tig and 4 + tig); FP32 split pairs
  double aG0 = 0.0, aG1 = 0.0;
  uint32_t aS[4] = {0, 0, 0, 0}, aS2[4] = {0, 0, 0, 0};
  if constexpr (F64) {
    aG0 = sG[gq * 8 + tig];
    aG1 = sG[gq * 8 + 4 + tig];
  } else {
    split_G(sG, gq, tig, NT, aS, aS2);
  }

  int it = 0;
  for (long long t = blockIdx.x; t < T; t += GS, ++it) {
    const int s = it % NSTAGE, fb = it & 1;
    const unsigned parity = (it / NSTAGE) & 1;
    // tiles t, t + grid, t + 2 grid: carried in registers for a work list (loaded
    // ahead), recomputed from t for a single solve
    int2 t3 = make_int2(-1, -1);
    if constexpr (BATCH) {
      t3 = tile_at(t + 3 * GS);
    } else {
      t0 = tile_at(t);
      t1 = tile_at(t + GS);
      t2 = tile_at(t + 2 * GS);
    }
    const bool has_next = t1.x >= 0;
    const int emnext = emask_at(t1);
    const int src2 = src_load(t2);
    const real fnext = face_load(has_next ? src1 : -1, t1.x);
    PW nxt;
    pw_load(t1, nxt);
    // One thread polls the stage's mbarrier (its acquire makes the copied data
    // visible; the barrier below orders every other thread after it), so the
    // other warps do not spend issue slots spinning.
    if (tid == 0 && !wait_phase(&bar[s], parity, P.flag)) abort_flag = 1;
    // After this barrier every thread has finished the previous element, so its
    // stage (reused for tile t + (NSTAGE - 1) grid), the partial gradients and
    // face buffer fb^1 are free.
    __syncthreads();
    if (abort_flag) {  // wait (bounded) for the copies still in flight, then leave
      if (warp == 0 && lane == 0)
        for (int k = 1; k < NSTAGE - 1; ++k)
          if (tile_at(t + k * GS).x >= 0) wait_phase(&bar[(it + k) % NSTAGE], ((it + k) / NSTAGE) & 1, nullptr);
      return;
    }
    {
      const int2 ti_ = NSTAGE == 2 ? t1 : tile_at(t + (NSTAGE - 1) * GS);
      if (warp == 0 && ti_.x >= 0) issue(ti_, (it + NSTAGE - 1) % NSTAGE);
    }
    const K1N8<real>& Q = prm(t0.x);
    const long long e = t0.y;
    const real* d = stg + s * K1_STAGE;
    const real* sPhi = PHIR ? sphi + fb * N3 : d;  // PhiLay
    const real* sJa = d + PSZ;                      // 9 fields (Lay), index (al*3 + c)
    const real* sfc = sface + fb * 6 * N2;
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
      real cu[2], cm[3][2];
      if constexpr (F64) {
        double du[2] = {0, 0}, dm[3][2] = {{0, 0}, {0, 0}, {0, 0}};
#pragma unroll
        for (int kc = 0; kc < 2; ++kc) {
          const int nn = bnode(al, wt8, kc, gq, tig), nd = Lay<real>::at(nn);
          const double u = sPhi[PhiLay<real>::at(nn)];
          const double a = kc ? aG1 : aG0;
          dmma(du[0], du[1], a, u);
#pragma unroll
          for (int c = 0; c < 3; ++c)
            if ((comps >> c) & 1) dmma(dm[c][0], dm[c][1], a, sJa[(al * 3 + c) * FS + nd] * u);
        }
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          cu[b] = du[b];
#pragma unroll
          for (int c = 0; c < 3; ++c) cm[c][b] = dm[c][b];
        }
      } else {
        // the three-term split carries FP32's 24 bits, so only the two-term
        // form takes the operand relative to its pencil value at node PREF
        constexpr bool OFS = NT == 2;
        const int nn0 = bn(al, wt8, 2 * tig, gq), nn1 = bn(al, wt8, 2 * tig + 1, gq);
        const int nd0 = Lay<real>::at(nn0), nd1 = Lay<real>::at(nn1);
        const float u0 = sPhi[PhiLay<real>::at(nn0)], u1 = sPhi[PhiLay<real>::at(nn1)];
        const int nnr = OFS ? bn(al, wt8, PREF, gq) : 0, ndr = Lay<real>::at(nnr);
        const float ur = OFS ? sPhi[PhiLay<real>::at(nnr)] : 0.f;
        float fu[4] = {0, 0, 0, 0}, fm[3][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
        mma_split<NT>(fu, aS, aS2, u0 - ur, u1 - ur);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if ((comps >> c) & 1) {
            const real* mc = sJa + (al * 3 + c) * FS;
            if constexpr (OFS) {
              const float pr = mc[ndr] * ur;
              mma_split<NT>(fm[c], aS, aS2, fmaf(mc[nd0], u0, -pr), fmaf(mc[nd1], u1, -pr));
            } else {
              mma_split<NT>(fm[c], aS, aS2, mc[nd0] * u0, mc[nd1] * u1);
            }
          }
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          cu[b] = fu[b] + fu[b + 2];
#pragma unroll
          for (int c = 0; c < 3; ++c) cm[c][b] = fm[c][b] + fm[c][b + 2];
        }
      }
      const int sface_f = gq == 0 ? 2 * al : gq == 7 ? 2 * al + 1 : -1;
      const bool sat = sface_f >= 0 && ((mask >> sface_f) & 1);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int nno = onode(al, wt8, b, gq, tig), no = Lay<real>::at(nno);
        real jump = 0;
        if (sat) jump = (gq ? inv2H : -inv2H) * (sfc[sface_f * N2 + opq(al, wt8, b, tig)] - sPhi[PhiLay<real>::at(nno)]);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if ((comps >> c) & 1) {
            const real m = sJa[(al * 3 + c) * FS + no];
            real r = (real)0.5 * cm[c][b] + (real)0.5 * m * cu[b];
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
      real u;
      if constexpr (PHIR) u = cur.phi;
      else u = sPhi[tphi];
      real g0 = (sg[tpad] + sg[3 * FS + tpad]) + sg[6 * FS + tpad];
      real g1 = (sg[FS + tpad] + sg[4 * FS + tpad]) + sg[7 * FS + tpad];
      real g2 = (sg[2 * FS + tpad] + sg[5 * FS + tpad]) + sg[8 * FS + tpad];
      g0 *= cur.invJ; g1 *= cur.invJ; g2 *= cur.invJ;
      if constexpr (GR) {
        Q.gout[n] = g0;
        Q.gout[Q.nn + n] = g1;
        Q.gout[2 * Q.nn + n] = g2;
      } else {
      real cc[10];
#pragma unroll
      for (int c = 0; c < 10; ++c) cc[c] = SC ? d[PSZ + 9 * FS + c * N3 + tid] : cur.c[c];
      const real a = cc[0];
      const real b0 = cc[1], b1 = cc[2], b2 = cc[3];
      const real K0 = cc[4], K1v = cc[5], K2 = cc[6], K3 = cc[7], K4 = cc[8], K5 = cc[9];
      const real Pi = cur.Pi;
      const real F0 = b0 * Pi + (K0 * g0 + K1v * g1 + K2 * g2);
      const real F1 = b1 * Pi + (K1v * g0 + K3 * g1 + K4 * g2);
      const real F2 = b2 * Pi + (K2 * g0 + K4 * g1 + K5 * g2);
      real phid = b0 * g0 + b1 * g1 + b2 * g2 + a * Pi;
      if (bnd && Q.bc_on) k1_boundary<real>(Q, e, ti, tj, tk, n, u, Pi, g0, g1, g2, cc, phid);
      {  // flux in the element-block layout (Lay) read by K2
        const long long fo = e * FS + tpad, fstr = Q.Ne * FS;
        Q.F[fo] = F0;
        Q.F[fstr + fo] = F1;
        Q.F[2 * fstr + fo] = F2;
      }
      if (P.epi)
        n8_rk<real>(P.stage, Q.dt, phid, u, cur.y, cur.acc, cur.comp, n, Q.y, Q.acc, Q.out, comp_on ? Q.comp : nullptr,
                    P.flag);
      else
        Q.Phidot[n] = phid;
      }  // !GR
    }
    if (has_next && tid < 6 * N2) sface[(fb ^ 1) * 6 * N2 + tid] = fnext;
    if constexpr (PHIR)
      if (has_next) sphi[(fb ^ 1) * N3 + tphi] = nxt.phi;
    cur = nxt;
    emcur = emnext;
    src1 = src2;
    if constexpr (BATCH) {
      t0 = t1;
      t1 = t2;
      t2 = t3;
    }
  }
}

// ---------------------------------------------------------------------------
template <typename real>
struct K2N8 {
  long long Ne, nn;
  long long e0;  // single-solve launches: the first element (see K1N8)
  const real* F0;
  const real* F1;
  const real* F2;
  const real* Ja;
  const real* invdetJ;
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
  unsigned* flag;
  float Gh[64];
};

// K2 staged fields: 0..2 F, 3..11 Ja.  Register prefetch: invJ, y, acc, comp.
// Two shapes (K2Shape): 512 threads (one node per thread, warps w and w + 8
// split the fields of pencil tile w & 7, a ring of NSTAGE stages) or 256
// threads (two nodes per thread, each warp does both halves of its tile, one
// stage whose next copy is issued as soon as the contraction pass has read
// it) -- the 256-thread shape fits two CTAs on an SM for FP64.  Partial
// divergences: one field per (axis, half) in the 512-thread shape; one per axis
// in the 256-thread shape, whose threads add the two halves in registers.
constexpr int K2_NF = 12;
template <typename real>
struct K2Shape {
  static constexpr int THR = std::is_same<real, double>::value ? 256 : 512;
  static constexpr int NS = THR == 512 ? n8::NSTAGE : 1;          // stages
  static constexpr int OCC = std::is_same<real, double>::value ? 2 : n8::Occ<real>::k2;
  static constexpr int NSD = THR == 512 ? 6 : 3;                  // partial-divergence fields
  static constexpr size_t STAGE = (size_t)K2_NF * n8::Lay<real>::FS;
};
template <typename real>
constexpr size_t k2_smem() {
  return (K2Shape<real>::NS * K2Shape<real>::STAGE + K2Shape<real>::NSD * n8::Lay<real>::FS + 2 * 6 * 3 * n8::N2) *
             sizeof(real) +
         n8::N2 * sizeof(double) + 64;
}

template <typename real, int NT, bool BATCH>
__global__ void __launch_bounds__(K2Shape<real>::THR, K2Shape<real>::OCC)
    k_cons_k2_n8(const K2N8<real> P, const K2N8<real>* __restrict__ plist, const int2* __restrict__ tiles,
                 long long ntiles) {
  using namespace n8;
  constexpr bool F64 = std::is_same<real, double>::value;
  constexpr int THR = K2Shape<real>::THR, NS = K2Shape<real>::NS;
  constexpr int NPT = N3 / THR;                 // nodes per thread in the node pass
  constexpr int NFACE = 6 * 3 * N2;             // 1152 neighbour face values
  constexpr int NFR = (NFACE + THR - 1) / THR;  // face values per thread
  constexpr int NHALF = THR == 512 ? 1 : 2;     // halves of its tile a warp does
  constexpr int FS = Lay<real>::FS, NSD = K2Shape<real>::NSD;
  constexpr size_t K2_STAGE = K2Shape<real>::STAGE;
  extern __shared__ __align__(128) unsigned char smraw[];
  double* sG = reinterpret_cast<double*>(smraw);                   // 64
  real* stg = reinterpret_cast<real*>(sG + N2);
  real* sdiv = stg + NS * K2_STAGE;                                // NSD partial divergences (Lay)
  real* sface = sdiv + NSD * FS;                                   // 2 x 6 x 3 x 64
  uint64_t* bar = reinterpret_cast<uint64_t*>(sface + 2 * NFACE);
  __shared__ int abort_flag;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tig = lane & 3, wt8 = warp & 7;
  const real inv2H = (real)(1.0 / (2.0 * P.H[0]));
  const bool comp_on = !F64 && P.epi && P.comp != nullptr;  // FP32 state only
  const bool need_y = P.epi && (P.stage <= 2 || (comp_on && P.stage == 3));
  const bool need_acc = P.epi && P.stage >= 1;
  const bool need_comp = comp_on && P.stage == 3;
  const unsigned tx_bytes = (unsigned)(K2_NF * FS * sizeof(real));
  const long long T = ntiles;
  const long long GS = gridDim.x;
  auto tile_at = [&](long long t) -> int2 {
    if (t >= T) return make_int2(-1, -1);
    if constexpr (BATCH) return tiles[t];
    else return make_int2(0, (int)(P.e0 + t));
  };
  auto prm = [&](int sidx) -> const K2N8<real>& {
    if constexpr (BATCH) return plist[sidx];
    else return P;
  };

  if (tid < N2) sG[tid] = P.G[tid];
  if (tid == 0) {
    abort_flag = 0;
    for (int k = 0; k < NS; ++k) mbar_init(&bar[k], 1);
    fence_barrier_init();
  }
  __syncthreads();

  auto issue = [&](int2 tl, int s) {
    const K2N8<real>& Q = prm(tl.x);
    const long long e = tl.y;
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[s], tx_bytes);
    }
    __syncwarp();
    real* d = stg + s * K2_STAGE;
    if (lane < K2_NF) {
      const real* src = lane < 3 ? (lane == 0 ? Q.F0 : lane == 1 ? Q.F1 : Q.F2) + e * FS
                                 : Q.Ja + ((long long)(lane - 3) * Q.Ne + e) * FS;
      bulk_g2s(d + lane * FS, src, FS * (unsigned)sizeof(real), &bar[s]);
    }
  };
  // neighbour flux face traces: [f][c][pq], 1152 values, NFR per thread; the
  // face sources are loaded one iteration ahead of the traces (see K1)
  auto src_load = [&](int2 tl, int src[NFR]) {
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = tid + r * THR;
      src[r] = (tl.x >= 0 && idx < NFACE) ? ::wt::bc_src(prm(tl.x).fsrc[idx / (3 * N2) + 6 * tl.y], prm(tl.x).Ne) : -1;
    }
  };
  auto face_load = [&](const int src[NFR], int sidx, real fv[NFR]) {
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = tid + r * THR;
      real v = 0;
      if (src[r] >= 0) {
        const K2N8<real>& Q = prm(sidx);
        const int rem = idx % (3 * N2), c = rem >> 6, pq = rem & 63;
        const real* Fc = c == 0 ? Q.F0 : c == 1 ? Q.F1 : Q.F2;
        v = Fc[(long long)(src[r] >> 6) * FS + Lay<real>::at(nbr_face_node(src[r], pq & 7, pq >> 3, N))];
      }
      fv[r] = v;
    }
  };
  auto emask_at = [&](int2 tl) -> int { return tl.x >= 0 ? prm(tl.x).emask[tl.y] : 0; };
  struct PW {
    real invJ, y, acc, comp;
  };
  auto pw_load = [&](int2 tl, PW w[NPT]) {
    if (tl.x < 0) return;
    const K2N8<real>& Q = prm(tl.x);
#pragma unroll
    for (int r = 0; r < NPT; ++r) {
      const long long n = (long long)tl.y * N3 + tid + r * THR;
      w[r].invJ = Q.invdetJ[n];
      w[r].y = need_y ? Q.y[n] : (real)0;
      w[r].acc = need_acc ? Q.acc[n] : (real)0;
      w[r].comp = need_comp ? Q.comp[n] : (real)0;
    }
  };

  int2 t0 = tile_at(blockIdx.x), t1 = tile_at(blockIdx.x + GS), t2 = tile_at(blockIdx.x + 2 * GS);
  PW cur[NPT];
  int emcur = 0, src1[NFR];
#pragma unroll
  for (int r = 0; r < NFR; ++r) src1[r] = -1;
  if (t0.x >= 0) {
    if (warp == 0)
      for (int k = 0; k < (NS > 1 ? NS - 1 : 1); ++k) {
        const int2 tk_ = tile_at(blockIdx.x + k * GS);
        if (tk_.x >= 0) issue(tk_, k);
      }
    emcur = emask_at(t0);
    int src0[NFR];
    src_load(t0, src0);
    real fv[NFR];
    face_load(src0, t0.x, fv);
#pragma unroll
    for (int r = 0; r < NFR; ++r)
      if (tid + r * THR < NFACE) sface[tid + r * THR] = fv[r];
    pw_load(t0, cur);
    src_load(t1, src1);
  }
  __syncthreads();
  double aG0 = 0.0, aG1 = 0.0;
  uint32_t aS[4] = {0, 0, 0, 0}, aS2[4] = {0, 0, 0, 0};
  if constexpr (F64) {
    aG0 = sG[gq * 8 + tig];
    aG1 = sG[gq * 8 + 4 + tig];
  } else {
    split_G(sG, gq, tig, NT, aS, aS2);
  }

  int it = 0;
  for (long long t = blockIdx.x; t < T; t += GS, ++it) {
    const int s = it % NS, fb = it & 1;
    const unsigned parity = (it / NS) & 1;
    // tiles t, t + grid, t + 2 grid: carried in registers for a work list (loaded
    // ahead), recomputed from t for a single solve
    int2 t3 = make_int2(-1, -1);
    if constexpr (BATCH) {
      t3 = tile_at(t + 3 * GS);
    } else {
      t0 = tile_at(t);
      t1 = tile_at(t + GS);
      t2 = tile_at(t + 2 * GS);
    }
    const bool has_next = t1.x >= 0;
    const int emnext = emask_at(t1);
    int src2[NFR];
    src_load(t2, src2);
    real fnext[NFR];
    face_load(src1, t1.x, fnext);
    PW nxt[NPT];
    pw_load(t1, nxt);
    // One thread polls the stage's mbarrier (its acquire makes the copied data
    // visible; the barrier below orders every other thread after it), so the
    // other warps do not spend issue slots spinning.
    if (tid == 0 && !wait_phase(&bar[s], parity, P.flag)) abort_flag = 1;
    __syncthreads();  // the previous element is finished: its stage and the buffers are free (see K1)
    if (abort_flag) {  // wait (bounded) for the copies still in flight, then leave
      if (warp == 0 && lane == 0)
        for (int k = 1; k < NS - 1; ++k)
          if (tile_at(t + k * GS).x >= 0) wait_phase(&bar[(it + k) % NS], ((it + k) / NS) & 1, nullptr);
      return;
    }
    if constexpr (NS > 1) {
      const int2 ti_ = NS == 2 ? t1 : tile_at(t + (NS - 1) * GS);
      if (warp == 0 && ti_.x >= 0) issue(ti_, (it + NS - 1) % NS);
    }
    const K2N8<real>& Q = prm(t0.x);
    const long long e = t0.y;
    const real* d = stg + s * K2_STAGE;
    const real* sF = d;           // 3 fields
    const real* sJa = d + 3 * FS;  // 9 fields
    const real* sfc = sface + fb * NFACE;
    const int mask = emcur & 63;
    const int bnd = emcur >> 6;
    // per-axis partial divergences (sdiv[al*2 + half], or sdiv[al] with the two
    // halves added in registers): no barrier between axes
#pragma unroll
    for (int al = 0; al < 3; ++al) {
      const real* m0 = sJa + (al * 3 + 0) * FS;
      const real* m1 = sJa + (al * 3 + 1) * FS;
      const real* m2 = sJa + (al * 3 + 2) * FS;
      real rsum[2] = {0, 0};
#pragma unroll
      for (int hh = 0; hh < NHALF; ++hh) {
        const int half = THR == 512 ? (warp >> 3) : hh;
        real cx[2], cy[2];
        if constexpr (F64) {
          double dx[2] = {0, 0}, dy[2] = {0, 0};
#pragma unroll
          for (int kc = 0; kc < 2; ++kc) {
            const int nd = Lay<real>::at(bnode(al, wt8, kc, gq, tig));
            const double a = kc ? aG1 : aG0;
            if (half == 0) {
              // contravariant flux Ja^al . F and F_0
              const double f0 = sF[nd];
              const double ft = m0[nd] * f0 + m1[nd] * sF[FS + nd] + m2[nd] * sF[2 * FS + nd];
              dmma(dx[0], dx[1], a, ft);
              dmma(dy[0], dy[1], a, f0);
            } else {
              dmma(dx[0], dx[1], a, sF[FS + nd]);
              dmma(dy[0], dy[1], a, sF[2 * FS + nd]);
            }
          }
          cx[0] = dx[0]; cx[1] = dx[1]; cy[0] = dy[0]; cy[1] = dy[1];
        } else {
          constexpr bool OFS = NT == 2;  // operand offset only for the two-term split (see K1)
          constexpr int NQ = OFS ? 3 : 2;
          const int nd[3] = {Lay<real>::at(bn(al, wt8, 2 * tig, gq)), Lay<real>::at(bn(al, wt8, 2 * tig + 1, gq)),
                             Lay<real>::at(bn(al, wt8, PREF, gq))};
          float vx[3] = {0, 0, 0}, vy[3] = {0, 0, 0};
#pragma unroll
          for (int q = 0; q < NQ; ++q) {
            if (half == 0) {
              const float f0 = sF[nd[q]];
              vx[q] = m0[nd[q]] * f0 + m1[nd[q]] * sF[FS + nd[q]] + m2[nd[q]] * sF[2 * FS + nd[q]];
              vy[q] = f0;
            } else {
              vx[q] = sF[FS + nd[q]];
              vy[q] = sF[2 * FS + nd[q]];
            }
          }
          float fx[4] = {0, 0, 0, 0}, fy[4] = {0, 0, 0, 0};
          mma_split<NT>(fx, aS, aS2, vx[0] - vx[2], vx[1] - vx[2]);
          mma_split<NT>(fy, aS, aS2, vy[0] - vy[2], vy[1] - vy[2]);
          cx[0] = fx[0] + fx[2]; cx[1] = fx[1] + fx[3];
          cy[0] = fy[0] + fy[2]; cy[1] = fy[1] + fy[3];
        }
        // half 1 adds the centred-flux SAT of an interior al-face on its rows
        const int sface_f = gq == 0 ? 2 * al : gq == 7 ? 2 * al + 1 : -1;
        const bool sat = half == 1 && sface_f >= 0 && ((mask >> sface_f) & 1);
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          const int no = Lay<real>::at(onode(al, wt8, b, gq, tig));
          real r;
          if (half == 0) {
            r = (real)0.5 * cx[b] + (real)0.5 * m0[no] * cy[b];
          } else {
            r = (real)0.5 * m1[no] * cx[b] + (real)0.5 * m2[no] * cy[b];
          }
          if (sat) {
            const int pq = opq(al, wt8, b, tig);
            const real sacc = m0[no] * (sfc[(sface_f * 3 + 0) * N2 + pq] - sF[no]) +
                              m1[no] * (sfc[(sface_f * 3 + 1) * N2 + pq] - sF[FS + no]) +
                              m2[no] * (sfc[(sface_f * 3 + 2) * N2 + pq] - sF[2 * FS + no]);
            r += (gq ? inv2H : -inv2H) * sacc;
          }
          if constexpr (NHALF == 2) rsum[b] = hh ? rsum[b] + r : r;
          else sdiv[(al * 2 + half) * FS + no] = r;
        }
      }
      if constexpr (NHALF == 2) {
#pragma unroll
        for (int b = 0; b < 2; ++b) sdiv[al * FS + Lay<real>::at(onode(al, wt8, b, gq, tig))] = rsum[b];
      }
    }
    __syncthreads();
    // one stage: the contraction pass has read it, so the next copy can start
    if constexpr (NS == 1) {
      if (warp == 0 && t1.x >= 0) issue(t1, 0);
    }
#pragma unroll
    for (int r = 0; r < NPT; ++r) {
      const int node = tid + r * THR;
      const int ti = node & 7, tj = (node >> 3) & 7, tk = node >> 6;
      const int tpad = Lay<real>::at(node);
      const long long n = e * N3 + node;
      real dv;
      if constexpr (NSD == 3)
        dv = (sdiv[tpad] + sdiv[FS + tpad]) + sdiv[2 * FS + tpad];
      else
        dv = ((sdiv[tpad] + sdiv[2 * FS + tpad]) + sdiv[4 * FS + tpad]) +
             ((sdiv[FS + tpad] + sdiv[3 * FS + tpad]) + sdiv[5 * FS + tpad]);
      dv *= cur[r].invJ;
      if (bnd && Q.bc_on) {
        const int idx3[3] = {ti, tj, tk};
        for (int f = 0; f < 6; ++f) {
          if (Q.bdry[f + 6 * e] == 0) continue;
          const int ax = f >> 1;
          if (idx3[ax] != ((f & 1) ? 7 : 0)) continue;
          const int p = ax == 0 ? tj : ti, q = ax == 2 ? tj : tk;
          dv += Q.bbuf[(long long)::wt::bc_slot(Q.bslot[f + 6 * e], Q.nbf) * N2 + p + 8 * q];
        }
      }
      if (P.epi)
        n8_rk<real>(P.stage, Q.dt, dv, cur[r].y, cur[r].y, cur[r].acc, cur[r].comp, n, Q.y, Q.acc, Q.out,
                    comp_on ? Q.comp : nullptr, P.flag);
      else
        Q.Pidot[n] = dv;
    }
    if (has_next) {
#pragma unroll
      for (int r = 0; r < NFR; ++r)
        if (tid + r * THR < NFACE) sface[(fb ^ 1) * NFACE + tid + r * THR] = fnext[r];
    }
#pragma unroll
    for (int r = 0; r < NPT; ++r) cur[r] = nxt[r];
    emcur = emnext;
#pragma unroll
    for (int r = 0; r < NFR; ++r) src1[r] = src2[r];
    if constexpr (BATCH) {
      t0 = t1;
      t1 = t2;
      t2 = t3;
    }
  }
}

// ---------------------------------------------------------------------------
// Fused RK4 stage kernel FK_s (FP64, n = 8): on each element, the K2 half of
// stage s (split-form divergence of F_s, centred-flux SAT, boundary terms, the
// Pi stage update) and the K1 half of stage s + 1 (split-form gradient of
// Phi_{s+1}, flux F_{s+1}, boundary terms, the Phi stage update) -- the
// integrator fused into the right-hand side (IDEAS.md:48-50 of the reference;
// the arithmetic is that of wave3d_curved_rhs!, src/wave3d_curved.jl:205-258).
// No grid-wide barrier is needed between the halves:
//   * K2_s of element e reads F_s of e and of its neighbours' faces: all of F_s
//     was written by the previous launch (F ping-pongs: this launch writes
//     F_{s+1} into the other buffer while neighbours still read F_s);
//   * K1_{s+1} of e reads Phi_{s+1} of e and of its neighbours' faces (written
//     by the previous launch) and Pi_{s+1} of e only, which its own K2 half has
//     just formed -- it stays in a register (one node per thread in both node
//     passes), so Pi_{s+1} is never stored;
//   * the boundary buffer: each thread reads its node's slots in the K2 half
//     before the K1 half rewrites them.
// Only the node passes depend on each other, so the two contraction passes run
// side by side: warps 0-7 contract the divergence (tile w, both halves of its
// fields, as the 256-thread k_cons_k2_n8<double>), warps 8-15 the gradient
// (tile w - 8, all nine components); one barrier later every thread does the
// divergence node pass and then the gradient node pass of its node.  Two CTA
// barriers per element, as in one of the two-kernel launches.  The metric terms
// Ja staged for the divergence are read by the gradient too, and 1/J once.  Per
// node and stage the fused kernel moves 33 words against 44 for the two
// kernels (F 3 + Ja 9 + 1/J 1 + Pi RK 3 + Phi 1 + coefficients 10 + Phi RK 3 +
// F_{s+1} 3).
// CTA: 512 threads, one per SM (217 KB of shared memory); the flux and metric
// terms (12 blocks) in a two-stage ring, issued one element ahead; the ten
// coefficient blocks (read only by the node pass) single-buffered, issued once
// the previous element's node pass is done; neighbour face traces of F_s and
// Phi_{s+1} and Phi_{s+1} itself by per-thread cp.async one element ahead; 1/J
// and the RK states prefetched into registers one element ahead.  Each partial
// sum is formed by the instructions k_cons_k2_n8<double> and
// k_cons_k1_n8<double> use and added in their order, so the fused step equals
// the two-kernel step bit for bit.
// Measured on the 64^3 x 8^3 solve: 262 DRAM bytes per node and launch (the two
// kernels: 364); the RK4 step 1-7 % faster than the two-kernel step timed right
// after it on the same GPU.  The kernels are bound by latency and issue (16
// warps per SM, about 41 % issue active) rather than by DRAM bandwidth, so
// the gain is smaller than the bytes saved.
struct FKN8 {
  K2N8<double> a;  // stage s: F_s in (a.F0..F2), the Pi stage update
  K1N8<double> b;  // stage s + 1: Phi_{s+1} in (b.Phi), F_{s+1} out (b.F), the Phi stage update
};
constexpr int FK_NA = 12;  // ring stage: F (3) + Ja (9) blocks
constexpr size_t fk_smem() {
  return (2 * FK_NA * 512 + 10 * 512 + 12 * 512 + 2 * 6 * 3 * 64 + 2 * 6 * 64 + 2 * 512) * sizeof(double) +
         64 * sizeof(double) + 64;
}
static_assert(fk_smem() + 64 + 1024 <= 233472, "the fused stage kernel's CTA must fit an SM");

namespace n8 {
// per-thread 8-byte asynchronous copy global -> shared, zero-filled when !valid
// (src must still be a valid address); commit / wait for all groups but the
// newest / wait for all (cp_async_wait_all)
__device__ __forceinline__ void cp_async8z(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
}  // namespace n8

// RK4 stage update of an FP64 field for stages 0..2 (n8_rk without the FP32
// compensation) returning the stage value; it is also written to out unless out
// is NULL (the fused step keeps Pi's stage value in a register and never reads
// it back).
__device__ __forceinline__ double n8_rk_out(int stage, double dt, double k, double yv, double accv, long long n,
                                            double* acc, double* out) {
  double o;
  if (stage == 0) {
    o = yv + (0.5 * dt) * k;
    acc[n] = yv + (dt / 6.0) * k;
  } else if (stage == 1) {
    o = yv + (0.5 * dt) * k;
    acc[n] = accv + (dt / 3.0) * k;
  } else {
    o = yv + dt * k;
    acc[n] = accv + (dt / 3.0) * k;
  }
  if (out) out[n] = o;
  return o;
}

__global__ void __launch_bounds__(n8::THREADS, 1) k_cons_fk_n8(const FKN8 P) {
  using namespace n8;
  using real = double;
  constexpr int FS = Lay<double>::FS;
  constexpr int NFACE = 6 * 3 * N2;                     // flux face values
  constexpr int NFR = (NFACE + THREADS - 1) / THREADS;  // per thread
  constexpr int NPF = 6 * N2;                           // Phi face values
  const K2N8<double>& A = P.a;
  const K1N8<double>& B = P.b;
  extern __shared__ __align__(128) unsigned char smraw[];
  double* sG = reinterpret_cast<double*>(smraw);  // 64
  double* stg = sG + N2;                          // 2 x 12 blocks: F (3), Ja (9)
  double* sC = stg + 2 * FK_NA * FS;              // 10 coefficient blocks (node order)
  double* sdiv = sC + 10 * N3;                    // 3 partial divergences [al] (Lay)
  double* sg = sdiv + 3 * FS;                     // 9 partial gradients [al * 3 + c] (Lay)
  double* sfF = sg + 9 * FS;                      // 2 x 1152 flux face traces [f][c][pq]
  double* sfP = sfF + 2 * NFACE;                  // 2 x 384 Phi face traces [f][pq]
  double* sphi = sfP + 2 * NPF;                   // 2 x 512 Phi_{s+1} (Lay)
  uint64_t* bar = reinterpret_cast<uint64_t*>(sphi + 2 * N3);  // [0], [1] ring, [2] coefficients
  __shared__ int abort_flag;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tig = lane & 3, wt8 = warp & 7;
  const bool divw = warp < 8;  // divergence-contraction warp (else gradient)
  const real inv2H = (real)(1.0 / (2.0 * A.H[0]));
  const int sa = A.stage, sb = B.stage;  // sb = sa + 1
  const bool needQy = sa <= 2, needQacc = sa >= 1;
  const bool needPy = sb == 1 || sb == 2;
  const unsigned txA = (unsigned)(FK_NA * FS * sizeof(real)), txC = (unsigned)(10 * N3 * sizeof(real));
  const int ti = tid & 7, tj = (tid >> 3) & 7, tk = tid >> 6;
  const int tpad = Lay<real>::at(tid);
  const long long T = A.Ne, GS = gridDim.x;

  if (tid < N2) sG[tid] = A.G[tid];
  if (tid == 0) {
    abort_flag = 0;
    for (int k = 0; k < 3; ++k) mbar_init(&bar[k], 1);
    fence_barrier_init();
  }
  __syncthreads();

  // warp 0: F_s and Ja of element e into ring stage s
  auto issueA = [&](long long e, int s) {
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[s], txA);
    }
    __syncwarp();
    real* d = stg + s * FK_NA * FS;
    if (lane < FK_NA) {
      const real* src = lane < 3 ? (lane == 0 ? A.F0 : lane == 1 ? A.F1 : A.F2) + e * FS
                                 : A.Ja + ((long long)(lane - 3) * A.Ne + e) * FS;
      bulk_g2s(d + lane * FS, src, FS * (unsigned)sizeof(real), &bar[s]);
    }
  };
  // warp 0: the ten coefficient blocks of element e
  auto issueC = [&](long long e) {
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[2], txC);
    }
    __syncwarp();
    if (lane < 10) bulk_g2s(sC + lane * N3, B.c10 + lane * B.nn + e * N3, N3 * (unsigned)sizeof(real), &bar[2]);
  };
  // face sources of element e (-1: none or past the end), loaded one iteration
  // before the traces they address
  auto srcF_load = [&](long long e, int src[NFR]) {
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = tid + r * THREADS;
      src[r] = (e < T && idx < NFACE) ? ::wt::bc_src(A.fsrc[idx / (3 * N2) + 6 * e], A.Ne) : -1;
    }
  };
  auto srcP_load = [&](long long e) -> int { return (e < T && tid < NPF) ? ::wt::bc_src(B.fsrc[(tid >> 6) + 6 * e], B.Ne) : -1; };
  auto faceF_load = [&](const int src[NFR], real fv[NFR]) {
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = tid + r * THREADS;
      real v = 0;
      if (src[r] >= 0) {
        const int rem = idx % (3 * N2), c = rem >> 6, pq = rem & 63;
        const real* Fc = c == 0 ? A.F0 : c == 1 ? A.F1 : A.F2;
        v = Fc[(long long)(src[r] >> 6) * FS + Lay<real>::at(nbr_face_node(src[r], pq & 7, pq >> 3, N))];
      }
      fv[r] = v;
    }
  };
  auto faceP_load = [&](int src) -> real {
    if (src < 0) return (real)0;
    const int pq = tid & 63;
    return B.Phi[(long long)(src >> 6) * N3 + nbr_face_node(src, pq & 7, pq >> 3, N)];
  };
  struct PW {
    real invJ, Qy, Qacc, Py, Pacc;
  };
  auto pw_load = [&](long long e, PW& w) {
    const long long n = e * N3 + tid;
    w.invJ = A.invdetJ[n];
    w.Qy = needQy ? A.y[n] : (real)0;
    w.Qacc = needQacc ? A.acc[n] : (real)0;
    w.Py = needPy ? B.y[n] : (real)0;
    w.Pacc = B.acc[n];  // stage s + 1 >= 1 reads the accumulator
  };

  PW cur;
  int emcur = 0, srcF1[NFR], srcP1 = -1;
#pragma unroll
  for (int r = 0; r < NFR; ++r) srcF1[r] = -1;
  {
    const long long t0 = blockIdx.x;
    if (t0 < T) {
      if (warp == 0) issueA(t0, 0);
      emcur = A.emask[t0];
      int s0[NFR];
      srcF_load(t0, s0);
      real fv[NFR];
      faceF_load(s0, fv);
#pragma unroll
      for (int r = 0; r < NFR; ++r)
        if (tid + r * THREADS < NFACE) sfF[tid + r * THREADS] = fv[r];
      const real pv = faceP_load(srcP_load(t0));
      if (tid < NPF) sfP[tid] = pv;
      pw_load(t0, cur);
      sphi[tpad] = B.Phi[t0 * N3 + tid];
      srcF_load(t0 + GS, srcF1);
      srcP1 = srcP_load(t0 + GS);
    }
  }
  __syncthreads();
  const double aG0 = sG[gq * 8 + tig], aG1 = sG[gq * 8 + 4 + tig];

  int it = 0;
  for (long long t = blockIdx.x; t < T; t += GS, ++it) {
    const int s = it & 1, fb = it & 1;
    const unsigned parity = (it >> 1) & 1;
    const long long t1 = t + GS;
    const bool has_next = t1 < T;
    const int emnext = has_next ? A.emask[t1] : 0;
    int srcF2[NFR];
    srcF_load(t + 2 * GS, srcF2);
    const int srcP2 = srcP_load(t + 2 * GS);
    // the next element's neighbour face traces and its Phi_{s+1} go straight into
    // the buffers fb ^ 1 by per-thread asynchronous copies (zero-filled where a
    // face has no neighbour; srcF1, srcP1 are -1 past the end); the previous
    // group -- this element's -- is complete after the wait, and visible to
    // every thread after the barrier below
    {
      double* dF = sfF + (fb ^ 1) * NFACE;
#pragma unroll
      for (int r = 0; r < NFR; ++r) {
        const int idx = tid + r * THREADS;
        if (idx < NFACE) {
          const real* g = A.F0;
          if (srcF1[r] >= 0) {
            const int rem = idx % (3 * N2), c = rem >> 6, pq = rem & 63;
            const real* Fc = c == 0 ? A.F0 : c == 1 ? A.F1 : A.F2;
            g = Fc + (long long)(srcF1[r] >> 6) * FS + Lay<real>::at(nbr_face_node(srcF1[r], pq & 7, pq >> 3, N));
          }
          cp_async8z(dF + idx, g, srcF1[r] >= 0);
        }
      }
      if (tid < NPF) {
        const real* g = B.Phi;
        if (srcP1 >= 0) {
          const int pq = tid & 63;
          g = B.Phi + (long long)(srcP1 >> 6) * N3 + nbr_face_node(srcP1, pq & 7, pq >> 3, N);
        }
        cp_async8z(sfP + (fb ^ 1) * NPF + tid, g, srcP1 >= 0);
      }
      cp_async8z(sphi + (fb ^ 1) * N3 + tpad, B.Phi + (has_next ? t1 : t) * N3 + tid, has_next);
      cp_async_commit();
      cp_async_wait_prior();
    }
    PW nxt;
    if (has_next) pw_load(t1, nxt);
    if (tid == 0 && !wait_phase(&bar[s], parity, A.flag)) abort_flag = 1;
    // every thread has finished the previous element: ring stage s ^ 1, the
    // coefficient buffer and the face / Phi buffers fb ^ 1 are free
    __syncthreads();
    if (abort_flag) {  // no bulk copy of this CTA is in flight (the coefficient copy was waited for)
      cp_async_wait_all();
      return;
    }
    if (warp == 0) {
      issueC(t);
      if (has_next) issueA(t1, s ^ 1);
    }
    const long long e = t;
    const real* d = stg + s * FK_NA * FS;
    const real* sF = d;
    const real* sJa = d + 3 * FS;
    const int mask = emcur & 63, bnd = emcur >> 6;

    if (divw) {
      // ---- divergence of F_s (K2 half), tile wt8: per axis the two halves of its
      // fields, added in registers into sdiv[al] ----
      const real* sfc = sfF + fb * NFACE;
#pragma unroll
      for (int al = 0; al < 3; ++al) {
        const real* m0 = sJa + (al * 3 + 0) * FS;
        const real* m1 = sJa + (al * 3 + 1) * FS;
        const real* m2 = sJa + (al * 3 + 2) * FS;
        real rsum[2] = {0, 0};
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          double dx[2] = {0, 0}, dy[2] = {0, 0};
#pragma unroll
          for (int kc = 0; kc < 2; ++kc) {
            const int nd = Lay<real>::at(bnode(al, wt8, kc, gq, tig));
            const double a = kc ? aG1 : aG0;
            if (hh == 0) {
              const double f0 = sF[nd];
              const double ft = m0[nd] * f0 + m1[nd] * sF[FS + nd] + m2[nd] * sF[2 * FS + nd];
              dmma(dx[0], dx[1], a, ft);
              dmma(dy[0], dy[1], a, f0);
            } else {
              dmma(dx[0], dx[1], a, sF[FS + nd]);
              dmma(dy[0], dy[1], a, sF[2 * FS + nd]);
            }
          }
          const int sface_f = gq == 0 ? 2 * al : gq == 7 ? 2 * al + 1 : -1;
          const bool sat = hh == 1 && sface_f >= 0 && ((mask >> sface_f) & 1);
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            const int no = Lay<real>::at(onode(al, wt8, b, gq, tig));
            real r;
            if (hh == 0) {
              r = (real)0.5 * dx[b] + (real)0.5 * m0[no] * dy[b];
            } else {
              r = (real)0.5 * m1[no] * dx[b] + (real)0.5 * m2[no] * dy[b];
            }
            if (sat) {
              const int pq = opq(al, wt8, b, tig);
              const real sacc = m0[no] * (sfc[(sface_f * 3 + 0) * N2 + pq] - sF[no]) +
                                m1[no] * (sfc[(sface_f * 3 + 1) * N2 + pq] - sF[FS + no]) +
                                m2[no] * (sfc[(sface_f * 3 + 2) * N2 + pq] - sF[2 * FS + no]);
              r += (gq ? inv2H : -inv2H) * sacc;
            }
            rsum[b] = hh ? rsum[b] + r : r;
          }
        }
#pragma unroll
        for (int b = 0; b < 2; ++b) sdiv[al * FS + Lay<real>::at(onode(al, wt8, b, gq, tig))] = rsum[b];
      }
    } else {
      // ---- split-form gradient of Phi_{s+1} (K1 half), tile wt8: all nine partials ----
      const real* sPhi = sphi + fb * N3;
      const real* sfc = sfP + fb * NPF;
#pragma unroll
      for (int al = 0; al < 3; ++al) {
        double du[2] = {0, 0}, dm[3][2] = {{0, 0}, {0, 0}, {0, 0}};
#pragma unroll
        for (int kc = 0; kc < 2; ++kc) {
          const int nd = Lay<real>::at(bnode(al, wt8, kc, gq, tig));
          const double u = sPhi[nd];
          const double a = kc ? aG1 : aG0;
          dmma(du[0], du[1], a, u);
#pragma unroll
          for (int c = 0; c < 3; ++c) dmma(dm[c][0], dm[c][1], a, sJa[(al * 3 + c) * FS + nd] * u);
        }
        const int sface_f = gq == 0 ? 2 * al : gq == 7 ? 2 * al + 1 : -1;
        const bool sat = sface_f >= 0 && ((mask >> sface_f) & 1);
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          const int no = Lay<real>::at(onode(al, wt8, b, gq, tig));
          real jump = 0;
          if (sat) jump = (gq ? inv2H : -inv2H) * (sfc[sface_f * N2 + opq(al, wt8, b, tig)] - sPhi[no]);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const real m = sJa[(al * 3 + c) * FS + no];
            real r = (real)0.5 * dm[c][b] + (real)0.5 * m * du[b];
            if (sat) r += m * jump;
            sg[(al * 3 + c) * FS + no] = r;
          }
        }
      }
    }
    if (tid == 0 && !wait_phase(&bar[2], (unsigned)(it & 1), A.flag)) abort_flag = 1;
    __syncthreads();
    if (abort_flag) {  // wait (bounded) for the next element's ring copy, then leave
      if (tid == 0 && has_next) wait_phase(&bar[s ^ 1], ((it + 1) >> 1) & 1, nullptr);
      cp_async_wait_all();
      return;
    }
    {
      const long long n = e * N3 + tid;
      // ---- divergence node pass: boundary terms, Pi stage update (K2 half) ----
      real dv = (sdiv[tpad] + sdiv[FS + tpad]) + sdiv[2 * FS + tpad];
      dv *= cur.invJ;
      if (bnd && A.bc_on) {
        const int idx3[3] = {ti, tj, tk};
        for (int f = 0; f < 6; ++f) {
          if (A.bdry[f + 6 * e] == 0) continue;
          const int ax = f >> 1;
          if (idx3[ax] != ((f & 1) ? 7 : 0)) continue;
          const int p = ax == 0 ? tj : ti, q = ax == 2 ? tj : tk;
          dv += A.bbuf[(long long)::wt::bc_slot(A.bslot[f + 6 * e], A.nbf) * N2 + p + 8 * q];
        }
      }
      const real Pi = n8_rk_out(sa, A.dt, dv, cur.Qy, cur.Qacc, n, A.acc, A.out);  // Pi_{s+1}
      // ---- gradient node pass: flux F_{s+1}, Phidot, boundary terms, Phi stage update (K1 half) ----
      const real u = sphi[fb * N3 + tpad];
      real g0 = (sg[tpad] + sg[3 * FS + tpad]) + sg[6 * FS + tpad];
      real g1 = (sg[FS + tpad] + sg[4 * FS + tpad]) + sg[7 * FS + tpad];
      real g2 = (sg[2 * FS + tpad] + sg[5 * FS + tpad]) + sg[8 * FS + tpad];
      g0 *= cur.invJ; g1 *= cur.invJ; g2 *= cur.invJ;
      real cc[10];
#pragma unroll
      for (int c = 0; c < 10; ++c) cc[c] = sC[c * N3 + tid];
      const real a = cc[0];
      const real b0 = cc[1], b1 = cc[2], b2 = cc[3];
      const real K0 = cc[4], K1v = cc[5], K2 = cc[6], K3 = cc[7], K4 = cc[8], K5 = cc[9];
      const real F0 = b0 * Pi + (K0 * g0 + K1v * g1 + K2 * g2);
      const real F1 = b1 * Pi + (K1v * g0 + K3 * g1 + K4 * g2);
      const real F2 = b2 * Pi + (K2 * g0 + K4 * g1 + K5 * g2);
      real phid = b0 * g0 + b1 * g1 + b2 * g2 + a * Pi;
      if (bnd && B.bc_on) k1_boundary<real>(B, e, ti, tj, tk, n, u, Pi, g0, g1, g2, cc, phid);
      {
        const long long fo = e * FS + tpad, fstr = B.Ne * FS;
        B.F[fo] = F0;
        B.F[fstr + fo] = F1;
        B.F[2 * fstr + fo] = F2;
      }
      n8_rk<real>(sb, B.dt, phid, u, cur.Py, cur.Pacc, (real)0, n, B.y, B.acc, B.out, nullptr, B.flag);
    }
    cur = nxt;
    emcur = emnext;
#pragma unroll
    for (int r = 0; r < NFR; ++r) srcF1[r] = srcF2[r];
    srcP1 = srcP2;
  }
}

// ---------------------------------------------------------------------------
// FP32 CUDA-core form (WT_FP32_CUDA_CORES) of the two n = 8 kernels: one
// thread per (axis, pencil) -- 3 x 64 = 192 threads -- does the 8x8
// contractions of its pencil as FFMAs whose operator entries come from the
// kernel's constant bank (the parameter block).  Exact FP32 arithmetic with
// about a quarter of the instructions of the split-BF16 form.  The staging,
// tables, face traces, prefetch and bounded waits are those of the kernels
// above; element blocks use the LayC layout.
namespace n8 {
// Element-block layout of the FP32 CUDA-core form: the node index with bits
// 0-4 XOR-ed by bits 5-7 (bit0 ^= b6, bit1 ^= b7, bit2 ^= b5, bit3 ^= b6,
// bit4 ^= b7), so that a warp reading one node of each of 32 pencils along any
// axis, or 32 nodes in order, touches 32 distinct banks.
struct LayC {
  static constexpr int FS = 512;
  __host__ __device__ __forceinline__ static int at(int n) {
    const int j2 = (n >> 5) & 1, k0 = (n >> 6) & 1, k1 = (n >> 7) & 1;
    return n ^ ((k0 * 9) ^ (k1 * 18) ^ (j2 * 4));
  }
};
constexpr int CTHR = 192;
// per-thread 4-byte asynchronous copy global -> shared (zero-filled when !valid)
__device__ __forceinline__ void cp_async4(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// index into a per-CTA table of the 6 x 64 face nodes for face source fs and
// this face's point pq: the neighbour face's point after the orientation
__device__ __forceinline__ int face_slot(int fs, int pq) {
  int pn, qn;
  face_perm((fs >> 3) & 7, pq & 7, pq >> 3, N, pn, qn);
  return ((fs & 7) << 6) + pn + 8 * qn;
}
// node at position pos of pencil pc along axis al; pc = a + 8 b numbers the
// other two axes in increasing order, so it is also the pencil's face index
__device__ __forceinline__ int pnode(int al, int pc, int pos) {
  const int a = pc & 7, b = pc >> 3;
  return al == 0 ? pos + 8 * a + 64 * b : al == 1 ? a + 8 * pos + 64 * b : a + 8 * b + 64 * pos;
}
// out[l] = sum_m G[l][m] v[m]
__device__ __forceinline__ void contract8(const float* G, const float v[8], float out[8]) {
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    float acc = G[l * 8] * v[0];
#pragma unroll
    for (int m = 1; m < 8; ++m) acc = fmaf(G[l * 8 + m], v[m], acc);
    out[l] = acc;
  }
}
}  // namespace n8

// K1c: the nine Ja blocks in one stage (read by the contraction pass) and the
// node-pass fields in a second buffer (ten coefficients, Pi, 1/J, y, acc, comp),
// each single-buffered and bulk-copied as soon as the pass that reads it is done,
// so that three CTAs fit on an SM.
constexpr size_t K1C_STAGE = 9 * (size_t)n8::LayC::FS;
// node-pass buffer: c10 (10), Pi, invJ, [y], acc, comp -- the compensated form
// reads the state's high part from the Phi pencils and holds no y
template <bool CP>
constexpr size_t k1c_b() { return (CP ? 14 : 15) * (size_t)n8::N3; }
constexpr size_t K2C_STAGE = (size_t)K2_NF * n8::LayC::FS;
constexpr int K1C_OCC = 3, K2C_OCC = 3;
constexpr int K2C_NS = 2;  // K2c flux + Ja stages (one stage at four CTAs per SM leaves 80 registers: spills)
template <bool CP = false>
constexpr size_t k1c_smem() {
  // CP adds one (single-buffered) copy of the small parts Phit: pencils and face traces
  return (K1C_STAGE + k1c_b<CP>() + 9 * n8::LayC::FS + 2 * 6 * n8::N2 + 2 * n8::N3 +
          (CP ? 6 * n8::N2 + n8::N3 : 0)) * sizeof(float) + 64;
}
// per CTA: dynamic + static (a few words) + the 1 KB the SM reserves; 228 KB per SM
static_assert(3 * (k1c_smem<true>() + 64 + 1024) <= 233472, "three compensated K1c CTAs must fit an SM");
// K2c node-pass fields (1/J and the RK state: invJ, y, acc, comp), one bulk-copied buffer
constexpr size_t K2C_B = 4 * (size_t)n8::N3;
constexpr size_t k2c_smem() {
  return (K2C_NS * K2C_STAGE + 3 * n8::LayC::FS + 2 * 6 * 3 * n8::N2 + K2C_B) * sizeof(float) + 64;
}

// CP: the compensated FP32 form (see K1N8::cp): Phi + Phit in FP64 through the
// contractions, the RK4 epilogue of n8_rk_cp.
template <bool BATCH, bool GR = false, bool CP = false>  // GR: gradient only (see k_cons_k1_n8)
__global__ void __launch_bounds__(n8::CTHR, K1C_OCC)
    k_cons_k1_n8c(const __grid_constant__ K1N8<float> P, const K1N8<float>* __restrict__ plist,
                  const int2* __restrict__ tiles, long long ntiles) {
  using namespace n8;
  using real = float;
  constexpr int THR = CTHR, FSC = LayC::FS;
  constexpr int NPT = (N3 + THR - 1) / THR;   // node slots per thread (3, the last one partly)
  constexpr int NFT = 6 * N2;                 // 384 neighbour Phi face values
  constexpr int NFR = (NFT + THR - 1) / THR;  // 2 per thread
  // node-pass buffer fields (sB)
  constexpr int IY = 12, IACC = CP ? 12 : 13, ICOMP = CP ? 13 : 14;
  extern __shared__ __align__(128) unsigned char smraw[];
  real* sJa = reinterpret_cast<real*>(smraw);  // 9 fields (LayC), index al*3 + c
  real* sB = sJa + K1C_STAGE;                  // node order: c10 (10), Pi, invJ, [y], acc, comp
  real* sg = sB + k1c_b<CP>();                 // 9 partial gradients [al*3 + c] (LayC)
  real* sface = sg + 9 * FSC;                  // 2 x 384
  real* sphi = sface + 2 * NFT;                // 2 x 512 (LayC)
  real* sfaceT = sphi + 2 * N3;                // CP: 384 small parts of the face traces
  real* sphiT = sfaceT + (CP ? NFT : 0);       // CP: 512 small parts (LayC)
  uint64_t* bar = reinterpret_cast<uint64_t*>(sphiT + (CP ? N3 : 0));  // [0] Ja stage, [1] sB
  __shared__ int abort_flag;
  __shared__ __align__(16) double sJa0[2][9];  // CP: the element-constant metric part, double-buffered
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int al = tid >> 6, pc = tid & 63;  // contraction: axis (warp-uniform) and pencil
  // node of the neighbour's face-trace point for face source fs and this face's point pq
  // (computed, not tabled: three compensated CTAs need the table's shared memory)
  auto fnode = [](int fs, int pq) -> int {
    const int slot = face_slot(fs, pq);
    const int fn = slot >> 6;
    return face_node(faxis(fn), frow(fn, N), slot & 7, (slot >> 3) & 7, N);
  };
  const real inv2H = (real)(1.0 / (2.0 * P.H[0]));
  const bool comp_on = P.epi && P.comp != nullptr;
  // the compensated form reads the state's high part from the Phi pencils and the low part at every stage
  const bool need_y = !CP && P.epi && (P.stage == 1 || P.stage == 2 || (comp_on && P.stage == 3));
  const bool need_acc = P.epi && P.stage >= 1;
  const bool need_comp = comp_on && (CP || P.stage == 3);
  const unsigned txA = (unsigned)(K1C_STAGE * sizeof(real));
  const unsigned txB = (unsigned)((GR ? 1 : 12 + need_y + need_acc + need_comp) * N3 * sizeof(real));
  const double inv2Hd = 1.0 / (2.0 * P.H[0]);
  const long long T = ntiles;
  const long long GS = gridDim.x;
  auto tile_at = [&](long long t) -> int2 {
    if (t >= T) return make_int2(-1, -1);
    if constexpr (BATCH) return tiles[t];
    else return make_int2(0, (int)(P.e0 + t));
  };
  auto prm = [&](int sidx) -> const K1N8<real>& {
    if constexpr (BATCH) return plist[sidx];
    else return P;
  };
  int addr[8];
#pragma unroll
  for (int pos = 0; pos < 8; ++pos) addr[pos] = LayC::at(pnode(al, pc, pos));

  if (tid == 0) {
    abort_flag = 0;
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();

  // warp 0 copies the Ja blocks (issueA) or the node-pass fields (issueB) of tile tl
  auto issueA = [&](int2 tl) {
    const K1N8<real>& Q = prm(tl.x);
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[0], txA);
    }
    __syncwarp();
    const real* ja = CP ? Q.dJa : Q.Ja;
    if (lane < 9)
      bulk_g2s(sJa + lane * FSC, ja + ((long long)lane * Q.Ne + tl.y) * FSC, FSC * (unsigned)sizeof(real), &bar[0]);
  };
  auto issueB = [&](int2 tl) {
    const K1N8<real>& Q = prm(tl.x);
    const long long o = (long long)tl.y * N3;
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[1], txB);
    }
    __syncwarp();
    const unsigned nb = N3 * (unsigned)sizeof(real);
    const real* src = nullptr;
    if (GR) {
      if (lane == 11) src = Q.invdetJ + o;
    } else if (lane < 10) src = Q.c10 + lane * Q.nn + o;
    else if (lane == 10) src = Q.Pi + o;
    else if (lane == 11) src = Q.invdetJ + o;
    else if (lane == IY && !CP && need_y) src = Q.y + o;
    else if (lane == IACC && need_acc) src = Q.acc + o;
    else if (lane == ICOMP && need_comp) src = Q.comp + o;
    if (src) bulk_g2s(sB + lane * N3, src, nb, &bar[1]);
  };
  // face-trace slot r of this thread: value tid + r * THR = (face, pq) of the 384
  auto src_load = [&](int2 tl, int src[NFR]) {
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = tid + r * THR;
      src[r] = (tl.x >= 0 && idx < NFT) ? ::wt::bc_src(prm(tl.x).fsrc[(idx >> 6) + 6 * tl.y], prm(tl.x).Ne) : -1;
    }
  };
  // neighbour Phi face traces and this element's Phi of tile tl straight into
  // shared buffer b (asynchronous copies: no registers held)
  auto async_load = [&](int2 tl, const int src[NFR], int b) {
    const K1N8<real>& Q = prm(tl.x);
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = tid + r * THR;
      if (idx < NFT) {
        const bool ok = src[r] >= 0;
        const real* g = ok ? Q.Phi + (long long)(src[r] >> 6) * N3 + fnode(src[r], idx & 63) : Q.Phi;
        cp_async4(sface + b * NFT + idx, g, ok);
      }
    }
#pragma unroll
    for (int r = 0; r < NPT; ++r) {
      const int node = tid + r * THR;
      if (node < N3) cp_async4(sphi + b * N3 + LayC::at(node), Q.Phi + (long long)tl.y * N3 + node, true);
    }
    if constexpr (CP) {
      if (tid < 9) cp_async8(&sJa0[b][tid], Q.Ja0 + 9 * (long long)tl.y + tid);
    }
  };
  // CP: the small parts Phit of the same values into the single buffers sfaceT, sphiT
  // (zero-filled where there is no neighbour or no Phit)
  auto async_loadT = [&](int2 tl, const int src[NFR]) {
    const K1N8<real>& Q = prm(tl.x);
    const bool have = Q.Phit != nullptr;
    const real* base = have ? Q.Phit : Q.Phi;
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const int idx = tid + r * THR;
      if (idx < NFT) {
        const bool ok = have && src[r] >= 0;
        const real* g = ok ? base + (long long)(src[r] >> 6) * N3 + fnode(src[r], idx & 63) : base;
        cp_async4(sfaceT + idx, g, ok);
      }
    }
#pragma unroll
    for (int r = 0; r < NPT; ++r) {
      const int node = tid + r * THR;
      if (node < N3) cp_async4(sphiT + LayC::at(node), base + (long long)tl.y * N3 + node, have);
    }
  };
  auto emask_at = [&](int2 tl) -> int { return tl.x >= 0 ? prm(tl.x).emask[tl.y] : 0; };

  int2 t0 = tile_at(blockIdx.x), t1 = tile_at(blockIdx.x + GS), t2 = tile_at(blockIdx.x + 2 * GS);
  int emcur = 0, src1[NFR];
#pragma unroll
  for (int r = 0; r < NFR; ++r) src1[r] = -1;
  if (t0.x >= 0) {
    if (warp == 0) issueA(t0);
    emcur = emask_at(t0);
    int src0[NFR];
    src_load(t0, src0);
    async_load(t0, src0, 0);
    if constexpr (CP) async_loadT(t0, src0);
    src_load(t1, src1);
    cp_async_wait_all();
  }
  __syncthreads();

  int it = 0;
  for (long long t = blockIdx.x; t < T; t += GS, ++it) {
    const int fb = it & 1;
    const unsigned parity = it & 1;
    int2 t3 = make_int2(-1, -1);
    if constexpr (BATCH) {
      t3 = tile_at(t + 3 * GS);
    } else {
      t0 = tile_at(t);
      t1 = tile_at(t + GS);
      t2 = tile_at(t + 2 * GS);
    }
    const bool has_next = t1.x >= 0;
    const int emnext = emask_at(t1);
    int src2[NFR];
    src_load(t2, src2);
    if (tid == 0 && !wait_phase(&bar[0], parity, P.flag)) abort_flag = 1;
    __syncthreads();  // the previous element is finished: sB and buffers fb^1 are free
    if (abort_flag) return;  // the only copy in flight is the one waited for
    if (warp == 0) issueB(t0);  // lands while the contraction pass runs
    if (has_next) async_load(t1, src1, fb ^ 1);
    const K1N8<real>& Q = prm(t0.x);
    const long long e = t0.y;
    const real* sPhi = sphi + fb * N3;
    const real* sfc = sface + fb * NFT;
    const int mask = emcur & 63;
    const int bnd = emcur >> 6;
    // ---- contractions: thread (al, pc); the operator in the constant bank is
    // 0.5 G (scaling by 1/2 is exact) ----
    if constexpr (CP) {
      // The state u = Phi + Phit enters the derivative in FP64: FP32 rounding of
      // it, or of the contraction of it, would be amplified by the second
      // derivative in Pi-dot.  With Ja = Ja0 + dJa (Ja0 element-constant, FP64):
      //   0.5 D(Ja u) + 0.5 Ja D u = (2 Ja0 + dJa) (0.5 D u) + 0.5 D(dJa u),
      // so the only contraction left in FP32 acts on dJa u, which is as small as
      // the metric terms' variation over the element; its rounding error is that
      // much smaller than the one of 0.5 D(Ja u) in FP32.  Once 0.5 D u has been
      // formed in FP64 it is a gradient-sized value, and FP32 suffices for the rest.
      const real* sPhiT = sphiT;
      float cu[8], uf[8], jmp0, jmp1;
      {
        double u[8];
#pragma unroll
        for (int pos = 0; pos < 8; ++pos) u[pos] = (double)sPhi[addr[pos]] + (double)sPhiT[addr[pos]];
#pragma unroll
        for (int l = 0; l < 8; ++l) {
          double acc = P.Gd[l * 8] * u[0];
#pragma unroll
          for (int m = 1; m < 8; ++m) acc = fma(P.Gd[l * 8 + m], u[m], acc);
          cu[l] = (float)acc;  // 0.5 D u
        }
        // centred-flux SAT of an interior al-face: jump on the face row (formed in FP64)
        const bool sat0 = (mask >> (2 * al)) & 1, sat1 = (mask >> (2 * al + 1)) & 1;
        const int f0 = (2 * al) * N2 + pc, f1 = (2 * al + 1) * N2 + pc;
        jmp0 = sat0 ? (float)(-inv2Hd * (((double)sfc[f0] + (double)sfaceT[f0]) - u[0])) : 0.f;
        jmp1 = sat1 ? (float)(inv2Hd * (((double)sfc[f1] + (double)sfaceT[f1]) - u[7])) : 0.f;
#pragma unroll
        for (int pos = 0; pos < 8; ++pos) uf[pos] = (float)u[pos];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const real* mc = sJa + (al * 3 + c) * FSC;
        const float m0 = (float)sJa0[fb][al * 3 + c];
        float w[8];
#pragma unroll
        for (int pos = 0; pos < 8; ++pos) w[pos] = mc[addr[pos]] * uf[pos];
        real* gout = sg + (al * 3 + c) * FSC;
#pragma unroll
        for (int l = 0; l < 8; ++l) {
          float o = P.Gh[l * 8] * w[0];
#pragma unroll
          for (int m = 1; m < 8; ++m) o = fmaf(P.Gh[l * 8 + m], w[m], o);  // 0.5 D(dJa u)
          const float dl = mc[addr[l]];
          float r = fmaf(2.f * m0 + dl, cu[l], o);
          if (l == 0) r = fmaf(m0 + dl, jmp0, r);
          if (l == 7) r = fmaf(m0 + dl, jmp1, r);
          gout[addr[l]] = r;
        }
      }
    } else {
      float u[8], cu[8], w[8], o[8];
#pragma unroll
      for (int pos = 0; pos < 8; ++pos) u[pos] = sPhi[addr[pos]];
      contract8(P.Gh, u, cu);  // 0.5 D u
      // centred-flux SAT of an interior al-face: jump on the face row
      const bool sat0 = (mask >> (2 * al)) & 1, sat1 = (mask >> (2 * al + 1)) & 1;
      const real jmp0 = sat0 ? -inv2H * (sfc[(2 * al) * N2 + pc] - u[0]) : (real)0;
      const real jmp1 = sat1 ? inv2H * (sfc[(2 * al + 1) * N2 + pc] - u[7]) : (real)0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const real* mc = sJa + (al * 3 + c) * FSC;
        float m[8];
#pragma unroll
        for (int pos = 0; pos < 8; ++pos) {
          m[pos] = mc[addr[pos]];
          w[pos] = m[pos] * u[pos];
        }
        contract8(P.Gh, w, o);  // 0.5 D (Ja u)
        real* gout = sg + (al * 3 + c) * FSC;
#pragma unroll
        for (int l = 0; l < 8; ++l) {
          real r = fmaf(m[l], cu[l], o[l]);  // 0.5 D(Ja u) + 0.5 Ja D u
          if (l == 0) r += m[0] * jmp0;
          if (l == 7) r += m[7] * jmp1;
          gout[addr[l]] = r;
        }
      }
    }
    if (tid == 0 && !wait_phase(&bar[1], parity, P.flag)) abort_flag = 1;
    __syncthreads();  // partial gradients and sB complete; the Ja stage is free
    if (abort_flag) return;
    if (warp == 0 && has_next) issueA(t1);  // lands while the node pass runs
    if constexpr (CP) {
      if (has_next) async_loadT(t1, src1);  // the small parts are read by the contraction pass only
    }
    // ---- node phase ----
#pragma unroll
    for (int rr = 0; rr < NPT; ++rr) {
      const int node = tid + rr * THR;
      if (node >= N3) continue;
      const int ti = node & 7, tj = (node >> 3) & 7, tk = node >> 6;
      const int at = LayC::at(node);
      const long long n = e * N3 + node;
      const real u = sPhi[at];  // CP: the state's high part
      const real invJ = sB[11 * N3 + node];
      real g0 = (sg[at] + sg[3 * FSC + at]) + sg[6 * FSC + at];
      real g1 = (sg[FSC + at] + sg[4 * FSC + at]) + sg[7 * FSC + at];
      real g2 = (sg[2 * FSC + at] + sg[5 * FSC + at]) + sg[8 * FSC + at];
      g0 *= invJ; g1 *= invJ; g2 *= invJ;
      if constexpr (GR) {
        Q.gout[n] = g0;
        Q.gout[Q.nn + n] = g1;
        Q.gout[2 * Q.nn + n] = g2;
        continue;
      }
      real cc[10];
#pragma unroll
      for (int c = 0; c < 10; ++c) cc[c] = sB[c * N3 + node];
      const real a = cc[0];
      const real b0 = cc[1], b1 = cc[2], b2 = cc[3];
      const real K0 = cc[4], K1v = cc[5], K2 = cc[6], K3 = cc[7], K4 = cc[8], K5 = cc[9];
      const real Pi = sB[10 * N3 + node];
      const real F0 = b0 * Pi + (K0 * g0 + K1v * g1 + K2 * g2);
      const real F1 = b1 * Pi + (K1v * g0 + K3 * g1 + K4 * g2);
      const real F2 = b2 * Pi + (K2 * g0 + K4 * g1 + K5 * g2);
      real phid = b0 * g0 + b1 * g1 + b2 * g2 + a * Pi;
      if (bnd && Q.bc_on) {
        // the whole stage value where a boundary term reads Phi itself
        const real uf = CP && Q.Phit ? u + Q.Phit[n] : u;
        k1_boundary<real>(Q, e, ti, tj, tk, n, uf, Pi, g0, g1, g2, cc, phid);
      }
      {  // flux in the LayC element-block layout read by K2
        const long long fo = e * FSC + at, fstr = Q.Ne * FSC;
        Q.F[fo] = F0;
        Q.F[fstr + fo] = F1;
        Q.F[2 * fstr + fo] = F2;
      }
      const real accv = need_acc ? sB[IACC * N3 + node] : (real)0;
      const real compv = need_comp ? sB[ICOMP * N3 + node] : (real)0;
      if constexpr (CP) {
        if (P.epi)
          n8_rk_cp(P.stage, Q.dt, phid, u, accv, compv, n, Q.y, Q.acc, Q.out, Q.comp, Q.hcopy, P.flag);
        else
          Q.Phidot[n] = phid;
      } else {
        const real yv = need_y ? sB[IY * N3 + node] : (real)0;
        if (P.epi)
          n8_rk<real>(P.stage, Q.dt, phid, u, yv, accv, compv, n, Q.y, Q.acc, Q.out, comp_on ? Q.comp : nullptr,
                      P.flag);
        else
          Q.Phidot[n] = phid;
      }
    }
    cp_async_wait_all();  // this thread's copies into buffers fb^1 (the barrier above the next element publishes them)
    emcur = emnext;
#pragma unroll
    for (int r = 0; r < NFR; ++r) src1[r] = src2[r];
    if constexpr (BATCH) {
      t0 = t1;
      t1 = t2;
      t2 = t3;
    }
  }
}

template <bool BATCH>
__global__ void __launch_bounds__(n8::CTHR, K2C_OCC)
    k_cons_k2_n8c(const __grid_constant__ K2N8<float> P, const K2N8<float>* __restrict__ plist,
                  const int2* __restrict__ tiles, long long ntiles) {
  using namespace n8;
  using real = float;
  constexpr int THR = CTHR, NS = K2C_NS, FSC = LayC::FS;
  constexpr int NPT = (N3 + THR - 1) / THR;  // 3 node slots per thread
  constexpr int NFACE = 6 * 3 * N2;          // 1152 neighbour flux face values
  constexpr int NFR = NFACE / THR;           // 6 per thread
  extern __shared__ __align__(128) unsigned char smraw[];
  real* stg = reinterpret_cast<real*>(smraw);  // NS stages x 12 fields
  real* sdiv = stg + NS * K2C_STAGE;           // 3 partial divergences (LayC)
  real* sface = sdiv + 3 * FSC;                // 2 x 1152
  real* sB = sface + 2 * NFACE;                // node-pass fields: invJ, y, acc, comp (node order)
  uint64_t* bar = reinterpret_cast<uint64_t*>(sB + K2C_B);  // NS stage barriers, then the sB barrier
  __shared__ int abort_flag;
  __shared__ short ftab[6 * N2];  // LayC offset of face-trace point pq on face fn of an element block
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int al = tid >> 6, pc = tid & 63;
  const real inv2H = (real)(1.0 / (2.0 * P.H[0]));
  const bool comp_on = P.epi && P.comp != nullptr;
  const bool need_y = P.epi && (P.stage <= 2 || (comp_on && P.stage == 3));
  const bool need_acc = P.epi && P.stage >= 1;
  const bool need_comp = comp_on && P.stage == 3;
  const unsigned tx_bytes = (unsigned)(K2C_STAGE * sizeof(real));
  const unsigned txB = (unsigned)((1 + need_y + need_acc + need_comp) * N3 * sizeof(real));
  const long long T = ntiles;
  const long long GS = gridDim.x;
  auto tile_at = [&](long long t) -> int2 {
    if (t >= T) return make_int2(-1, -1);
    if constexpr (BATCH) return tiles[t];
    else return make_int2(0, (int)(P.e0 + t));
  };
  auto prm = [&](int sidx) -> const K2N8<real>& {
    if constexpr (BATCH) return plist[sidx];
    else return P;
  };
  int addr[8];
#pragma unroll
  for (int pos = 0; pos < 8; ++pos) addr[pos] = LayC::at(pnode(al, pc, pos));

  for (int i = tid; i < 6 * N2; i += THR)
    ftab[i] = (short)LayC::at(face_node(faxis(i >> 6), frow(i >> 6, N), i & 7, (i >> 3) & 7, N));
  if (tid == 0) {
    abort_flag = 0;
    for (int k = 0; k <= NS; ++k) mbar_init(&bar[k], 1);
    fence_barrier_init();
  }
  __syncthreads();

  auto issue = [&](int2 tl, int s) {
    const K2N8<real>& Q = prm(tl.x);
    const long long e = tl.y;
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[s], tx_bytes);
    }
    __syncwarp();
    real* d = stg + s * K2C_STAGE;
    if (lane < K2_NF) {
      const real* src = lane < 3 ? (lane == 0 ? Q.F0 : lane == 1 ? Q.F1 : Q.F2) + e * FSC
                                 : Q.Ja + ((long long)(lane - 3) * Q.Ne + e) * FSC;
      bulk_g2s(d + lane * FSC, src, FSC * (unsigned)sizeof(real), &bar[s]);
    }
  };
  // face-trace slot r of this thread is face r, flux component tid >> 6 (warp-
  // uniform), point tid & 63: sface[(r * 3 + c) * 64 + pq] = sface[r * THR + tid]
  auto src_load = [&](int2 tl, int src[NFR]) {
#pragma unroll
    for (int r = 0; r < NFR; ++r) src[r] = tl.x >= 0 ? ::wt::bc_src(prm(tl.x).fsrc[r + 6 * tl.y], prm(tl.x).Ne) : -1;
  };
  // neighbour flux face traces of tile tl straight into shared buffer b
  auto async_faces = [&](int2 tl, const int src[NFR], int b) {
    const K2N8<real>& Q = prm(tl.x);
    const int c = tid >> 6, pq = tid & 63;
    const real* Fc = c == 0 ? Q.F0 : c == 1 ? Q.F1 : Q.F2;
#pragma unroll
    for (int r = 0; r < NFR; ++r) {
      const bool ok = src[r] >= 0;
      const real* g = ok ? Fc + (long long)(src[r] >> 6) * FSC + ftab[face_slot(src[r], pq)] : Fc;
      cp_async4(sface + b * NFACE + r * THR + tid, g, ok);
    }
  };
  auto emask_at = [&](int2 tl) -> int { return tl.x >= 0 ? prm(tl.x).emask[tl.y] : 0; };
  // warp 0 copies the node-pass fields of tile tl into sB
  auto issueB = [&](int2 tl) {
    const K2N8<real>& Q = prm(tl.x);
    const long long o = (long long)tl.y * N3;
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect_tx(&bar[NS], txB);
    }
    __syncwarp();
    const unsigned nb = N3 * (unsigned)sizeof(real);
    if (lane == 0) bulk_g2s(sB, Q.invdetJ + o, nb, &bar[NS]);
    else if (lane == 1 && need_y) bulk_g2s(sB + N3, Q.y + o, nb, &bar[NS]);
    else if (lane == 2 && need_acc) bulk_g2s(sB + 2 * N3, Q.acc + o, nb, &bar[NS]);
    else if (lane == 3 && need_comp) bulk_g2s(sB + 3 * N3, Q.comp + o, nb, &bar[NS]);
  };

  int2 t0 = tile_at(blockIdx.x), t1 = tile_at(blockIdx.x + GS), t2 = tile_at(blockIdx.x + 2 * GS);
  int emcur = 0, src1[NFR];
#pragma unroll
  for (int r = 0; r < NFR; ++r) src1[r] = -1;
  if (t0.x >= 0) {
    if (warp == 0) issue(t0, 0);
    emcur = emask_at(t0);
    int src0[NFR];
    src_load(t0, src0);
    async_faces(t0, src0, 0);
    src_load(t1, src1);
    cp_async_wait_all();
  }
  __syncthreads();

  int it = 0;
  for (long long t = blockIdx.x; t < T; t += GS, ++it) {
    const int s = it % NS, fb = it & 1;
    const unsigned parity = (it / NS) & 1;
    int2 t3 = make_int2(-1, -1);
    if constexpr (BATCH) {
      t3 = tile_at(t + 3 * GS);
    } else {
      t0 = tile_at(t);
      t1 = tile_at(t + GS);
      t2 = tile_at(t + 2 * GS);
    }
    const bool has_next = t1.x >= 0;
    const int emnext = emask_at(t1);
    int src2[NFR];
    src_load(t2, src2);
    if (tid == 0 && !wait_phase(&bar[s], parity, P.flag)) abort_flag = 1;
    __syncthreads();  // the previous element is finished: stage (it+1) % NS, sB and face buffer fb^1 are free
    if (abort_flag) {
      return;  // NS = 2: the only copy in flight is the one waited for
    }
    if (warp == 0) {
      if (NS > 1 && t1.x >= 0) issue(t1, (it + 1) % NS);
      issueB(t0);  // lands while the contraction below runs
    }
    if (has_next) async_faces(t1, src1, fb ^ 1);
    const K2N8<real>& Q = prm(t0.x);
    const long long e = t0.y;
    const real* d = stg + s * K2C_STAGE;
    const real* sF = d;
    const real* sJa = d + 3 * FSC;
    const real* sfc = sface + fb * NFACE;
    const int mask = emcur & 63;
    const int bnd = emcur >> 6;
    // ---- contractions: thread (al, pc) ----
    {
      const real* m0 = sJa + (al * 3 + 0) * FSC;
      const real* m1 = sJa + (al * 3 + 1) * FSC;
      const real* m2 = sJa + (al * 3 + 2) * FSC;
      // r = 0.5 D(Ja^al . F) + 0.5 sum_c Ja^al_c D(F_c), one component live at a time
      // (the operator in the constant bank is 0.5 G; scaling by 1/2 is exact)
      float v[8], o[8], r[8];
#pragma unroll
      for (int pos = 0; pos < 8; ++pos) {
        const int ad = addr[pos];
        v[pos] = m0[ad] * sF[ad] + m1[ad] * sF[FSC + ad] + m2[ad] * sF[2 * FSC + ad];
      }
      contract8(P.Gh, v, r);  // 0.5 D (Ja^al . F)
      const bool sat0 = (mask >> (2 * al)) & 1, sat1 = (mask >> (2 * al + 1)) & 1;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const real* mc = sJa + (al * 3 + c) * FSC;
        const real* fc = sF + c * FSC;
        float fv[8];
#pragma unroll
        for (int pos = 0; pos < 8; ++pos) fv[pos] = fc[addr[pos]];
        contract8(P.Gh, fv, o);  // 0.5 D F_c
#pragma unroll
        for (int l = 0; l < 8; ++l) r[l] = fmaf(mc[addr[l]], o[l], r[l]);
        // centred-flux SAT of an interior al-face on the face rows
        if (sat0) r[0] -= inv2H * mc[addr[0]] * (sfc[((2 * al) * 3 + c) * N2 + pc] - fv[0]);
        if (sat1) r[7] += inv2H * mc[addr[7]] * (sfc[((2 * al + 1) * 3 + c) * N2 + pc] - fv[7]);
      }
#pragma unroll
      for (int l = 0; l < 8; ++l) sdiv[al * FSC + addr[l]] = r[l];
    }
    if (tid == 0 && !wait_phase(&bar[NS], it & 1, P.flag)) abort_flag = 1;
    __syncthreads();
    if (abort_flag) return;
    if (NS == 1 && warp == 0 && t1.x >= 0) issue(t1, 0);  // one stage: refilled once the contraction has read it
#pragma unroll
    for (int rr = 0; rr < NPT; ++rr) {
      const int node = tid + rr * THR;
      if (node >= N3) continue;
      const int ti = node & 7, tj = (node >> 3) & 7, tk = node >> 6;
      const int at = LayC::at(node);
      const long long n = e * N3 + node;
      real dv = (sdiv[at] + sdiv[FSC + at]) + sdiv[2 * FSC + at];
      dv *= sB[node];
      if (bnd && Q.bc_on) {
        const int idx3[3] = {ti, tj, tk};
        for (int f = 0; f < 6; ++f) {
          if (Q.bdry[f + 6 * e] == 0) continue;
          const int ax = f >> 1;
          if (idx3[ax] != ((f & 1) ? 7 : 0)) continue;
          const int p = ax == 0 ? tj : ti, q = ax == 2 ? tj : tk;
          dv += Q.bbuf[(long long)::wt::bc_slot(Q.bslot[f + 6 * e], Q.nbf) * N2 + p + 8 * q];
        }
      }
      const real yv = need_y ? sB[N3 + node] : (real)0, accv = need_acc ? sB[2 * N3 + node] : (real)0;
      const real compv = need_comp ? sB[3 * N3 + node] : (real)0;
      if (P.epi)
        n8_rk<real>(P.stage, Q.dt, dv, yv, yv, accv, compv, n, Q.y, Q.acc, Q.out, comp_on ? Q.comp : nullptr, P.flag);
      else
        Q.Pidot[n] = dv;
    }
    cp_async_wait_all();  // this thread's face copies into buffer fb^1
    emcur = emnext;
#pragma unroll
    for (int r = 0; r < NFR; ++r) src1[r] = src2[r];
    if constexpr (BATCH) {
      t0 = t1;
      t1 = t2;
      t2 = t3;
    }
  }
}

// padded element-block copy of the nine metric-term fields for the n = 8 path
template <typename real, typename L>
__global__ void k_pad_fields(long long Ne, int nf, const real* __restrict__ src, real* __restrict__ dst) {
  const long long total = (long long)nf * Ne * n8::N3;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
    const long long f = x / (Ne * n8::N3);
    const long long r = x - f * Ne * n8::N3;
    const long long e = r / n8::N3;
    const int t = (int)(r - e * n8::N3);
    dst[(f * Ne + e) * L::FS + L::at(t)] = src[x];
  }
}

// Split of the FP64 metric terms for the compensated FP32 form: per element
// the mean of each of the nine fields (FP64), and every node's deviation from
// it rounded to FP32 (n = 8: in the LayC element blocks of the CUDA-core
// kernels; otherwise node order).  FP32 rounding then perturbs the metric
// terms by the deviation's ulp, not the field's.
__global__ void k_split_metric_mean(int N3, long long Ne, long long nn, const double* __restrict__ Ja,
                                    double* __restrict__ Ja0) {
  const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;  // one warp per (element, field)
  const int lane = threadIdx.x & 31;
  if (w >= 9 * Ne) return;  // whole warps leave together
  const long long e = w / 9;
  const int c = (int)(w - 9 * e);
  const double* src = Ja + c * nn + e * N3;
  double sum = 0.0;
  for (int t = lane; t < N3; t += 32) sum += src[t];
  for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if (lane == 0) Ja0[9 * e + c] = sum / N3;
}

template <bool LAYC>
__global__ void k_split_metric_dev(int N3, long long Ne, long long nn, const double* __restrict__ Ja,
                                   const double* __restrict__ Ja0, float* __restrict__ dJa) {
  const long long total = 9 * nn;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
    const long long c = x / nn, r = x - c * nn, e = r / N3;
    const int t = (int)(r - e * N3);
    const float v = (float)(Ja[x] - Ja0[9 * e + c]);
    if (LAYC)
      dJa[(c * Ne + e) * n8::LayC::FS + n8::LayC::at(t)] = v;
    else
      dJa[x] = v;
  }
}

int launch_split_metric(const DevMesh& m, cudaStream_t s) {
  const int N3 = m.N * m.N * m.N;
  const long long warps = 9 * m.Ne;
  k_split_metric_mean<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(N3, m.Ne, m.nn, m.Ja, m.Ja0);
  if (m.N == 8)
    k_split_metric_dev<true><<<4096, 256, 0, s>>>(N3, m.Ne, m.nn, m.Ja, m.Ja0, (float*)m.dJa);
  else
    k_split_metric_dev<false><<<4096, 256, 0, s>>>(N3, m.Ne, m.nn, m.Ja, m.Ja0, (float*)m.dJa);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// element-block layout of the mesh's n = 8 kernels: 0 = Lay<real>, 1 = LayC (FP32 CUDA-core form)
static int n8_layout(const DevMesh& m) {
  return m.precision == 1 && (m.fp32_form == WT_FP32_CUDA_CORES || m.fp32_form == WT_FP32_COMPENSATED) ? 1 : 0;
}
static long long n8_fs(const DevMesh& m) {
  return m.precision == 0 ? n8::Lay<double>::FS : n8_layout(m) ? n8::LayC::FS : n8::Lay<float>::FS;
}

int launch_pad_metric_n8(DevMesh& m, cudaStream_t s) {
  if (m.precision == 0)
    k_pad_fields<double, n8::Lay<double>><<<4096, 256, 0, s>>>(m.Ne, 9, (const double*)m.Ja_r, (double*)m.Ja_n8);
  else if (n8_layout(m))
    k_pad_fields<float, n8::LayC><<<4096, 256, 0, s>>>(m.Ne, 9, (const float*)m.Ja_r, (float*)m.Ja_n8);
  else
    k_pad_fields<float, n8::Lay<float>><<<4096, 256, 0, s>>>(m.Ne, 9, (const float*)m.Ja_r, (float*)m.Ja_n8);
  m.ja_n8_layout = n8_layout(m);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// words per field of the element-block layouts (the larger, FP32, one: an
// allocation of this size serves both precisions)
long long n8_padded_field_size(long long Ne) { return Ne * n8::FS; }
long long n8_flux_block(const DevMesh& m) { return n8_fs(m); }

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

template <typename real>
static K1N8<real> k1n8_params(const DevMesh& m, const DevCoef& c, const void* Phi, const void* Pi, void* F,
                              void* Phidot, void* bbuf, const ConsBC& bc, const RKStage& rk, unsigned* flag) {
  K1N8<real> P;
  P.Ne = m.Ne; P.nn = m.nn; P.e0 = 0;
  P.Phi = (const real*)Phi; P.Pi = (const real*)Pi; P.c10 = (const real*)c.c10;
  P.Ja = (const real*)m.Ja_n8; P.invdetJ = (const real*)m.invdetJ_r;
  P.nbr = m.nbr; P.nbrf = m.nbrf; P.bdry = m.bdry; P.bslot = m.bslot; P.G = m.G; P.H = m.H;
  P.emask = m.emask; P.fsrc = m.fsrc;
  P.F = (real*)F; P.Phidot = (real*)Phidot; P.bbuf = (real*)bbuf;
  P.bc_on = bc.on; P.exc_tag = bc.exc_tag; P.nbf = m.nbf; P.kind = bc.kinds[0]; P.sigma = bc.sigma;
  P.bnorm = (const real*)m.bnorm;
  P.gPhi = (const real*)bc.gPhi; P.gPi = (const real*)bc.gPi;
  P.gDx = (const real*)bc.gDx; P.gDy = (const real*)bc.gDy; P.gDz = (const real*)bc.gDz;
  P.epi = rk.on; P.stage = rk.stage; P.dt = rk.dt;
  P.y = (real*)rk.y; P.acc = (real*)rk.acc; P.out = (real*)rk.out; P.comp = (real*)rk.comp; P.flag = flag;
  for (int i = 0; i < 64; ++i) P.Gh[i] = (float)(0.5 * m.ops.G[i]);
  P.gout = nullptr;
  P.cp = m.precision == WT_F32 && m.fp32_form == WT_FP32_COMPENSATED ? 1 : 0;
  P.Phit = (const real*)rk.phit;
  P.dJa = (const real*)m.dJa;
  P.Ja0 = m.Ja0;
  P.hcopy = (real*)rk.hcopy;
  for (int i = 0; i < 64; ++i) P.Gd[i] = 0.5 * m.ops.G[i];
  return P;
}

template <typename real>
static K2N8<real> k2n8_params(const DevMesh& m, const void* F, void* Pidot, const void* bbuf, const ConsBC& bc,
                              const RKStage& rk, unsigned* flag) {
  K2N8<real> P;
  P.Ne = m.Ne; P.nn = m.nn; P.e0 = 0;
  const long long fs = m.Ne * n8_fs(m);
  P.F0 = (const real*)F; P.F1 = (const real*)F + fs; P.F2 = (const real*)F + 2 * fs;
  P.Ja = (const real*)m.Ja_n8; P.invdetJ = (const real*)m.invdetJ_r;
  P.nbr = m.nbr; P.nbrf = m.nbrf; P.bdry = m.bdry; P.bslot = m.bslot; P.G = m.G; P.H = m.H;
  P.emask = m.emask; P.fsrc = m.fsrc;
  P.bbuf = (const real*)bbuf; P.bc_on = bc.on; P.nbf = m.nbf;
  P.Pidot = (real*)Pidot;
  P.epi = rk.on; P.stage = rk.stage; P.dt = rk.dt;
  P.y = (real*)rk.y; P.acc = (real*)rk.acc; P.out = (real*)rk.out; P.comp = (real*)rk.comp; P.flag = flag;
  for (int i = 0; i < 64; ++i) P.Gh[i] = (float)(0.5 * m.ops.G[i]);
  return P;
}

// Launch K1 (which = 1) or K2 (which = 2) of one instantiation: a single solve
// (plist == nullptr, ntiles = P.Ne) or a work list over the solves of plist.
template <typename real, int NT, bool BATCH>
static int n8_launch(int which, const void* hP, const void* plist, const int2* tiles, long long ntiles, cudaStream_t s) {
  static bool attr1 = false, attr2 = false;
  if (which == 1) {
    if (!attr1) {
      if (cudaFuncSetAttribute(k_cons_k1_n8<real, NT, BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)k1_smem<real>()) != cudaSuccess)
        return -2;
      attr1 = true;
    }
    const long long cap = (long long)sm_count() * n8::Occ<real>::k1;
    const long long grid = ntiles < cap ? ntiles : cap;
    if (grid <= 0) return 0;
    k_cons_k1_n8<real, NT, BATCH><<<(unsigned)grid, n8::THREADS, k1_smem<real>(), s>>>(
        *(const K1N8<real>*)hP, (const K1N8<real>*)plist, tiles, ntiles);
  } else {
    if (!attr2) {
      if (cudaFuncSetAttribute(k_cons_k2_n8<real, NT, BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)k2_smem<real>()) != cudaSuccess)
        return -2;
      attr2 = true;
    }
    const long long cap = (long long)sm_count() * K2Shape<real>::OCC;
    const long long grid = ntiles < cap ? ntiles : cap;
    if (grid <= 0) return 0;
    k_cons_k2_n8<real, NT, BATCH><<<(unsigned)grid, K2Shape<real>::THR, k2_smem<real>(), s>>>(
        *(const K2N8<real>*)hP, (const K2N8<real>*)plist, tiles, ntiles);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <bool BATCH, bool CP>
static int n8c_launch(int which, const void* hP, const void* plist, const int2* tiles, long long ntiles,
                      cudaStream_t s) {
  static bool attr1 = false, attr2 = false;
  const int occ = which == 1 ? K1C_OCC : K2C_OCC;
  const long long cap = (long long)sm_count() * occ;
  const long long grid = ntiles < cap ? ntiles : cap;
  if (which == 1) {
    constexpr size_t smem = k1c_smem<CP>();
    if (!attr1) {
      // three CTAs per SM need (nearly) all of the SM's shared memory
      if (cudaFuncSetAttribute(k_cons_k1_n8c<BATCH, false, CP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem) != cudaSuccess ||
          cudaFuncSetAttribute(k_cons_k1_n8c<BATCH, false, CP>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
        return -2;
      attr1 = true;
    }
    if (grid <= 0) return 0;
    k_cons_k1_n8c<BATCH, false, CP><<<(unsigned)grid, n8::CTHR, smem, s>>>(
        *(const K1N8<float>*)hP, (const K1N8<float>*)plist, tiles, ntiles);
  } else {
    if (!attr2) {
      if (cudaFuncSetAttribute(k_cons_k2_n8c<BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k2c_smem()) !=
              cudaSuccess ||
          cudaFuncSetAttribute(k_cons_k2_n8c<BATCH>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
        return -2;
      attr2 = true;
    }
    if (grid <= 0) return 0;
    k_cons_k2_n8c<BATCH><<<(unsigned)grid, n8::CTHR, k2c_smem(), s>>>(*(const K2N8<float>*)hP,
                                                                       (const K2N8<float>*)plist, tiles, ntiles);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <bool BATCH>
static int n8_dispatch(int which, int precision, int fp32_form, const void* hP, const void* plist, const int2* tiles,
                       long long ntiles, cudaStream_t s) {
  if (precision == 0) return n8_launch<double, 0, BATCH>(which, hP, plist, tiles, ntiles, s);
  if (fp32_form == WT_FP32_COMPENSATED) return n8c_launch<BATCH, true>(which, hP, plist, tiles, ntiles, s);
  if (fp32_form == WT_FP32_CUDA_CORES) return n8c_launch<BATCH, false>(which, hP, plist, tiles, ntiles, s);
  if (fp32_form == WT_FP32_BF16X2) return n8_launch<float, 2, BATCH>(which, hP, plist, tiles, ntiles, s);
  return n8_launch<float, 3, BATCH>(which, hP, plist, tiles, ntiles, s);
}

int launch_cons_k1_n8(const DevMesh& m, const DevCoef& c, const void* Phi, const void* Pi, void* F, void* Phidot,
                      void* bbuf, const ConsBC& bc, const RKStage& rk, unsigned* flag, cudaStream_t s, long long e0,
                      long long e1) {
  if (e1 < 0) e1 = m.Ne;
  if (m.precision == 0) {
    K1N8<double> P = k1n8_params<double>(m, c, Phi, Pi, F, Phidot, bbuf, bc, rk, flag);
    P.e0 = e0;
    return n8_dispatch<false>(1, 0, m.fp32_form, &P, nullptr, nullptr, e1 - e0, s);
  }
  K1N8<float> P = k1n8_params<float>(m, c, Phi, Pi, F, Phidot, bbuf, bc, rk, flag);
  P.e0 = e0;
  return n8_dispatch<false>(1, 1, m.fp32_form, &P, nullptr, nullptr, e1 - e0, s);
}

int launch_cons_fk_n8(const DevMesh& m, const DevCoef& c, const void* Fin, void* Fout, const void* Phi, void* bbuf,
                      const ConsBC& bc, const RKStage& rkQ, const RKStage& rkP, cudaStream_t s) {
  if (m.precision != 0 || rkQ.stage < 0 || rkQ.stage > 2 || rkP.stage != rkQ.stage + 1 || !rkQ.on || !rkP.on)
    return -4;
  FKN8 P;
  P.a = k2n8_params<double>(m, Fin, nullptr, bbuf, bc, rkQ, m.errflag);
  P.b = k1n8_params<double>(m, c, Phi, nullptr, Fout, nullptr, bbuf, bc, rkP, m.errflag);
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_cons_fk_n8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fk_smem()) != cudaSuccess)
      return -2;
    attr = true;
  }
  const long long cap = sm_count(), grid = m.Ne < cap ? m.Ne : cap;
  if (grid <= 0) return 0;
  k_cons_fk_n8<<<(unsigned)grid, n8::THREADS, fk_smem(), s>>>(P);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_cons_k2_n8(const DevMesh& m, const void* F, void* Pidot, const void* bbuf, const ConsBC& bc,
                      const RKStage& rk, unsigned* flag, cudaStream_t s, long long e0, long long e1) {
  if (e1 < 0) e1 = m.Ne;
  if (m.precision == 0) {
    K2N8<double> P = k2n8_params<double>(m, F, Pidot, bbuf, bc, rk, flag);
    P.e0 = e0;
    return n8_dispatch<false>(2, 0, m.fp32_form, &P, nullptr, nullptr, e1 - e0, s);
  }
  K2N8<float> P = k2n8_params<float>(m, F, Pidot, bbuf, bc, rk, flag);
  P.e0 = e0;
  return n8_dispatch<false>(2, 1, m.fp32_form, &P, nullptr, nullptr, e1 - e0, s);
}

// Gradient-only launch (the energy's split-form gradient, apply_gradient3d! with the
// centred-flux SAT) through the n = 8 kernels: gout = 3 fields of nn words.
template <typename real, int NT>
static int launch_grad_n8_t(const K1N8<real>& P, bool cuda_core, cudaStream_t s) {
  if constexpr (std::is_same<real, float>::value) {
    if (cuda_core) {
      static bool attr = false;
      if (!attr) {
        if (cudaFuncSetAttribute(k_cons_k1_n8c<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)k1c_smem()) != cudaSuccess ||
            cudaFuncSetAttribute(k_cons_k1_n8c<false, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
          return -2;
        attr = true;
      }
      const long long cap = (long long)sm_count() * K1C_OCC, grid = P.Ne < cap ? P.Ne : cap;
      k_cons_k1_n8c<false, true><<<(unsigned)grid, n8::CTHR, k1c_smem(), s>>>(P, nullptr, nullptr, P.Ne);
      return cudaGetLastError() == cudaSuccess ? 0 : -2;
    }
  }
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_cons_k1_n8<real, NT, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)k1_smem<real>()) != cudaSuccess)
      return -2;
    attr = true;
  }
  const long long cap = (long long)sm_count() * n8::Occ<real>::k1, grid = P.Ne < cap ? P.Ne : cap;
  k_cons_k1_n8<real, NT, false, true><<<(unsigned)grid, n8::THREADS, k1_smem<real>(), s>>>(P, nullptr, nullptr, P.Ne);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_grad_n8(const DevMesh& m, const void* Phi, void* grad, unsigned* flag, cudaStream_t s) {
  DevCoef none;
  ConsBC bc;
  RKStage rk;
  if (m.precision == 0) {
    K1N8<double> P = k1n8_params<double>(m, none, Phi, nullptr, nullptr, nullptr, nullptr, bc, rk, flag);
    P.gout = (double*)grad;
    return launch_grad_n8_t<double, 0>(P, false, s);
  }
  K1N8<float> P = k1n8_params<float>(m, none, Phi, nullptr, nullptr, nullptr, nullptr, bc, rk, flag);
  P.gout = (float*)grad;
  if (m.fp32_form == WT_FP32_BF16X2) return launch_grad_n8_t<float, 2>(P, false, s);
  return launch_grad_n8_t<float, 3>(P, m.fp32_form == WT_FP32_CUDA_CORES || m.fp32_form == WT_FP32_COMPENSATED, s);
}

// Self-test of the bounded-wait failure path: one thread polls an mbarrier the
// way the pipelined kernels do -- at most `polls` times, then it sets bit 1 of
// the status word and returns.  With arrive = 1 the barrier's phase completes
// first (a plain arrive) and the wait succeeds.  Nothing faults and nothing
// waits without a bound.
__global__ void k_wait_selftest(long long polls, int arrive, unsigned* flag) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  n8::mbar_init(&bar, 1);
  n8::fence_barrier_init();
  if (arrive) n8::mbar_expect_tx(&bar, 0u);
  for (long long it = 0; it < polls; ++it)
    if (n8::mbar_try_wait(&bar, 0)) return;
  atomicOr(flag, 2u);
}

int launch_wait_selftest(long long polls, int arrive, unsigned* flag, cudaStream_t s) {
  k_wait_selftest<<<1, 32, 0, s>>>(polls, arrive, flag);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// ---- face-plane halo of a z-slab partition ---------------------------------------------
// Pack (pack = 1) or unpack (pack = 0) the face plane `row` (0: the -z face, N - 1:
// the +z face) of the L elements from e0: per element and face point pq = p + N q,
// the Phi the next stage reads, its small part (phit != NULL: the compensated FP32
// form), then the three flux components (element blocks of B words in layout lay:
// 0 node order, 1 Lay<double>, 2 Lay<float>, 3 LayC).  buf: [component][element][pq].
template <typename real>
__global__ void k_halo_face(int N, long long e0, long long L, int row, real* phi, real* phit, real* F, long long Ne,
                            long long B, int lay, real* buf, int pack) {
  const long long N2 = (long long)N * N, N3 = N2 * N, tot = L * N2;
  const int nc = phit ? 5 : 4;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < tot; v += (long long)gridDim.x * blockDim.x) {
    const long long l = v / N2;
    const int pq = (int)(v - l * N2), p = pq % N, q = pq / N;
    const long long e = e0 + l;
    const int node = p + N * (q + N * row);
    const int fo = lay == 1 ? n8::Lay<double>::at(node) : lay == 2 ? n8::Lay<float>::at(node)
                 : lay == 3 ? n8::LayC::at(node) : node;
    real* ptr[5];
    int c = 0;
    ptr[c++] = phi + e * N3 + node;
    if (phit) ptr[c++] = phit + e * N3 + node;
    for (int k = 0; k < 3; ++k) ptr[c++] = F + (long long)k * Ne * B + e * B + fo;
    for (int k = 0; k < nc; ++k) {
      real* b = buf + (long long)k * tot + v;
      if (pack) *b = *ptr[k];
      else *ptr[k] = *b;
    }
  }
}

int launch_halo_face(const DevMesh& m, long long e0, long long L, int row, void* phi, void* phit, void* F, long long B,
                     int lay, void* buf, int pack, cudaStream_t s) {
  const long long tot = L * m.N * m.N;
  if (tot <= 0) return 0;
  const unsigned blocks = (unsigned)((tot + 255) / 256 < 4096 ? (tot + 255) / 256 : 4096);
  if (m.precision == 0)
    k_halo_face<double><<<blocks, 256, 0, s>>>(m.N, e0, L, row, (double*)phi, (double*)phit, (double*)F, m.Ne, B, lay,
                                               (double*)buf, pack);
  else
    k_halo_face<float><<<blocks, 256, 0, s>>>(m.N, e0, L, row, (float*)phi, (float*)phit, (float*)F, m.Ne, B, lay,
                                              (float*)buf, pack);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// element-block layout of the flux the n = 8 kernels of this mesh write (see k_halo_face)
int n8_flux_layout(const DevMesh& m) { return m.precision == 0 ? 1 : n8_layout(m) ? 3 : 2; }

// ---- work-list batching -------------------------------------------------------------
size_t cons_n8_param_size(int precision, int which) {
  if (precision == 0) return which == 1 ? sizeof(K1N8<double>) : sizeof(K2N8<double>);
  return which == 1 ? sizeof(K1N8<float>) : sizeof(K2N8<float>);
}

void cons_n8_fill_params(int which, const SolveStage& ss, unsigned* flag, void* dst) {
  const DevMesh& m = *ss.m;
  if (m.precision == 0) {
    if (which == 1)
      *(K1N8<double>*)dst = k1n8_params<double>(m, *ss.c, ss.Phi, ss.Pi, ss.F, nullptr, ss.bbuf, ss.bc, ss.rkP, flag);
    else
      *(K2N8<double>*)dst = k2n8_params<double>(m, ss.F, nullptr, ss.bbuf, ss.bc, ss.rkQ, flag);
  } else {
    if (which == 1)
      *(K1N8<float>*)dst = k1n8_params<float>(m, *ss.c, ss.Phi, ss.Pi, ss.F, nullptr, ss.bbuf, ss.bc, ss.rkP, flag);
    else
      *(K2N8<float>*)dst = k2n8_params<float>(m, ss.F, nullptr, ss.bbuf, ss.bc, ss.rkQ, flag);
  }
}

int launch_cons_n8_batch(int which, int precision, int fp32_form, const void* hP0, const void* plist, const int2* tiles,
                         long long ntiles, cudaStream_t s) {
  return n8_dispatch<true>(which, precision, fp32_form, hP0, plist, tiles, ntiles, s);
}

// this file's bounds word (bounds-check build; 0 otherwise)
WT_BOUNDS_TAKE(bounds_take_n8)

}  // namespace wt
