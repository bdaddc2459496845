// wt_common.cuh -- internal declarations shared by the CUDA translation units of
// libwavetoy_b200.so.  Not part of the public ABI (include/wavetoy_b200.h is).
//
// Data layout in HBM (one mesh, N GLL nodes per axis, Ne elements, nn = N^3 Ne):
//   * every scalar field is (N,N,N,Ne) element-major, i fastest: one element is a
//     contiguous block of N^3 values (4 KB for N=8 in FP64), so a CTA that owns an
//     element reads it with fully coalesced 128-bit loads;
//   * multi-component fields are structure-of-arrays: component c of field X
//     lives at X + c*nn (the reference's separate Julia arrays);
//   * connectivity is int32 [f + 6 e], 0-based, -1 = no neighbour;
//   * streamed per-node coefficients are stored in the state precision `real`
//     (double for the plain form, float for the FP32 form); geometry is computed
//     and kept in FP64 and converted once.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include <initializer_list>

#include "../../include/wavetoy_b200.h"

#ifndef WT_NO_NVTX
#include <nvtx3/nvToolsExt.h>
#endif

#define WT_MAXN 8

struct wt_ctx;  // the public context (include/wavetoy_b200.h)

namespace wt {

// ---- NVTX ranges (host side) ---------------------------------------------------------
// The C entry points, the RK4 stages, graph captures and replays are named
// ranges on an Nsight Systems timeline, and `ncu --nvtx --nvtx-include` can pick
// kernels by them.  NVTX v3 is header-only: with no tool attached a range costs
// a test of a null function pointer.  -DWT_NO_NVTX compiles them out.
struct NvtxRange {
#ifndef WT_NO_NVTX
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
#else
  explicit NvtxRange(const char*) {}
#endif
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// ---- bounds-check build (-DWT_BOUNDS_CHECK) ------------------------------------------
// The kernels index memory through four host-built tables: face sources
// (fsrc: 64 * neighbour element + 8 * orientation + neighbour face), neighbour
// elements (nbr), boundary slots (bslot) and, for batches, (solve, element)
// tiles built from the member list.  Every value read from the first three
// passes through one of these checks where it is loaded, so every access that
// depends on it is covered.  In the bounds-check build a value outside its
// table's range sets a bit of this translation unit's bounds word (1:
// element, 2: boundary slot) and is replaced by "no neighbour" (-1) or slot
// 0, which every buffer holds; the kernel goes on and no access leaves its
// buffer.  wt_ctx_bounds_status reads and clears the words.  In the normal
// build the checks compile to nothing.
#ifdef WT_BOUNDS_CHECK
static __device__ unsigned int wt_bounds_word;  // one per translation unit
__device__ __forceinline__ int bc_src(int v, long long Ne) {
  if (v < 0 || (long long)(v >> 6) < Ne) return v;
  atomicOr(&wt_bounds_word, 1u);
  return -1;
}
__device__ __forceinline__ int bc_elem(int v, long long Ne) {
  if (v < Ne) return v;
  atomicOr(&wt_bounds_word, 1u);
  return -1;
}
__device__ __forceinline__ int bc_slot(int v, int nbf) {
  if (v >= 0 && v < (nbf > 0 ? nbf : 1)) return v;
  atomicOr(&wt_bounds_word, 2u);
  return 0;
}
// defines `unsigned int fn()`: this translation unit's bounds word, cleared
#define WT_BOUNDS_TAKE(fn)                                              \
  unsigned int fn() {                                                   \
    unsigned int v = 0, z = 0;                                          \
    cudaMemcpyFromSymbol(&v, wt::wt_bounds_word, sizeof(v));            \
    cudaMemcpyToSymbol(wt::wt_bounds_word, &z, sizeof(z));              \
    return v;                                                           \
  }
#else
__device__ __forceinline__ int bc_src(int v, long long) { return v; }
__device__ __forceinline__ int bc_elem(int v, long long) { return v; }
__device__ __forceinline__ int bc_slot(int v, int) { return v; }
#define WT_BOUNDS_TAKE(fn) \
  unsigned int fn() { return 0; }
#endif
// the bounds words of the kernel translation units (wt_cons.cu, wt_cons_n8.cu, wt_second.cu, wt_geom.cu)
unsigned int bounds_take_cons();
unsigned int bounds_take_n8();
unsigned int bounds_take_second();
unsigned int bounds_take_geom();

// ---- host-side GLL operators (product code, independent of the oracle) -----
struct HostOps {
  int N = 0;
  std::vector<double> x, H, G;  // x, H on [0,1]; G[i*N+p]
};
HostOps gll_operators(int N);

// ---- device-side mesh --------------------------------------------------------
struct DevMesh {
  int N = 0;
  long long Ne = 0, nn = 0;
  int precision = 0;   // 0 = double, 1 = float
  int fp32_form = WT_FP32_COMPENSATED;  // FP32 meshes: WT_FP32_* of include/wavetoy_b200.h
  int ja_n8_layout = 0;  // layout Ja_n8 holds (0: Lay<real>, 1: LayC of the FP32 CUDA-core form)
  int affine = 1;      // 1 if every Jacobian is diagonal and constant per element
  int M[3] = {0, 0, 0};
  // connectivity
  int32_t* nbr = nullptr;   // [f + 6e]
  int32_t* nbrf = nullptr;
  int32_t* bdry = nullptr;
  int32_t* handed = nullptr;  // [e]
  std::vector<int32_t> h_nbr, h_nbrf, h_bdry;
  // operators on device: G (N*N), GT (transposed), H (N), x (N) -- double
  double* G = nullptr;
  double* H = nullptr;
  double* x = nullptr;
  HostOps ops;
  // FP64 geometry
  double* coords = nullptr;  // [a + 3n]
  double* jac = nullptr;     // [a + 3b + 9n]
  double* invjac = nullptr;  // [al + 3be + 9n]
  double* detjac = nullptr;
  double* Hphys = nullptr;
  double* Ja = nullptr;      // 9 fields, field-major
  double* invdetJ = nullptr;
  double* Hd = nullptr;
  double* dinvjac = nullptr; // lazily: [a + 3c + 9d + 27n]
  // streamed copies in the state precision
  void* Ja_r = nullptr;      // 9 fields
  void* invdetJ_r = nullptr;
  void* sdiag = nullptr;     // [3e + d] element-constant axis scale invjac[d,d] at node 0
  void* Ja_n8 = nullptr;     // n = 8: metric terms in the n8 element-block layout (FP64 512, FP32 544 words per element), state precision
  // FP32 meshes (the compensated form's gradient): Ja split into an element-constant
  // FP64 part Ja0 [9e + c] (the element's mean) and an FP32 deviation dJa
  // (9 fields; n = 8: LayC element blocks, otherwise node order)
  double* Ja0 = nullptr;
  void* dJa = nullptr;
  // per element: bits 0-5 faces that get the centred-flux SAT (interior face with a
  // neighbour), bit 6 element has an outer face
  int32_t* emask = nullptr;
  // per (f,e): 64 * neighbour element + 8 * orientation + neighbour face for SAT faces, -1 otherwise
  int32_t* fsrc = nullptr;
  int has_ori = 0;           // some face has orientation != 0 (multi-patch mesh)
  // boundary faces: slot per (f,e) with bdry != 0, -1 otherwise
  int32_t* bslot = nullptr;
  int nbf = 0;
  void* bnorm = nullptr;     // per boundary-face node: (nx, ny, nz, wt_curv, wF/Hphys) in real
  // lines along each axis (for line-local Kreiss-Oliger): element lists
  int line_ok[3] = {0, 0, 0};
  int nlines[3] = {0, 0, 0};
  int line_len[3] = {0, 0, 0};      // elements per line (all lines equal length)
  int line_closed[3] = {0, 0, 0};   // periodic lines
  int32_t* lines[3] = {nullptr, nullptr, nullptr};  // [line*len + pos] element ids
  // device status word of the owning context: bit 0 non-finite state, bit 1 a
  // bounded wait in a pipelined kernel gave up
  unsigned int* errflag = nullptr;
};

// Kernel-side view of the mesh (passed by value).
struct MeshView {
  int N;
  long long Ne, nn;
  const int32_t* nbr;
  const int32_t* nbrf;
  const int32_t* bdry;
  const double* G;
  const double* H;
};

inline MeshView view(const DevMesh& m) {
  MeshView v;
  v.N = m.N; v.Ne = m.Ne; v.nn = m.nn; v.nbr = m.nbr; v.nbrf = m.nbrf; v.bdry = m.bdry;
  v.G = m.G; v.H = m.H;
  return v;
}

// ---- device-side background coefficients --------------------------------------
struct DevCoef {
  long long nn = 0;
  double* c11 = nullptr;  // 11 fields FP64 (sample_background3d! layout)
  void* c10 = nullptr;    // 10 streamed fields in `real`: a, b1, b2, b3, K11, K12, K13, K22, K23, K33
  int precision = 0;
};

// ---- face helpers -----------------------------------------------------------------
__host__ __device__ inline int faxis(int f) { return f >> 1; }
__host__ __device__ inline int frow(int f, int N) { return (f & 1) ? N - 1 : 0; }
__host__ __device__ inline double fsign(int f) { return (f & 1) ? 1.0 : -1.0; }
__host__ __device__ inline int face_node(int ax, int r, int p, int q, int N) {
  // local node index of face node (p,q) of the face with axis ax at row r
  return ax == 0 ? r + N * (p + N * q) : ax == 1 ? p + N * (r + N * q) : p + N * (q + N * r);
}
// Face orientation: the neighbour's face node (pn, qn) that coincides with this
// face's node (p, q), for the D4 element ori (bit 2: swap p and q; bit 0:
// reverse the first index; bit 1: reverse the second).  ori = 0 is the
// identity (aligned patches); the library infers ori from the node
// coordinates when it builds the topology.  Encodings: nbrf[f + 6e] = fn |
// ori << 3; fsrc[f + 6e] = 64 nbr + 8 ori + fn.
__host__ __device__ inline void face_perm(int ori, int p, int q, int N, int& pn, int& qn) {
  const int a = (ori & 4) ? q : p, b = (ori & 4) ? p : q;
  pn = (ori & 1) ? N - 1 - a : a;
  qn = (ori & 2) ? N - 1 - b : b;
}
// neighbour face node for face source fs = 64 nbr + 8 ori + fn (node within the neighbour element)
__host__ __device__ inline int nbr_face_node(int fs, int p, int q, int N) {
  const int fn = fs & 7;
  int pn, qn;
  face_perm((fs >> 3) & 7, p, q, N, pn, qn);
  return face_node(faxis(fn), frow(fn, N), pn, qn, N);
}

// set the context's last-error message and return code (wt_capi.cu)
int ctx_fail(::wt_ctx* ctx, int code, const std::string& msg);
// a device allocation the context tracks (and wt_ctx_inject_alloc_failure can fail), and its release
int ctx_alloc(::wt_ctx* ctx, void** p, size_t bytes);
void ctx_free(::wt_ctx* ctx, void* p);

// ---- meshes built from node coordinates (wt_patches.cu, host) ----------------------
// D4 orientation under which face (e,f)'s nodes coincide with face (en,fn)'s
// (within tol; with shift, up to one constant translation); -1 if none
int infer_orientation(int N, const double* X, long long e, int f, long long en, int fn, double tol, bool shift);
// neighbours (-1: none) and nbrf = fn | ori << 3 of every face, by matching coordinates; -1 on inconsistency
int match_faces(int N, long long Ne, const double* X, double tol, std::vector<int32_t>& nbr,
                std::vector<int32_t>& nbrf);
// jac[a + 3 b + 9 n] = SBP derivative of the node coordinates along xi_b
void coords_jacobian(int N, long long Ne, const double* X, const std::vector<double>& G, double* jac);
// node coordinates of a WT_MESH_* multi-patch mesh; scale = the domain's size; -1 bad parameters, -2 bad kind
int build_patch_mesh(int kind, int N, int M, const double p[3], const std::vector<double>& xg,
                     std::vector<double>& X, double& scale);

// ---- error reporting ----------------------------------------------------------------
struct Status {
  int code = 0;
  std::string msg;
};

// ---- launchers implemented in the .cu files -------------------------------------------
// geometry (wt_geom.cu)
// analytic (warped) cube geometry; a z-slab mesh passes its first layer z0 within
// the whole mesh of Mz layers (0: the mesh is the whole cube)
int launch_geom_analytic(DevMesh& m, double x0, double x1, double A, cudaStream_t s, int z0 = 0, int Mz = 0);
int launch_geom_derived(DevMesh& m, cudaStream_t s);
int launch_metric(DevMesh& m, cudaStream_t s);
int launch_dinvjac(DevMesh& m, cudaStream_t s);
int launch_boundary_normals(DevMesh& m, cudaStream_t s);
int launch_streamed_geometry(DevMesh& m, cudaStream_t s);
// kinds 4, 5 (spacetime-metric backgrounds) are sampled at time *d_t + toff
int launch_background(const DevMesh& m, DevCoef& c, int kind, const double* p, cudaStream_t s,
                      const double* d_t = nullptr, double toff = 0.0);
int launch_advance_time(double* d_t, double dt, cudaStream_t s);
// out = y + dt * sum_{j < nk} a_j k_j (nk <= 8)
int launch_erk_combine(long long n, int precision, double dt, const void* y, void* out, int nk, const void* const* k,
                       const double* a, cudaStream_t s);
int launch_coef_combine(const DevMesh& m, DevCoef& c, cudaStream_t s);
int launch_min_spacing(const DevMesh& m, double* out, cudaStream_t s);
int launch_initial(const DevMesh& m, int kind, const double* dparams, int np, double t, void* u, void* ut,
                   cudaStream_t s, bool f64 = false);  // f64: evaluate in FP64 whatever the mesh precision

// conservative first-order system (wt_cons.cu)
struct ConsBC {
  int on = 0;          // boundary pass requested
  int curv = 0;        // curvilinear pass (single kind) vs affine per-side kinds
  int kinds[6] = {0, 0, 0, 0, 0, 0};
  double sigma = 1.0;
  int exc_tag = 0;
  const void* gPhi = nullptr;
  const void* gPi = nullptr;
  const void* gDx = nullptr;
  const void* gDy = nullptr;
  const void* gDz = nullptr;
};
struct RKStage {
  int on = 0;          // fused RK4 epilogue instead of writing the RHS
  int stage = 0;       // 0..3
  double dt = 0.0;
  void* y = nullptr;   // state (read; written at stage 3)
  void* acc = nullptr; // accumulator
  void* out = nullptr; // next stage input
  // FP32 state only: per-node compensation of the stage-3 sum y + increment
  // (Kahan); with it, acc holds the step increment alone
  void* comp = nullptr;
  unsigned int* nonfinite = nullptr;  // set to 1 if the stage-3 update is not finite
  // compensated FP32 form (WT_FP32_COMPENSATED): the small part K1 adds to its
  // Phi input (the state's low part at stage 0, the previous stage's output
  // after it), and the copy of the state's high part stage 2 writes for stage 3
  const void* phit = nullptr;
  void* hcopy = nullptr;
};
// K1: gradient, flux F, Phidot (+ affine/curv BC increments), optional RK epilogue for Phi.
// e0, e1: the elements [e0, e1) the launch covers (e1 < 0: to the last element)
int launch_cons_k1(const DevMesh& m, const DevCoef& c, const void* Phi, const void* Pi, void* F, void* Phidot,
                   void* bbuf, void* grad_out, int use_metric, const ConsBC& bc, const RKStage& rk,
                   cudaStream_t s, bool n8 = false, long long e0 = 0, long long e1 = -1);
// K2: divergence of F (+ boundary increments), optional RK epilogue for Pi.
int launch_cons_k2(const DevMesh& m, const void* F, void* Pidot, const void* bbuf, int use_metric,
                   const ConsBC& bc, const RKStage& rk, unsigned int* nonfinite, cudaStream_t s, bool n8 = false,
                   long long e0 = 0, long long e1 = -1);
int launch_apply_D(const DevMesh& m, const void* u, void* out, int d, cudaStream_t s);
// n = 8 curvilinear path: persistent, bulk-copy-pipelined, tensor cores (wt_cons_n8.cu)
// [e0, e1): the elements the launch covers (e1 < 0: to the last element)
int launch_cons_k1_n8(const DevMesh& m, const DevCoef& c, const void* Phi, const void* Pi, void* F, void* Phidot,
                      void* bbuf, const ConsBC& bc, const RKStage& rk, unsigned* flag, cudaStream_t s,
                      long long e0 = 0, long long e1 = -1);
int launch_cons_k2_n8(const DevMesh& m, const void* F, void* Pidot, const void* bbuf, const ConsBC& bc,
                      const RKStage& rk, unsigned* flag, cudaStream_t s, long long e0 = 0, long long e1 = -1);
// Fused RK4 stage (FP64): K2 of stage rkQ.stage (0..2, F_s in Fin) and K1 of
// stage rkP.stage = rkQ.stage + 1 (Phi_{s+1} in Phi, F_{s+1} into Fout) in one
// launch; Fin and Fout must differ.  rkQ.out may be NULL (Pi's stage value is
// then not stored).
int launch_cons_fk_n8(const DevMesh& m, const DevCoef& c, const void* Fin, void* Fout, const void* Phi, void* bbuf,
                      const ConsBC& bc, const RKStage& rkQ, const RKStage& rkP, cudaStream_t s);
int launch_pad_metric_n8(DevMesh& m, cudaStream_t s);
// FP32 meshes: m.Ja0 (element means of the FP64 metric terms) and m.dJa (FP32 deviations)
int launch_split_metric(const DevMesh& m, cudaStream_t s);
// whether the generic (any n) kernels run the compensated FP32 form on this mesh
bool cons_gen_cp_supported(const DevMesh& m);
// whether the batch has pipelined kernels (launch variant 2) for order N
bool cons_gen_pipe_available(int N);
// bounded-wait self-test (see k_wait_selftest)
int launch_wait_selftest(long long polls, int arrive, unsigned* flag, cudaStream_t s);
// the split-form gradient of Phi through the n = 8 kernels (3 fields of nn words into grad)
int launch_grad_n8(const DevMesh& m, const void* Phi, void* grad, unsigned* flag, cudaStream_t s);
long long n8_padded_field_size(long long Ne);
// values per element block of a flux component written by the n = 8 kernels (component c at F + c Ne block)
long long n8_flux_block(const DevMesh& m);
// its element-block layout: 1 Lay<double>, 2 Lay<float>, 3 LayC (0: node order, the generic kernels)
int n8_flux_layout(const DevMesh& m);
// face plane `row` of the L elements from e0 (Phi stage input, [small part], three flux
// components) into buf (pack = 1) or back (pack = 0); see k_halo_face
int launch_halo_face(const DevMesh& m, long long e0, long long L, int row, void* phi, void* phit, void* F, long long B,
                     int lay, void* buf, int pack, cudaStream_t s);
// True when an RHS evaluation takes the n = 8 pipelined path (both kernels take
// the same path: K1 then writes F in the padded layout K2 reads).
bool cons_n8_path(const DevMesh& m, const DevCoef& c, int use_metric, const ConsBC& bc, const RKStage& rkP,
                  const RKStage& rkQ, std::initializer_list<const void*> ptrs);

// ---- work-list batching of many solves (one launch per kernel and group) ----
// Everything one solve contributes to one RK4 stage: its mesh, coefficients,
// stage inputs, scratch, boundary data and the stage updates of Phi and Pi.
struct SolveStage {
  const DevMesh* m = nullptr;
  const DevCoef* c = nullptr;
  const void* Phi = nullptr;
  const void* Pi = nullptr;
  void* F = nullptr;
  void* bbuf = nullptr;
  ConsBC bc;
  RKStage rkP, rkQ;
};
// n = 8 pipelined kernels: parameter block size / fill / launch over a work
// list of (solve, element) tiles; hP0 is the host copy of the first block
// (stage-wide values), plist the device array of all blocks.
size_t cons_n8_param_size(int precision, int which);
void cons_n8_fill_params(int which, const SolveStage& ss, unsigned* flag, void* dst);
int launch_cons_n8_batch(int which, int precision, int fp32_form, const void* hP0, const void* plist, const int2* tiles,
                         long long ntiles, cudaStream_t s);
// generic kernels (any N, curvilinear form): epb_variant 0 = default elements
// per CTA, 1 = twice that (when it fits 1024 threads); chosen by the autotuner
size_t cons_gen_param_size(int precision, int which);
void cons_gen_fill_params(int which, const SolveStage& ss, unsigned* flag, void* dst);
int launch_cons_gen_batch(int which, int N, int precision, int epb_variant, int cp, const void* plist, const int2* tiles,
                          long long ntiles, cudaStream_t s);
// dst += koT * sum_d D_d^6 field; scratch (2 nn words, may be NULL when every
// axis has straight element lines) serves meshes without them
int launch_ko_add(const DevMesh& m, void* dst, const void* field, double koT, cudaStream_t s, void* scratch);
int launch_div3d(const DevMesh& m, const void* F, void* out, cudaStream_t s);

// second-order forms (wt_second.cu)
int launch_sipg(const DevMesh& m, const void* u, const void* ut, void* utt, void* trace, const double bvals[6],
                double tau, double inv_R, cudaStream_t s);
int launch_strong(const DevMesh& m, const void* u, const void* ut, void* utt, double tau, double inv_R,
                  cudaStream_t s);
int launch_lap_strong_cons(const DevMesh& m, const void* u, void* Lu, double h, double tau, cudaStream_t s);
// scalar wave on a prescribed 4-metric (wt_second.cu)
int launch_curved4(const DevMesh& m, const void* u, const void* ud, void* udd, const void* ginv, const void* gam,
                   double h, int conservative, double tau, cudaStream_t s);
int launch_curved4_background(const DevMesh& m, int kind, const double* p, double t, void* ginv, void* gam,
                              cudaStream_t s);

// reductions and vector updates (wt_reduce.cu)
int launch_energy(const DevMesh& m, const DevCoef& c, const void* Pi, const void* grad, int use_metric,
                  double* partial, int nblocks, cudaStream_t s, int lapse = 0);
int launch_dot_weighted(const DevMesh& m, const void* a, const void* b, const void* c, const void* d,
                        int weight_kind, int mode, double* partial, int nblocks, cudaStream_t s);
int launch_sumsq(long long n, int precision, const void* a, double* partial, int nblocks, cudaStream_t s);
int launch_scale(long long n, int precision, void* a, double s, cudaStream_t st);
int launch_fill(long long n, int precision, void* a, double v, cudaStream_t st);
int launch_copy(long long n, int precision, void* dst, const void* src, cudaStream_t st);
int launch_gather(int precision, int count, const void* field, const int64_t* nodes, double* out, cudaStream_t s);
// hi = (float)a, lo = (float)(a - hi)
int launch_split_f64(long long n, const double* a, float* hi, float* lo, cudaStream_t st);
int launch_rk_update(long long n, int precision, int stage, double dt, void* y, void* acc, void* out,
                     const void* k, cudaStream_t st, void* comp = nullptr);
int launch_axpy(long long n, int precision, void* y, double a, const void* x, cudaStream_t st);
int launch_alt_sign(const DevMesh& m, void* v, cudaStream_t st);
int launch_finite_check(long long n, int precision, const void* a, unsigned int* flag, cudaStream_t st);
int reduce_blocks();

}  // namespace wt
