// wt_capi.cu -- host runtime behind the C ABI of include/wavetoy_b200.h.
//
// Owns device memory for meshes, background coefficients and workspaces,
// validates arguments (ArgumentError in the reference -> WT_EINVAL with a
// message), orders launches on the context stream and replays the RK4 step as
// a CUDA graph.  No CPU fallback exists: every numeric entry point runs the
// kernels of wt_cons.cu / wt_second.cu / wt_reduce.cu.
#include "wt_common.cuh"
#include "../../include/wavetoy_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <string>
#include <vector>

struct wt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;      // stream launches go to
  cudaStream_t own_stream = nullptr;  // the context's own stream
  std::string err;
  long long launches = 0;
  unsigned int* d_flag = nullptr;
  double* d_partial = nullptr;
  int nblocks = 0;
  // per-kernel timing (CUDA events around K1/K2 launches on the launching stream)
  int prof_on = 0;
  std::vector<cudaEvent_t> prof_ev[3];  // [kernel: K1, K2, fused stage] start/stop pairs
  cudaEvent_t ord_a = nullptr, ord_b = nullptr;  // order the graph stream with the caller's stream
  double* noalloc_scratch = nullptr;  // device address of the wt_rhs_curved_noalloc array (first call)
  // device memory of the objects the context owns (meshes, coefficients,
  // workspaces, batches, served requests): live allocations by address
  std::unordered_map<void*, size_t> live;
  long long live_bytes = 0, total_allocs = 0;
  long long fail_after = -1;  // host-side fault injection: allocations left before one fails (< 0: none)
};

static void prof_mark(wt_ctx* ctx, int which) {
  if (!ctx->prof_on) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  cudaEvent_t ev;
  if (cudaEventCreate(&ev) != cudaSuccess) return;
  cudaEventRecord(ev, ctx->stream);
  ctx->prof_ev[which].push_back(ev);
}

struct wt_mesh {
  wt_ctx* ctx = nullptr;
  wt::DevMesh m;
  std::vector<void*> owned;
};

struct wt_coef {
  wt_ctx* ctx = nullptr;
  wt_mesh* mesh = nullptr;
  wt::DevCoef c;
  // time-dependent (spacetime-metric) backgrounds: kind, parameters and the
  // time the coefficients hold (on the host, and on the device for kernels
  // captured in a CUDA graph)
  int kind = -1;
  double p[16] = {};
  bool td = false;
  mutable double t = 0.0;
  double* d_t = nullptr;
};

struct wt_ws {
  wt_ctx* ctx = nullptr;
  wt_mesh* mesh = nullptr;
  double mu = 0.0, inv_mu5 = 0.0;
  bool mu_done = false;  // mu is computed on first use (Kreiss-Oliger or wt_workspace_mu)
  void* F = nullptr;      // 3 nn
  void* F2 = nullptr;     // FP64 n = 8 fused stages: the second flux buffer (F ping-pongs between launches)
  int fused = 1;          // FP64 n = 8 RK4 steps through the fused stage kernel (wt_workspace_set_fused)
  void* bbuf = nullptr;   // nbf N^2
  void* grad = nullptr;   // 3 nn
  void* kP = nullptr;     // nn (Phidot / u_t slope)
  void* kQ = nullptr;     // nn
  void* S0 = nullptr;     // stage buffers
  void* S1 = nullptr;
  void* SQ = nullptr;
  void* accP = nullptr;
  void* accQ = nullptr;
  void* trace = nullptr;  // 6 N^2 Ne
  void* zero = nullptr;   // nn zeros
  void* Lu = nullptr;     // nn
  // FP32 state: the low parts the FP32 state arrays lost (the state is
  // Phi + compP, Pi + compQ): Kahan compensation of the RK4 step sums, kept
  // while the caller keeps stepping the same state buffers
  void* compP = nullptr;
  void* compQ = nullptr;
  const void* comp_for[2] = {nullptr, nullptr};
  void* erk = nullptr;    // explicit RK stage slopes: 2 x erk_stages x nn (Phi slopes, then Pi slopes)
  int erk_stages = 0;
  long long flux_block = 0;  // values per element block of F as the last fused stage wrote it (halo copies)
  int flux_lay = 0;          // and its element-block layout (wt::n8_flux_layout; 0: node order)
  int halo_cp = 0;        // the last fused stage ran the compensated FP32 form (its halo adds Phit)
  // host-buffer evolution (evolve_host): device state, staging pair for the
  // copies to the host, per-sample energy partial sums -- kept between calls
  void* evo[4] = {nullptr, nullptr, nullptr, nullptr};
  double* evoE = nullptr;
  size_t evoE_len = 0;
};

namespace {

int fail(wt_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int cuda_fail(wt_ctx* ctx, cudaError_t e, const char* where) {
  return fail(ctx, WT_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

size_t rsize(int precision) { return precision == 0 ? sizeof(double) : sizeof(float); }

template <typename T>
int dalloc(wt_ctx* ctx, T** p, size_t bytes, std::vector<void*>* owner) {
  if (bytes == 0) bytes = 16;
  if (ctx->fail_after >= 0 && ctx->fail_after-- == 0)  // wt_ctx_inject_alloc_failure: fail as cudaMalloc would
    return fail(ctx, WT_ENOMEM, std::string("device allocation of ") + std::to_string(bytes) +
                                    " bytes failed: injected failure");
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, WT_ENOMEM, std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " +
                                    cudaGetErrorString(e));
  }
  ctx->live[(void*)*p] = bytes;
  ctx->live_bytes += (long long)bytes;
  ctx->total_allocs += 1;
  if (owner) owner->push_back((void*)*p);
  return 0;
}

// free an allocation of dalloc (NULL: nothing)
void dfree(wt_ctx* ctx, void* p) {
  if (!p) return;
  auto it = ctx->live.find(p);
  if (it != ctx->live.end()) {
    ctx->live_bytes -= (long long)it->second;
    ctx->live.erase(it);
  }
  cudaFree(p);
}

#define WT_TRY(x)            \
  do {                       \
    int _rc = (x);           \
    if (_rc != 0) return _rc; \
  } while (0)

int lrc(wt_ctx* ctx, int rc, const char* where) {
  if (rc == 0) return 0;
  if (rc == -4) return fail(ctx, WT_ENOTSUP, std::string(where) + ": configuration not supported");
  if (rc == -3) return fail(ctx, WT_ENOMEM, std::string(where) + ": out of device memory");
  cudaError_t e = cudaGetLastError();
  return fail(ctx, WT_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Boundary-face slots, line tables and device copies of the connectivity.
int finish_topology(wt_mesh* mh) {
  wt::DevMesh& m = mh->m;
  wt_ctx* ctx = mh->ctx;
  const long long Ne = m.Ne;
  std::vector<int32_t> slot(6 * Ne, -1);
  int nbf = 0;
  for (long long e = 0; e < Ne; ++e)
    for (int f = 0; f < 6; ++f)
      if (m.h_bdry[f + 6 * e] != 0) slot[f + 6 * e] = nbf++;
  m.nbf = nbf;
  WT_TRY(dalloc(ctx, &m.nbr, 6 * Ne * sizeof(int32_t), &mh->owned));
  WT_TRY(dalloc(ctx, &m.nbrf, 6 * Ne * sizeof(int32_t), &mh->owned));
  WT_TRY(dalloc(ctx, &m.bdry, 6 * Ne * sizeof(int32_t), &mh->owned));
  WT_TRY(dalloc(ctx, &m.bslot, 6 * Ne * sizeof(int32_t), &mh->owned));
  cudaMemcpyAsync(m.nbr, m.h_nbr.data(), 6 * Ne * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(m.nbrf, m.h_nbrf.data(), 6 * Ne * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(m.bdry, m.h_bdry.data(), 6 * Ne * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(m.bslot, slot.data(), 6 * Ne * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream);
  {
    std::vector<int32_t> emask(Ne, 0), fsrc(6 * Ne, -1);
    for (long long e = 0; e < Ne; ++e)
      for (int f = 0; f < 6; ++f) {
        const long long i = f + 6 * e;
        if (m.h_bdry[i] != 0) emask[e] |= 64;
        else if (m.h_nbr[i] >= 0) {
          emask[e] |= 1 << f;
          fsrc[i] = 64 * m.h_nbr[i] + m.h_nbrf[i];  // h_nbrf = fn | ori << 3
          if (m.h_nbrf[i] >> 3) m.has_ori = 1;
        }
      }
    WT_TRY(dalloc(ctx, &m.emask, Ne * sizeof(int32_t), &mh->owned));
    WT_TRY(dalloc(ctx, &m.fsrc, 6 * Ne * sizeof(int32_t), &mh->owned));
    cudaMemcpyAsync(m.emask, emask.data(), Ne * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(m.fsrc, fsrc.data(), 6 * Ne * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream);
    cudaError_t ce = cudaStreamSynchronize(ctx->stream);  // host vectors go out of scope
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "topology upload");
  }
  // lines along each axis: follow face 2d+1 neighbours whose matching face is 2d
  for (int d = 0; d < 3; ++d) {
    std::vector<char> seen(Ne, 0);
    std::vector<int32_t> all;
    int len = -1, nl = 0, closed = -1;
    bool ok = true;
    auto fwd = [&](long long e) -> long long {
      int en = m.h_nbr[2 * d + 1 + 6 * e];
      if (en < 0 || m.h_nbrf[2 * d + 1 + 6 * e] != 2 * d || m.h_bdry[2 * d + 1 + 6 * e] != 0) return -1;
      return en;
    };
    auto has_back = [&](long long e) -> bool {
      int en = m.h_nbr[2 * d + 6 * e];
      return en >= 0 && m.h_nbrf[2 * d + 6 * e] == 2 * d + 1 && m.h_bdry[2 * d + 6 * e] == 0;
    };
    // a face that couples to a neighbour (apply_D!'s SAT) but does not continue
    // a straight line: a line may not end there (multi-patch meshes)
    auto coupled = [&](long long e, int f) -> bool { return m.h_nbr[f + 6 * e] >= 0 && m.h_bdry[f + 6 * e] == 0; };
    for (long long e = 0; e < Ne && ok; ++e)
      if ((coupled(e, 2 * d + 1) && fwd(e) < 0) || (coupled(e, 2 * d) && !has_back(e))) ok = false;
    for (long long e0 = 0; e0 < Ne && ok; ++e0) {
      if (seen[e0] || has_back(e0)) continue;
      std::vector<int32_t> ln;
      for (long long e = e0; e >= 0 && !seen[e]; e = fwd(e)) { seen[e] = 1; ln.push_back((int32_t)e); }
      if (len < 0) len = (int)ln.size();
      if ((int)ln.size() != len || closed == 1) ok = false;
      closed = 0;
      all.insert(all.end(), ln.begin(), ln.end());
      ++nl;
    }
    for (long long e0 = 0; e0 < Ne && ok; ++e0) {  // periodic (closed) lines
      if (seen[e0]) continue;
      std::vector<int32_t> ln;
      long long e = e0;
      while (e >= 0 && !seen[e]) { seen[e] = 1; ln.push_back((int32_t)e); e = fwd(e); }
      if (e != e0) { ok = false; break; }
      if (len < 0) len = (int)ln.size();
      if ((int)ln.size() != len || closed == 0) ok = false;
      closed = 1;
      all.insert(all.end(), ln.begin(), ln.end());
      ++nl;
    }
    m.line_ok[d] = ok && len > 0 ? 1 : 0;
    if (m.line_ok[d]) {
      m.nlines[d] = nl; m.line_len[d] = len; m.line_closed[d] = closed == 1;
      WT_TRY(dalloc(ctx, &m.lines[d], all.size() * sizeof(int32_t), &mh->owned));
      cudaMemcpyAsync(m.lines[d], all.data(), all.size() * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream);
    }
  }
  return 0;
}

int alloc_geometry(wt_mesh* mh) {
  wt::DevMesh& m = mh->m;
  wt_ctx* ctx = mh->ctx;
  const long long nn = m.nn;
  const int N = m.N;
  m.ops = wt::gll_operators(N);
  WT_TRY(dalloc(ctx, &m.G, N * N * sizeof(double), &mh->owned));
  WT_TRY(dalloc(ctx, &m.H, N * sizeof(double), &mh->owned));
  WT_TRY(dalloc(ctx, &m.x, N * sizeof(double), &mh->owned));
  cudaMemcpyAsync(m.G, m.ops.G.data(), N * N * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(m.H, m.ops.H.data(), N * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(m.x, m.ops.x.data(), N * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  WT_TRY(dalloc(ctx, &m.coords, 3 * nn * sizeof(double), &mh->owned));
  WT_TRY(dalloc(ctx, &m.jac, 9 * nn * sizeof(double), &mh->owned));
  WT_TRY(dalloc(ctx, &m.invjac, 9 * nn * sizeof(double), &mh->owned));
  WT_TRY(dalloc(ctx, &m.detjac, nn * sizeof(double), &mh->owned));
  WT_TRY(dalloc(ctx, &m.Hphys, nn * sizeof(double), &mh->owned));
  WT_TRY(dalloc(ctx, &m.Ja, 9 * nn * sizeof(double), &mh->owned));
  WT_TRY(dalloc(ctx, &m.invdetJ, nn * sizeof(double), &mh->owned));
  WT_TRY(dalloc(ctx, &m.Hd, nn * sizeof(double), &mh->owned));
  WT_TRY(dalloc(ctx, &m.handed, m.Ne * sizeof(int32_t), &mh->owned));
  const size_t rs = rsize(m.precision);
  if (m.precision == 0) {
    m.Ja_r = m.Ja;
    m.invdetJ_r = m.invdetJ;
  } else {
    WT_TRY(dalloc(ctx, &m.Ja_r, 9 * nn * rs, &mh->owned));
    WT_TRY(dalloc(ctx, &m.invdetJ_r, nn * rs, &mh->owned));
  }
  WT_TRY(dalloc(ctx, &m.sdiag, 3 * m.Ne * rs, &mh->owned));
  WT_TRY(dalloc(ctx, &m.bnorm, (size_t)5 * (m.nbf > 0 ? m.nbf : 1) * N * N * rs, &mh->owned));
  return 0;
}

int derive_geometry(wt_mesh* mh) {
  wt::DevMesh& m = mh->m;
  cudaStream_t s = mh->ctx->stream;
  WT_TRY(lrc(mh->ctx, wt::launch_geom_derived(m, s), "geometry"));
  WT_TRY(lrc(mh->ctx, wt::launch_metric(m, s), "metric terms"));
  WT_TRY(lrc(mh->ctx, wt::launch_streamed_geometry(m, s), "streamed geometry"));
  if (m.N == 8) {  // padded element blocks (state precision) for the pipelined n = 8 kernels
    WT_TRY(dalloc(mh->ctx, &m.Ja_n8, 9 * (size_t)wt::n8_padded_field_size(m.Ne) * rsize(m.precision), &mh->owned));
    WT_TRY(lrc(mh->ctx, wt::launch_pad_metric_n8(m, s), "padded metric terms"));
  }
  if (m.precision == WT_F32) {  // the compensated form's split metric terms
    WT_TRY(dalloc(mh->ctx, &m.Ja0, 9 * (size_t)m.Ne * sizeof(double), &mh->owned));
    const size_t nd = m.N == 8 ? (size_t)wt::n8_padded_field_size(m.Ne) : (size_t)m.nn;
    WT_TRY(dalloc(mh->ctx, &m.dJa, 9 * nd * sizeof(float), &mh->owned));
    WT_TRY(lrc(mh->ctx, wt::launch_split_metric(m, s), "split metric terms"));
  }
  WT_TRY(lrc(mh->ctx, wt::launch_boundary_normals(m, s), "boundary normals"));
  mh->ctx->launches += 6;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(mh->ctx, e, "mesh set-up");
  return 0;
}

void free_mesh(wt_mesh* mh) {
  for (void* p : mh->owned) dfree(mh->ctx, p);
  mh->owned.clear();
}

int ensure(wt_ws* ws, void** p, size_t bytes) {
  if (*p) return 0;
  return dalloc(ws->ctx, p, bytes, nullptr);
}

int ws_buffers(wt_ws* ws) {
  const wt::DevMesh& m = ws->mesh->m;
  const size_t rs = rsize(m.precision);
  size_t nb = (size_t)m.nn * rs;
  if (m.N == 8) nb = std::max(nb, (size_t)wt::n8_padded_field_size(m.Ne) * rs);  // padded flux layout
  WT_TRY(ensure(ws, &ws->F, 3 * nb));
  WT_TRY(ensure(ws, &ws->bbuf, (size_t)(m.nbf > 0 ? m.nbf : 1) * m.N * m.N * rs));
  return 0;
}

int ws_step_buffers(wt_ws* ws) {
  const wt::DevMesh& m = ws->mesh->m;
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  WT_TRY(ws_buffers(ws));
  WT_TRY(ensure(ws, &ws->S0, nb));
  WT_TRY(ensure(ws, &ws->S1, nb));
  WT_TRY(ensure(ws, &ws->SQ, nb));
  WT_TRY(ensure(ws, &ws->accP, nb));
  WT_TRY(ensure(ws, &ws->accQ, nb));
  if (m.precision == WT_F32) {
    WT_TRY(ensure(ws, &ws->compP, nb));
    WT_TRY(ensure(ws, &ws->compQ, nb));
    WT_TRY(ensure(ws, &ws->kP, nb));  // the compensated form's copy of Phi's high part (stage 2 -> 3)
  }
  return 0;
}

// Zero the FP32 compensation when the caller steps other state buffers than
// last time (a new solve or new initial data in other arrays).
void comp_track(wt_ws* ws, const void* Phi, const void* Pi) {
  if (!ws->compP) return;
  if (ws->comp_for[0] == Phi && ws->comp_for[1] == Pi) return;
  const size_t nb = (size_t)ws->mesh->m.nn * sizeof(float);
  cudaMemsetAsync(ws->compP, 0, nb, ws->ctx->stream);
  cudaMemsetAsync(ws->compQ, 0, nb, ws->ctx->stream);
  ws->comp_for[0] = Phi;
  ws->comp_for[1] = Pi;
}

int ws_k_buffers(wt_ws* ws) {
  const wt::DevMesh& m = ws->mesh->m;
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  WT_TRY(ensure(ws, &ws->kP, nb));
  WT_TRY(ensure(ws, &ws->kQ, nb));
  return 0;
}

int reduce_to_host(wt_ctx* ctx, double* out) {
  std::vector<double> h(ctx->nblocks);
  cudaMemcpyAsync(h.data(), ctx->d_partial, ctx->nblocks * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "reduction");
  double s = 0.0;
  for (double v : h) s += v;
  *out = s;
  return 0;
}

int make_bc(wt_ctx* ctx, const wt_bc_desc* bc, int use_metric, wt::ConsBC& out) {
  out = wt::ConsBC();
  if (!bc) return 0;
  for (int f = 0; f < 6; ++f) {
    if (bc->kinds[f] < 1 || bc->kinds[f] > 4)
      return fail(ctx, WT_EINVAL, "unknown boundary condition kind " + std::to_string(bc->kinds[f]) +
                                      " (expected 1 dirichlet, 2 sommerfeld, 3 excision, 4 full_dirichlet)");
  }
  out.on = 1;
  out.curv = use_metric ? 1 : 0;
  for (int f = 0; f < 6; ++f) out.kinds[f] = bc->kinds[f];
  out.sigma = bc->sigma;
  out.exc_tag = bc->excision_tag;
  out.gPhi = bc->gPhi; out.gPi = bc->gPi; out.gDx = bc->gDx; out.gDy = bc->gDy; out.gDz = bc->gDz;
  if (use_metric && bc->kinds[0] == WT_BC_EXCISION && bc->excision_tag == 0) out.on = 0;
  return 0;
}

// Entry points that evaluate the analytic map, sample a background at the
// nodes or use the FP64 Jacobians need the set-up geometry.
int need_setup_geometry(const wt_mesh* mh, const char* what) {
  if (mh->m.coords && mh->m.jac) return 0;
  return fail(mh->ctx, WT_EINVAL, std::string(what) + ": the mesh's set-up geometry was released");
}

int check_ws(wt_ctx* ctx, wt_ws* ws) {
  if (!ctx) return WT_EINVAL;
  if (!ws) return fail(ctx, WT_EINVAL, "workspace is NULL");
  if (ws->ctx != ctx) return fail(ctx, WT_EINVAL, "workspace belongs to another context");
  return 0;
}

// mu of make_wave3d_workspace: 30 power-iteration steps v <- D_1^2 v / ||D_1^2 v||
// from the alternating-sign start (src/wave3d_curved.jl:163-175).  Computed on
// first use; it synchronises the stream, so it runs outside graph capture.
int ensure_mu(wt_ws* ws) {
  if (ws->mu_done) return 0;
  wt_ctx* ctx = ws->ctx;
  const wt::DevMesh& m = ws->mesh->m;
  WT_TRY(ws_k_buffers(ws));
  cudaStream_t s = ctx->stream;
  int rc = lrc(ctx, wt::launch_alt_sign(m, ws->kP, s), "mu");
  double mu2 = 0.0;
  for (int it = 0; it < 30 && !rc; ++it) {
    rc = lrc(ctx, wt::launch_apply_D(m, ws->kP, ws->kQ, 0, s), "mu");
    if (!rc) rc = lrc(ctx, wt::launch_apply_D(m, ws->kQ, ws->kP, 0, s), "mu");
    if (!rc) rc = lrc(ctx, wt::launch_sumsq(m.nn, m.precision, ws->kP, ctx->d_partial, ctx->nblocks, s), "mu");
    double ss = 0.0;
    if (!rc) rc = reduce_to_host(ctx, &ss);
    ctx->launches += 3;
    if (rc) break;
    mu2 = std::sqrt(ss);
    if (!(mu2 > 0)) break;
    rc = lrc(ctx, wt::launch_scale(m.nn, m.precision, ws->kP, mu2, s), "mu");
    ctx->launches += 1;
  }
  if (rc) return rc;
  ws->mu = std::sqrt(mu2);
  ws->inv_mu5 = ws->mu > 0 ? std::pow(1.0 / ws->mu, 5) : 0.0;
  ws->mu_done = true;
  return 0;
}

// One RHS evaluation of the conservative system (non-fused).
int rhs_curved_impl(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, const void* Phi, const void* Pi, void* Phid,
                    void* Pid, double eps_ko, const wt::ConsBC& bc, int use_metric) {
  const wt::DevMesh& m = ws->mesh->m;
  wt::RKStage rk;
  const bool n8 = wt::cons_n8_path(m, coef->c, use_metric, bc, rk, rk, {Phi, Pi, ws->F, Phid, Pid});
  WT_TRY(lrc(ctx, wt::launch_cons_k1(m, coef->c, Phi, Pi, ws->F, Phid, ws->bbuf, nullptr, use_metric, bc, rk,
                                     ctx->stream, n8), "rhs K1"));
  WT_TRY(lrc(ctx, wt::launch_cons_k2(m, ws->F, Pid, ws->bbuf, use_metric, bc, rk, nullptr, ctx->stream, n8),
             "rhs K2"));
  ctx->launches += 2;
  if (eps_ko != 0.0) {
    const double koT = eps_ko * ws->inv_mu5;
    // the flux scratch is free once K2 has run
    WT_TRY(lrc(ctx, wt::launch_ko_add(m, Phid, Phi, koT, ctx->stream, ws->F), "Kreiss-Oliger"));
    WT_TRY(lrc(ctx, wt::launch_ko_add(m, Pid, Pi, koT, ctx->stream, ws->F), "Kreiss-Oliger"));
    ctx->launches += 6;
  }
  return 0;
}

}  // namespace

namespace wt {
// error reporting on a context for the other host translation units (the server)
int ctx_fail(wt_ctx* ctx, int code, const std::string& msg) { return fail(ctx, code, msg); }
// tracked device allocations for the other host translation units (the server's state buffers)
int ctx_alloc(wt_ctx* ctx, void** p, size_t bytes) { return dalloc(ctx, p, bytes, nullptr); }
void ctx_free(wt_ctx* ctx, void* p) { dfree(ctx, p); }
}  // namespace wt

extern "C" {

int wt_ctx_create(int device, wt_ctx** out) {
  if (!out) return WT_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return WT_ECUDA;
  }
  if (device < 0 || device >= ndev) return WT_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return WT_ECUDA;
  auto* c = new wt_ctx();
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return WT_ECUDA; }
  c->stream = c->own_stream;
  c->nblocks = wt::reduce_blocks();
  if (cudaMalloc(&c->d_flag, sizeof(unsigned int)) != cudaSuccess ||
      cudaMalloc(&c->d_partial, c->nblocks * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(c->d_flag);
    cudaStreamDestroy(c->own_stream);
    delete c;
    return WT_ENOMEM;
  }
  cudaMemset(c->d_flag, 0, sizeof(unsigned int));
  cudaEventCreateWithFlags(&c->ord_a, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&c->ord_b, cudaEventDisableTiming);
  *out = c;
  return 0;
}

int wt_ctx_destroy(wt_ctx* ctx) {
  if (!ctx) return WT_EINVAL;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->d_flag);
  cudaFree(ctx->d_partial);
  cudaEventDestroy(ctx->ord_a);
  cudaEventDestroy(ctx->ord_b);
  cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return 0;
}

const char* wt_last_error(const wt_ctx* ctx) { return ctx ? ctx->err.c_str() : "NULL context"; }

int wt_ctx_synchronize(wt_ctx* ctx) {
  if (!ctx) return WT_EINVAL;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "synchronize");
}

int wt_ctx_get_stream(wt_ctx* ctx, void** stream) {
  if (!ctx || !stream) return WT_EINVAL;
  *stream = (void*)ctx->stream;
  return 0;
}

int wt_ctx_set_stream(wt_ctx* ctx, void* stream) {
  if (!ctx) return WT_EINVAL;
  cudaStreamSynchronize(ctx->stream);
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return 0;
}

int wt_ctx_launch_count(const wt_ctx* ctx, long long* count) {
  if (!ctx || !count) return WT_EINVAL;
  *count = ctx->launches;
  return 0;
}

int wt_ctx_memory(const wt_ctx* ctx, long long* live_bytes, long long* live_allocs, long long* total_allocs) {
  if (!ctx) return WT_EINVAL;
  if (live_bytes) *live_bytes = ctx->live_bytes;
  if (live_allocs) *live_allocs = (long long)ctx->live.size();
  if (total_allocs) *total_allocs = ctx->total_allocs;
  return 0;
}

int wt_build_flags(int* flags) {
  if (!flags) return WT_EINVAL;
  *flags = 0;
#ifdef WT_BOUNDS_CHECK
  *flags |= WT_BUILD_BOUNDS_CHECK;
#endif
#ifndef WT_NO_NVTX
  *flags |= WT_BUILD_NVTX;
#endif
  return 0;
}

int wt_mesh_debug_set_table(wt_mesh* mesh, int table, long long e, int f, int value) {
  if (!mesh) return WT_EINVAL;
#ifndef WT_BOUNDS_CHECK
  (void)table; (void)e; (void)f; (void)value;
  return fail(mesh->ctx, WT_ENOTSUP, "wt_mesh_debug_set_table: only in the bounds-check build (-DWT_BOUNDS_CHECK)");
#else
  const wt::DevMesh& m = mesh->m;
  if (e < 0 || e >= m.Ne || f < 0 || f > 5 || (table != WT_TABLE_FACE_SOURCE && table != WT_TABLE_BOUNDARY_SLOT))
    return fail(mesh->ctx, WT_EINVAL, "wt_mesh_debug_set_table: bad table, element or face");
  int32_t* t = table == WT_TABLE_FACE_SOURCE ? m.fsrc : m.bslot;
  if (!t) return fail(mesh->ctx, WT_EINVAL, "wt_mesh_debug_set_table: the mesh has no such table");
  const int32_t v = value;
  cudaError_t err = cudaMemcpyAsync(t + f + 6 * e, &v, sizeof(v), cudaMemcpyHostToDevice, mesh->ctx->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(mesh->ctx->stream);
  return err == cudaSuccess ? 0 : cuda_fail(mesh->ctx, err, "wt_mesh_debug_set_table");
#endif
}

int wt_ctx_bounds_status(wt_ctx* ctx, unsigned int* word) {
  if (!ctx || !word) return WT_EINVAL;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "wt_ctx_bounds_status");
  *word = wt::bounds_take_cons() | wt::bounds_take_n8() | wt::bounds_take_second() | wt::bounds_take_geom();
  return 0;
}

int wt_ctx_inject_alloc_failure(wt_ctx* ctx, long long after) {
  if (!ctx) return WT_EINVAL;
  ctx->fail_after = after < 0 ? -1 : after;
  return 0;
}

int wt_ctx_profile(wt_ctx* ctx, int enable) {
  if (!ctx) return WT_EINVAL;
  ctx->prof_on = enable ? 1 : 0;
  return 0;
}

int wt_ctx_profile_read(wt_ctx* ctx, double ms[3], long long count[3]) {
  if (!ctx || !ms || !count) return WT_EINVAL;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "profile");
  for (int k = 0; k < 3; ++k) {
    ms[k] = 0.0;
    count[k] = 0;
    auto& v = ctx->prof_ev[k];
    for (size_t i = 0; i + 1 < v.size(); i += 2) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, v[i], v[i + 1]) == cudaSuccess) { ms[k] += t; ++count[k]; }
    }
    for (auto ev : v) cudaEventDestroy(ev);
    v.clear();
  }
  return 0;
}

int wt_ctx_nonfinite(wt_ctx* ctx, int* flag) {
  if (!ctx || !flag) return WT_EINVAL;
  unsigned int h = 0;
  cudaMemcpyAsync(&h, ctx->d_flag, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemsetAsync(ctx->d_flag, 0, sizeof(unsigned int), ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "nonfinite flag");
  *flag = (h & 1u) ? 1 : 0;
  if (h & 2u) return fail(ctx, WT_ETIMEOUT, "a bounded wait for staged data gave up in a pipelined kernel");
  return 0;
}

int wt_ctx_selftest_wait(wt_ctx* ctx, int arrive, long long polls) {
  if (!ctx) return WT_EINVAL;
  if (polls < 1 || polls > (1LL << 24)) return fail(ctx, WT_EINVAL, "wt_ctx_selftest_wait: polls must be in 1..2^24");
  int bad = 0;
  WT_TRY(wt_ctx_nonfinite(ctx, &bad));  // start from a clear status word
  WT_TRY(lrc(ctx, wt::launch_wait_selftest(polls, arrive, ctx->d_flag, ctx->stream), "wait self-test"));
  ctx->launches += 1;
  return wt_ctx_nonfinite(ctx, &bad);
}

// ---- reference element ------------------------------------------------------------
int wt_gll_operators(int N, double* x, double* H, double* G) {
  if (N < 2 || N > WT_MAXN || !x || !H || !G) return WT_EINVAL;
  wt::HostOps o = wt::gll_operators(N);
  std::memcpy(x, o.x.data(), N * sizeof(double));
  std::memcpy(H, o.H.data(), N * sizeof(double));
  std::memcpy(G, o.G.data(), N * N * sizeof(double));
  return 0;
}

// ---- mesh -------------------------------------------------------------------
// The analytic (warped) cube of desc, restricted to nz element layers along z
// starting at layer z0 of the whole mesh (modulo M[2] for a periodic mesh).
// Faces between layers of the slab couple as in the whole mesh; a z face whose
// neighbour layer lies outside the slab gets no neighbour and no tag (a cut),
// unless it is an outer face of the whole mesh.
static int create_analytic(wt_ctx* ctx, const wt_mesh_desc* d, int z0, int nz, wt_mesh** out) {
  cudaSetDevice(ctx->device);
  auto* mh = new wt_mesh();
  mh->ctx = ctx;
  wt::DevMesh& m = mh->m;
  m.errflag = ctx->d_flag;
  m.N = d->N;
  m.M[0] = d->M[0];
  m.M[1] = d->M[1];
  m.M[2] = nz;
  m.Ne = (long long)d->M[0] * d->M[1] * nz;
  m.nn = m.Ne * d->N * d->N * d->N;
  m.precision = d->precision;
  m.affine = d->warp_A == 0.0;
  m.h_nbr.assign(6 * m.Ne, -1);
  m.h_nbrf.assign(6 * m.Ne, 0);
  m.h_bdry.assign(6 * m.Ne, 0);
  const int Mx = d->M[0], My = d->M[1], Mz = d->M[2];
  const int ML[3] = {Mx, My, nz};
  for (long long e = 0; e < m.Ne; ++e) {
    int c[3] = {(int)(e % Mx), (int)((e / Mx) % My), (int)(e / ((long long)Mx * My))};
    for (int f = 0; f < 6; ++f) {
      const int ax = f >> 1;
      int cc[3] = {c[0], c[1], c[2]};
      cc[ax] += (f & 1) ? 1 : -1;
      if (cc[ax] < 0 || cc[ax] >= ML[ax]) {
        const bool whole = ax < 2 || nz == Mz;  // this axis spans the whole mesh
        if (!whole) {
          const int g = z0 + cc[2];  // the neighbour layer in the whole mesh
          if (!d->periodic && (g < 0 || g >= Mz)) m.h_bdry[f + 6 * e] = d->outer_tag == 0 ? f + 1 : d->outer_tag;
          continue;  // otherwise a cut face: no neighbour, no tag
        }
        if (!d->periodic) {
          m.h_bdry[f + 6 * e] = d->outer_tag == 0 ? f + 1 : d->outer_tag;
          continue;
        }
        cc[ax] = (cc[ax] + ML[ax]) % ML[ax];
      }
      m.h_nbr[f + 6 * e] = (int32_t)(cc[0] + (long long)Mx * (cc[1] + (long long)My * cc[2]));
      m.h_nbrf[f + 6 * e] = f ^ 1;
    }
  }
  int rc = finish_topology(mh);
  if (!rc) rc = alloc_geometry(mh);
  if (!rc) rc = lrc(ctx, wt::launch_geom_analytic(m, d->x0, d->x1, d->warp_A, ctx->stream, z0, Mz), "geometry");
  if (!rc) rc = derive_geometry(mh);
  if (rc) { free_mesh(mh); delete mh; return rc; }
  ctx->launches += 1;
  *out = mh;
  return 0;
}

static int check_mesh_desc(wt_ctx* ctx, const wt_mesh_desc* d) {
  if (d->N < 2 || d->N > WT_MAXN) return fail(ctx, WT_EINVAL, "N must be in 2..8, got " + std::to_string(d->N));
  if (d->M[0] < 1 || d->M[1] < 1 || d->M[2] < 1) return fail(ctx, WT_EINVAL, "element counts must be >= 1");
  if (d->precision != WT_F64 && d->precision != WT_F32) return fail(ctx, WT_EINVAL, "precision must be WT_F64 or WT_F32");
  if (!(d->x1 > d->x0)) return fail(ctx, WT_EINVAL, "x1 must exceed x0");
  return 0;
}

int wt_mesh_create(wt_ctx* ctx, const wt_mesh_desc* d, wt_mesh** out) {
  wt::NvtxRange nvtx_("wt_mesh_create");
  if (!ctx) return WT_EINVAL;
  if (!d || !out) return fail(ctx, WT_EINVAL, "wt_mesh_create: NULL argument");
  *out = nullptr;
  WT_TRY(check_mesh_desc(ctx, d));
  return create_analytic(ctx, d, 0, d->M[2], out);
}

int wt_mesh_create_slab(wt_ctx* ctx, const wt_mesh_desc* d, int z0, int nz, wt_mesh** out) {
  if (!ctx) return WT_EINVAL;
  if (!d || !out) return fail(ctx, WT_EINVAL, "wt_mesh_create_slab: NULL argument");
  *out = nullptr;
  WT_TRY(check_mesh_desc(ctx, d));
  const int Mz = d->M[2];
  if (nz < 1 || nz > Mz) return fail(ctx, WT_EINVAL, "wt_mesh_create_slab: nz must be in 1..M[2]");
  if (d->periodic ? (z0 < -Mz || z0 >= Mz) : (z0 < 0 || z0 + nz > Mz))
    return fail(ctx, WT_EINVAL, "wt_mesh_create_slab: layers [z0, z0 + nz) outside the mesh (periodic meshes: "
                                "-M[2] <= z0 < M[2])");
  return create_analytic(ctx, d, z0, nz, out);
}

}  // extern "C"

// A mesh from host coordinates, Jacobian and 0-based topology (nbrf = fn | ori << 3).
static int create_from_host(wt_ctx* ctx, int N, long long Ne, const double* coords, const double* jac,
                            std::vector<int32_t>& nbr, std::vector<int32_t>& nbrf, std::vector<int32_t>& bdry,
                            int precision, wt_mesh** out) {
  cudaSetDevice(ctx->device);
  auto* mh = new wt_mesh();
  mh->ctx = ctx;
  wt::DevMesh& m = mh->m;
  m.errflag = ctx->d_flag;
  m.N = N; m.Ne = Ne; m.nn = Ne * N * N * N; m.precision = precision; m.affine = 0;
  m.h_nbr.swap(nbr); m.h_nbrf.swap(nbrf); m.h_bdry.swap(bdry);
  int rc = finish_topology(mh);
  if (!rc) rc = alloc_geometry(mh);
  if (!rc) {
    cudaMemcpyAsync(m.coords, coords, 3 * m.nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(m.jac, jac, 9 * m.nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
    rc = derive_geometry(mh);
  }
  if (rc) { free_mesh(mh); delete mh; return rc; }
  *out = mh;
  return 0;
}

extern "C" {

int wt_mesh_create_arrays(wt_ctx* ctx, int N, long long Ne, const double* coords, const double* jac,
                          const int32_t* neighbour, const int32_t* neighbour_face, const int8_t* orientation,
                          const int8_t* bdry, int precision, wt_mesh** out) {
  (void)orientation;  // inferred from the coordinates
  if (!ctx) return WT_EINVAL;
  if (!out || !coords || !jac || !neighbour || !neighbour_face || !bdry)
    return fail(ctx, WT_EINVAL, "wt_mesh_create_arrays: NULL argument");
  *out = nullptr;
  if (N < 2 || N > WT_MAXN) return fail(ctx, WT_EINVAL, "N must be in 2..8");
  if (Ne < 1) return fail(ctx, WT_EINVAL, "Ne must be >= 1");
  if (precision != WT_F64 && precision != WT_F32) return fail(ctx, WT_EINVAL, "bad precision");
  std::vector<int32_t> nbr(6 * Ne), nbrf(6 * Ne), bd(6 * Ne);
  double scale = 0.0;
  for (long long i = 0; i < 3 * Ne * N * N * N; ++i) scale = std::max(scale, std::fabs(coords[i]));
  const double tol = 1e-9 * (scale > 0.0 ? scale : 1.0);
  for (long long i = 0; i < 6 * Ne; ++i) {
    const int en = neighbour[i];
    if (en < 0 || en > Ne) return fail(ctx, WT_EINVAL, "neighbour index out of range");
    nbr[i] = en - 1;
    const int fn = neighbour_face[i];
    if (en > 0 && (fn < 1 || fn > 6)) return fail(ctx, WT_EINVAL, "neighbour_face out of range");
    bd[i] = bdry[i];
    nbrf[i] = 0;
    if (en > 0) {
      const long long e = i / 6;
      const int f = (int)(i % 6);
      int ori = wt::infer_orientation(N, coords, e, f, en - 1, fn - 1, tol, false);
      if (ori < 0) ori = wt::infer_orientation(N, coords, e, f, en - 1, fn - 1, tol, true);  // periodic faces
      if (ori < 0)
        return fail(ctx, WT_EINVAL, "face " + std::to_string(f + 1) + " of element " + std::to_string(e + 1) +
                                        " does not coincide with its neighbour's face under any orientation");
      nbrf[i] = (fn - 1) | (ori << 3);
    }
  }
  return create_from_host(ctx, N, Ne, coords, jac, nbr, nbrf, bd, precision, out);
}

}  // extern "C"

// Host arrays of a WT_MESH_* patch mesh (0-based topology, nbrf = fn | ori << 3);
// "" or the reason it was refused.
static std::string patch_arrays(const wt_patch_desc* d, std::vector<double>& X, std::vector<double>& J,
                                std::vector<int32_t>& nbr, std::vector<int32_t>& nbrf, std::vector<int32_t>& bd) {
  if (d->N < 2 || d->N > WT_MAXN) return "N must be in 2..8";
  if (d->M < 1 || d->M > 64) return "M must be in 1..64";
  if (d->precision != WT_F64 && d->precision != WT_F32) return "bad precision";
  if (d->outer_tag == 0 || (d->kind == WT_MESH_RADIAL_SHELL && d->inner_tag == 0))
    return "outer_tag (and the radial shell's inner_tag) must be nonzero";
  const wt::HostOps ops = wt::gll_operators(d->N);
  double scale = 1.0;
  const int brc = wt::build_patch_mesh(d->kind, d->N, d->M, d->p, ops.x, X, scale);
  if (brc == -2) return "unknown mesh kind " + std::to_string(d->kind);
  if (brc) return "bad mesh parameters for kind " + std::to_string(d->kind);
  const long long N3 = (long long)d->N * d->N * d->N, Ne = (long long)X.size() / (3 * N3);
  if (wt::match_faces(d->N, Ne, X.data(), 1e-9 * scale, nbr, nbrf)) return "inconsistent face matching";
  bd.assign(6 * Ne, 0);
  for (long long i = 0; i < 6 * Ne; ++i) {
    if (nbr[i] >= 0) continue;
    int tag = d->outer_tag;
    if (d->kind == WT_MESH_RADIAL_SHELL) {  // inner or outer sphere: the radius of the face's first node
      const long long e = i / 6;
      const int f = (int)(i % 6);
      const double* x = &X[3 * (e * N3 + wt::face_node(wt::faxis(f), wt::frow(f, d->N), 0, 0, d->N))];
      if (std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]) < 0.5 * (d->p[0] + d->p[1])) tag = d->inner_tag;
    }
    bd[i] = tag;
  }
  J.assign(9 * N3 * Ne, 0.0);
  wt::coords_jacobian(d->N, Ne, X.data(), ops.G, J.data());
  return "";
}

extern "C" {

int wt_mesh_create_patches(wt_ctx* ctx, const wt_patch_desc* d, wt_mesh** out) {
  if (!ctx) return WT_EINVAL;
  if (!d || !out) return fail(ctx, WT_EINVAL, "wt_mesh_create_patches: NULL argument");
  *out = nullptr;
  std::vector<double> X, J;
  std::vector<int32_t> nbr, nbrf, bd;
  const std::string why = patch_arrays(d, X, J, nbr, nbrf, bd);
  if (!why.empty()) return fail(ctx, WT_EINVAL, "wt_mesh_create_patches: " + why);
  const long long Ne = (long long)nbr.size() / 6;
  return create_from_host(ctx, d->N, Ne, X.data(), J.data(), nbr, nbrf, bd, d->precision, out);
}

int wt_patch_mesh_arrays(const wt_patch_desc* d, long long* Ne, double* coords, double* jac, int32_t* neighbour,
                         int32_t* neighbour_face, int32_t* orientation, int32_t* bdry) {
  if (!d || !Ne) return WT_EINVAL;
  std::vector<double> X, J;
  std::vector<int32_t> nbr, nbrf, bd;
  if (!patch_arrays(d, X, J, nbr, nbrf, bd).empty()) return WT_EINVAL;
  const long long ne = (long long)nbr.size() / 6;
  *Ne = ne;
  if (!coords) return 0;
  std::memcpy(coords, X.data(), X.size() * sizeof(double));
  if (jac) std::memcpy(jac, J.data(), J.size() * sizeof(double));
  for (long long i = 0; i < 6 * ne; ++i) {
    if (neighbour) neighbour[i] = nbr[i] + 1;
    if (neighbour_face) neighbour_face[i] = nbr[i] < 0 ? 0 : (nbrf[i] & 7) + 1;
    if (orientation) orientation[i] = nbr[i] < 0 ? 0 : nbrf[i] >> 3;
    if (bdry) bdry[i] = bd[i];
  }
  return 0;
}

int wt_mesh_destroy(wt_mesh* mh) {
  if (!mh) return WT_EINVAL;
  cudaStreamSynchronize(mh->ctx->stream);
  free_mesh(mh);
  delete mh;
  return 0;
}

int wt_mesh_info(const wt_mesh* mh, int* N, long long* Ne, int* precision) {
  if (!mh) return WT_EINVAL;
  if (N) *N = mh->m.N;
  if (Ne) *Ne = mh->m.Ne;
  if (precision) *precision = mh->m.precision;
  return 0;
}

int wt_mesh_get(const wt_mesh* mh, const char* name, void* host_out) {
  if (!mh || !name || !host_out) return WT_EINVAL;
  const wt::DevMesh& m = mh->m;
  wt_ctx* ctx = mh->ctx;
  std::string s(name);
  const void* src = nullptr;
  size_t bytes = 0;
  if (s == "coords") { src = m.coords; bytes = 3 * m.nn * sizeof(double); }
  else if (s == "jac") { src = m.jac; bytes = 9 * m.nn * sizeof(double); }
  else if (s == "invjac") { src = m.invjac; bytes = 9 * m.nn * sizeof(double); }
  else if (s == "detjac") { src = m.detjac; bytes = m.nn * sizeof(double); }
  else if (s == "Hphys") { src = m.Hphys; bytes = m.nn * sizeof(double); }
  else if (s == "Hd") { src = m.Hd; bytes = m.nn * sizeof(double); }
  else if (s == "invdetJ") { src = m.invdetJ; bytes = m.nn * sizeof(double); }
  else if (s == "Ja") { src = m.Ja; bytes = 9 * m.nn * sizeof(double); }
  else if (s == "x") { std::memcpy(host_out, m.ops.x.data(), m.N * sizeof(double)); return 0; }
  else if (s == "H") { std::memcpy(host_out, m.ops.H.data(), m.N * sizeof(double)); return 0; }
  else if (s == "G") { std::memcpy(host_out, m.ops.G.data(), m.N * m.N * sizeof(double)); return 0; }
  else if (s == "bdry") { std::memcpy(host_out, m.h_bdry.data(), 6 * m.Ne * sizeof(int32_t)); return 0; }
  else if (s == "neighbour") {
    int32_t* o = (int32_t*)host_out;
    for (long long i = 0; i < 6 * m.Ne; ++i) o[i] = m.h_nbr[i] + 1;
    return 0;
  } else if (s == "neighbour_face" || s == "orientation") {  // 1-based face; D4 code of face_perm
    int32_t* o = (int32_t*)host_out;
    const bool face = s == "neighbour_face";
    for (long long i = 0; i < 6 * m.Ne; ++i)
      o[i] = m.h_nbr[i] < 0 ? 0 : face ? (m.h_nbrf[i] & 7) + 1 : m.h_nbrf[i] >> 3;
    return 0;
  } else if (s == "handedness") { src = m.handed; bytes = m.Ne * sizeof(int32_t); }
  else return fail(ctx, WT_EINVAL, "wt_mesh_get: unknown array '" + s + "'");
  if (!src) return fail(ctx, WT_EINVAL, "wt_mesh_get: '" + s + "' was released with the set-up geometry");
  cudaMemcpyAsync(host_out, src, bytes, cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "wt_mesh_get");
}

int wt_mesh_set_bdry(wt_mesh* mh, const int32_t* bdry) {
  if (!mh || !bdry) return WT_EINVAL;
  wt::DevMesh& m = mh->m;
  // the set of boundary faces must not change (slots and normals are precomputed)
  for (long long i = 0; i < 6 * m.Ne; ++i)
    if ((bdry[i] != 0) != (m.h_bdry[i] != 0))
      return fail(mh->ctx, WT_EINVAL, "wt_mesh_set_bdry may only relabel existing outer faces");
  std::memcpy(m.h_bdry.data(), bdry, 6 * m.Ne * sizeof(int32_t));
  cudaMemcpyAsync(m.bdry, m.h_bdry.data(), 6 * m.Ne * sizeof(int32_t), cudaMemcpyHostToDevice, mh->ctx->stream);
  cudaError_t e = cudaStreamSynchronize(mh->ctx->stream);
  return e == cudaSuccess ? 0 : cuda_fail(mh->ctx, e, "wt_mesh_set_bdry");
}

int wt_mesh_set_fp32_form(wt_mesh* mh, int form) {
  if (!mh) return WT_EINVAL;
  if (form != WT_FP32_CUDA_CORES && form != WT_FP32_BF16X3 && form != WT_FP32_BF16X2 && form != WT_FP32_COMPENSATED)
    return fail(mh->ctx, WT_EINVAL, "unknown FP32 form " + std::to_string(form));
  wt::DevMesh& m = mh->m;
  m.fp32_form = form;
  // the FP32 CUDA-core n = 8 kernels read the metric terms in their own layout
  const int want = m.precision == WT_F32 && (form == WT_FP32_CUDA_CORES || form == WT_FP32_COMPENSATED) ? 1 : 0;
  if (m.N == 8 && m.Ja_n8 && m.ja_n8_layout != want) {
    WT_TRY(lrc(mh->ctx, wt::launch_pad_metric_n8(m, mh->ctx->stream), "n = 8 metric layout"));
    cudaError_t e = cudaStreamSynchronize(mh->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(mh->ctx, e, "wt_mesh_set_fp32_form");
  }
  return 0;
}

int wt_mesh_release_setup_geometry(wt_mesh* mh) {
  if (!mh) return WT_EINVAL;
  wt::DevMesh& m = mh->m;
  cudaStreamSynchronize(mh->ctx->stream);
  std::vector<void*> drop = {m.coords, m.jac, m.invjac, m.detjac};
  if (m.precision != WT_F64) {  // FP32 meshes stream their own copies of Ja and 1/J
    drop.push_back(m.Ja);
    drop.push_back(m.invdetJ);
  }
  for (void* p : drop) {
    if (!p) continue;
    auto it = std::find(mh->owned.begin(), mh->owned.end(), p);
    if (it != mh->owned.end()) mh->owned.erase(it);
    dfree(mh->ctx, p);
  }
  m.coords = m.jac = m.invjac = m.detjac = nullptr;
  if (m.precision != WT_F64) m.Ja = m.invdetJ = nullptr;
  return 0;
}

int wt_mesh_min_spacing(wt_mesh* mh, double* h) {
  if (!mh || !h) return WT_EINVAL;
  WT_TRY(need_setup_geometry(mh, "wt_mesh_min_spacing"));
  mh->ctx->launches += 1;
  return lrc(mh->ctx, wt::launch_min_spacing(mh->m, h, mh->ctx->stream), "min spacing");
}

// ---- background ------------------------------------------------------------------
static int coef_alloc(wt_ctx* ctx, wt_mesh* mesh, wt_coef** out) {
  auto* c = new wt_coef();
  c->ctx = ctx; c->mesh = mesh;
  c->c.nn = mesh->m.nn;
  c->c.precision = mesh->m.precision;
  if (dalloc(ctx, &c->c.c11, 11 * c->c.nn * sizeof(double), nullptr) ||
      dalloc(ctx, &c->c.c10, 10 * c->c.nn * rsize(c->c.precision), nullptr)) {
    dfree(ctx, c->c.c11);
    delete c;
    return WT_ENOMEM;
  }
  *out = c;
  return 0;
}

int wt_background_set(wt_ctx* ctx, wt_mesh* mesh, const wt_background_desc* desc, wt_coef** out) {
  wt::NvtxRange nvtx_("wt_background_set");
  if (!ctx) return WT_EINVAL;
  if (!mesh || !desc || !out) return fail(ctx, WT_EINVAL, "wt_background_set: NULL argument");
  if (desc->kind < 0 || desc->kind > 5) return fail(ctx, WT_EINVAL, "unknown background kind");
  if (desc->kind == WT_BG_ADM_PERTURBED && !(desc->p[3] > 0))
    return fail(ctx, WT_EINVAL, "ADM background needs a positive Gaussian width p[3]");
  const bool td = desc->kind == WT_BG_GAUGE_WAVE || desc->kind == WT_BG_SINE_SHIFT;
  if (td && (!(std::fabs(desc->p[0]) < 1.0) || !(desc->p[1] > 0.0) || !std::isfinite(desc->p[2])))
    return fail(ctx, WT_EINVAL, "metric backgrounds need |A| < 1, d > 0 and a finite t0 (p[0..2])");
  WT_TRY(need_setup_geometry(mesh, "wt_background_set"));
  wt_coef* c = nullptr;
  WT_TRY(coef_alloc(ctx, mesh, &c));
  c->kind = desc->kind;
  std::memcpy(c->p, desc->p, sizeof(c->p));
  c->td = td;
  if (td) {
    c->t = desc->p[2];
    if (dalloc(ctx, (void**)&c->d_t, sizeof(double), nullptr)) { wt_coef_destroy(c); return WT_ENOMEM; }
    cudaMemcpyAsync(c->d_t, &c->t, sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  }
  int rc = lrc(ctx, wt::launch_background(mesh->m, c->c, desc->kind, desc->p, ctx->stream, c->d_t, 0.0),
               "background");
  if (!rc) rc = lrc(ctx, wt::launch_coef_combine(mesh->m, c->c, ctx->stream), "background");
  ctx->launches += 2;
  if (!rc) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "background");
  }
  if (rc) { wt_coef_destroy(c); return rc; }
  *out = c;
  return 0;
}

int wt_background_set_arrays(wt_ctx* ctx, wt_mesh* mesh, const double* coef11, wt_coef** out) {
  if (!ctx) return WT_EINVAL;
  if (!mesh || !coef11 || !out) return fail(ctx, WT_EINVAL, "wt_background_set_arrays: NULL argument");
  wt_coef* c = nullptr;
  WT_TRY(coef_alloc(ctx, mesh, &c));
  cudaMemcpyAsync(c->c.c11, coef11, 11 * c->c.nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  int rc = lrc(ctx, wt::launch_coef_combine(mesh->m, c->c, ctx->stream), "background");
  ctx->launches += 1;
  if (!rc) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "background");
  }
  if (rc) { wt_coef_destroy(c); return rc; }
  *out = c;
  return 0;
}

int wt_coef_get(const wt_coef* c, double* coef11) {
  if (!c || !coef11) return WT_EINVAL;
  cudaMemcpyAsync(coef11, c->c.c11, 11 * c->c.nn * sizeof(double), cudaMemcpyDeviceToHost, c->ctx->stream);
  cudaError_t e = cudaStreamSynchronize(c->ctx->stream);
  return e == cudaSuccess ? 0 : cuda_fail(c->ctx, e, "wt_coef_get");
}

int wt_coef_destroy(wt_coef* c) {
  if (!c) return WT_EINVAL;
  cudaStreamSynchronize(c->ctx->stream);
  dfree(c->ctx, c->c.c11);
  dfree(c->ctx, c->c.c10);
  dfree(c->ctx, c->d_t);
  delete c;
  return 0;
}

int wt_coef_set_time(wt_ctx* ctx, wt_coef* c, double t) {
  if (!ctx) return WT_EINVAL;
  if (!c) return fail(ctx, WT_EINVAL, "wt_coef_set_time: NULL argument");
  if (!c->td) return fail(ctx, WT_EINVAL, "wt_coef_set_time: the coefficients are not time-dependent");
  if (!std::isfinite(t)) return fail(ctx, WT_EINVAL, "wt_coef_set_time: t must be finite");
  WT_TRY(need_setup_geometry(c->mesh, "wt_coef_set_time"));
  c->t = t;
  cudaMemcpyAsync(c->d_t, &c->t, sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  int rc = lrc(ctx, wt::launch_background(c->mesh->m, c->c, c->kind, c->p, ctx->stream, c->d_t, 0.0), "background");
  if (!rc) rc = lrc(ctx, wt::launch_coef_combine(c->mesh->m, c->c, ctx->stream), "background");
  ctx->launches += 2;
  if (!rc) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "wt_coef_set_time");
  }
  return rc;
}

int wt_coef_get_time(const wt_coef* c, double* t) {
  if (!c || !t) return WT_EINVAL;
  *t = c->td ? c->t : 0.0;
  return 0;
}

// ---- initial data ---------------------------------------------------------------
int wt_initial_data(wt_ctx* ctx, wt_mesh* mesh, int kind, const double* params, int nparams, double t, void* u,
                    void* ut) {
  wt::NvtxRange nvtx_("wt_initial_data");
  if (!ctx) return WT_EINVAL;
  if (!mesh || !u || (nparams > 0 && !params)) return fail(ctx, WT_EINVAL, "wt_initial_data: NULL argument");
  if (kind < 0 || kind > 4) return fail(ctx, WT_EINVAL, "wt_initial_data: unknown kind");
  if (nparams < 0 || nparams > 4096) return fail(ctx, WT_EINVAL, "wt_initial_data: bad parameter count");
  if (kind == WT_IC_GAUSSIANS && (nparams < 1 || 1 + 5 * (int)params[0] > nparams))
    return fail(ctx, WT_EINVAL, "wt_initial_data: Gaussian count does not match the parameters");
  WT_TRY(need_setup_geometry(mesh, "wt_initial_data"));
  double* dp = nullptr;
  WT_TRY(dalloc(ctx, &dp, (nparams > 0 ? nparams : 1) * sizeof(double), nullptr));
  if (nparams > 0) cudaMemcpyAsync(dp, params, nparams * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  int rc = lrc(ctx, wt::launch_initial(mesh->m, kind, dp, nparams, t, u, ut, ctx->stream), "initial data");
  ctx->launches += 1;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  dfree(ctx, dp);
  if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, "initial data");
  return rc;
}

int wt_initial_state(wt_ctx* ctx, wt_ws* ws, int kind, const double* params, int nparams, double t, void* Phi,
                     void* Pi) {
  wt::NvtxRange nvtx_("wt_initial_state");
  WT_TRY(check_ws(ctx, ws));
  if (!Phi || !Pi) return fail(ctx, WT_EINVAL, "wt_initial_state: NULL argument");
  wt_mesh* mesh = ws->mesh;
  if (mesh->m.precision == WT_F64) return wt_initial_data(ctx, mesh, kind, params, nparams, t, Phi, Pi);
  if (kind < 0 || kind > 4) return fail(ctx, WT_EINVAL, "wt_initial_state: unknown kind");
  if (nparams < 0 || nparams > 4096 || (nparams > 0 && !params))
    return fail(ctx, WT_EINVAL, "wt_initial_state: bad parameters");
  if (kind == WT_IC_GAUSSIANS && (nparams < 1 || 1 + 5 * (int)params[0] > nparams))
    return fail(ctx, WT_EINVAL, "wt_initial_state: Gaussian count does not match the parameters");
  WT_TRY(need_setup_geometry(mesh, "wt_initial_state"));
  WT_TRY(ws_step_buffers(ws));
  const long long nn = mesh->m.nn;
  double *dp = nullptr, *tmp = nullptr;
  WT_TRY(dalloc(ctx, &dp, (nparams > 0 ? nparams : 1) * sizeof(double), nullptr));
  if (dalloc(ctx, &tmp, 2 * (size_t)nn * sizeof(double), nullptr)) {
    dfree(ctx, dp);
    return WT_ENOMEM;
  }
  if (nparams > 0) cudaMemcpyAsync(dp, params, nparams * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  int rc = lrc(ctx, wt::launch_initial(mesh->m, kind, dp, nparams, t, tmp, tmp + nn, ctx->stream, true),
               "initial state");
  if (!rc) rc = lrc(ctx, wt::launch_split_f64(nn, tmp, (float*)Phi, (float*)ws->compP, ctx->stream), "state split");
  if (!rc) rc = lrc(ctx, wt::launch_split_f64(nn, tmp + nn, (float*)Pi, (float*)ws->compQ, ctx->stream), "state split");
  ctx->launches += 3;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  dfree(ctx, dp);
  dfree(ctx, tmp);
  if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, "initial state");
  if (!rc) {
    ws->comp_for[0] = Phi;
    ws->comp_for[1] = Pi;
  }
  return rc;
}

// ---- workspace ---------------------------------------------------------------------
int wt_workspace_create(wt_ctx* ctx, wt_mesh* mesh, wt_ws** out) {
  if (!ctx) return WT_EINVAL;
  if (!mesh || !out) return fail(ctx, WT_EINVAL, "wt_workspace_create: NULL argument");
  auto* ws = new wt_ws();
  ws->ctx = ctx; ws->mesh = mesh;
  int rc = ws_buffers(ws);
  if (rc) { wt_workspace_destroy(ws); return rc; }
  *out = ws;
  return 0;
}

int wt_workspace_destroy(wt_ws* ws) {
  if (!ws) return WT_EINVAL;
  cudaStreamSynchronize(ws->ctx->stream);
  void* bufs[] = {ws->F, ws->F2, ws->bbuf, ws->grad, ws->kP, ws->kQ, ws->S0, ws->S1, ws->SQ, ws->accP, ws->accQ,
                  ws->trace, ws->zero, ws->Lu, ws->compP, ws->compQ, ws->erk, ws->evo[0], ws->evo[1],
                  ws->evo[2], ws->evo[3], ws->evoE};
  for (void* p : bufs) dfree(ws->ctx, p);
  delete ws;
  return 0;
}

int wt_workspace_set_fused(wt_ws* ws, int on) {
  if (!ws) return WT_EINVAL;
  ws->fused = on ? 1 : 0;
  return 0;
}

int wt_workspace_mu(wt_ws* ws, double* mu) {
  if (!ws || !mu) return WT_EINVAL;
  WT_TRY(ensure_mu(ws));
  *mu = ws->mu;
  return 0;
}

int wt_workspace_set_mu(wt_ws* ws, double mu) {
  if (!ws) return WT_EINVAL;
  if (!(mu > 0) || !std::isfinite(mu)) return fail(ws->ctx, WT_EINVAL, "wt_workspace_set_mu: mu must be positive");
  WT_TRY(ws_k_buffers(ws));  // ensure_mu allocates these with the estimate; the RK4 paths rely on it
  ws->mu = mu;
  ws->inv_mu5 = std::pow(1.0 / mu, 5);
  ws->mu_done = true;
  return 0;
}

int wt_state_set_f64(wt_ctx* ctx, wt_ws* ws, const double* Phi64, const double* Pi64, void* Phi, void* Pi) {
  WT_TRY(check_ws(ctx, ws));
  if (!Phi64 || !Pi64 || !Phi || !Pi) return fail(ctx, WT_EINVAL, "wt_state_set_f64: NULL argument");
  const wt::DevMesh& m = ws->mesh->m;
  if (m.precision == WT_F64) {
    cudaMemcpyAsync(Phi, Phi64, (size_t)m.nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
    cudaError_t e = cudaMemcpyAsync(Pi, Pi64, (size_t)m.nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "wt_state_set_f64");
  }
  WT_TRY(ws_step_buffers(ws));
  WT_TRY(lrc(ctx, wt::launch_split_f64(m.nn, Phi64, (float*)Phi, (float*)ws->compP, ctx->stream), "state split"));
  WT_TRY(lrc(ctx, wt::launch_split_f64(m.nn, Pi64, (float*)Pi, (float*)ws->compQ, ctx->stream), "state split"));
  ctx->launches += 2;
  ws->comp_for[0] = Phi;  // the low parts belong to this state pair: stepping it keeps them
  ws->comp_for[1] = Pi;
  return 0;
}

// ---- host checkpoints of a stepped state ----------------------------------------------
// Layout: Phi, Pi in the mesh precision, then (FP32 meshes) the low parts compP,
// compQ as float -- zeros when the workspace holds none for this state pair.
int wt_state_checkpoint_size(const wt_ws* ws, long long* bytes) {
  if (!ws || !bytes) return WT_EINVAL;
  const wt::DevMesh& m = ws->mesh->m;
  *bytes = (long long)m.nn * (long long)(m.precision == WT_F64 ? 2 * sizeof(double) : 4 * sizeof(float));
  return 0;
}

int wt_state_checkpoint_save(wt_ctx* ctx, wt_ws* ws, const void* Phi, const void* Pi, void* host, long long bytes) {
  wt::NvtxRange nvtx_("wt_state_checkpoint_save");
  WT_TRY(check_ws(ctx, ws));
  if (!Phi || !Pi || !host) return fail(ctx, WT_EINVAL, "wt_state_checkpoint_save: NULL argument");
  long long need = 0;
  wt_state_checkpoint_size(ws, &need);
  if (bytes != need)
    return fail(ctx, WT_EINVAL, "wt_state_checkpoint_save: the buffer must hold " + std::to_string(need) + " bytes");
  const wt::DevMesh& m = ws->mesh->m;
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  char* h = (char*)host;
  cudaMemcpyAsync(h, Phi, nb, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(h + nb, Pi, nb, cudaMemcpyDeviceToHost, ctx->stream);
  if (m.precision != WT_F64) {
    const size_t cb = (size_t)m.nn * sizeof(float);
    const bool held = ws->compP && ws->comp_for[0] == Phi && ws->comp_for[1] == Pi;
    if (held) {
      cudaMemcpyAsync(h + 2 * nb, ws->compP, cb, cudaMemcpyDeviceToHost, ctx->stream);
      cudaMemcpyAsync(h + 2 * nb + cb, ws->compQ, cb, cudaMemcpyDeviceToHost, ctx->stream);
    } else {
      std::memset(h + 2 * nb, 0, 2 * cb);  // stepping this pair would start from zero low parts
    }
  }
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "wt_state_checkpoint_save");
}

int wt_state_checkpoint_load(wt_ctx* ctx, wt_ws* ws, void* Phi, void* Pi, const void* host, long long bytes) {
  wt::NvtxRange nvtx_("wt_state_checkpoint_load");
  WT_TRY(check_ws(ctx, ws));
  if (!Phi || !Pi || !host) return fail(ctx, WT_EINVAL, "wt_state_checkpoint_load: NULL argument");
  long long need = 0;
  wt_state_checkpoint_size(ws, &need);
  if (bytes != need)
    return fail(ctx, WT_EINVAL, "wt_state_checkpoint_load: the buffer must hold " + std::to_string(need) + " bytes");
  const wt::DevMesh& m = ws->mesh->m;
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  const char* h = (const char*)host;
  if (m.precision != WT_F64) WT_TRY(ws_step_buffers(ws));  // the low parts' home
  cudaMemcpyAsync(Phi, h, nb, cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(Pi, h + nb, nb, cudaMemcpyHostToDevice, ctx->stream);
  if (m.precision != WT_F64) {
    const size_t cb = (size_t)m.nn * sizeof(float);
    cudaMemcpyAsync(ws->compP, h + 2 * nb, cb, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(ws->compQ, h + 2 * nb + cb, cb, cudaMemcpyHostToDevice, ctx->stream);
    ws->comp_for[0] = Phi;  // the low parts belong to this state pair: stepping it keeps them
    ws->comp_for[1] = Pi;
  }
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "wt_state_checkpoint_load");
}

// ---- RHS ----------------------------------------------------------------------------
int wt_rhs_curved(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, const void* Phi, const void* Pi, void* Phidot,
                  void* Pidot, double eps_ko, const wt_bc_desc* bc, int use_metric) {
  wt::NvtxRange nvtx_("wt_rhs_curved");
  WT_TRY(check_ws(ctx, ws));
  if (!coef || !Phi || !Pi || !Phidot || !Pidot) return fail(ctx, WT_EINVAL, "wt_rhs_curved: NULL argument");
  if (coef->mesh != ws->mesh) return fail(ctx, WT_EINVAL, "coefficients belong to another mesh");
  wt::ConsBC b;
  WT_TRY(make_bc(ctx, bc, use_metric, b));
  if (eps_ko != 0.0) WT_TRY(ensure_mu(ws));
  return rhs_curved_impl(ctx, ws, coef, Phi, Pi, Phidot, Pidot, eps_ko, b, use_metric);
}

int wt_apply_D(wt_ctx* ctx, wt_ws* ws, const void* u, void* Du, int d) {
  wt::NvtxRange nvtx_("wt_apply_D");
  WT_TRY(check_ws(ctx, ws));
  if (!u || !Du) return fail(ctx, WT_EINVAL, "wt_apply_D: NULL argument");
  if (d < 1 || d > 3) return fail(ctx, WT_EINVAL, "wt_apply_D: d must be 1, 2 or 3");
  ctx->launches += 1;
  return lrc(ctx, wt::launch_apply_D(ws->mesh->m, u, Du, d - 1, ctx->stream), "apply_D");
}

int wt_ko_add(wt_ctx* ctx, wt_ws* ws, void* dst, const void* field, double eps_ko) {
  WT_TRY(check_ws(ctx, ws));
  if (!dst || !field) return fail(ctx, WT_EINVAL, "wt_ko_add: NULL argument");
  WT_TRY(ensure_mu(ws));
  WT_TRY(ws_buffers(ws));
  ctx->launches += 3;
  return lrc(ctx, wt::launch_ko_add(ws->mesh->m, dst, field, eps_ko * ws->inv_mu5, ctx->stream, ws->F),
             "Kreiss-Oliger");
}

int wt_gradient3d(wt_ctx* ctx, wt_ws* ws, const void* u, void* g1, void* g2, void* g3) {
  WT_TRY(check_ws(ctx, ws));
  if (!u || !g1 || !g2 || !g3) return fail(ctx, WT_EINVAL, "wt_gradient3d: NULL argument");
  const wt::DevMesh& m = ws->mesh->m;
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  WT_TRY(ensure(ws, &ws->grad, 3 * nb));
  wt::DevCoef nocoef;
  wt::ConsBC bc;
  wt::RKStage rk;
  WT_TRY(lrc(ctx, wt::launch_cons_k1(m, nocoef, u, nullptr, nullptr, nullptr, nullptr, ws->grad, 1, bc, rk,
                                     ctx->stream), "gradient3d"));
  cudaMemcpyAsync(g1, ws->grad, nb, cudaMemcpyDeviceToDevice, ctx->stream);
  cudaMemcpyAsync(g2, (char*)ws->grad + nb, nb, cudaMemcpyDeviceToDevice, ctx->stream);
  cudaMemcpyAsync(g3, (char*)ws->grad + 2 * nb, nb, cudaMemcpyDeviceToDevice, ctx->stream);
  ctx->launches += 1;
  return 0;
}

int wt_divergence3d(wt_ctx* ctx, wt_ws* ws, const void* F1, const void* F2, const void* F3, void* out) {
  WT_TRY(check_ws(ctx, ws));
  if (!F1 || !F2 || !F3 || !out) return fail(ctx, WT_EINVAL, "wt_divergence3d: NULL argument");
  const wt::DevMesh& m = ws->mesh->m;
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  cudaMemcpyAsync(ws->F, F1, nb, cudaMemcpyDeviceToDevice, ctx->stream);
  cudaMemcpyAsync((char*)ws->F + nb, F2, nb, cudaMemcpyDeviceToDevice, ctx->stream);
  cudaMemcpyAsync((char*)ws->F + 2 * nb, F3, nb, cudaMemcpyDeviceToDevice, ctx->stream);
  ctx->launches += 1;
  return lrc(ctx, wt::launch_div3d(m, ws->F, out, ctx->stream), "divergence3d");
}

int wt_rhs_sipg(wt_ctx* ctx, wt_ws* ws, const void* u, const void* ut, void* utt, const double bdry_values[6],
                double tau, double sommerfeld_R) {
  wt::NvtxRange nvtx_("wt_rhs_sipg");
  WT_TRY(check_ws(ctx, ws));
  if (!u || !ut || !utt || !bdry_values) return fail(ctx, WT_EINVAL, "wt_rhs_sipg: NULL argument");
  const wt::DevMesh& m = ws->mesh->m;
  if (!m.affine) return fail(ctx, WT_ENOTSUP, "wt_rhs_sipg: this build supports axis-aligned affine meshes only");
  WT_TRY(ensure(ws, &ws->trace, (size_t)6 * m.N * m.N * m.Ne * rsize(m.precision)));
  const double inv_R = (std::isfinite(sommerfeld_R) && sommerfeld_R > 0) ? 1.0 / sommerfeld_R : 0.0;
  ctx->launches += 2;
  return lrc(ctx, wt::launch_sipg(m, u, ut, utt, ws->trace, bdry_values, tau, inv_R, ctx->stream), "rhs_sipg");
}

int wt_rhs_strong(wt_ctx* ctx, wt_ws* ws, const void* u, const void* ut, void* utt, double tau,
                  double sommerfeld_R) {
  wt::NvtxRange nvtx_("wt_rhs_strong");
  WT_TRY(check_ws(ctx, ws));
  if (!u || !ut || !utt) return fail(ctx, WT_EINVAL, "wt_rhs_strong: NULL argument");
  WT_TRY(need_setup_geometry(ws->mesh, "wt_rhs_strong"));
  wt::DevMesh& m = ws->mesh->m;
  if (!m.dinvjac) {
    WT_TRY(dalloc(ctx, &m.dinvjac, 27 * (size_t)m.nn * sizeof(double), &ws->mesh->owned));
    WT_TRY(lrc(ctx, wt::launch_dinvjac(m, ctx->stream), "make_metric_derivs"));
    ctx->launches += 1;
  }
  const double inv_R = (std::isfinite(sommerfeld_R) && sommerfeld_R > 0) ? 1.0 / sommerfeld_R : 0.0;
  ctx->launches += 1;
  return lrc(ctx, wt::launch_strong(m, u, ut, utt, tau, inv_R, ctx->stream), "rhs_strong");
}

int wt_lap_strong_cons(wt_ctx* ctx, wt_ws* ws, const void* u, void* Lu, double h, double tau) {
  WT_TRY(check_ws(ctx, ws));
  if (!u || !Lu) return fail(ctx, WT_EINVAL, "wt_lap_strong_cons: NULL argument");
  if (!(h > 0)) return fail(ctx, WT_EINVAL, "wt_lap_strong_cons: h must be positive");
  if (!ws->mesh->m.affine) return fail(ctx, WT_EINVAL, "wt_lap_strong_cons: uniform Cartesian meshes only");
  ctx->launches += 1;
  return lrc(ctx, wt::launch_lap_strong_cons(ws->mesh->m, u, Lu, h, tau, ctx->stream), "lap_strong_cons");
}

// ---- reductions ---------------------------------------------------------------------------
int wt_curved4_background(wt_ctx* ctx, wt_mesh* mesh, int kind, const double* params, double t, void* ginv,
                          void* gamma) {
  if (!ctx) return WT_EINVAL;
  if (!mesh || !ginv || !gamma) return fail(ctx, WT_EINVAL, "wt_curved4_background: NULL argument");
  if (kind != WT_CURVED4_MINKOWSKI && kind != WT_CURVED4_GAUGE_WAVE)
    return fail(ctx, WT_EINVAL, "wt_curved4_background: unknown metric kind");
  double p[2] = {0.0, 1.0};
  if (kind == WT_CURVED4_GAUGE_WAVE) {
    if (!params) return fail(ctx, WT_EINVAL, "wt_curved4_background: the gauge wave needs (A, d)");
    p[0] = params[0];
    p[1] = params[1];
    if (!(p[1] != 0.0) || !(std::fabs(p[0]) < 1.0))
      return fail(ctx, WT_EINVAL, "wt_curved4_background: gauge wave needs |A| < 1 and d != 0");
  }
  WT_TRY(need_setup_geometry(mesh, "wt_curved4_background"));
  ctx->launches += 1;
  return lrc(ctx, wt::launch_curved4_background(mesh->m, kind, p, t, ginv, gamma, ctx->stream), "curved4 background");
}

int wt_rhs_curved4(wt_ctx* ctx, wt_ws* ws, const void* phi, const void* phidot, void* phiddot, const void* ginv,
                   const void* gamma, double h, int conservative, double tau) {
  wt::NvtxRange nvtx_("wt_rhs_curved4");
  WT_TRY(check_ws(ctx, ws));
  if (!phi || !phidot || !phiddot || !ginv || !gamma) return fail(ctx, WT_EINVAL, "wt_rhs_curved4: NULL argument");
  if (!(h > 0)) return fail(ctx, WT_EINVAL, "wt_rhs_curved4: h must be positive");
  if (!ws->mesh->m.affine) return fail(ctx, WT_EINVAL, "wt_rhs_curved4: uniform Cartesian meshes only");
  ctx->launches += 1;
  return lrc(ctx, wt::launch_curved4(ws->mesh->m, phi, phidot, phiddot, ginv, gamma, h, conservative ? 1 : 0, tau,
                                     ctx->stream), "rhs_curved4");
}

// The energy's per-block partial sums into ctx->d_partial (asynchronous).
static int energy_partials(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, const void* Phi, const void* Pi,
                           int use_metric, int lapse = 0) {
  const wt::DevMesh& m = ws->mesh->m;
  WT_TRY(ensure(ws, &ws->grad, 3 * (size_t)m.nn * rsize(m.precision)));
  wt::DevCoef nocoef;
  wt::ConsBC bc;
  wt::RKStage rk;
  auto a16 = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
  if (m.N == 8 && use_metric && m.Ja_n8 && a16(Phi) && a16(ws->grad) && a16(m.invdetJ_r))
    WT_TRY(lrc(ctx, wt::launch_grad_n8(m, Phi, ws->grad, m.errflag, ctx->stream), "energy gradient"));
  else
    WT_TRY(lrc(ctx, wt::launch_cons_k1(m, nocoef, Phi, nullptr, nullptr, nullptr, nullptr, ws->grad, use_metric, bc,
                                       rk, ctx->stream), "energy gradient"));
  WT_TRY(lrc(ctx, wt::launch_energy(m, coef->c, Pi, ws->grad, use_metric, ctx->d_partial, ctx->nblocks, ctx->stream,
                                     lapse), "energy"));
  ctx->launches += 2;
  return 0;
}

int wt_energy(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, const void* Phi, const void* Pi, int use_metric,
              double* E) {
  wt::NvtxRange nvtx_("wt_energy");
  WT_TRY(check_ws(ctx, ws));
  if (!coef || !Phi || !Pi || !E) return fail(ctx, WT_EINVAL, "wt_energy: NULL argument");
  WT_TRY(energy_partials(ctx, ws, coef, Phi, Pi, use_metric));
  return reduce_to_host(ctx, E);
}

int wt_energy_lapse(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, const void* Phi, const void* Pi, int use_metric,
                    double* E) {
  wt::NvtxRange nvtx_("wt_energy_lapse");
  WT_TRY(check_ws(ctx, ws));
  if (!coef || !Phi || !Pi || !E) return fail(ctx, WT_EINVAL, "wt_energy_lapse: NULL argument");
  if (coef->mesh != ws->mesh) return fail(ctx, WT_EINVAL, "coefficients belong to another mesh");
  WT_TRY(energy_partials(ctx, ws, coef, Phi, Pi, use_metric, 1));
  return reduce_to_host(ctx, E);
}

int wt_energy_sipg(wt_ctx* ctx, wt_ws* ws, const void* u, const void* ut, double tau, double* E) {
  wt::NvtxRange nvtx_("wt_energy_sipg");
  WT_TRY(check_ws(ctx, ws));
  if (!u || !ut || !E) return fail(ctx, WT_EINVAL, "wt_energy_sipg: NULL argument");
  const wt::DevMesh& m = ws->mesh->m;
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  if (!ws->zero) {
    WT_TRY(ensure(ws, &ws->zero, nb));
    cudaMemsetAsync(ws->zero, 0, nb, ctx->stream);
  }
  WT_TRY(ensure(ws, &ws->Lu, nb));
  const double bz[6] = {0, 0, 0, 0, 0, 0};
  WT_TRY(wt_rhs_sipg(ctx, ws, u, ws->zero, ws->Lu, bz, tau, 0.0));
  double K = 0, V = 0;
  WT_TRY(lrc(ctx, wt::launch_dot_weighted(m, ut, ut, nullptr, nullptr, 0, 0, ctx->d_partial, ctx->nblocks,
                                          ctx->stream), "energy_sipg"));
  WT_TRY(reduce_to_host(ctx, &K));
  WT_TRY(lrc(ctx, wt::launch_dot_weighted(m, u, ws->Lu, nullptr, nullptr, 0, 0, ctx->d_partial, ctx->nblocks,
                                          ctx->stream), "energy_sipg"));
  WT_TRY(reduce_to_host(ctx, &V));
  ctx->launches += 2;
  *E = K / 2 - V / 2;
  return 0;
}

int wt_l2_diff(wt_ctx* ctx, wt_ws* ws, const void* a, const void* b, int use_metric, double* out) {
  wt::NvtxRange nvtx_("wt_l2_diff");
  WT_TRY(check_ws(ctx, ws));
  if (!a || !out) return fail(ctx, WT_EINVAL, "wt_l2_diff: NULL argument");
  double s = 0;
  WT_TRY(lrc(ctx, wt::launch_dot_weighted(ws->mesh->m, a, b, nullptr, nullptr, use_metric ? 1 : 0, 1, ctx->d_partial,
                                          ctx->nblocks, ctx->stream), "l2"));
  ctx->launches += 1;
  WT_TRY(reduce_to_host(ctx, &s));
  *out = std::sqrt(s);
  return 0;
}

// ---- time stepping ------------------------------------------------------------------------
// Time-dependent coefficients: sample at the coefficients' time + toff (stage times of RK4).
static int coef_resample(wt_ctx* ctx, const wt_coef* coef, double toff, cudaStream_t s) {
  wt::DevCoef c = coef->c;
  WT_TRY(lrc(ctx, wt::launch_background(coef->mesh->m, c, coef->kind, coef->p, s, coef->d_t, toff), "background"));
  WT_TRY(lrc(ctx, wt::launch_coef_combine(coef->mesh->m, c, s), "background"));
  ctx->launches += 2;
  return 0;
}

// The Phi side of fused RK4 stage st (eps_ko = 0).  Plain forms: K1 reads the
// state at stage 0 and the previous stage's output after it.  Compensated FP32
// form: K1 reads the state's high part (stage 3: the copy stage 2 made of it,
// since stage 3 overwrites the state while neighbours still read it) plus a
// small part -- the state's low part at stage 0, the previous stage's output
// (low part + increment) after it.
struct PhiStage {
  const void* in;
  const void* phit;
  void* hcopy;
};
static PhiStage phi_stage(const wt_ws* ws, void* Phi, int st, bool cp) {
  void* SP[2] = {ws->S0, ws->S1};
  if (!cp) return {st == 0 ? Phi : SP[(st - 1) % 2], nullptr, nullptr};
  return {st == 3 ? ws->kP : Phi, st == 0 ? ws->compP : SP[(st - 1) % 2], st == 2 ? ws->kP : nullptr};
}

// Whether the fused stages of this mesh run the compensated FP32 form: the
// default FP32 form, through the kernels that implement it.
static bool compensated(const wt::DevMesh& m, bool n8) {
  return m.precision == WT_F32 && m.fp32_form == WT_FP32_COMPENSATED && (n8 || wt::cons_gen_cp_supported(m));
}

// One half of fused RK4 stage st (eps_ko = 0): part 1 launches K1 (flux, boundary
// terms, the Phi stage update), part 2 K2 (divergence, the Pi stage update).
static int rk4_stage_part(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, int st,
                          int part, const wt::ConsBC& b, int use_metric, long long e0 = 0, long long e1 = -1) {
  const wt::DevMesh& m = ws->mesh->m;
  cudaStream_t s = ctx->stream;
  void* SP[2] = {ws->S0, ws->S1};
  const void* inQ = st == 0 ? Pi : ws->SQ;
  wt::RKStage rkP, rkQ;
  rkP.stage = rkQ.stage = st;
  rkP.dt = rkQ.dt = dt;
  rkP.y = Phi; rkP.acc = ws->accP; rkP.out = SP[st % 2]; rkP.comp = ws->compP;
  rkQ.y = Pi; rkQ.acc = ws->accQ; rkQ.out = ws->SQ; rkQ.comp = ws->compQ;
  rkP.nonfinite = rkQ.nonfinite = st == 3 ? ctx->d_flag : nullptr;
  rkP.on = rkQ.on = 1;
  const bool n8 = wt::cons_n8_path(m, coef->c, use_metric, b, rkP, rkQ, {Phi, inQ, ws->F});
  const bool cp = compensated(m, n8);  // its buffers (kP: the high-part copy) come with ws_step_buffers
  const PhiStage ps = phi_stage(ws, Phi, st, cp);
  const void* inP = ps.in;
  rkP.phit = ps.phit;
  rkP.hcopy = ps.hcopy;
  ws->halo_cp = cp ? 1 : 0;
  ws->flux_block = n8 ? wt::n8_flux_block(m) : (long long)m.N * m.N * m.N;
  ws->flux_lay = n8 ? wt::n8_flux_layout(m) : 0;
  static const char* kNames[2][4] = {{"rk4 stage 0 K1", "rk4 stage 1 K1", "rk4 stage 2 K1", "rk4 stage 3 K1"},
                                     {"rk4 stage 0 K2", "rk4 stage 1 K2", "rk4 stage 2 K2", "rk4 stage 3 K2"}};
  wt::NvtxRange nv(kNames[part - 1][st]);
  if (part == 1) {
    prof_mark(ctx, 0);
    WT_TRY(lrc(ctx, wt::launch_cons_k1(m, coef->c, inP, inQ, ws->F, nullptr, ws->bbuf, nullptr, use_metric, b, rkP,
                                       s, n8, e0, e1), "rk4 K1"));
    prof_mark(ctx, 0);
  } else {
    prof_mark(ctx, 1);
    WT_TRY(lrc(ctx, wt::launch_cons_k2(m, ws->F, nullptr, ws->bbuf, use_metric, b, rkQ, rkQ.nonfinite, s, n8, e0, e1),
               "rk4 K2"));
    prof_mark(ctx, 1);
  }
  ctx->launches += 1;
  return 0;
}

// The RK4 step of an FP64 n = 8 solve through the fused stage kernel: K1_0,
// FK_0, FK_1, FK_2 (each the K2 half of stage s and the K1 half of stage s + 1),
// K2_3 -- five launches instead of eight, the flux ping-ponging between ws->F
// and ws->F2.  Time-dependent backgrounds are re-sampled before the launch
// whose K1 half reads them (the K2 halves read no coefficients).  The results
// equal those of the two-kernel stages bit for bit.
static bool fused_path(const wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double eps_ko,
                       const wt::ConsBC& b, int use_metric) {
  const wt::DevMesh& m = ws->mesh->m;
  if (!ws->fused || eps_ko != 0.0 || m.precision != WT_F64 || m.N != 8 || !ws->F2) return false;
  wt::RKStage r;
  r.on = 1;
  r.y = Phi; r.acc = ws->accP; r.out = ws->S0;
  wt::RKStage q = r;
  q.y = Pi; q.acc = ws->accQ; q.out = ws->SQ;
  return wt::cons_n8_path(m, coef->c, use_metric, b, r, q, {Phi, Pi, ws->F, ws->F2, ws->S1});
}

static int step_curved_fused(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt,
                             const wt::ConsBC& b, int use_metric) {
  const wt::DevMesh& m = ws->mesh->m;
  cudaStream_t s = ctx->stream;
  void* SP[2] = {ws->S0, ws->S1};
  void* FB[2] = {ws->F, ws->F2};
  const double toff[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};  // RK4 stage times
  auto rkP = [&](int st) {
    wt::RKStage r;
    r.on = 1; r.stage = st; r.dt = dt;
    r.y = Phi; r.acc = ws->accP; r.out = SP[st % 2];
    return r;
  };
  auto rkQ = [&](int st) {
    wt::RKStage r;
    r.on = 1; r.stage = st; r.dt = dt;
    r.y = Pi; r.acc = ws->accQ; r.out = nullptr;  // Pi's stage value stays in the fused kernel's registers
    return r;
  };
  ws->halo_cp = 0;
  ws->flux_block = wt::n8_flux_block(m);
  ws->flux_lay = wt::n8_flux_layout(m);
  if (coef->td) WT_TRY(coef_resample(ctx, coef, toff[0], s));
  {
    wt::NvtxRange nv("rk4 stage 0 K1");
    prof_mark(ctx, 0);
    WT_TRY(lrc(ctx, wt::launch_cons_k1(m, coef->c, Phi, Pi, FB[0], nullptr, ws->bbuf, nullptr, use_metric, b, rkP(0),
                                       s, true), "rk4 K1"));
    prof_mark(ctx, 0);
  }
  ctx->launches += 1;
  static const char* kNames[3] = {"rk4 fused stage 0-1", "rk4 fused stage 1-2", "rk4 fused stage 2-3"};
  for (int st = 0; st < 3; ++st) {
    if (coef->td) WT_TRY(coef_resample(ctx, coef, toff[st + 1], s));
    wt::NvtxRange nv(kNames[st]);
    prof_mark(ctx, 2);
    WT_TRY(lrc(ctx, wt::launch_cons_fk_n8(m, coef->c, FB[st % 2], FB[(st + 1) % 2], SP[st % 2], ws->bbuf, b, rkQ(st),
                                          rkP(st + 1), s), "rk4 fused stage"));
    prof_mark(ctx, 2);
    ctx->launches += 1;
  }
  {
    wt::NvtxRange nv("rk4 stage 3 K2");
    prof_mark(ctx, 1);
    WT_TRY(lrc(ctx, wt::launch_cons_k2(m, FB[1], nullptr, ws->bbuf, use_metric, b, rkQ(3), nullptr, s, true),
               "rk4 K2"));
    prof_mark(ctx, 1);
  }
  ctx->launches += 1;
  if (coef->td) {
    WT_TRY(lrc(ctx, wt::launch_advance_time(coef->d_t, dt, s), "background time"));
    ctx->launches += 1;
  }
  return 0;
}

static int step_curved_once(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt,
                            double eps_ko, const wt::ConsBC& b, int use_metric) {
  if (fused_path(ws, coef, Phi, Pi, eps_ko, b, use_metric))
    return step_curved_fused(ctx, ws, coef, Phi, Pi, dt, b, use_metric);
  const wt::DevMesh& m = ws->mesh->m;
  cudaStream_t s = ctx->stream;
  void* SP[2] = {ws->S0, ws->S1};
  const double toff[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};  // RK4 stage times
  for (int st = 0; st < 4; ++st) {
    if (coef->td) WT_TRY(coef_resample(ctx, coef, toff[st], s));
    const void* inP = st == 0 ? Phi : SP[(st - 1) % 2];
    const void* inQ = st == 0 ? Pi : ws->SQ;
    if (eps_ko == 0.0) {
      WT_TRY(rk4_stage_part(ctx, ws, coef, Phi, Pi, dt, st, 1, b, use_metric));
      WT_TRY(rk4_stage_part(ctx, ws, coef, Phi, Pi, dt, st, 2, b, use_metric));
    } else {
      WT_TRY(rhs_curved_impl(ctx, ws, coef, inP, inQ, ws->kP, ws->kQ, eps_ko, b, use_metric));
      WT_TRY(lrc(ctx, wt::launch_rk_update(m.nn, m.precision, st, dt, Phi, ws->accP, SP[st % 2], ws->kP, s,
                                           ws->compP), "rk4"));
      WT_TRY(lrc(ctx, wt::launch_rk_update(m.nn, m.precision, st, dt, Pi, ws->accQ, ws->SQ, ws->kQ, s, ws->compQ),
                 "rk4"));
      ctx->launches += 2;
    }
  }
  if (coef->td) {
    WT_TRY(lrc(ctx, wt::launch_advance_time(coef->d_t, dt, s), "background time"));
    ctx->launches += 1;
  }
  return 0;
}

// Butcher tableaus of the fixed-step explicit Runge-Kutta methods that
// pick_integrator_first_order selects (src/evolve.jl:43-48; evolve3d calls them
// with adaptive = false, src/evolve.jl:1311): the classic RK4 and Tsit5
// (Ch. Tsitouras, "Runge-Kutta pairs of order 5(4) satisfying only the first
// column simplifying assumption", Comput. Math. Appl. 62 (2011) 770-775: the
// fifth-order solution).  Tsit5's seventh stage has weight 0 (it only serves
// the embedded error estimate and the first-same-as-last reuse), so a fixed
// step evaluates six stages.
struct ErkTableau {
  int s = 0;
  double c[WT_ERK_MAX_STAGES] = {};
  double A[WT_ERK_MAX_STAGES][WT_ERK_MAX_STAGES] = {};
  double b[WT_ERK_MAX_STAGES] = {};
};

static const ErkTableau* erk_tableau(int method) {
  static ErkTableau rk4, tsit5;
  static bool init = false;
  if (!init) {
    rk4.s = 4;
    const double c4[4] = {0.0, 0.5, 0.5, 1.0};
    const double b4[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    for (int i = 0; i < 4; ++i) { rk4.c[i] = c4[i]; rk4.b[i] = b4[i]; }
    rk4.A[1][0] = 0.5; rk4.A[2][1] = 0.5; rk4.A[3][2] = 1.0;
    tsit5.s = 7;
    const double c7[7] = {0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0, 1.0};
    for (int i = 0; i < 7; ++i) tsit5.c[i] = c7[i];
    const double a[7][6] = {
        {0, 0, 0, 0, 0, 0},
        {0.161, 0, 0, 0, 0, 0},
        {-0.008480655492356989, 0.335480655492357, 0, 0, 0, 0},
        {2.897153057105493, -6.359448489975075, 4.3622954328695815, 0, 0, 0},
        {5.325864828439257, -11.748883564062828, 7.4955393428898365, -0.09249506636175525, 0, 0},
        {5.86145544294642, -12.92096931784711, 8.159367898576159, -0.071584973281401, -0.028269050394068383, 0},
        {0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081, 2.324710524099774}};
    for (int i = 0; i < 7; ++i)
      for (int j = 0; j < 6; ++j) tsit5.A[i][j] = a[i][j];
    for (int j = 0; j < 6; ++j) tsit5.b[j] = a[6][j];  // first same as last: b = the last row
    tsit5.b[6] = 0.0;
    init = true;
  }
  return method == WT_ERK_RK4 ? &rk4 : method == WT_ERK_TSIT5 ? &tsit5 : nullptr;
}

// One fixed step of an explicit RK method (general tableau, stage slopes kept
// in ws->erk): stage states y + dt sum_j a_ij k_j, the RHS at the stage time
// (time-dependent backgrounds re-sampled), then y += dt sum_j b_j k_j.
static int step_erk_once(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt,
                         const ErkTableau& T, double eps_ko, const wt::ConsBC& b, int use_metric) {
  const wt::DevMesh& m = ws->mesh->m;
  cudaStream_t s = ctx->stream;
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  char* base = static_cast<char*>(ws->erk);  // the Phi slopes of the T.s stages, then the Pi slopes
  const void* kP[WT_ERK_MAX_STAGES];
  const void* kQ[WT_ERK_MAX_STAGES];
  for (int j = 0; j < T.s; ++j) { kP[j] = base + j * nb; kQ[j] = base + (T.s + j) * nb; }
  int last = T.s - 1;
  while (last > 0 && T.b[last] == 0.0) --last;  // stages past the last nonzero weight do not contribute
  for (int st = 0; st <= last; ++st) {
    const void* inP = Phi;
    const void* inQ = Pi;
    if (st > 0) {
      WT_TRY(lrc(ctx, wt::launch_erk_combine(m.nn, m.precision, dt, Phi, ws->S0, st, kP, T.A[st], s), "RK stage"));
      WT_TRY(lrc(ctx, wt::launch_erk_combine(m.nn, m.precision, dt, Pi, ws->SQ, st, kQ, T.A[st], s), "RK stage"));
      ctx->launches += 2;
      inP = ws->S0;
      inQ = ws->SQ;
    }
    if (coef->td) WT_TRY(coef_resample(ctx, coef, T.c[st] * dt, s));
    WT_TRY(rhs_curved_impl(ctx, ws, coef, inP, inQ, (void*)kP[st], (void*)kQ[st], eps_ko, b, use_metric));
  }
  WT_TRY(lrc(ctx, wt::launch_erk_combine(m.nn, m.precision, dt, Phi, Phi, last + 1, kP, T.b, s), "RK step"));
  WT_TRY(lrc(ctx, wt::launch_erk_combine(m.nn, m.precision, dt, Pi, Pi, last + 1, kQ, T.b, s), "RK step"));
  ctx->launches += 2;
  if (coef->td) {
    WT_TRY(lrc(ctx, wt::launch_advance_time(coef->d_t, dt, s), "background time"));
    ctx->launches += 1;
  }
  return 0;
}

}  // extern "C"

// Capture one step (any stream may be the caller's, including the legacy
// default stream, which cannot be captured): capture and replay on the
// context's own stream, ordered after / before the caller's stream by events.
template <typename F>
static int replay_graph(wt_ctx* ctx, int nsteps, F&& one_step) {
  cudaStream_t user = ctx->stream, own = ctx->own_stream;
  cudaEventRecord(ctx->ord_a, user);
  cudaStreamWaitEvent(own, ctx->ord_a, 0);
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const long long before = ctx->launches;
  ctx->stream = own;
  int rc = 0;
  cudaError_t e;
  {
    wt::NvtxRange nv("graph capture");
    e = cudaStreamBeginCapture(own, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { ctx->stream = user; return cuda_fail(ctx, e, "graph capture"); }
    rc = one_step();
    e = cudaStreamEndCapture(own, &graph);
  }
  ctx->stream = user;
  if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "graph capture");
  e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) { cudaGraphDestroy(graph); return cuda_fail(ctx, e, "graph instantiate"); }
  const long long per = ctx->launches - before;
  ctx->launches = before;
  {
    wt::NvtxRange nv("graph replay");
    for (int i = 0; i < nsteps && e == cudaSuccess; ++i) e = cudaGraphLaunch(exec, own);
  }
  ctx->launches += per * nsteps;
  cudaEventRecord(ctx->ord_b, own);
  cudaStreamWaitEvent(user, ctx->ord_b, 0);
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "graph launch");
}

extern "C" {

int wt_step_rk4_curved(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, int nsteps,
                       double eps_ko, const wt_bc_desc* bc, int use_metric) {
  wt::NvtxRange nvtx_("wt_step_rk4_curved");
  WT_TRY(check_ws(ctx, ws));
  if (!coef || !Phi || !Pi) return fail(ctx, WT_EINVAL, "wt_step_rk4_curved: NULL argument");
  if (nsteps < 0) return fail(ctx, WT_EINVAL, "nsteps must be >= 0");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(ctx, WT_EINVAL, "dt must be positive and finite");
  wt::ConsBC b;
  WT_TRY(make_bc(ctx, bc, use_metric, b));
  WT_TRY(ws_step_buffers(ws));
  {  // the fused stages' second flux buffer (FP64 n = 8 whole-step calls only)
    const wt::DevMesh& m = ws->mesh->m;
    if (m.precision == WT_F64 && m.N == 8 && ws->fused && eps_ko == 0.0)
      WT_TRY(ensure(ws, &ws->F2, 3 * (size_t)wt::n8_padded_field_size(m.Ne) * sizeof(double)));
  }
  if (eps_ko != 0.0) WT_TRY(ensure_mu(ws));
  if (coef->td) WT_TRY(need_setup_geometry(coef->mesh, "wt_step_rk4_curved (time-dependent background)"));
  comp_track(ws, Phi, Pi);
  int rc = 0;
  if (nsteps <= 2) {
    for (int i = 0; i < nsteps && !rc; ++i) rc = step_curved_once(ctx, ws, coef, Phi, Pi, dt, eps_ko, b, use_metric);
  } else {
    // capture one step as a CUDA graph and replay it
    rc = replay_graph(ctx, nsteps,
                      [&]() { return step_curved_once(ctx, ws, coef, Phi, Pi, dt, eps_ko, b, use_metric); });
  }
  if (!rc && coef->td) coef->t += nsteps * dt;  // the device copy was advanced step by step
  return rc;
}

}  // extern "C"

// One half of RK4 stage `stage` on the elements [e0, e1) (e1 < 0: all).
static int stage_curved_range(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt,
                              int stage, int part, long long e0, long long e1, const wt_bc_desc* bc, int use_metric) {
  if (!coef || !Phi || !Pi) return fail(ctx, WT_EINVAL, "wt_rk4_stage_curved: NULL argument");
  if (stage < 0 || stage > 3 || (part != 1 && part != 2))
    return fail(ctx, WT_EINVAL, "wt_rk4_stage_curved: stage must be 0..3 and part 1 or 2");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(ctx, WT_EINVAL, "dt must be positive and finite");
  if (coef->mesh != ws->mesh) return fail(ctx, WT_EINVAL, "coefficients belong to another mesh");
  wt::ConsBC b;
  WT_TRY(make_bc(ctx, bc, use_metric, b));
  WT_TRY(ws_step_buffers(ws));
  if (coef->td) WT_TRY(need_setup_geometry(coef->mesh, "wt_rk4_stage_curved (time-dependent background)"));
  comp_track(ws, Phi, Pi);
  const double toff[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};
  if (coef->td && part == 1) WT_TRY(coef_resample(ctx, coef, toff[stage], ctx->stream));
  WT_TRY(rk4_stage_part(ctx, ws, coef, Phi, Pi, dt, stage, part, b, use_metric, e0, e1));
  if (coef->td && part == 2 && stage == 3) {
    WT_TRY(lrc(ctx, wt::launch_advance_time(coef->d_t, dt, ctx->stream), "background time"));
    ctx->launches += 1;
    coef->t += dt;
  }
  return 0;
}

extern "C" {

int wt_rk4_stage_curved(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, int stage,
                        int part, const wt_bc_desc* bc, int use_metric) {
  wt::NvtxRange nvtx_("wt_rk4_stage_curved");
  WT_TRY(check_ws(ctx, ws));
  return stage_curved_range(ctx, ws, coef, Phi, Pi, dt, stage, part, 0, -1, bc, use_metric);
}

int wt_rk4_stage_curved_layers(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt,
                               int stage, int part, int layer0, int nlayers, const wt_bc_desc* bc, int use_metric) {
  wt::NvtxRange nvtx_("wt_rk4_stage_curved_layers");
  WT_TRY(check_ws(ctx, ws));
  const wt::DevMesh& m = ws->mesh->m;
  if (m.M[2] <= 0 || (long long)m.M[0] * m.M[1] * m.M[2] != m.Ne)
    return fail(ctx, WT_EINVAL, "wt_rk4_stage_curved_layers: the mesh has no element layers (analytic cubes only)");
  if (layer0 < 0 || nlayers < 0 || layer0 + nlayers > m.M[2])
    return fail(ctx, WT_EINVAL, "wt_rk4_stage_curved_layers: layers outside the mesh");
  const long long L = (long long)m.M[0] * m.M[1];
  return stage_curved_range(ctx, ws, coef, Phi, Pi, dt, stage, part, layer0 * L, (layer0 + nlayers) * L, bc,
                            use_metric);
}

int wt_rk4_stage_curved_ko(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, int stage,
                           double eps_ko, const wt_bc_desc* bc, int use_metric) {
  wt::NvtxRange nvtx_("wt_rk4_stage_curved_ko");
  WT_TRY(check_ws(ctx, ws));
  if (!coef || !Phi || !Pi) return fail(ctx, WT_EINVAL, "wt_rk4_stage_curved_ko: NULL argument");
  if (stage < 0 || stage > 3) return fail(ctx, WT_EINVAL, "wt_rk4_stage_curved_ko: stage must be 0..3");
  if (eps_ko == 0.0 || !std::isfinite(eps_ko))
    return fail(ctx, WT_EINVAL, "wt_rk4_stage_curved_ko: eps_ko must be nonzero (eps_ko = 0: wt_rk4_stage_curved)");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(ctx, WT_EINVAL, "dt must be positive and finite");
  if (coef->mesh != ws->mesh) return fail(ctx, WT_EINVAL, "coefficients belong to another mesh");
  wt::ConsBC b;
  WT_TRY(make_bc(ctx, bc, use_metric, b));
  WT_TRY(ws_step_buffers(ws));
  WT_TRY(ws_k_buffers(ws));
  WT_TRY(ensure_mu(ws));
  if (coef->td) WT_TRY(need_setup_geometry(coef->mesh, "wt_rk4_stage_curved_ko (time-dependent background)"));
  comp_track(ws, Phi, Pi);
  const wt::DevMesh& m = ws->mesh->m;
  cudaStream_t s = ctx->stream;
  void* SP[2] = {ws->S0, ws->S1};
  const double toff[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};
  if (coef->td) WT_TRY(coef_resample(ctx, coef, toff[stage], s));
  // the stage of step_curved_once with eps_ko != 0: RHS with dissipation, then both updates
  const void* inP = stage == 0 ? Phi : SP[(stage - 1) % 2];
  const void* inQ = stage == 0 ? Pi : ws->SQ;
  WT_TRY(rhs_curved_impl(ctx, ws, coef, inP, inQ, ws->kP, ws->kQ, eps_ko, b, use_metric));
  WT_TRY(lrc(ctx, wt::launch_rk_update(m.nn, m.precision, stage, dt, Phi, ws->accP, SP[stage % 2], ws->kP, s,
                                       ws->compP), "rk4"));
  WT_TRY(lrc(ctx, wt::launch_rk_update(m.nn, m.precision, stage, dt, Pi, ws->accQ, ws->SQ, ws->kQ, s, ws->compQ),
             "rk4"));
  ctx->launches += 2;
  if (coef->td && stage == 3) {
    WT_TRY(lrc(ctx, wt::launch_advance_time(coef->d_t, dt, s), "background time"));
    ctx->launches += 1;
    coef->t += dt;
  }
  return 0;
}

int wt_halo_state_copy(wt_ctx* ctx, wt_ws* ws, void* Phi, void* Pi, int stage, int layer, int count, void* buf,
                       int pack) {
  wt::NvtxRange nvtx_("wt_halo_state_copy");
  WT_TRY(check_ws(ctx, ws));
  if (!Phi || !Pi || !buf) return fail(ctx, WT_EINVAL, "wt_halo_state_copy: NULL argument");
  const wt::DevMesh& m = ws->mesh->m;
  if (stage < 0 || stage > 3) return fail(ctx, WT_EINVAL, "wt_halo_state_copy: stage must be 0..3");
  if (count < 1 || layer < 0 || layer + count > m.M[2])
    return fail(ctx, WT_EINVAL, "wt_halo_state_copy: layers outside the mesh");
  WT_TRY(ws_step_buffers(ws));
  const size_t es = rsize(m.precision);
  const long long L = (long long)m.M[0] * m.M[1], N3 = (long long)m.N * m.N * m.N;
  // the state the next stage reads: the stage outputs, or the caller's Phi and Pi after stage 3
  char* f[2] = {(char*)(stage < 3 ? (stage % 2 ? ws->S1 : ws->S0) : Phi), (char*)(stage < 3 ? ws->SQ : Pi)};
  const size_t off = (size_t)(layer * L * N3) * es, len = (size_t)(count * L * N3) * es;
  for (int k = 0; k < 2; ++k) {
    char* b = (char*)buf + k * len;
    cudaError_t e = pack ? cudaMemcpyAsync(b, f[k] + off, len, cudaMemcpyDeviceToDevice, ctx->stream)
                         : cudaMemcpyAsync(f[k] + off, b, len, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "wt_halo_state_copy");
  }
  return 0;
}

int wt_halo_size(const wt_ws* ws, long long* values) {
  if (!ws || !values) return WT_EINVAL;
  const wt::DevMesh& m = ws->mesh->m;
  if (!ws->flux_block) return fail(ws->ctx, WT_EINVAL, "wt_halo_size: no fused stage has run on this workspace yet");
  const long long L = (long long)m.M[0] * m.M[1];
  *values = L * ((ws->halo_cp ? 2 : 1) * (long long)m.N * m.N * m.N + 3 * ws->flux_block);
  return 0;
}

int wt_halo_copy(wt_ctx* ctx, wt_ws* ws, void* Phi, int stage, int layer, void* buf, int pack) {
  wt::NvtxRange nvtx_("wt_halo_copy");
  WT_TRY(check_ws(ctx, ws));
  if (!Phi || !buf) return fail(ctx, WT_EINVAL, "wt_halo_copy: NULL argument");
  const wt::DevMesh& m = ws->mesh->m;
  if (stage < 0 || stage > 3) return fail(ctx, WT_EINVAL, "wt_halo_copy: stage must be 0..3");
  if (layer < 0 || layer >= m.M[2]) return fail(ctx, WT_EINVAL, "wt_halo_copy: no such element layer");
  if (!ws->flux_block) return fail(ctx, WT_EINVAL, "wt_halo_copy: no fused stage has run on this workspace yet");
  const size_t es = rsize(m.precision);
  const long long L = (long long)m.M[0] * m.M[1], N3 = (long long)m.N * m.N * m.N, B = ws->flux_block;
  // the Phi the next stage reads (the caller's Phi after stage 3) -- for the
  // compensated FP32 form its high part and its small part -- then the three
  // flux components
  const PhiStage ps = phi_stage(ws, Phi, (stage + 1) % 4, ws->halo_cp != 0);
  std::vector<char*> seg;
  std::vector<size_t> len;
  seg.push_back((char*)ps.in + (size_t)(layer * L * N3) * es);
  len.push_back((size_t)(L * N3) * es);
  if (ws->halo_cp) {
    seg.push_back((char*)ps.phit + (size_t)(layer * L * N3) * es);
    len.push_back((size_t)(L * N3) * es);
  }
  for (int c = 0; c < 3; ++c) {
    seg.push_back((char*)ws->F + (size_t)(c * m.Ne * B + layer * L * B) * es);
    len.push_back((size_t)(L * B) * es);
  }
  size_t off = 0;
  for (size_t k = 0; k < seg.size(); ++k) {
    char* b = (char*)buf + off;
    cudaError_t e = pack ? cudaMemcpyAsync(b, seg[k], len[k], cudaMemcpyDeviceToDevice, ctx->stream)
                         : cudaMemcpyAsync(seg[k], b, len[k], cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "wt_halo_copy");
    off += len[k];
  }
  return 0;
}

int wt_halo_face_size(const wt_ws* ws, long long* values) {
  if (!ws || !values) return WT_EINVAL;
  const wt::DevMesh& m = ws->mesh->m;
  if (!ws->flux_block)
    return fail(ws->ctx, WT_EINVAL, "wt_halo_face_size: no fused stage has run on this workspace yet");
  *values = (long long)m.M[0] * m.M[1] * m.N * m.N * (ws->halo_cp ? 5 : 4);
  return 0;
}

int wt_halo_face_copy(wt_ctx* ctx, wt_ws* ws, void* Phi, int stage, int layer, int face, void* buf, int pack) {
  wt::NvtxRange nvtx_("wt_halo_face_copy");
  WT_TRY(check_ws(ctx, ws));
  if (!Phi || !buf) return fail(ctx, WT_EINVAL, "wt_halo_face_copy: NULL argument");
  const wt::DevMesh& m = ws->mesh->m;
  if (stage < 0 || stage > 3) return fail(ctx, WT_EINVAL, "wt_halo_face_copy: stage must be 0..3");
  if (layer < 0 || layer >= m.M[2]) return fail(ctx, WT_EINVAL, "wt_halo_face_copy: no such element layer");
  if (face != 4 && face != 5) return fail(ctx, WT_EINVAL, "wt_halo_face_copy: face must be 4 (-z) or 5 (+z)");
  if (!ws->flux_block) return fail(ctx, WT_EINVAL, "wt_halo_face_copy: no fused stage has run on this workspace yet");
  // the Phi the next stage reads (compensated FP32 form: its high part and its
  // small part) and the three flux components, on the face plane only
  const PhiStage ps = phi_stage(ws, Phi, (stage + 1) % 4, ws->halo_cp != 0);
  const long long L = (long long)m.M[0] * m.M[1];
  return lrc(ctx, wt::launch_halo_face(m, layer * L, L, face == 5 ? m.N - 1 : 0, (void*)ps.in,
                                       ws->halo_cp ? (void*)ps.phit : nullptr, ws->F, ws->flux_block, ws->flux_lay,
                                       buf, pack, ctx->stream), "wt_halo_face_copy");
}

}  // extern "C"

// nsteps steps of the explicit tableau T (wt_step_erk_curved and _tableau)
static int erk_run(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, int nsteps,
                   const ErkTableau& Tab, double eps_ko, const wt_bc_desc* bc, int use_metric) {
  const ErkTableau* T = &Tab;
  if (!coef || !Phi || !Pi) return fail(ctx, WT_EINVAL, "wt_step_erk_curved: NULL argument");
  if (nsteps < 0) return fail(ctx, WT_EINVAL, "nsteps must be >= 0");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(ctx, WT_EINVAL, "dt must be positive and finite");
  wt::ConsBC b;
  WT_TRY(make_bc(ctx, bc, use_metric, b));
  WT_TRY(ws_step_buffers(ws));
  const wt::DevMesh& m = ws->mesh->m;
  if (ws->erk_stages < T->s) {  // room for this tableau's slopes
    dfree(ctx, ws->erk);
    ws->erk = nullptr;
    ws->erk_stages = 0;
    WT_TRY(dalloc(ctx, &ws->erk, 2 * (size_t)T->s * (size_t)m.nn * rsize(m.precision), nullptr));
    ws->erk_stages = T->s;
  }
  if (eps_ko != 0.0) WT_TRY(ensure_mu(ws));
  if (coef->td) WT_TRY(need_setup_geometry(coef->mesh, "wt_step_erk_curved (time-dependent background)"));
  int rc = 0;
  if (nsteps <= 2) {
    for (int i = 0; i < nsteps && !rc; ++i) rc = step_erk_once(ctx, ws, coef, Phi, Pi, dt, *T, eps_ko, b, use_metric);
  } else {
    rc = replay_graph(ctx, nsteps,
                      [&]() { return step_erk_once(ctx, ws, coef, Phi, Pi, dt, *T, eps_ko, b, use_metric); });
  }
  if (!rc && coef->td) coef->t += nsteps * dt;
  return rc;
}

extern "C" {

int wt_step_erk_curved(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, int nsteps,
                       int method, double eps_ko, const wt_bc_desc* bc, int use_metric) {
  wt::NvtxRange nvtx_("wt_step_erk_curved");
  WT_TRY(check_ws(ctx, ws));
  const ErkTableau* T = erk_tableau(method);
  if (!T) return fail(ctx, WT_EINVAL, "wt_step_erk_curved: unknown method " + std::to_string(method));
  if (method == WT_ERK_RK4)  // the fused low-storage stages
    return wt_step_rk4_curved(ctx, ws, coef, Phi, Pi, dt, nsteps, eps_ko, bc, use_metric);
  return erk_run(ctx, ws, coef, Phi, Pi, dt, nsteps, *T, eps_ko, bc, use_metric);
}

int wt_step_erk_curved_tableau(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt,
                               int nsteps, int stages, const double* c, const double* A, const double* b,
                               double eps_ko, const wt_bc_desc* bc, int use_metric) {
  wt::NvtxRange nvtx_("wt_step_erk_curved_tableau");
  WT_TRY(check_ws(ctx, ws));
  if (stages < 1 || stages > WT_ERK_MAX_STAGES || !c || !A || !b)
    return fail(ctx, WT_EINVAL, "wt_step_erk_curved_tableau: stages must be in 1..16, c, A, b not NULL");
  auto T = std::make_unique<ErkTableau>();
  T->s = stages;
  for (int i = 0; i < stages; ++i) {
    T->c[i] = c[i];
    T->b[i] = b[i];
    if (!std::isfinite(c[i]) || !std::isfinite(b[i]))
      return fail(ctx, WT_EINVAL, "wt_step_erk_curved_tableau: c and b must be finite");
    for (int j = 0; j < stages; ++j) {
      const double a = A[i * stages + j];
      if (!std::isfinite(a) || (j >= i && a != 0.0))
        return fail(ctx, WT_EINVAL, "wt_step_erk_curved_tableau: A must be finite and strictly lower triangular "
                                    "(an explicit method)");
      T->A[i][j] = a;
    }
  }
  return erk_run(ctx, ws, coef, Phi, Pi, dt, nsteps, *T, eps_ko, bc, use_metric);
}

int wt_erk_tableau(int method, int* stages, double* c, double* A, double* b) {
  const ErkTableau* T = erk_tableau(method);
  if (!T || !stages) return WT_EINVAL;
  *stages = T->s;
  for (int i = 0; i < T->s; ++i) {
    if (c) c[i] = T->c[i];
    if (b) b[i] = T->b[i];
    if (A)
      for (int j = 0; j < T->s; ++j) A[i * T->s + j] = T->A[i][j];
  }
  return 0;
}

static int step_sipg_once(wt_ctx* ctx, wt_ws* ws, void* u, void* ut, double dt, const double bv[6], double tau,
                          double R, double eps_ko) {
  const wt::DevMesh& m = ws->mesh->m;
  cudaStream_t s = ctx->stream;
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  for (int st = 0; st < 4; ++st) {
    const void* inU = st == 0 ? u : ws->S0;
    const void* inV = st == 0 ? ut : ws->SQ;
    WT_TRY(wt_rhs_sipg(ctx, ws, inU, inV, ws->kQ, bv, tau, R));
    cudaMemcpyAsync(ws->kP, inV, nb, cudaMemcpyDeviceToDevice, s);
    if (eps_ko != 0.0) {
      const double koT = eps_ko * ws->inv_mu5;
      WT_TRY(lrc(ctx, wt::launch_ko_add(m, ws->kP, inU, koT, s, ws->F), "Kreiss-Oliger"));
      WT_TRY(lrc(ctx, wt::launch_ko_add(m, ws->kQ, inV, koT, s, ws->F), "Kreiss-Oliger"));
      ctx->launches += 6;
    }
    WT_TRY(lrc(ctx, wt::launch_rk_update(m.nn, m.precision, st, dt, u, ws->accP, ws->S0, ws->kP, s), "rk4"));
    WT_TRY(lrc(ctx, wt::launch_rk_update(m.nn, m.precision, st, dt, ut, ws->accQ, ws->SQ, ws->kQ, s), "rk4"));
    ctx->launches += 2;
  }
  return 0;
}

int wt_step_rk4_sipg(wt_ctx* ctx, wt_ws* ws, void* u, void* ut, double dt, int nsteps, const double bdry_values[6],
                     double tau, double sommerfeld_R, double eps_ko) {
  wt::NvtxRange nvtx_("wt_step_rk4_sipg");
  WT_TRY(check_ws(ctx, ws));
  if (!u || !ut || !bdry_values) return fail(ctx, WT_EINVAL, "wt_step_rk4_sipg: NULL argument");
  if (nsteps < 0 || !(dt > 0)) return fail(ctx, WT_EINVAL, "bad nsteps/dt");
  if (!ws->mesh->m.affine) return fail(ctx, WT_ENOTSUP, "SIPG stepping supports affine meshes only");
  WT_TRY(ws_step_buffers(ws));
  WT_TRY(ws_k_buffers(ws));
  WT_TRY(ws_buffers(ws));  // Kreiss-Oliger scratch (allocated before any graph capture)
  if (eps_ko != 0.0) WT_TRY(ensure_mu(ws));
  const wt::DevMesh& m = ws->mesh->m;
  WT_TRY(ensure(ws, &ws->trace, (size_t)6 * m.N * m.N * m.Ne * rsize(m.precision)));
  if (nsteps <= 2) {
    for (int i = 0; i < nsteps; ++i) WT_TRY(step_sipg_once(ctx, ws, u, ut, dt, bdry_values, tau, sommerfeld_R, eps_ko));
    return 0;
  }
  return replay_graph(ctx, nsteps,
                      [&]() { return step_sipg_once(ctx, ws, u, ut, dt, bdry_values, tau, sommerfeld_R, eps_ko); });
}

// ---- device-side diagnostics and snapshots ------------------------------------------
int wt_gather_nodes(wt_ctx* ctx, wt_mesh* mesh, const void* field, const int64_t* nodes, int count,
                    double* host_out) {
  if (!ctx) return WT_EINVAL;
  if (!mesh || !field || (count > 0 && (!nodes || !host_out)) || count < 0)
    return fail(ctx, WT_EINVAL, "wt_gather_nodes: bad argument");
  for (int q = 0; q < count; ++q)
    if (nodes[q] < 0 || nodes[q] >= mesh->m.nn) return fail(ctx, WT_EINVAL, "wt_gather_nodes: node out of range");
  if (count == 0) return 0;
  int64_t* dn = nullptr;
  double* dv = nullptr;
  WT_TRY(dalloc(ctx, &dn, count * sizeof(int64_t), nullptr));
  if (dalloc(ctx, &dv, count * sizeof(double), nullptr)) { dfree(ctx, dn); return WT_ENOMEM; }
  cudaMemcpyAsync(dn, nodes, count * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream);
  int rc = lrc(ctx, wt::launch_gather(mesh->m.precision, count, field, dn, dv, ctx->stream), "gather");
  ctx->launches += 1;
  if (!rc) cudaMemcpyAsync(host_out, dv, count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  dfree(ctx, dn);
  dfree(ctx, dv);
  if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, "gather");
  return rc;
}

namespace {
// Snapshot file: a 64-byte little-endian header, then Phi and Pi as raw
// arrays in the mesh precision, (N,N,N,Ne) node order.
struct SnapHeader {
  char magic[8];        // "WTB2SNP1"
  uint32_t version;     // 1
  uint32_t N;
  uint64_t Ne;
  uint32_t precision;   // WT_F64 / WT_F32
  uint32_t nfields;     // 2: Phi, Pi
  double t;
  uint8_t reserved[24];
};
static_assert(sizeof(SnapHeader) == 64, "snapshot header is 64 bytes");
}  // namespace

int wt_snapshot_save(wt_ctx* ctx, wt_mesh* mesh, const void* Phi, const void* Pi, double t, const char* path) {
  if (!ctx) return WT_EINVAL;
  if (!mesh || !Phi || !Pi || !path) return fail(ctx, WT_EINVAL, "wt_snapshot_save: NULL argument");
  const wt::DevMesh& m = mesh->m;
  SnapHeader hd;
  std::memset(&hd, 0, sizeof(hd));
  std::memcpy(hd.magic, "WTB2SNP1", 8);
  hd.version = 1; hd.N = (uint32_t)m.N; hd.Ne = (uint64_t)m.Ne; hd.precision = (uint32_t)m.precision;
  hd.nfields = 2; hd.t = t;
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  std::vector<char> buf(nb);
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return fail(ctx, WT_EINVAL, std::string("wt_snapshot_save: cannot open ") + path);
  int rc = std::fwrite(&hd, sizeof(hd), 1, fp) == 1 ? 0 : WT_EINVAL;
  for (const void* f : {Phi, Pi}) {
    if (rc) break;
    cudaMemcpyAsync(buf.data(), f, nb, cudaMemcpyDeviceToHost, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "wt_snapshot_save"); break; }
    if (std::fwrite(buf.data(), 1, nb, fp) != nb) rc = fail(ctx, WT_EINVAL, "wt_snapshot_save: write failed");
  }
  if (std::fclose(fp) != 0 && !rc) rc = fail(ctx, WT_EINVAL, "wt_snapshot_save: close failed");
  return rc;
}

int wt_snapshot_load(wt_ctx* ctx, wt_mesh* mesh, void* Phi, void* Pi, double* t, const char* path) {
  if (!ctx) return WT_EINVAL;
  if (!mesh || !Phi || !Pi || !path) return fail(ctx, WT_EINVAL, "wt_snapshot_load: NULL argument");
  const wt::DevMesh& m = mesh->m;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(ctx, WT_EINVAL, std::string("wt_snapshot_load: cannot open ") + path);
  SnapHeader hd;
  int rc = 0;
  if (std::fread(&hd, sizeof(hd), 1, fp) != 1 || std::memcmp(hd.magic, "WTB2SNP1", 8) != 0 || hd.version != 1)
    rc = fail(ctx, WT_EINVAL, "wt_snapshot_load: not a snapshot file");
  else if (hd.N != (uint32_t)m.N || hd.Ne != (uint64_t)m.Ne || hd.precision != (uint32_t)m.precision ||
           hd.nfields != 2)
    rc = fail(ctx, WT_EINVAL, "wt_snapshot_load: snapshot does not match the mesh (N, Ne or precision)");
  const size_t nb = (size_t)m.nn * rsize(m.precision);
  std::vector<char> buf(rc ? 0 : nb);
  for (void* f : {Phi, Pi}) {
    if (rc) break;
    if (std::fread(buf.data(), 1, nb, fp) != nb) { rc = fail(ctx, WT_EINVAL, "wt_snapshot_load: file too short"); break; }
    cudaMemcpyAsync(f, buf.data(), nb, cudaMemcpyHostToDevice, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "wt_snapshot_load");
  }
  std::fclose(fp);
  if (!rc && t) *t = hd.t;
  return rc;
}

}  // extern "C"

// host-buffer evolve for state words of `prec` (the mesh precision)
static int evolve_host(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi_host, void* Pi_host, int prec,
                       const char* name, double dt, int steps_per_sample, int nsamples, double eps_ko,
                       const wt_bc_desc* bc, int use_metric, double* energy) {
  WT_TRY(check_ws(ctx, ws));
  if (!coef || !Phi_host || !Pi_host) return fail(ctx, WT_EINVAL, std::string(name) + ": NULL argument");
  if (ws->mesh->m.precision != prec)
    return fail(ctx, WT_ENOTSUP,
                std::string(name) + (prec == WT_F64 ? " takes FP64 host buffers; use an FP64 mesh"
                                                    : " takes FP32 host buffers; use an FP32 mesh"));
  if (steps_per_sample < 1 || nsamples < 1) return fail(ctx, WT_EINVAL, "steps_per_sample, nsamples must be >= 1");
  const wt::DevMesh& m = ws->mesh->m;
  const size_t nb = (size_t)m.nn * rsize(prec);
  // device state (dP, dQ) and a staging copy of the last sample (sP, sQ), kept
  // in the workspace between calls: each sample is copied device to device on
  // the compute stream and from the staging pair to the host on two copy
  // streams, so the device-to-host copy of sample s overlaps the steps of
  // sample s + 1.  Nothing in the loop waits on the host: the energies go to a
  // device array (per-block partial sums, summed on the host at the end in the
  // order wt_energy sums them) and the non-finite flag is read every 16
  // samples and at the end.
  for (void*& p : ws->evo) WT_TRY(ensure(ws, &p, nb));
  const size_t elen = energy ? (size_t)nsamples * ctx->nblocks : 0;
  if (elen > ws->evoE_len) {
    dfree(ctx, ws->evoE);
    ws->evoE = nullptr;
    ws->evoE_len = 0;
    WT_TRY(dalloc(ctx, &ws->evoE, elen * sizeof(double), nullptr));
    ws->evoE_len = elen;
  }
  void *dP = ws->evo[0], *dQ = ws->evo[1], *sP = ws->evo[2], *sQ = ws->evo[3];
  // one copy stream per field, so that the two device-to-host copies can run on
  // separate copy engines at the same time
  cudaStream_t cs = nullptr, cs2 = nullptr;
  cudaEvent_t staged = nullptr, copied = nullptr, copied2 = nullptr;
  int rc = 0;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&cs2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&staged, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&copied, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&copied2, cudaEventDisableTiming) != cudaSuccess)
    rc = fail(ctx, WT_ECUDA, std::string(name) + ": stream or event creation failed");
  if (!rc) {
    cudaMemcpyAsync(dP, Phi_host, nb, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dQ, Pi_host, nb, cudaMemcpyHostToDevice, ctx->stream);
  }
  auto check_finite = [&]() -> int {
    int bad = 0;
    int r = wt_ctx_nonfinite(ctx, &bad);
    if (!r && bad) r = fail(ctx, WT_ENONFINITE, "state became non-finite during evolution");
    return r;
  };
  for (int sidx = 0; sidx < nsamples && !rc; ++sidx) {
    rc = wt_step_rk4_curved(ctx, ws, coef, dP, dQ, dt, steps_per_sample, eps_ko, bc, use_metric);
    if (rc) break;
    if (energy) {
      rc = energy_partials(ctx, ws, coef, dP, dQ, use_metric);
      if (rc) break;
      cudaMemcpyAsync(ws->evoE + (size_t)sidx * ctx->nblocks, ctx->d_partial, ctx->nblocks * sizeof(double),
                      cudaMemcpyDeviceToDevice, ctx->stream);
    }
    if (sidx % 16 == 15 && (rc = check_finite())) break;
    if (sidx > 0) {  // the previous sample has left the staging pair
      cudaStreamWaitEvent(ctx->stream, copied, 0);
      cudaStreamWaitEvent(ctx->stream, copied2, 0);
    }
    cudaMemcpyAsync(sP, dP, nb, cudaMemcpyDeviceToDevice, ctx->stream);
    cudaMemcpyAsync(sQ, dQ, nb, cudaMemcpyDeviceToDevice, ctx->stream);
    cudaEventRecord(staged, ctx->stream);
    cudaStreamWaitEvent(cs, staged, 0);
    cudaStreamWaitEvent(cs2, staged, 0);
    cudaMemcpyAsync(Phi_host, sP, nb, cudaMemcpyDeviceToHost, cs);
    cudaMemcpyAsync(Pi_host, sQ, nb, cudaMemcpyDeviceToHost, cs2);
    cudaEventRecord(copied, cs);
    cudaEventRecord(copied2, cs2);
  }
  for (cudaStream_t c : {cs, cs2})
    if (c) {
      cudaError_t e = cudaStreamSynchronize(c);
      if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, name);
    }
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, name);
  if (!rc) rc = check_finite();
  if (!rc && energy) {
    std::vector<double> h(elen);
    e = cudaMemcpy(h.data(), ws->evoE, elen * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, name);
    for (int sidx = 0; sidx < nsamples && !rc; ++sidx) {
      double sum = 0.0;
      for (int k = 0; k < ctx->nblocks; ++k) sum += h[(size_t)sidx * ctx->nblocks + k];
      energy[sidx] = sum;
    }
  }
  if (staged) cudaEventDestroy(staged);
  if (copied) cudaEventDestroy(copied);
  if (copied2) cudaEventDestroy(copied2);
  if (cs) cudaStreamDestroy(cs);
  if (cs2) cudaStreamDestroy(cs2);
  return rc;
}

extern "C" {

int wt_evolve_curved_host(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, double* Phi_host, double* Pi_host, double dt,
                          int steps_per_sample, int nsamples, double eps_ko, const wt_bc_desc* bc, int use_metric,
                          double* energy) {
  wt::NvtxRange nvtx_("wt_evolve_curved_host");
  return evolve_host(ctx, ws, coef, Phi_host, Pi_host, WT_F64, "wt_evolve_curved_host", dt, steps_per_sample,
                     nsamples, eps_ko, bc, use_metric, energy);
}

int wt_evolve_curved_host_f32(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, float* Phi_host, float* Pi_host, double dt,
                              int steps_per_sample, int nsamples, double eps_ko, const wt_bc_desc* bc, int use_metric,
                              double* energy) {
  wt::NvtxRange nvtx_("wt_evolve_curved_host_f32");
  return evolve_host(ctx, ws, coef, Phi_host, Pi_host, WT_F32, "wt_evolve_curved_host_f32", dt, steps_per_sample,
                     nsamples, eps_ko, bc, use_metric, energy);
}

}  // extern "C"

// ---- batches of independent solves -----------------------------------------------------
// Many solves of uneven element counts and orders advance together: solves are
// grouped by (n, precision, kernel path); each group is one work list of
// (solve, element) tiles over which one persistent (n = 8) or element-parallel
// kernel launch runs per RK4 stage, every tile reading its solve's parameter
// block (meshes, coefficients, state, scratch, dt).  One RK4 step of all
// groups is captured once as a CUDA graph and replayed; adding or removing a
// solve only rebuilds the work lists, parameter blocks and graph.
struct wt_batch {
  wt_ctx* ctx = nullptr;
  struct Member {
    bool active = false;
    wt_ws* ws = nullptr;
    const wt_coef* coef = nullptr;
    void* Phi = nullptr;
    void* Pi = nullptr;
    double dt = 0.0;
    wt::ConsBC bc;
    bool cp = false;  // the member's stages run the compensated FP32 form
  };
  std::vector<Member> members;
  struct Group {
    int N = 0, precision = 0, fp32_form = 0;
    bool n8 = false;
    std::vector<int> slots;
    long long ntiles = 0;
    int2* d_tiles = nullptr;
    char* d_k1 = nullptr;
    char* d_k2 = nullptr;
    std::vector<char> h_k1, h_k2;  // [stage][solve] parameter blocks
    size_t k1sz = 0, k2sz = 0;
    int epb_variant = 0;
  };
  std::vector<Group> groups;
  bool dirty = true;
  int autotune = 1;
  int force_var[2] = {-1, -1};  // wt_batch_set_variant: fixed launch variants of K1 / K2 (-1: tuned)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long launches_per_step = 0;
  // one stream per group inside the captured step: the groups share no buffer,
  // so their launches form parallel branches of the graph and run side by side
  std::vector<cudaStream_t> gstreams;
  std::vector<cudaEvent_t> gjoin;
  cudaEvent_t fork = nullptr;
};

namespace {

void batch_release(wt_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  for (cudaStream_t st : b->gstreams) cudaStreamDestroy(st);
  for (cudaEvent_t ev : b->gjoin) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  b->gstreams.clear();
  b->gjoin.clear();
  b->fork = nullptr;
  for (auto& g : b->groups) {
    dfree(b->ctx, g.d_tiles);
    dfree(b->ctx, g.d_k1);
    dfree(b->ctx, g.d_k2);
  }
  b->groups.clear();
}

// the per-solve inputs of RK4 stage st (the same buffers step_curved_once uses)
wt::SolveStage batch_stage(wt_batch* b, const wt_batch::Member& mb, int st) {
  wt_ws* ws = mb.ws;
  wt::SolveStage ss;
  ss.m = &ws->mesh->m;
  ss.c = &mb.coef->c;
  void* SP[2] = {ws->S0, ws->S1};
  const PhiStage ps = phi_stage(ws, mb.Phi, st, mb.cp);
  ss.Phi = ps.in;
  ss.Pi = st == 0 ? mb.Pi : ws->SQ;
  ss.F = ws->F;
  ss.bbuf = ws->bbuf;
  ss.bc = mb.bc;
  ss.rkP.on = ss.rkQ.on = 1;
  ss.rkP.stage = ss.rkQ.stage = st;
  ss.rkP.dt = ss.rkQ.dt = mb.dt;
  ss.rkP.y = mb.Phi; ss.rkP.acc = ws->accP; ss.rkP.out = SP[st % 2]; ss.rkP.comp = ws->compP;
  ss.rkP.phit = ps.phit; ss.rkP.hcopy = ps.hcopy;
  ss.rkQ.y = mb.Pi; ss.rkQ.acc = ws->accQ; ss.rkQ.out = ws->SQ; ss.rkQ.comp = ws->compQ;
  ss.rkP.nonfinite = ss.rkQ.nonfinite = st == 3 ? b->ctx->d_flag : nullptr;
  return ss;
}

int batch_launch(wt_batch* b, wt_batch::Group& g, int which, int st, cudaStream_t s) {
  const size_t ns = g.slots.size();
  if (g.n8) {
    const size_t sz = which == 1 ? g.k1sz : g.k2sz;
    const char* h = (which == 1 ? g.h_k1.data() : g.h_k2.data()) + st * ns * sz;
    const char* d = (which == 1 ? g.d_k1 : g.d_k2) + st * ns * sz;
    return wt::launch_cons_n8_batch(which, g.precision, g.fp32_form, h, d, g.d_tiles, g.ntiles, s);
  }
  const size_t sz = which == 1 ? g.k1sz : g.k2sz;
  const char* d = (which == 1 ? g.d_k1 : g.d_k2) + st * ns * sz;
  const int cp = g.precision == WT_F32 && g.fp32_form == WT_FP32_COMPENSATED;
  const int variant = (g.epb_variant >> (2 * (which - 1))) & 3;  // bits 0-1: K1, bits 2-3: K2
  return wt::launch_cons_gen_batch(which, g.N, g.precision, variant, cp, d, g.d_tiles, g.ntiles, s);
}

// Members of a group with a time-dependent background: re-sample it at the stage
// time before the group's K1 of stage st (as step_curved_once does), and after
// stage 3 advance the time it holds by the member's dt.
int batch_group_td(wt_batch* b, const wt_batch::Group& g, int st, bool after, cudaStream_t s) {
  for (int slot : g.slots) {
    const auto& mb = b->members[slot];
    if (!mb.coef->td) continue;
    if (!after) {
      const double toff[4] = {0.0, 0.5 * mb.dt, 0.5 * mb.dt, mb.dt};
      WT_TRY(coef_resample(b->ctx, mb.coef, toff[st], s));
    } else {
      WT_TRY(lrc(b->ctx, wt::launch_advance_time(mb.coef->d_t, mb.dt, s), "background time"));
      b->ctx->launches += 1;
    }
  }
  return 0;
}

int batch_one_step(wt_batch* b, cudaStream_t s) {
  if (b->groups.size() <= 1 || b->gstreams.size() != b->groups.size()) {
    for (int st = 0; st < 4; ++st) {
      for (auto& g : b->groups) {
        WT_TRY(batch_group_td(b, g, st, false, s));
        WT_TRY(lrc(b->ctx, batch_launch(b, g, 1, st, s), "batch K1"));
      }
      for (auto& g : b->groups) WT_TRY(lrc(b->ctx, batch_launch(b, g, 2, st, s), "batch K2"));
    }
    for (auto& g : b->groups) WT_TRY(batch_group_td(b, g, 3, true, s));
    return 0;
  }
  // fork: each group's eight launches in order on its own stream, joined at the end
  if (cudaEventRecord(b->fork, s) != cudaSuccess) return fail(b->ctx, WT_ECUDA, "batch fork");
  for (size_t k = 0; k < b->groups.size(); ++k) {
    cudaStream_t gs = b->gstreams[k];
    cudaStreamWaitEvent(gs, b->fork, 0);
    for (int st = 0; st < 4; ++st) {
      WT_TRY(batch_group_td(b, b->groups[k], st, false, gs));
      WT_TRY(lrc(b->ctx, batch_launch(b, b->groups[k], 1, st, gs), "batch K1"));
      WT_TRY(lrc(b->ctx, batch_launch(b, b->groups[k], 2, st, gs), "batch K2"));
    }
    WT_TRY(batch_group_td(b, b->groups[k], 3, true, gs));
    cudaEventRecord(b->gjoin[k], gs);
    cudaStreamWaitEvent(s, b->gjoin[k], 0);
  }
  return 0;
}

// Time K1 and K2 of stage 0 of a generic group in each launch variant -- the
// generic kernels at two elements-per-CTA counts and, for n = 4 and 6, the
// pipelined kernels -- and keep the fastest of each (stage 0 writes only stage
// scratch, never the solution state).  epb_variant: bits 0-1 K1's choice, bits
// 2-3 K2's.  A variant fixed by wt_batch_set_variant is kept untimed.
int batch_tune_group(wt_batch* b, wt_batch::Group& g) {
  cudaStream_t s = b->ctx->own_stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int choice = 0, rc = 0;
  const int nvar = wt::cons_gen_pipe_available(g.N) ? 3 : 2;
  for (int which = 1; which <= 2 && !rc; ++which) {
    const int sh = 2 * (which - 1);
    if (b->force_var[which - 1] >= 0) {
      choice |= (b->force_var[which - 1] < nvar ? b->force_var[which - 1] : 0) << sh;
      continue;
    }
    float best = 1e30f;
    int best_v = 0;
    for (int v = 0; v < nvar && !rc; ++v) {
      g.epb_variant = (choice & ~(3 << sh)) | (v << sh);
      for (int rep = 0; rep < 2 && !rc; ++rep) rc = batch_launch(b, g, which, 0, s);  // warm up
      cudaEventRecord(e0, s);
      for (int rep = 0; rep < 4 && !rc; ++rep) rc = batch_launch(b, g, which, 0, s);
      cudaEventRecord(e1, s);
      if (rc) break;
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) { best = ms; best_v = v; }
    }
    choice |= best_v << sh;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return lrc(b->ctx, rc, "batch autotune");
  g.epb_variant = choice;
  return 0;
}

int batch_rebuild(wt_batch* b) {
  wt_ctx* ctx = b->ctx;
  batch_release(b);
  // group the active members
  for (int slot = 0; slot < (int)b->members.size(); ++slot) {
    const auto& mb = b->members[slot];
    if (!mb.active) continue;
    auto& mbw = b->members[slot];
    const wt::DevMesh& m = mb.ws->mesh->m;
    mbw.cp = false;
    const wt::SolveStage s0 = batch_stage(b, mb, 0);
    const bool n8 = wt::cons_n8_path(m, mb.coef->c, 1, mb.bc, s0.rkP, s0.rkQ,
                                     {mb.Phi, mb.Pi, mb.ws->F, mb.ws->S0, mb.ws->S1, mb.ws->SQ});
    mbw.cp = compensated(m, n8);
    const int form = m.precision == WT_F32 ? m.fp32_form : 0;
    wt_batch::Group* g = nullptr;
    for (auto& x : b->groups)
      if (x.N == m.N && x.precision == m.precision && x.n8 == n8 && x.fp32_form == form) g = &x;
    if (!g) {
      b->groups.emplace_back();
      g = &b->groups.back();
      g->N = m.N; g->precision = m.precision; g->n8 = n8; g->fp32_form = form;
    }
    g->slots.push_back(slot);
  }
  for (auto& g : b->groups) {
    const size_t ns = g.slots.size();
    std::vector<int2> tiles;
    for (size_t i = 0; i < ns; ++i) {
      const long long Ne = b->members[g.slots[i]].ws->mesh->m.Ne;
      for (long long e = 0; e < Ne; ++e) tiles.push_back(make_int2((int)i, (int)e));
    }
    g.ntiles = (long long)tiles.size();
    g.k1sz = g.n8 ? wt::cons_n8_param_size(g.precision, 1) : wt::cons_gen_param_size(g.precision, 1);
    g.k2sz = g.n8 ? wt::cons_n8_param_size(g.precision, 2) : wt::cons_gen_param_size(g.precision, 2);
    g.h_k1.assign(4 * ns * g.k1sz, 0);
    g.h_k2.assign(4 * ns * g.k2sz, 0);
    for (int st = 0; st < 4; ++st)
      for (size_t i = 0; i < ns; ++i) {
        const wt::SolveStage ss = batch_stage(b, b->members[g.slots[i]], st);
        void* p1 = g.h_k1.data() + (st * ns + i) * g.k1sz;
        void* p2 = g.h_k2.data() + (st * ns + i) * g.k2sz;
        if (g.n8) {
          wt::cons_n8_fill_params(1, ss, ctx->d_flag, p1);
          wt::cons_n8_fill_params(2, ss, ctx->d_flag, p2);
        } else {
          wt::cons_gen_fill_params(1, ss, ss.rkP.nonfinite, p1);
          wt::cons_gen_fill_params(2, ss, ss.rkQ.nonfinite, p2);
        }
      }
    WT_TRY(dalloc(ctx, &g.d_tiles, tiles.size() * sizeof(int2), nullptr));
    WT_TRY(dalloc(ctx, &g.d_k1, g.h_k1.size(), nullptr));
    WT_TRY(dalloc(ctx, &g.d_k2, g.h_k2.size(), nullptr));
    cudaMemcpy(g.d_tiles, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice);
    cudaMemcpy(g.d_k1, g.h_k1.data(), g.h_k1.size(), cudaMemcpyHostToDevice);
    cudaError_t e = cudaMemcpy(g.d_k2, g.h_k2.data(), g.h_k2.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch parameter upload");
  }
  if (b->autotune) {
    cudaStreamSynchronize(ctx->stream);  // the tuning launches run on the context's own stream
    for (auto& g : b->groups)
      if (!g.n8) WT_TRY(batch_tune_group(b, g));
  } else {
    for (auto& g : b->groups) {  // untuned: the fixed variants, else the default one
      const int nvar = wt::cons_gen_pipe_available(g.N) ? 3 : 2;
      int v[2];
      for (int w = 0; w < 2; ++w) v[w] = b->force_var[w] >= 0 && b->force_var[w] < nvar ? b->force_var[w] : 0;
      g.epb_variant = g.n8 ? 0 : v[0] | (v[1] << 2);
    }
  }
  // capture one RK4 step of every group (several groups: parallel branches)
  cudaStream_t own = ctx->own_stream;
  if (b->groups.size() > 1) {
    if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
      return fail(ctx, WT_ECUDA, "batch: event creation failed");
    for (size_t k = 0; k < b->groups.size(); ++k) {
      cudaStream_t gs = nullptr;
      cudaEvent_t ev = nullptr;
      if (cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
        return fail(ctx, WT_ECUDA, "batch: stream or event creation failed");
      b->gstreams.push_back(gs);
      b->gjoin.push_back(ev);
    }
  }
  cudaError_t e = cudaStreamBeginCapture(own, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph capture");
  int rc = batch_one_step(b, own);
  e = cudaStreamEndCapture(own, &b->graph);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph capture");
  e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph instantiate");
  b->launches_per_step = 8 * (long long)b->groups.size();
  for (const auto& mb : b->members)
    if (mb.active && mb.coef->td) b->launches_per_step += 9;  // 4 re-samplings of 2 launches + the time step
  b->dirty = false;
  return 0;
}

}  // namespace

extern "C" {

int wt_batch_create(wt_ctx* ctx, wt_batch** out) {
  if (!ctx) return WT_EINVAL;
  if (!out) return fail(ctx, WT_EINVAL, "wt_batch_create: NULL argument");
  auto* b = new wt_batch();
  b->ctx = ctx;
  *out = b;
  return 0;
}

int wt_batch_destroy(wt_batch* b) {
  if (!b) return WT_EINVAL;
  cudaStreamSynchronize(b->ctx->own_stream);
  cudaStreamSynchronize(b->ctx->stream);
  batch_release(b);
  delete b;
  return 0;
}

int wt_batch_add(wt_batch* b, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, const wt_bc_desc* bc,
                 int* slot) {
  if (!b) return WT_EINVAL;
  wt_ctx* ctx = b->ctx;
  WT_TRY(check_ws(ctx, ws));
  if (!coef || !Phi || !Pi || !slot) return fail(ctx, WT_EINVAL, "wt_batch_add: NULL argument");
  if (coef->mesh != ws->mesh) return fail(ctx, WT_EINVAL, "coefficients belong to another mesh");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(ctx, WT_EINVAL, "dt must be positive and finite");
  // a time-dependent background is re-sampled at every stage inside the batch's graph
  if (coef->td) WT_TRY(need_setup_geometry(coef->mesh, "wt_batch_add (time-dependent background)"));
  wt_batch::Member mb;
  WT_TRY(make_bc(ctx, bc, 1, mb.bc));
  WT_TRY(ws_step_buffers(ws));
  comp_track(ws, Phi, Pi);
  mb.active = true;
  mb.ws = ws;
  mb.coef = coef;
  mb.Phi = Phi;
  mb.Pi = Pi;
  mb.dt = dt;
  for (const auto& x : b->members)
    if (x.active && x.ws == ws) return fail(ctx, WT_EINVAL, "a workspace can serve one batch member at a time");
  int s = -1;
  for (int i = 0; i < (int)b->members.size(); ++i)
    if (!b->members[i].active) { s = i; break; }
  if (s < 0) { s = (int)b->members.size(); b->members.emplace_back(); }
  b->members[s] = mb;
  b->dirty = true;
  *slot = s;
  return 0;
}

int wt_batch_remove(wt_batch* b, int slot) {
  if (!b) return WT_EINVAL;
  if (slot < 0 || slot >= (int)b->members.size() || !b->members[slot].active)
    return fail(b->ctx, WT_EINVAL, "wt_batch_remove: no such member");
  b->members[slot].active = false;
  b->dirty = true;
  return 0;
}

int wt_batch_set_autotune(wt_batch* b, int on) {
  if (!b) return WT_EINVAL;
  b->autotune = on ? 1 : 0;
  b->dirty = true;
  return 0;
}

int wt_batch_set_variant(wt_batch* b, int k1, int k2) {
  if (!b) return WT_EINVAL;
  if (k1 < -1 || k1 > 2 || k2 < -1 || k2 > 2)
    return fail(b->ctx, WT_EINVAL, "wt_batch_set_variant: variants are -1 (tuned), 0, 1 or 2");
  b->force_var[0] = k1;
  b->force_var[1] = k2;
  b->dirty = true;
  return 0;
}

int wt_batch_step(wt_batch* b, int nsteps) {
  wt::NvtxRange nvtx_("wt_batch_step");
  if (!b) return WT_EINVAL;
  wt_ctx* ctx = b->ctx;
  if (nsteps < 0) return fail(ctx, WT_EINVAL, "nsteps must be >= 0");
  // re-sampling a time-dependent background reads the set-up coordinates: refuse
  // before any launch if a member's mesh released them after it joined
  for (const auto& mb : b->members)
    if (mb.active && mb.coef->td) WT_TRY(need_setup_geometry(mb.coef->mesh, "wt_batch_step (time-dependent background)"));
  if (b->dirty) WT_TRY(batch_rebuild(b));
  if (nsteps == 0 || b->groups.empty()) return 0;
  cudaStream_t user = ctx->stream, own = ctx->own_stream;
  cudaEventRecord(ctx->ord_a, user);
  cudaStreamWaitEvent(own, ctx->ord_a, 0);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < nsteps && e == cudaSuccess; ++i) e = cudaGraphLaunch(b->exec, own);
  cudaEventRecord(ctx->ord_b, own);
  cudaStreamWaitEvent(user, ctx->ord_b, 0);
  ctx->launches += b->launches_per_step * nsteps;
  for (const auto& mb : b->members)  // the host copy of a time-dependent background's time
    if (mb.active && mb.coef->td) mb.coef->t += nsteps * mb.dt;
  return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "batch graph launch");
}

int wt_batch_info(wt_batch* b, int* nsolves, long long* nodes, int* ngroups) {
  if (!b) return WT_EINVAL;
  int n = 0;
  long long nn = 0;
  for (const auto& mb : b->members)
    if (mb.active) { ++n; nn += mb.ws->mesh->m.nn; }
  if (nsolves) *nsolves = n;
  if (nodes) *nodes = nn;
  if (ngroups) {
    if (b->dirty) WT_TRY(batch_rebuild(b));
    *ngroups = (int)b->groups.size();
  }
  return 0;
}

int wt_batch_group_info(wt_batch* b, int group, int* N, int* precision, int* n8_path, int* epb_variant,
                        long long* tiles) {
  if (!b) return WT_EINVAL;
  if (b->dirty) WT_TRY(batch_rebuild(b));
  if (group < 0 || group >= (int)b->groups.size()) return fail(b->ctx, WT_EINVAL, "no such group");
  const auto& g = b->groups[group];
  if (N) *N = g.N;
  if (precision) *precision = g.precision;
  if (n8_path) *n8_path = g.n8 ? 1 : 0;
  if (epb_variant) *epb_variant = g.epb_variant;
  if (tiles) *tiles = g.ntiles;
  return 0;
}

}  // extern "C"

// ---- allocation-free RHS -------------------------------------------------------------
// Some callers cannot allocate device memory at the moment they evaluate the
// RHS: a host runtime that owns the device memory pool of the process (and
// frees nothing it did not hand out), code that runs inside a memory budget
// fixed before the time loop starts, or a loop that cannot afford the
// device-wide synchronisation cudaMalloc and cudaFree may cause.  For them
// wt_rhs_curved_noalloc evaluates the same conservative RHS as wt_rhs_curved
// without a workspace: the two scratch buffers the RHS needs (the flux F
// between the gradient and the divergence pass, and the boundary-face
// increments) live in one fixed array of device memory that the library
// declares at file scope.  Every GPU that loads the library holds the array
// (8.4 MiB) until the process exits.
//
// The array's name is only a host-side stand-in for the symbol; its device
// address is looked up by cudaGetSymbolAddress, with the context's device
// current, on the first call made through each wt_ctx, and that address is
// what the kernels receive.  Keeping it per context (not per device for the
// whole process) means a context created after cudaDeviceReset looks the
// address up again instead of reusing one from before the reset.
//
// Every call uses the same array and it keeps the contents of the last call.
// Nothing in it has to start at zero: the gradient pass writes every flux
// entry and every boundary-face entry that the divergence pass of the same
// call reads.  Calls whose kernels overlap on the GPU (different streams, or
// different contexts on one device, without ordering between them) race on the
// array and produce wrong results.
namespace {

constexpr long long kNoallocMaxNodes = WT_NOALLOC_MAX_NODES;
// flux: three components of max(nodes, padded n=8 element blocks) doubles
constexpr long long kNoallocFluxDoubles = (kNoallocMaxNodes / 512) * 544;
constexpr long long kNoallocBdryDoubles = WT_NOALLOC_MAX_BOUNDARY_NODES;
constexpr long long kNoallocDoubles = 3 * kNoallocFluxDoubles + kNoallocBdryDoubles;

static __device__ __align__(256) double wt_noalloc_scratch[kNoallocDoubles];

// Device address of the scratch array for ctx (set-up on the context's first call).
int noalloc_scratch(wt_ctx* ctx, double** out) {
  if (!ctx->noalloc_scratch) {
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "wt_rhs_curved_noalloc set-up (cudaGetDevice)");
    e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "wt_rhs_curved_noalloc set-up (cudaSetDevice)");
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, wt_noalloc_scratch);
    cudaSetDevice(prev);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return cuda_fail(ctx, e, "wt_rhs_curved_noalloc set-up (cudaGetSymbolAddress)");
    }
    ctx->noalloc_scratch = (double*)p;
  }
  *out = ctx->noalloc_scratch;
  return 0;
}

}  // namespace

extern "C" {

int wt_rhs_curved_noalloc(wt_ctx* ctx, const wt_coef* coef, const void* Phi, const void* Pi, void* Phidot,
                          void* Pidot, double eps_ko, double mu, const wt_bc_desc* bc, int use_metric) {
  wt::NvtxRange nvtx_("wt_rhs_curved_noalloc");
  if (!ctx) return WT_EINVAL;
  if (!coef || !Phi || !Pi || !Phidot || !Pidot) return fail(ctx, WT_EINVAL, "wt_rhs_curved_noalloc: NULL argument");
  if (coef->ctx != ctx) return fail(ctx, WT_EINVAL, "coefficients belong to another context");
  const wt::DevMesh& m = coef->mesh->m;
  if ((long long)m.nn > kNoallocMaxNodes)
    return fail(ctx, WT_EINVAL, "wt_rhs_curved_noalloc: mesh has " + std::to_string((long long)m.nn) +
                                    " nodes; the fixed scratch array holds at most " +
                                    std::to_string(kNoallocMaxNodes) + " (use wt_rhs_curved)");
  const long long bnodes = (long long)m.nbf * m.N * m.N;
  if (bnodes > kNoallocBdryDoubles)
    return fail(ctx, WT_EINVAL, "wt_rhs_curved_noalloc: mesh has " + std::to_string(bnodes) +
                                    " boundary-face nodes; the fixed scratch array holds at most " +
                                    std::to_string(kNoallocBdryDoubles) + " (use wt_rhs_curved)");
  if (eps_ko != 0.0 && !(mu > 0.0 && std::isfinite(mu)))
    return fail(ctx, WT_EINVAL, "wt_rhs_curved_noalloc: mu must be positive and finite when eps_ko != 0 "
                                "(pass wt_workspace_mu of a workspace on the same mesh)");
  wt::ConsBC b;
  WT_TRY(make_bc(ctx, bc, use_metric, b));
  double* scratch = nullptr;
  WT_TRY(noalloc_scratch(ctx, &scratch));
  void* F = scratch;
  void* bbuf = scratch + 3 * kNoallocFluxDoubles;
  wt::RKStage rk;
  const bool n8 = wt::cons_n8_path(m, coef->c, use_metric, b, rk, rk, {Phi, Pi, F, Phidot, Pidot});
  WT_TRY(lrc(ctx, wt::launch_cons_k1(m, coef->c, Phi, Pi, F, Phidot, bbuf, nullptr, use_metric, b, rk, ctx->stream,
                                     n8), "rhs K1"));
  WT_TRY(lrc(ctx, wt::launch_cons_k2(m, F, Pidot, bbuf, use_metric, b, rk, nullptr, ctx->stream, n8), "rhs K2"));
  ctx->launches += 2;
  if (eps_ko != 0.0) {
    const double koT = eps_ko * std::pow(1.0 / mu, 5);
    // the flux scratch is free once K2 has run
    WT_TRY(lrc(ctx, wt::launch_ko_add(m, Phidot, Phi, koT, ctx->stream, F), "Kreiss-Oliger"));
    WT_TRY(lrc(ctx, wt::launch_ko_add(m, Pidot, Pi, koT, ctx->stream, F), "Kreiss-Oliger"));
    ctx->launches += 6;
  }
  return 0;
}

}  // extern "C"
