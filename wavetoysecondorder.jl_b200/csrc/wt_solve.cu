// wt_solve.cu -- evolve3d in one call (host code).
//
// A client of the public C ABI, like the server: wt_evolve3d does the set-up of
// _evolve3d_conservative (src/evolve.jl:1149-1263: mesh, element operators,
// geometry and metric terms, coefficients, workspace, initial data), its time
// step (src/evolve.jl:1209-1213) and its sample loop (src/evolve.jl:1311-1352),
// with the integration on the device (wt_step_rk4_curved) and the per-sample
// diagnostics as device reductions.
#include "wavetoy_b200.h"
#include "wt_common.cuh"

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

namespace {

bool finite_pos(double v) { return std::isfinite(v) && v > 0; }

std::string check_desc(const wt_solve_desc* d) {
  if (!d) return "NULL descriptor";
  if (d->mesh_kind < 0 || d->mesh_kind > WT_MESH_RADIAL_SHELL) return "mesh_kind must be 0 or a WT_MESH_* kind";
  if (d->precision != WT_F64 && d->precision != WT_F32) return "precision must be WT_F64 or WT_F32";
  const int N = d->mesh_kind == 0 ? d->mesh.N : d->patch.N;
  if (N < 2 || N > WT_MAXN) return "N must be in 2..8";
  if (d->mesh_kind == 0 && (d->mesh.M[0] < 1 || d->mesh.M[1] < 1 || d->mesh.M[2] < 1)) return "M must be >= 1";
  if (d->mesh_kind != 0 && d->patch.M < 1) return "M must be >= 1";
  if (d->nic < 0 || d->nic > WT_SERVE_MAX_IC) return "nic must be in 0..WT_SERVE_MAX_IC";
  if (d->bc.gPhi || d->bc.gPi || d->bc.gDx || d->bc.gDy || d->bc.gDz) return "boundary data pointers must be NULL";
  if (!std::isfinite(d->t0) || !std::isfinite(d->t1) || d->t1 < d->t0) return "t0 <= t1, both finite";
  if (d->nt < 1) return "nt must be >= 1";
  if (!finite_pos(d->cfl) || !finite_pos(d->max_speed)) return "cfl and max_speed must be positive and finite";
  if (!std::isfinite(d->eps_ko) || d->eps_ko < 0) return "eps_ko must be >= 0 and finite";
  return "";
}

// The sampling of the reference's loop in the time type T: for each sample
// time ts[n] of range(t0, t1, nt), step while t < ts[n]; a step past t1 is
// shortened to end on t1.
template <typename T>
int schedule_t(double t0d, double t1d, int nt, double dtd, long long* steps, double* dt_last, double* ts_actual) {
  const T t0 = (T)t0d, t1 = (T)t1d, dt = (T)dtd;
  if (!(dt > 0)) return WT_EINVAL;
  if ((t1d - t0d) / dtd > 1e9) return WT_EINVAL;  // more steps than any solve takes (a host loop of them)
  T t = t0, last = dt;
  for (int n = 0; n < nt; ++n) {
    // the range's end points are exact; the points between them rounded once to T
    const T target = n == 0 ? t0 : n == nt - 1 ? t1 : (T)(t0d + (t1d - t0d) * (double)n / (double)(nt - 1));
    long long k = 0;
    while (t < target) {
      if (t + dt > t1) {
        last = t1 - t;
        t = t1;
      } else {
        t = t + dt;
      }
      ++k;
    }
    if (steps) steps[n] = k;
    if (ts_actual) ts_actual[n] = (double)t;
  }
  if (dt_last) *dt_last = (double)last;
  return 0;
}

// device objects of one call, released in reverse order
struct Solve {
  wt_ctx* ctx = nullptr;
  wt_mesh* mesh = nullptr;
  wt_coef* coef = nullptr;
  wt_ws* ws = nullptr;
  void* state = nullptr;  // Phi, Pi
  void* ref = nullptr;    // the exact solution at a sample time
  ~Solve() {
    if (ctx) wt_ctx_synchronize(ctx);
    if (ref) wt::ctx_free(ctx, ref);
    if (state) wt::ctx_free(ctx, state);
    if (ws) wt_workspace_destroy(ws);
    if (coef) wt_coef_destroy(coef);
    if (mesh) wt_mesh_destroy(mesh);
  }
};

#define WT_TRY_SOLVE(x)      \
  do {                       \
    int _rc = (x);           \
    if (_rc != 0) return _rc; \
  } while (0)

}  // namespace

extern "C" {

int wt_solve_desc_check(const wt_solve_desc* desc, char* msg, int msglen) {
  const std::string why = check_desc(desc);
  if (msg && msglen > 0) std::snprintf(msg, (size_t)msglen, "%s", why.c_str());
  return why.empty() ? 0 : WT_EINVAL;
}

int wt_solve_nodes(const wt_solve_desc* d, long long* nodes) {
  if (!nodes || !check_desc(d).empty()) return WT_EINVAL;
  if (d->mesh_kind == 0) {
    const long long N = d->mesh.N;
    *nodes = N * N * N * d->mesh.M[0] * d->mesh.M[1] * d->mesh.M[2];
  } else {
    const long long N = d->patch.N, M = d->patch.M;
    const long long per = d->mesh_kind == WT_MESH_CUBED_CUBE ? 7 : d->mesh_kind == WT_MESH_INFLATED_CUBE ? 13 : 6;
    *nodes = per * M * M * M * N * N * N;
  }
  return 0;
}

int wt_solve_schedule(double t0, double t1, int nt, double dt, int precision, long long* steps, double* dt_last,
                      double* ts_actual) {
  if (nt < 1 || !std::isfinite(t0) || !std::isfinite(t1) || t1 < t0 || !finite_pos(dt)) return WT_EINVAL;
  return precision == WT_F32 ? schedule_t<float>(t0, t1, nt, dt, steps, dt_last, ts_actual)
                             : schedule_t<double>(t0, t1, nt, dt, steps, dt_last, ts_actual);
}

int wt_slice_select(const double* xyz, long long nodes, double y, double z, double atol, long long capacity,
                    long long* node_out, double* xs_out, long long* count) {
  if (!xyz || nodes < 0 || !count || capacity < 0 || !(atol > 0)) return WT_EINVAL;
  std::vector<long long> idx;
  std::vector<double> xs;
  for (long long n = 0; n < nodes; ++n) {  // storage order: node i fastest, then j, k, element
    const double* p = xyz + 3 * n;
    if (!(std::fabs(p[1] - y) < atol && std::fabs(p[2] - z) < atol)) continue;
    bool isnew = true;
    for (double x0 : xs)
      if (std::fabs(x0 - p[0]) < atol) { isnew = false; break; }
    if (!isnew) continue;
    idx.push_back(n);
    xs.push_back(p[0]);
  }
  std::vector<size_t> perm(xs.size());
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) { return xs[a] < xs[b]; });
  *count = (long long)xs.size();
  for (size_t q = 0; q < perm.size() && (long long)q < capacity; ++q) {
    if (node_out) node_out[q] = idx[perm[q]];
    if (xs_out) xs_out[q] = xs[perm[q]];
  }
  return 0;
}

int wt_evolve3d(wt_ctx* ctx, const wt_solve_desc* d, void* Phi_host, void* Pi_host, double* ts_actual,
                double* energy, double* l2, wt_solve_slice* slice, wt_solve_info* info) {
  if (!ctx) return WT_EINVAL;
  wt::NvtxRange nv("wt_evolve3d");
  const std::string why = check_desc(d);
  if (!why.empty()) return wt::ctx_fail(ctx, WT_EINVAL, "wt_evolve3d: " + why);
  if (!Phi_host || !Pi_host) return wt::ctx_fail(ctx, WT_EINVAL, "wt_evolve3d: NULL state buffer");
  Solve S;
  S.ctx = ctx;
  // set-up (src/evolve.jl:1174-1196)
  if (d->mesh_kind == 0) {
    wt_mesh_desc md = d->mesh;
    md.precision = d->precision;
    WT_TRY_SOLVE(wt_mesh_create(ctx, &md, &S.mesh));
  } else {
    wt_patch_desc pd = d->patch;
    pd.kind = d->mesh_kind;
    pd.precision = d->precision;
    WT_TRY_SOLVE(wt_mesh_create_patches(ctx, &pd, &S.mesh));
  }
  int N = 0, prec = 0;
  long long Ne = 0;
  WT_TRY_SOLVE(wt_mesh_info(S.mesh, &N, &Ne, &prec));
  const long long nn = (long long)N * N * N * Ne;
  const size_t fb = (size_t)nn * (prec == WT_F64 ? sizeof(double) : sizeof(float));
  WT_TRY_SOLVE(wt_background_set(ctx, S.mesh, &d->bg, &S.coef));
  const bool td = d->bg.kind == WT_BG_GAUGE_WAVE || d->bg.kind == WT_BG_SINE_SHIFT;
  if (td) WT_TRY_SOLVE(wt_coef_set_time(ctx, S.coef, d->t0));
  WT_TRY_SOLVE(wt_workspace_create(ctx, S.mesh, &S.ws));
  WT_TRY_SOLVE(wt::ctx_alloc(ctx, &S.state, 2 * fb));
  if (d->ic_exact) WT_TRY_SOLVE(wt::ctx_alloc(ctx, &S.ref, fb));
  void* Phi = S.state;
  void* Pi = (char*)S.state + fb;
  const double* icp = d->nic ? d->ic : nullptr;
  WT_TRY_SOLVE(wt_initial_state(ctx, S.ws, d->ic_kind, icp, d->nic, d->t0, Phi, Pi));
  // the step (src/evolve.jl:1209-1213), in the solve's precision
  double dx = 0, mu = 0;
  WT_TRY_SOLVE(wt_mesh_min_spacing(S.mesh, &dx));
  double dt;
  if (prec == WT_F32)
    dt = (double)((float)d->cfl * (float)dx / (float)d->max_speed);
  else
    dt = d->cfl * dx / d->max_speed;
  if (d->eps_ko != 0) {
    WT_TRY_SOLVE(wt_workspace_mu(S.ws, &mu));
    const double lim = prec == WT_F32 ? (double)(1.4f / ((float)d->eps_ko * (float)mu)) : 1.4 / (d->eps_ko * mu);
    dt = std::fmin(dt, lim);
  }
  // the 1-D slice (src/evolve.jl:1322-1334): atol = sqrt(eps(T)), the mid-plane by default
  std::vector<int64_t> snodes;
  if (slice) {
    if (slice->capacity < 0 || (slice->capacity > 0 && (!slice->xs || !slice->Phi || !slice->Pi)))
      return wt::ctx_fail(ctx, WT_EINVAL, "wt_evolve3d: slice buffers missing for its capacity");
    const double mid = d->mesh_kind == 0 ? 0.5 * (d->mesh.x0 + d->mesh.x1) : 0.0;  // patch meshes are centred
    const double ys = std::isnan(slice->y) ? mid : slice->y, zs = std::isnan(slice->z) ? mid : slice->z;
    const double atol = prec == WT_F32 ? (double)std::sqrt(FLT_EPSILON) : std::sqrt(DBL_EPSILON);
    std::vector<double> xyz(3 * (size_t)nn);
    WT_TRY_SOLVE(wt_mesh_get(S.mesh, "coords", xyz.data()));
    std::vector<long long> sel((size_t)std::max<long long>(slice->capacity, 0));
    WT_TRY_SOLVE(wt_slice_select(xyz.data(), nn, ys, zs, atol, slice->capacity, sel.data(), slice->xs,
                                 &slice->count));
    if (slice->nodes)
      for (long long q = 0; q < std::min(slice->count, slice->capacity); ++q) slice->nodes[q] = sel[q];
    if (slice->count <= slice->capacity) snodes.assign(sel.begin(), sel.begin() + slice->count);
  }
  // no boundary conditions (bc3d = nothing, e.g. a periodic mesh) when every kind is 0
  bool any_kind = false;
  for (int f = 0; f < 6; ++f) any_kind = any_kind || d->bc.kinds[f] != 0;
  const wt_bc_desc* bc = any_kind ? &d->bc : nullptr;
  // the sample loop (src/evolve.jl:1311-1352)
  std::vector<long long> steps(d->nt);
  std::vector<double> ts(d->nt);
  double dt_last = dt;
  if (wt_solve_schedule(d->t0, d->t1, d->nt, dt, prec, steps.data(), &dt_last, ts.data()))
    return wt::ctx_fail(ctx, WT_EINVAL, "wt_evolve3d: (t1 - t0) / dt is too large");
  int last_sample = -1;  // the sample in which the final step is taken
  long long total = 0;
  for (int n = 0; n < d->nt; ++n)
    if (steps[n] > 0) last_sample = n;
  for (int n = 0; n < d->nt; ++n) {
    long long k = steps[n];
    const bool short_last = n == last_sample && dt_last != dt;
    if (short_last) --k;
    while (k > 0) {
      const int chunk = (int)(k < (1 << 30) ? k : (1 << 30));
      WT_TRY_SOLVE(wt_step_rk4_curved(ctx, S.ws, S.coef, Phi, Pi, dt, chunk, d->eps_ko, bc, d->use_metric));
      k -= chunk;
    }
    if (short_last)
      WT_TRY_SOLVE(wt_step_rk4_curved(ctx, S.ws, S.coef, Phi, Pi, dt_last, 1, d->eps_ko, bc, d->use_metric));
    total += steps[n];
    int bad = 0;
    WT_TRY_SOLVE(wt_ctx_nonfinite(ctx, &bad));  // the reference's all(isfinite, ...) per sample
    if (bad) return wt::ctx_fail(ctx, WT_ENONFINITE, "wt_evolve3d: the state became non-finite before sample " +
                                                         std::to_string(n));
    if (ts_actual) ts_actual[n] = ts[n];
    if (energy) WT_TRY_SOLVE(wt_energy(ctx, S.ws, S.coef, Phi, Pi, d->use_metric, &energy[n]));
    if (!snodes.empty()) {
      const int cnt = (int)snodes.size();
      WT_TRY_SOLVE(wt_gather_nodes(ctx, S.mesh, Phi, snodes.data(), cnt, slice->Phi + n * slice->capacity));
      WT_TRY_SOLVE(wt_gather_nodes(ctx, S.mesh, Pi, snodes.data(), cnt, slice->Pi + n * slice->capacity));
    }
    if (l2) {
      if (d->ic_exact) WT_TRY_SOLVE(wt_initial_data(ctx, S.mesh, d->ic_kind, icp, d->nic, ts[n], S.ref, nullptr));
      WT_TRY_SOLVE(wt_l2_diff(ctx, S.ws, Phi, d->ic_exact ? S.ref : nullptr, d->use_metric, &l2[n]));
    }
  }
  void* st = nullptr;
  WT_TRY_SOLVE(wt_ctx_get_stream(ctx, &st));
  cudaMemcpyAsync(Phi_host, Phi, fb, cudaMemcpyDeviceToHost, (cudaStream_t)st);
  cudaMemcpyAsync(Pi_host, Pi, fb, cudaMemcpyDeviceToHost, (cudaStream_t)st);
  const cudaError_t e = cudaStreamSynchronize((cudaStream_t)st);
  if (e != cudaSuccess) return wt::ctx_fail(ctx, WT_ECUDA, std::string("wt_evolve3d: ") + cudaGetErrorString(e));
  if (info) {
    info->dt = dt;
    info->dx = dx;
    info->mu = mu;
    info->steps = total;
  }
  return 0;
}

}  // extern "C"
