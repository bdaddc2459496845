// wt_serve.cu -- serving a stream of solve requests over one batch (host code).
//
// No counterpart in the reference, whose evolve3d (src/evolve.jl:1149-1358) runs
// one solve per call.  The server is a client of the public C ABI: admission
// builds a request's mesh, coefficients, workspace and state with wt_mesh_create,
// wt_background_set, wt_workspace_create and wt_initial_data (the set-up
// evolve3d does, src/evolve.jl:1174-1263), adds it to a wt_batch, and the batch
// advances every running request together (work-list kernels, one CUDA graph
// per RK4 step).  The scheduling rounds are described in include/wavetoy_b200.h.
#include "wavetoy_b200.h"
#include "wt_common.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

// device bytes per node of a running request (set-up geometry released): streamed
// coefficients and metric, workspace and state, with the allocator's rounding
int bytes_per_node(int precision, int n) {
  if (precision == WT_F64) return n == 8 ? 520 : 480;
  return n == 8 ? 340 : 300;  // FP32: with the compensated form's split metric terms and Phi copy
}
constexpr int kSetupBytesPerNode = 272;  // FP64 set-up geometry: held while a request is built, and
                                          // while it runs if its background is time-dependent

struct Req {
  wt_serve_request q{};
  int precision = WT_F64;
  long long nodes = 0;
  double cost = 0, service = 0, work = 0;
  // admitted
  wt_mesh* mesh = nullptr;
  wt_coef* coef = nullptr;
  wt_ws* ws = nullptr;
  void* state = nullptr;  // Phi then Pi, nodes values each
  int slot = -1, left = 0;
  double dt = 0, admitted = 0, finished = 0;
  bool finished_flag = false;
  int status = WT_REQ_WAITING;
  // preemption: the host checkpoint of the state (wt_state_checkpoint_save) and
  // the background time it was taken at; resumed from on the next admission
  std::vector<char> ckpt;
  double t_ckpt = 0;
  int preemptions = 0;
};

int form_of(const wt_serve_desc& d, const wt_serve_request& q) {
  if (d.precision != WT_SERVE_AUTO) return d.precision;
  return q.steps <= d.auto_fp32_max_steps ? WT_F32 : WT_F64;
}

long long nodes_of(const wt_serve_request& q) {
  const long long N = q.mesh.N;
  return (long long)q.mesh.M[0] * q.mesh.M[1] * q.mesh.M[2] * N * N * N;
}

size_t esize(int precision) { return precision == WT_F64 ? sizeof(double) : sizeof(float); }

// the admission order: a stable sort of the waiting requests by the policy's key
void order_queue(int order, double now, std::vector<int>& idx, const std::vector<double>& arrival,
                 const std::vector<double>& service, const std::vector<double>& work) {
  auto by = [&](auto key) {
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return key(a) < key(b); });
  };
  if (order == WT_SERVE_HRRN)
    by([&](int k) { return std::make_pair(-(now - arrival[k] + service[k]) / service[k], arrival[k]); });
  else if (order == WT_SERVE_SJF)
    by([&](int k) { return std::make_pair(work[k], arrival[k]); });
  else
    by([&](int k) { return arrival[k]; });
}

int check_desc(const wt_serve_desc* d) {
  if (!d) return -1;
  if (!(d->hbm_budget > 0) || d->tick < 1 || d->max_active < 0 || d->fill_nodes < 0) return -1;
  if (d->order < WT_SERVE_HRRN || d->order > WT_SERVE_FIFO) return -1;
  if (d->precision != WT_F64 && d->precision != WT_F32 && d->precision != WT_SERVE_AUTO) return -1;
  if (d->fp32_form < WT_FP32_CUDA_CORES || d->fp32_form > WT_FP32_COMPENSATED) return -1;
  if (d->preempt != 0 && d->preempt != 1) return -1;
  return 0;
}

// why a request is not servable, or empty
std::string check_request(const wt_serve_request* q) {
  if (!q) return "NULL request";
  if (!std::isfinite(q->arrival)) return "arrival must be finite";
  if (q->mesh.N < 2 || q->mesh.N > WT_MAXN) return "N must be in 2..8";
  if (q->mesh.M[0] < 1 || q->mesh.M[1] < 1 || q->mesh.M[2] < 1) return "M must be >= 1";
  if (q->steps < 1) return "steps must be >= 1";
  if (!(q->cfl > 0) || !(q->max_speed > 0) || !std::isfinite(q->cfl) || !std::isfinite(q->max_speed))
    return "cfl and max_speed must be positive and finite";
  if (q->nic < 0 || q->nic > WT_SERVE_MAX_IC) return "nic must be in 0..WT_SERVE_MAX_IC";
  if (q->bc.gPhi || q->bc.gPi || q->bc.gDx || q->bc.gDy || q->bc.gDz) return "boundary data pointers must be NULL";
  return "";
}

// whether a request of `cost` bytes could start with `u` bytes used and `na` requests
// running on `run` nodes, under desc's limits
bool fits_desc(const wt_serve_desc& d, double cost, double u, int na, long long run) {
  if (u + cost > d.hbm_budget) return false;
  if (d.max_active > 0 && na >= d.max_active) return false;
  if (d.fill_nodes > 0 && na > 0 && run >= d.fill_nodes) return false;
  return true;
}

// The victims of preemptive admission for a head request (head_work = nodes x steps
// left): the running requests never preempted before with at least twice its remaining
// work, most work first, as many as it takes to make room -- none if even all of them
// do not.  Indices into the running lists.
std::vector<int> choose_victims(const wt_serve_desc& d, double used, const std::vector<long long>& nodes,
                                const std::vector<double>& work, const std::vector<double>& cost,
                                const std::vector<int>& preemptions, double head_cost, double head_work) {
  std::vector<int> cand;
  for (size_t k = 0; k < nodes.size(); ++k)
    if (preemptions[k] == 0 && work[k] >= 2.0 * head_work) cand.push_back((int)k);
  std::stable_sort(cand.begin(), cand.end(), [&](int a, int b) { return work[a] > work[b]; });
  double u = used;
  int na = (int)nodes.size();
  long long run = 0;
  for (long long v : nodes) run += v;
  size_t n = 0;
  while (!fits_desc(d, head_cost, u, na, run) && n < cand.size()) {
    u -= cost[cand[n]];
    na -= 1;
    run -= nodes[cand[n]];
    ++n;
  }
  if (!fits_desc(d, head_cost, u, na, run)) return {};
  cand.resize(n);
  return cand;
}

#define WT_TRY_SERVE(x)      \
  do {                       \
    int _rc = (x);           \
    if (_rc != 0) return _rc; \
  } while (0)

}  // namespace

struct wt_server {
  wt_ctx* ctx = nullptr;
  wt_serve_desc d{};
  wt_batch* batch = nullptr;
  Clock::time_point t0;
  std::vector<Req> reqs;     // by rid
  std::vector<int> pending;  // not yet arrived, by (arrival, rid)
  std::vector<int> queue;    // arrived, waiting for admission
  std::vector<int> active;   // running, in admission order
  double used = 0, peak = 0;
  int done = 0, cancelled = 0;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

  // the admission keys of a request with `steps` left: work and estimated service time
  void estimate(Req& r, int steps) const {
    r.work = (double)r.nodes * steps;
    r.service = 2.0 * r.work / (r.precision == WT_F64 ? d.rate_f64 : d.rate_f32) + 0.05;
  }

  void release(Req& r, bool keep_state) {
    if (r.ws) wt_workspace_destroy(r.ws);
    if (r.coef) wt_coef_destroy(r.coef);
    if (r.mesh) wt_mesh_destroy(r.mesh);
    r.ws = nullptr;
    r.coef = nullptr;
    r.mesh = nullptr;
    if (!keep_state && r.state) {
      wt::ctx_free(ctx, r.state);
      r.state = nullptr;
    }
  }

  // build request r on the device and add it to the batch
  int admit(Req& r) {
    wt::NvtxRange nv("wt_serve admit");
    wt_mesh_desc md = r.q.mesh;
    md.precision = r.precision;
    int rc = wt_mesh_create(ctx, &md, &r.mesh);
    if (!rc && r.precision == WT_F32) rc = wt_mesh_set_fp32_form(r.mesh, d.fp32_form);
    if (!rc) rc = wt_background_set(ctx, r.mesh, &r.q.bg, &r.coef);
    if (!rc) rc = wt_workspace_create(ctx, r.mesh, &r.ws);
    const size_t fb = (size_t)r.nodes * esize(r.precision);
    if (!rc) rc = wt::ctx_alloc(ctx, &r.state, 2 * fb);
    void* Phi = r.state;
    void* Pi = r.state ? (void*)((char*)r.state + fb) : nullptr;
    const bool resume = !r.ckpt.empty();
    // (u, u_t) in FP64; an FP32 request keeps the low parts in its workspace
    if (!rc && !resume)
      rc = wt_initial_state(ctx, r.ws, r.q.ic_kind, r.q.nic ? r.q.ic : nullptr, r.q.nic, 0.0, Phi, Pi);
    if (!rc && resume) rc = wt_state_checkpoint_load(ctx, r.ws, Phi, Pi, r.ckpt.data(), (long long)r.ckpt.size());
    double h = 0;
    if (!rc) rc = wt_mesh_min_spacing(r.mesh, &h);
    if (!rc) {
      r.dt = r.q.cfl * h / r.q.max_speed;
      // a time-dependent background is re-sampled on the mesh every stage: keep its geometry
      const bool td = r.q.bg.kind == WT_BG_GAUGE_WAVE || r.q.bg.kind == WT_BG_SINE_SHIFT;
      if (!td) rc = wt_mesh_release_setup_geometry(r.mesh);
      else if (resume) rc = wt_coef_set_time(ctx, r.coef, r.t_ckpt);
    }
    if (!rc) rc = wt_batch_add(batch, r.ws, r.coef, Phi, Pi, r.dt, &r.q.bc, &r.slot);
    if (rc) {
      release(r, false);
      return rc;
    }
    if (!resume) r.left = r.q.steps;
    r.ckpt.clear();
    r.ckpt.shrink_to_fit();
    r.status = WT_REQ_RUNNING;
    return 0;
  }

  // take running request rid out of the batch and release its device memory
  int leave_batch(int rid, bool keep_state) {
    Req& r = reqs[rid];
    const int rc = wt_batch_remove(batch, r.slot);
    if (rc) return rc;
    release(r, keep_state);
    used -= r.cost;
    active.erase(std::find(active.begin(), active.end(), rid));
    return 0;
  }

  // whether request r could start with `u` bytes used, `na` requests running on `run` nodes
  bool fits(const Req& r, double u, int na, long long run) const { return fits_desc(d, r.cost, u, na, run); }
  long long running_nodes() const {
    long long run = 0;
    for (int k : active) run += reqs[k].nodes;
    return run;
  }

  // preemptive admission for the queue head r: the running requests with at least twice
  // its remaining work, most work first, if preempting them lets r start
  int make_room(const Req& r) {
    std::vector<long long> nodes;
    std::vector<double> work, cost;
    std::vector<int> pre;
    for (int k : active) {
      nodes.push_back(reqs[k].nodes);
      work.push_back((double)reqs[k].nodes * reqs[k].left);
      cost.push_back(reqs[k].cost);
      pre.push_back(reqs[k].preemptions);
    }
    const std::vector<int> running = active;  // preempt() edits active
    for (int k : choose_victims(d, used, nodes, work, cost, pre, r.cost, (double)r.nodes * r.left))
      WT_TRY_SERVE(preempt(running[k]));
    return 0;
  }

  int preempt(int rid) {
    Req& r = reqs[rid];
    long long nb = 0;
    int rc = wt_state_checkpoint_size(r.ws, &nb);
    if (rc) return rc;
    std::vector<char> ck((size_t)nb);
    const size_t fb = (size_t)r.nodes * esize(r.precision);
    void* Phi = r.state;
    void* Pi = (char*)r.state + fb;
    rc = wt_state_checkpoint_save(ctx, r.ws, Phi, Pi, ck.data(), nb);  // synchronises: the steps so far are done
    if (!rc && (r.q.bg.kind == WT_BG_GAUGE_WAVE || r.q.bg.kind == WT_BG_SINE_SHIFT))
      rc = wt_coef_get_time(r.coef, &r.t_ckpt);
    if (!rc) rc = leave_batch(rid, false);
    if (rc) return rc;
    r.ckpt.swap(ck);
    r.status = WT_REQ_PREEMPTED;
    r.preemptions += 1;
    estimate(r, r.left);
    queue.push_back(rid);  // ordered with the others at the next round
    return 0;
  }

  int cancel(int rid) {
    Req& r = reqs[rid];
    if (r.status == WT_REQ_RUNNING) {
      WT_TRY_SERVE(wt_ctx_synchronize(ctx));
      WT_TRY_SERVE(leave_batch(rid, false));
    } else {
      pending.erase(std::remove(pending.begin(), pending.end(), rid), pending.end());
      queue.erase(std::remove(queue.begin(), queue.end(), rid), queue.end());
      r.ckpt.clear();
      r.ckpt.shrink_to_fit();
    }
    r.status = WT_REQ_CANCELLED;
    ++cancelled;
    return 0;
  }

  int poll(int* nfin) {
    wt::NvtxRange nv("wt_serve_poll");
    int fin = 0;
    const double t = now();
    while (!pending.empty() && reqs[pending.front()].q.arrival <= t) {
      queue.push_back(pending.front());
      pending.erase(pending.begin());
    }
    if (queue.size() > 1) {
      std::vector<double> a(queue.size()), sv(queue.size()), w(queue.size());
      for (size_t k = 0; k < queue.size(); ++k) {
        const Req& r = reqs[queue[k]];
        a[k] = r.q.arrival;
        sv[k] = r.service;
        w[k] = r.work;
      }
      std::vector<int> idx(queue.size());
      std::iota(idx.begin(), idx.end(), 0);
      order_queue(d.order, t, idx, a, sv, w);
      std::vector<int> q2(queue.size());
      for (size_t k = 0; k < idx.size(); ++k) q2[k] = queue[idx[k]];
      queue.swap(q2);
    }
    // admission from the head of the queue
    while (!queue.empty()) {
      Req& r = reqs[queue.front()];
      if (d.preempt && !fits(r, used, (int)active.size(), running_nodes())) WT_TRY_SERVE(make_room(r));
      if (!fits(r, used, (int)active.size(), running_nodes())) break;
      used += r.cost;
      peak = std::max(peak, used);
      const int rid = queue.front();
      const int rc = admit(r);
      if (rc) {  // the request stays at the head of the queue; a later round retries it
        used -= r.cost;
        return rc;
      }
      queue.erase(queue.begin());
      r.admitted = now();
      active.push_back(rid);
    }
    if (active.empty()) {
      if (!pending.empty()) {
        const double wait = std::min(0.01, reqs[pending.front()].q.arrival - now());
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
      }
      if (nfin) *nfin = 0;
      return 0;
    }
    int k = d.tick;
    for (int rid : active) k = std::min(k, reqs[rid].left);
    int rc = wt_batch_step(batch, k);
    if (!rc) rc = wt_ctx_synchronize(ctx);
    if (rc) return rc;
    const double t_done = now();
    std::vector<int> still;
    for (int rid : active) {
      Req& r = reqs[rid];
      r.left -= k;
      if (r.left > 0) {
        still.push_back(rid);
        continue;
      }
      rc = wt_batch_remove(batch, r.slot);
      if (rc) return rc;
      r.finished = t_done;
      r.finished_flag = true;
      r.status = WT_REQ_FINISHED;
      release(r, d.keep_results != 0);
      used -= r.cost;
      ++done;
      ++fin;
    }
    active.swap(still);
    if (nfin) *nfin = fin;
    return 0;
  }
};

extern "C" {

int wt_serve_create(wt_ctx* ctx, const wt_serve_desc* desc, wt_server** out) {
  if (!ctx || !out) return WT_EINVAL;
  *out = nullptr;
  if (check_desc(desc))
    return wt::ctx_fail(ctx, WT_EINVAL, "wt_serve_create: bad descriptor (budget > 0, tick >= 1, "
                                        "max_active >= 0, fill_nodes >= 0, order, precision, fp32_form, preempt 0 or 1)");
  auto* s = new wt_server();
  s->ctx = ctx;
  s->d = *desc;
  if (!(s->d.rate_f64 > 0)) s->d.rate_f64 = 3e9;
  if (!(s->d.rate_f32 > 0)) s->d.rate_f32 = 6e9;
  const int rc = wt_batch_create(ctx, &s->batch);
  if (rc) {
    delete s;
    return rc;
  }
  s->t0 = Clock::now();
  *out = s;
  return 0;
}

int wt_serve_destroy(wt_server* s) {
  if (!s) return WT_EINVAL;
  wt_ctx_synchronize(s->ctx);
  if (s->batch) wt_batch_destroy(s->batch);
  for (auto& r : s->reqs) s->release(r, false);
  delete s;
  return 0;
}

int wt_serve_cost(const wt_serve_desc* desc, const wt_serve_request* req, double* bytes, int* precision) {
  if (check_desc(desc) || !req || !check_request(req).empty()) return WT_EINVAL;
  const int p = form_of(*desc, *req);
  if (bytes) *bytes = (double)nodes_of(*req) * (bytes_per_node(p, req->mesh.N) + kSetupBytesPerNode);
  if (precision) *precision = p;
  return 0;
}

int wt_serve_submit(wt_server* s, const wt_serve_request* req, int* rid) {
  if (!s) return WT_EINVAL;
  const std::string why = check_request(req);
  if (!why.empty()) return wt::ctx_fail(s->ctx, WT_EINVAL, "wt_serve_submit: " + why);
  Req r;
  r.q = *req;
  r.precision = form_of(s->d, *req);
  r.nodes = nodes_of(*req);
  r.cost = (double)r.nodes * (bytes_per_node(r.precision, req->mesh.N) + kSetupBytesPerNode);
  if (r.cost > s->d.hbm_budget)
    return wt::ctx_fail(s->ctx, WT_EINVAL, "wt_serve_submit: the request (" + std::to_string(r.nodes) +
                                               " nodes) does not fit the HBM budget");
  r.left = req->steps;
  s->estimate(r, req->steps);
  const int id = (int)s->reqs.size();
  s->reqs.push_back(r);
  // pending stays ordered by (arrival, rid)
  auto it = std::upper_bound(s->pending.begin(), s->pending.end(), id, [&](int a, int b) {
    return s->reqs[a].q.arrival < s->reqs[b].q.arrival;
  });
  s->pending.insert(it, id);
  if (rid) *rid = id;
  return 0;
}

int wt_serve_poll(wt_server* s, int* finished) {
  if (!s) return WT_EINVAL;
  return s->poll(finished);
}

int wt_serve_run(wt_server* s) {
  if (!s) return WT_EINVAL;
  while (!s->pending.empty() || !s->queue.empty() || !s->active.empty()) {
    const int rc = s->poll(nullptr);
    if (rc) return rc;
  }
  int bad = 0;
  const int rc = wt_ctx_nonfinite(s->ctx, &bad);
  if (rc) return rc;
  if (bad) return wt::ctx_fail(s->ctx, WT_ENONFINITE, "wt_serve_run: a served solve became non-finite");
  return 0;
}

int wt_serve_get_result(const wt_server* s, int rid, wt_serve_result* out) {
  if (!s || !out) return WT_EINVAL;
  if (rid < 0 || rid >= (int)s->reqs.size() || !s->reqs[rid].finished_flag)
    return wt::ctx_fail(s->ctx, WT_EINVAL, "wt_serve_get_result: request " + std::to_string(rid) + " has not finished");
  const Req& r = s->reqs[rid];
  out->precision = r.precision;
  out->nodes = r.nodes;
  out->steps = r.q.steps;
  out->dt = r.dt;
  out->arrival = r.q.arrival;
  out->admitted = r.admitted;
  out->finished = r.finished;
  return 0;
}

int wt_serve_result_state(wt_server* s, int rid, void* Phi, void* Pi) {
  if (!s) return WT_EINVAL;
  if (rid < 0 || rid >= (int)s->reqs.size() || !s->reqs[rid].finished_flag || !s->reqs[rid].state)
    return wt::ctx_fail(s->ctx, WT_EINVAL, "wt_serve_result_state: no kept state for request " + std::to_string(rid) +
                                               " (finished, with keep_results?)");
  if (!Phi || !Pi) return wt::ctx_fail(s->ctx, WT_EINVAL, "wt_serve_result_state: NULL buffer");
  const Req& r = s->reqs[rid];
  const size_t fb = (size_t)r.nodes * esize(r.precision);
  void* st = nullptr;
  const int rc = wt_ctx_get_stream(s->ctx, &st);
  if (rc) return rc;
  if (cudaMemcpyAsync(Phi, r.state, fb, cudaMemcpyDeviceToDevice, (cudaStream_t)st) != cudaSuccess ||
      cudaMemcpyAsync(Pi, (char*)r.state + fb, fb, cudaMemcpyDeviceToDevice, (cudaStream_t)st) != cudaSuccess)
    return wt::ctx_fail(s->ctx, WT_ECUDA, "wt_serve_result_state: copy failed");
  return 0;
}

int wt_serve_status(const wt_server* s, int rid, int* status, int* steps_left, int* preemptions) {
  if (!s) return WT_EINVAL;
  if (rid < 0 || rid >= (int)s->reqs.size())
    return wt::ctx_fail(s->ctx, WT_EINVAL, "wt_serve_status: no request " + std::to_string(rid));
  const Req& r = s->reqs[rid];
  if (status) *status = r.status;
  if (steps_left) *steps_left = r.left;
  if (preemptions) *preemptions = r.preemptions;
  return 0;
}

int wt_serve_cancel(wt_server* s, int rid) {
  if (!s) return WT_EINVAL;
  wt::NvtxRange nv("wt_serve_cancel");
  if (rid < 0 || rid >= (int)s->reqs.size())
    return wt::ctx_fail(s->ctx, WT_EINVAL, "wt_serve_cancel: no request " + std::to_string(rid));
  const int st = s->reqs[rid].status;
  if (st == WT_REQ_FINISHED || st == WT_REQ_CANCELLED)
    return wt::ctx_fail(s->ctx, WT_EINVAL, "wt_serve_cancel: request " + std::to_string(rid) + " has " +
                                               (st == WT_REQ_FINISHED ? "finished" : "been cancelled"));
  return s->cancel(rid);
}

int wt_serve_preempt(wt_server* s, int rid) {
  if (!s) return WT_EINVAL;
  wt::NvtxRange nv("wt_serve_preempt");
  if (rid < 0 || rid >= (int)s->reqs.size() || s->reqs[rid].status != WT_REQ_RUNNING)
    return wt::ctx_fail(s->ctx, WT_EINVAL, "wt_serve_preempt: request " + std::to_string(rid) + " is not running");
  return s->preempt(rid);
}

int wt_serve_info(const wt_server* s, int* waiting, int* active, int* done, double* used_bytes, double* peak_bytes) {
  if (!s) return WT_EINVAL;
  if (waiting) *waiting = (int)(s->pending.size() + s->queue.size());
  if (active) *active = (int)s->active.size();
  if (done) *done = s->done;
  if (used_bytes) *used_bytes = s->used;
  if (peak_bytes) *peak_bytes = s->peak;
  return 0;
}

int wt_serve_preempt_choice(const wt_serve_desc* desc, double used, int count, const long long* nodes,
                            const int* steps_left, const double* cost, const int* preemptions, long long head_nodes,
                            int head_steps_left, double head_cost, int* victims, int* nvictims) {
  if (check_desc(desc) || count < 0 || !nvictims) return WT_EINVAL;
  if (count > 0 && (!nodes || !steps_left || !cost || !preemptions || !victims)) return WT_EINVAL;
  std::vector<long long> nv(nodes, nodes + count);
  std::vector<double> work(count), cv(cost, cost + count);
  std::vector<int> pre(preemptions, preemptions + count);
  for (int k = 0; k < count; ++k) work[k] = (double)nodes[k] * steps_left[k];
  const std::vector<int> v =
      choose_victims(*desc, used, nv, work, cv, pre, head_cost, (double)head_nodes * head_steps_left);
  std::copy(v.begin(), v.end(), victims);
  *nvictims = (int)v.size();
  return 0;
}

int wt_serve_queue_order(int order, double now, int count, const double* arrival, const double* service,
                         const double* work, int* perm) {
  if (count < 0 || (count > 0 && (!arrival || !service || !work || !perm))) return WT_EINVAL;
  if (order < WT_SERVE_HRRN || order > WT_SERVE_FIFO) return WT_EINVAL;
  std::vector<double> a(arrival, arrival + count), sv(service, service + count), w(work, work + count);
  for (int k = 0; k < count; ++k)
    if (order == WT_SERVE_HRRN && !(sv[k] > 0)) return WT_EINVAL;
  std::vector<int> idx(count);
  std::iota(idx.begin(), idx.end(), 0);
  order_queue(order, now, idx, a, sv, w);
  std::copy(idx.begin(), idx.end(), perm);
  return 0;
}

}  // extern "C"
