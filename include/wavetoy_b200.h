/*
 * wavetoy_b200.h -- C ABI of the B200 (sm_100a) implementation of
 * WaveToySecondOrder.jl's 3D SBP-SAT right-hand side and RK4 time step.
 *
 * Conventions
 *   - Every function returns int: 0 = OK, < 0 = error (WT_E*); the message of
 *     the last error on a context is wt_last_error(ctx).
 *   - Fields are the reference's Julia arrays: (N,N,N,Ne), column-major, i
 *     fastest (index i + N*(j + N*(k + N*e)), 0-based).  Connectivity arrays
 *     given by callers are Julia's MeshConnectivity: (6,Ne), 1-based element
 *     and face numbers, 0 = no neighbour.  Faces 1..6 = (-x,+x,-y,+y,-z,+z).
 *   - State pointers passed to wt_rhs_* / wt_step_* are DEVICE pointers owned
 *     by the caller (CuArray interop), of the context's precision (double for
 *     WT_F64, float for WT_F32); calls are asynchronous on the context stream.
 *     Functions ending in _host take host pointers and synchronise.
 *   - A context owns one CUDA stream.  It is thread-compatible (one context
 *     per host thread), not thread-safe.
 *
 * Boundary-condition kinds (src/boundaries1d.jl:61-64):
 *   1 = Dirichlet, 2 = Sommerfeld, 3 = excision, 4 = full Dirichlet.
 * Outer-face tags (src/wave.jl:23, 567-571): 0 interior, 1..6 Dirichlet
 * against bdry_values[tag], 7 Sommerfeld, 8 excision.
 */
#ifndef WAVETOY_B200_H
#define WAVETOY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  WT_OK = 0,
  WT_EINVAL = -1,     /* bad argument (ArgumentError in the reference) */
  WT_ECUDA = -2,      /* CUDA runtime error */
  WT_ENOMEM = -3,     /* device allocation failed / over budget */
  WT_ENOTSUP = -4,    /* configuration not supported by this build */
  WT_ENONFINITE = -5, /* a NaN/Inf was detected (the reference's isfinite assert) */
  WT_ETIMEOUT = -6    /* a bounded device wait gave up */
};

enum { WT_F64 = 0, WT_F32 = 1 };
/* How an FP32 mesh steps (the precision forms of the large-solve study):
 *   WT_FP32_COMPENSATED (default): FP32 storage of the state, the RK4 stages,
 *     the coefficients, the metric terms and the flux; the state Phi is held
 *     as a compensated pair (the caller's FP32 array plus a low part the
 *     workspace keeps, as for Pi), every RK4 stage carries that low part, and
 *     K1 evaluates the split-form gradient of Phi in FP64 (CUDA cores) with the
 *     metric terms split into an element-constant FP64 part and an FP32
 *     deviation.  Rounding Phi to FP32 is what limits the plain forms: it is
 *     amplified by the second derivative in Pi-dot.  Applies to the RK4
 *     stepping without Kreiss-Oliger dissipation (eps_KO = 0), all n; the
 *     other FP32 paths (dissipative stages, Tsit5) run as WT_FP32_CUDA_CORES.
 *   WT_FP32_CUDA_CORES: FP32 everywhere, FFMA contractions (n = 8 kernels).
 *   WT_FP32_BF16X3 / WT_FP32_BF16X2: n = 8 contractions as split-precision
 *     BF16 on tensor cores with three-term operands (FP32 accuracy) or two-term
 *     hi + lo operands.
 * Other n use the generic CUDA-core kernels (compensated for the default). */
enum { WT_FP32_CUDA_CORES = 0, WT_FP32_BF16X3 = 1, WT_FP32_BF16X2 = 2, WT_FP32_COMPENSATED = 3 };
enum { WT_BC_DIRICHLET = 1, WT_BC_SOMMERFELD = 2, WT_BC_EXCISION = 3, WT_BC_FULL_DIRICHLET = 4 };
enum { WT_BG_MINKOWSKI = 0, WT_BG_CONSTANT_SHIFT = 1, WT_BG_ADM_PERTURBED = 2, WT_BG_RADIAL_SHIFT = 3,
       WT_BG_GAUGE_WAVE = 4, WT_BG_SINE_SHIFT = 5 };
/* prescribed 4-metrics of the fully second-order curved path */
enum { WT_CURVED4_MINKOWSKI = 0, WT_CURVED4_GAUGE_WAVE = 1 };

typedef struct wt_ctx wt_ctx;
typedef struct wt_mesh wt_mesh;
typedef struct wt_coef wt_coef;
typedef struct wt_ws wt_ws;
typedef struct wt_batch wt_batch;

/* ---- context ------------------------------------------------------------ */
/* No reference counterpart (Julia picks the backend per array); owns the
 * stream that KernelAbstractions' backend queue stands for. */
int wt_ctx_create(int device, wt_ctx** out);
int wt_ctx_destroy(wt_ctx* ctx);
const char* wt_last_error(const wt_ctx* ctx);
int wt_ctx_synchronize(wt_ctx* ctx);
/* the context's cudaStream_t, as void* */
int wt_ctx_get_stream(wt_ctx* ctx, void** stream);
/* Launch on a caller-owned cudaStream_t instead (e.g. the stream a CuArray or
 * torch tensor was produced on); NULL restores the context's own stream.  The
 * context never destroys a caller's stream. */
int wt_ctx_set_stream(wt_ctx* ctx, void* stream);
/* number of kernel launches this context has issued (evidence counter) */
int wt_ctx_launch_count(const wt_ctx* ctx, long long* count);
/* Device memory held by the objects of this context (meshes, coefficients,
 * workspaces, batches, served requests): live bytes, live allocations, and
 * the allocations made since the context was created (any may be NULL).
 * Host only.  No counterpart in the reference (Julia's GC owns its arrays). */
int wt_ctx_memory(const wt_ctx* ctx, long long* live_bytes, long long* live_allocs, long long* total_allocs);
/* Host-side fault injection: the device allocation `after` allocations from
 * now (0: the next one) fails once with WT_ENOMEM, as if cudaMalloc had
 * failed, without calling it; after < 0 cancels a pending injection.  The
 * failing call releases what it had allocated, and the context stays usable.
 * No device fault is involved.  No counterpart in the reference. */
int wt_ctx_inject_alloc_failure(wt_ctx* ctx, long long after);
/* How this library was built: WT_BUILD_BOUNDS_CHECK (compiled with
 * -DWT_BOUNDS_CHECK: every index a kernel reads from the mesh's neighbour,
 * face-source and boundary-slot tables is checked against the table's range
 * before use) and WT_BUILD_NVTX (NVTX ranges on the entry points).  Host only. */
enum { WT_BUILD_BOUNDS_CHECK = 1, WT_BUILD_NVTX = 2 };
int wt_build_flags(int* flags);
/* Synchronise, then read and clear the bounds word of the bounds-check build:
 * bit 0 = a neighbour element index out of range was read, bit 1 = a boundary
 * slot out of range.  The kernel replaced the value by "no neighbour" / slot 0
 * and made no access outside its buffers.  Always 0 in the normal build.  No
 * counterpart in the reference (its kernels run with @inbounds). */
int wt_ctx_bounds_status(wt_ctx* ctx, unsigned int* word);
/* Bounds-check build only (WT_ENOTSUP otherwise): overwrite entry (e, f) of a
 * mesh's device face-source table (64 * neighbour + 8 * orientation +
 * neighbour face, -1 = none) or boundary-slot table, so that a test can plant
 * an out-of-range index and see wt_ctx_bounds_status report it while every
 * access stays inside its buffer.  Synchronous. */
enum { WT_TABLE_FACE_SOURCE = 0, WT_TABLE_BOUNDARY_SLOT = 1 };
int wt_mesh_debug_set_table(wt_mesh* mesh, int table, long long e, int f, int value);
/* Read and clear the device non-finite flag that fused RK4 steps set when the
 * state stops being finite (the reference asserts all(isfinite, ...) per
 * sample, src/evolve.jl:1344); synchronous. */
int wt_ctx_nonfinite(wt_ctx* ctx, int* flag);
/* Self-test of the bounded-wait failure path (no counterpart in the reference):
 * one thread polls an mbarrier as the pipelined kernels do, at most `polls`
 * times (1..2^24), after arriving on it (arrive = 1: returns 0) or not
 * (arrive = 0: the wait gives up, sets the status word and the call returns
 * WT_ETIMEOUT); the context stays usable.  Nothing faults or waits unbounded. */
int wt_ctx_selftest_wait(wt_ctx* ctx, int arrive, long long polls);
/* Per-kernel timing for measurement: while enabled, the fused RK4 step records
 * CUDA events around each launch of its kernels (gradient/flux K1, divergence
 * K2, and the fused stage kernel of FP64 n = 8 solves) on the launching
 * stream; wt_ctx_profile_read synchronises and returns the summed milliseconds
 * and launch counts {K1, K2, fused stage}, then clears. */
int wt_ctx_profile(wt_ctx* ctx, int enable);
int wt_ctx_profile_read(wt_ctx* ctx, double ms[3], long long count[3]);

/* ---- reference element ----------------------------------------------------- */
/* HexSBPSAT.make_element(T, N) + make_operators(elem) (src/evolve.jl:1189):
 * GLL nodes x and SBP norm H (diagonal) on [0,1] and the differentiation
 * matrix G[i*N + p], with H G + (H G)^T = diag(-1,0,...,0,1) (README.md:14-19).
 * Host only; needs no device.  N in 2..8. */
int wt_gll_operators(int N, double* x, double* H, double* G);

/* ---- mesh + geometry ------------------------------------------------------ */
/* Analytic hex builder.  Replaces HexMeshes.make_uniform_hex(T, Mx, My, Mz,
 * x0, x1; periodic) / make_warped_uniform_hex(T, Mx, My, Mz, x0, x1, A;
 * periodic) (test/dirichlet_warped_tests.jl:23-40, src/evolve.jl:1174-1175)
 * followed by HexSBPSAT.make_element/make_operators/make_geometry and, for
 * curvilinear meshes, make_metric_terms3d (src/evolve.jl:1189-1196).  Warp:
 * X = s + A P(s), P = sin(2 pi s1) sin(2 pi s2) sin(2 pi s3) for all three
 * components.  Geometry and curl-form metric terms are computed on the device
 * in FP64. */
typedef struct {
  int N;            /* GLL nodes per axis, 2..8 */
  int M[3];         /* elements per axis */
  double x0, x1;    /* the cube [x0,x1]^3 */
  double warp_A;    /* warp amplitude; 0 = affine uniform hex */
  int periodic;     /* 1 = periodic connectivity */
  int outer_tag;    /* 0 = side tags 1..6; else this tag on every outer face */
  int precision;    /* WT_F64 or WT_F32: type of streamed fields and state */
} wt_mesh_desc;
int wt_mesh_create(wt_ctx* ctx, const wt_mesh_desc* desc, wt_mesh** out);

/* Generic mesh from host arrays mirroring MeshGeometry + MeshConnectivity:
 * coords (3,N,N,N,Ne), jac (3,3,N,N,N,Ne) = dx_a/dxi_b, neighbour /
 * neighbour_face (6,Ne) int32 1-based, orientation / bdry (6,Ne) int8.
 * Replaces HexSBPSAT.to_device(geom, backend) (src/evolve.jl:1191).
 * The face orientation of every interior face is inferred from the node
 * coordinates (the D4 map under which the two faces' nodes coincide, or differ
 * by one constant shift for periodic faces); `orientation` may be NULL and is
 * not read.  Faces that coincide under no such map give WT_EINVAL. */
int wt_mesh_create_arrays(wt_ctx* ctx, int N, long long Ne, const double* coords, const double* jac,
                          const int32_t* neighbour, const int32_t* neighbour_face,
                          const int8_t* orientation, const int8_t* bdry, int precision, wt_mesh** out);
/* Multi-patch curvilinear meshes of evolve3d's mesh kinds (src/evolve.jl:1176-1184;
 * the builders are HexMeshes' make_cubed_cube_mesh / make_inflated_cube_mesh /
 * make_radial_shell_mesh in the reference, restated with this library's own
 * maps): WT_MESH_CUBED_CUBE (p = {R}: [-1,1]^3 around a centre cube [-R,R]^3,
 * 7 M^3 elements), WT_MESH_INFLATED_CUBE (p = {L, R1, R2}: centre cube
 * [-L,L]^3, a layer to the sphere R1 and a shell to R2, 13 M^3 elements),
 * WT_MESH_RADIAL_SHELL (p = {R1, R2}: 6 M^3 elements).  Neighbours and face
 * orientations come from matching node coordinates; outer faces get
 * outer_tag, the radial shell's inner sphere inner_tag (the excision tag 8 in
 * evolve3d). */
enum { WT_MESH_CUBED_CUBE = 1, WT_MESH_INFLATED_CUBE = 2, WT_MESH_RADIAL_SHELL = 3 };
typedef struct {
  int kind;       /* WT_MESH_* */
  int N;          /* nodes per axis, 2..8 */
  int M;          /* elements per patch and axis */
  double p[3];    /* kind parameters (above) */
  int outer_tag;  /* tag of the outer faces (nonzero) */
  int inner_tag;  /* radial shell: tag of the inner faces (nonzero) */
  int precision;  /* WT_F64 or WT_F32 */
} wt_patch_desc;
int wt_mesh_create_patches(wt_ctx* ctx, const wt_patch_desc* desc, wt_mesh** out);
/* One z-slab of the analytic cube of desc, for a solve partitioned over GPUs
 * (no counterpart in the reference, which runs one device per solve): the nz
 * element layers z0 .. z0 + nz - 1 of the whole mesh (taken modulo M[2] when
 * desc->periodic; there -M[2] <= z0 < M[2]), with the geometry, metric terms
 * and face tags those elements have in the whole mesh.  A z face whose
 * neighbour layer lies outside the slab gets no neighbour and no tag (a cut):
 * a partition gives each slab one ghost layer beyond each cut and refreshes it
 * with wt_halo_copy after the first part of every RK4 stage
 * (wt_rk4_stage_curved), so that the slab's own layers advance exactly as in
 * the whole mesh.  Elements are numbered as in wt_mesh_create with M[2] = nz. */
int wt_mesh_create_slab(wt_ctx* ctx, const wt_mesh_desc* desc, int z0, int nz, wt_mesh** out);
/* The same mesh as host arrays (host only, no device work): *Ne, and when
 * coords != NULL also coords (3,N,N,N,Ne), jac (9 per node, may be NULL),
 * neighbour / neighbour_face (6,Ne, 1-based, 0 = none), orientation (6,Ne, the
 * D4 code described at wt_mesh_get) and bdry (6,Ne).  Call once with
 * coords = NULL for *Ne.  No counterpart in the reference (HexMeshes returns
 * the mesh object). */
int wt_patch_mesh_arrays(const wt_patch_desc* desc, long long* Ne, double* coords, double* jac, int32_t* neighbour,
                         int32_t* neighbour_face, int32_t* orientation, int32_t* bdry);
int wt_mesh_destroy(wt_mesh* mesh);
int wt_mesh_info(const wt_mesh* mesh, int* N, long long* Ne, int* precision);
/* Copy a geometry array to host (FP64): "coords" (3*nn), "jac", "invjac"
 * (9*nn), "detjac", "Hphys", "Hd", "invdetJ" (nn), "Ja" (9*nn, field-major:
 * Ja[(al*3+i)*nn + node] = J dxi_al/dx_i), "x","H" (N), "G" (N*N, G[i*N+p]);
 * int32 arrays: "bdry", "neighbour" (6*Ne, 1-based), "neighbour_face" (6*Ne,
 * 1-based, 0 where there is no neighbour), "orientation" (6*Ne: the D4 code
 * ori whose map (p,q) -> (p',q') is: swap if ori & 4, then reverse p' if
 * ori & 1 and q' if ori & 2), "handedness" (Ne). */
int wt_mesh_get(const wt_mesh* mesh, const char* name, void* host_out);
/* Override the outer-face tags (6,Ne) int32, e.g. to mark excision faces. */
int wt_mesh_set_bdry(wt_mesh* mesh, const int32_t* bdry);
/* Free the FP64 set-up geometry the RHS and RK4 path no longer read (node
 * coordinates, Jacobian, inverse, determinant; for FP32 meshes also the FP64
 * metric terms) to make room for more solves.  Afterwards background sampling,
 * initial data, min spacing, the strong form and reading those arrays return
 * WT_EINVAL.  No counterpart in the reference (Julia's GC owns its arrays). */
int wt_mesh_release_setup_geometry(wt_mesh* mesh);
/* Precision form of an FP32 mesh (WT_FP32_*; default WT_FP32_COMPENSATED).
 * Switching between the CUDA-core and the BF16 forms re-lays the mesh's
 * n = 8 metric blocks (synchronous).  No counterpart in the reference (its
 * T = Float32 path uses one form). */
int wt_mesh_set_fp32_form(wt_mesh* mesh, int form);
/* _min_node_spacing_3d (src/evolve.jl:60-69); synchronous. */
int wt_mesh_min_spacing(wt_mesh* mesh, double* h);

/* ---- ADM background --------------------------------------------------------*/
/* Analytic background sampled on the device: replaces AnalyticBackground3D +
 * make_coef3d + sample_background3d! (src/wave3d_curved.jl:45-124).
 *   MINKOWSKI: -   CONSTANT_SHIFT: p[0..2] = beta
 *   ADM_PERTURBED: alpha = 1 + p0 sin 2pi x, beta^i = p1 cos 2pi x_i,
 *     gamma_ij = d_ij + p2 exp(-|x-c|^2/p3)(d_ij + 0.5 s_ij), c = p4..p6,
 *     s = p7..p12 (s11,s12,s13,s22,s23,s33)
 *   RADIAL_SHIFT: beta_r linear from p0 at r=p2 to p1 at r=p3 (src/evolve.jl:1128-1145)
 * Time-dependent backgrounds from a spacetime metric (MetricBackground3D,
 * src/wave3d_curved.jl:56-71: ADM variables of the metric at (t, x, y, z)),
 * p[0] = A, p[1] = d, p[2] = the time t0 they are first sampled at; with
 * H = 1 - A sin(2 pi (x - t)/d) and c = cos(2 pi (x - t)/d):
 *   GAUGE_WAVE (SpacetimeMetrics.GaugeWave): alpha = sqrt(H), beta = 0,
 *     gamma = diag(H, 1, 1);
 *   SINE_SHIFT (SpacetimeMetrics.SineShift): alpha = 1, beta^x = -A c/(1 + A c),
 *     gamma = diag((1 + A c)^2, 1, 1)
 * (the decompositions evolve1d documents, src/evolve.jl:171-195, flat in y, z).
 * wt_step_rk4_curved re-samples them at every stage time, as evolve3d's rhs!
 * calls sample_background3d!(coef, bg, t) (src/evolve.jl:1289), and advances
 * the coefficients' time; wt_coef_set_time samples them at a given time. */
typedef struct {
  int kind;
  double p[16];
} wt_background_desc;
int wt_background_set(wt_ctx* ctx, wt_mesh* mesh, const wt_background_desc* desc, wt_coef** out);
/* Host-sampled 11-field bundle (alpha, sqrtg, b1, b2, b3, gu11, gu12, gu13,
 * gu22, gu23, gu33), each (N,N,N,Ne) FP64 -- the layout sample_background3d!
 * fills. */
int wt_background_set_arrays(wt_ctx* ctx, wt_mesh* mesh, const double* coef11, wt_coef** out);
int wt_coef_get(const wt_coef* coef, double* coef11_host);
/* Time-dependent coefficients (WT_BG_GAUGE_WAVE, WT_BG_SINE_SHIFT): sample at
 * time t (synchronous); the time they hold.  Static coefficients: set_time
 * returns WT_EINVAL, get_time gives 0. */
int wt_coef_set_time(wt_ctx* ctx, wt_coef* coef, double t);
int wt_coef_get_time(const wt_coef* coef, double* t);
int wt_coef_destroy(wt_coef* coef);

/* ---- initial data --------------------------------------------------------------*/
enum { WT_IC_EIGENMODE_CARTESIAN = 0, WT_IC_GAUSSIANS = 1, WT_IC_OUTGOING_PULSE = 2, WT_IC_PLANE_WAVE = 3,
       WT_IC_EIGENMODE_RADIAL = 4 };
/* Fill u (and ut, may be NULL) on the device at time t:
 *   EIGENMODE_CARTESIAN eigenmode_cartesian! (src/wave.jl:163-185): p = A, kx, ky, kz, omega, x0, x1
 *   GAUSSIANS  the :gaussian IC (src/evolve.jl:1260-1263), summed: p = count, then (cx, cy, cz, A, w) each
 *   OUTGOING_PULSE outgoing_pulse! (src/wave.jl:292-323): p = A, s0, sigma, cx, cy, cz
 *   PLANE_WAVE Phi_e / Pi_e of _background3d :minkowski/:constant_shift (src/evolve.jl:1115-1118): p = k, omega, s
 *   EIGENMODE_RADIAL eigenmode_radial! (src/wave.jl:207-226): p = A, R, n, cx, cy, cz */
int wt_initial_data(wt_ctx* ctx, wt_mesh* mesh, int kind, const double* params, int nparams, double t, void* u,
                    void* ut);

/* wt_initial_data of (Phi, Pi) = (u, u_t) for the solve that ws steps,
 * evaluated in FP64: an FP32 mesh's state then starts as the compensated
 * FP64 values (the rounded values in Phi, Pi, the low parts in the workspace),
 * as wt_state_set_f64 does.  Synchronous. */
int wt_initial_state(wt_ctx* ctx, wt_ws* ws, int kind, const double* params, int nparams, double t, void* Phi,
                     void* Pi);
/* Load a Float64 state (device arrays) into the state arrays a solve steps:
 * for an FP64 mesh a copy; for an FP32 mesh the FP32 arrays Phi, Pi get the
 * rounded values and the workspace keeps the low parts the rounding lost
 * (the compensated state that WT_FP32_COMPENSATED and the Kahan-compensated
 * RK4 sums carry), so that stepping Phi, Pi with this workspace starts from
 * the Float64 state itself.  Replaces the host-side Float64 -> T conversion
 * before the reference's evolve loop (src/evolve.jl:1270); asynchronous. */
int wt_state_set_f64(wt_ctx* ctx, wt_ws* ws, const double* Phi64, const double* Pi64, void* Phi, void* Pi);
/* Host checkpoints of a stepped state, word for word: Phi and Pi in the mesh
 * precision and, for an FP32 mesh, the low parts the workspace keeps for that
 * pair (zeros if it keeps none).  Loading a checkpoint into the state arrays of
 * a workspace on a mesh of the same N, Ne and precision, then stepping, gives
 * the values that stepping the saved solve gives, bit for bit.  bytes must equal
 * wt_state_checkpoint_size.  The serving engine's preemption keeps a
 * preempted request's state this way.  No counterpart in the reference, whose
 * evolve3d returns its final state only (src/evolve.jl:1361-1365).
 * Synchronous. */
int wt_state_checkpoint_size(const wt_ws* ws, long long* bytes);
int wt_state_checkpoint_save(wt_ctx* ctx, wt_ws* ws, const void* Phi, const void* Pi, void* host, long long bytes);
int wt_state_checkpoint_load(wt_ctx* ctx, wt_ws* ws, void* Phi, void* Pi, const void* host, long long bytes);

/* ---- workspace ---------------------------------------------------------------*/
/* Replaces make_wave3d_workspace (src/wave3d_curved.jl:158-178): device
 * scratch plus mu, the spectral radius of apply_D! along axis 1 from the
 * reference's 30-step power iteration (alternating-sign start).  mu is
 * computed on first use (wt_workspace_mu or any call with eps_ko != 0); that
 * first use synchronises the stream, so make it before capturing a graph. */
int wt_workspace_create(wt_ctx* ctx, wt_mesh* mesh, wt_ws** out);
int wt_workspace_destroy(wt_ws* ws);
int wt_workspace_mu(wt_ws* ws, double* mu);
/* Impose mu instead of estimating it (no counterpart in the reference): the
 * slabs of a partitioned solve take the whole mesh's value, since each slab's
 * own estimate differs from it. */
int wt_workspace_set_mu(wt_ws* ws, double mu);
/* Fused RK4 stages (the integrator-in-RHS idea of the reference's IDEAS.md:48-50;
 * no entry point of its own there): with on = 1 (the default) an FP64 n = 8
 * solve without Kreiss-Oliger dissipation steps through the fused stage kernel,
 * which runs the divergence half of stage s and the gradient half of stage
 * s + 1 in one launch (five launches per RK4 step instead of eight, 28 % fewer
 * DRAM bytes).  The results equal the two-kernel stages' bit for bit; on = 0
 * selects the two-kernel stages.  Takes effect at the next step call; the
 * second flux buffer (3 x 8 bytes per node) is allocated then. */
int wt_workspace_set_fused(wt_ws* ws, int on);

/* ---- right-hand sides (device pointers, async) ------------------------------*/
typedef struct {
  int kinds[6];       /* BC kind per side (-x,+x,-y,+y,-z,+z); curvilinear uses kinds[0] */
  double sigma;       /* penalty strength, 1 in the reference */
  int excision_tag;   /* faces with this tag get no SAT (curvilinear pass) */
  const void* gPhi;   /* optional data fields (device, NULL = none) */
  const void* gPi;
  const void* gDx;
  const void* gDy;
  const void* gDz;
} wt_bc_desc;

/* wave3d_curved_rhs!(Phidot, Pidot, Phi, Pi, coef; geom, ops, ws, eps_KO,
 * bc3d, metric) (src/wave3d_curved.jl:205-258) with the boundary passes
 * _apply_bc3d! / _apply_bc3d_curv! (src/boundaries3d.jl:58-232).
 * use_metric = 0 selects the affine per-axis path (metric === nothing),
 * 1 the curvilinear split-form path.  bc may be NULL (periodic). */
int wt_rhs_curved(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, const void* Phi, const void* Pi,
                  void* Phidot, void* Pidot, double eps_ko, const wt_bc_desc* bc, int use_metric);
/* No counterpart in the reference.  The RHS of wt_rhs_curved, evaluated
 * without a workspace and without allocating: for callers that may not
 * allocate device memory while they evaluate the RHS (a host runtime that owns
 * the process's device memory pool, a memory budget fixed before the time
 * loop, or a loop that must not pay for the device-wide synchronisation of
 * cudaMalloc/cudaFree).  Its scratch is one fixed device array of the library
 * (8.4 MiB, held on every GPU that loads the library until exit), so the mesh
 * may have at most WT_NOALLOC_MAX_NODES nodes and WT_NOALLOC_MAX_BOUNDARY_NODES
 * boundary-face nodes; larger meshes are rejected with WT_EINVAL.  mu is the
 * KO normalisation that wt_workspace_mu returns for a workspace on the same
 * mesh, used only when eps_ko != 0 (then a non-positive or non-finite mu is
 * rejected with WT_EINVAL; nothing else ties mu to the mesh).  The first call
 * through each wt_ctx looks up the array's device address on the context's
 * device (set-up); make that first call before any stream capture.  The
 * address belongs to the device's primary context: after cudaDeviceReset,
 * create a new wt_ctx.  All calls share the array: calls whose kernels overlap
 * on the GPU race and give wrong results. */
#define WT_NOALLOC_MAX_NODES 262144
#define WT_NOALLOC_MAX_BOUNDARY_NODES 262144
int wt_rhs_curved_noalloc(wt_ctx* ctx, const wt_coef* coef, const void* Phi, const void* Pi, void* Phidot,
                          void* Pidot, double eps_ko, double mu, const wt_bc_desc* bc, int use_metric);
/* HexSBPSAT.apply_D!(Du, u, d) (called at src/wave3d_curved.jl:169-170, 184-189, 219-221), d = 1..3. */
int wt_apply_D(wt_ctx* ctx, wt_ws* ws, const void* u, void* Du, int d);
/* dst += eps * mu^-5 * sum_d D_d^6 field: the three _ko_axis3! calls of one
 * field (src/wave3d_curved.jl:182-192, 241-248). */
int wt_ko_add(wt_ctx* ctx, wt_ws* ws, void* dst, const void* field, double eps_ko);
/* apply_gradient3d! (src/wave3d_curved.jl:223): split-form curvilinear gradient. */
int wt_gradient3d(wt_ctx* ctx, wt_ws* ws, const void* u, void* g1, void* g2, void* g3);
/* apply_divergence3d! (src/wave3d_curved.jl:237). */
int wt_divergence3d(wt_ctx* ctx, wt_ws* ws, const void* F1, const void* F2, const void* F3, void* out);

/* rhs_wave3d!(utt, u, ut, bdry_values; geom, ops, work, tau, sommerfeld_R)
 * (src/wave.jl:583-611): SIPG Laplacian (apply_laplacian!, README.md:57-80)
 * plus the tag-7 Sommerfeld pass (src/wave.jl:453-542).  Affine meshes.
 * sommerfeld_R <= 0 or infinite = plane-wave BGT-0. */
int wt_rhs_sipg(wt_ctx* ctx, wt_ws* ws, const void* u, const void* ut, void* utt, const double bdry_values[6],
                double tau, double sommerfeld_R);
/* wave_strong_rhs_mesh!(utt, u, ut, mesh, geom, dinvjac, ops; tau, sommerfeld_R)
 * (src/wave_strong_rhs.jl:296-341); dinvjac (make_metric_derivs, :376-391)
 * is built on the device on first use. */
int wt_rhs_strong(wt_ctx* ctx, wt_ws* ws, const void* u, const void* ut, void* utt, double tau,
                  double sommerfeld_R);
/* wave_lap_strong_conservative_mesh!(Lu, u, mesh, ops, h; tau)
 * (src/wave_lap_strong.jl:280-308): uniform Cartesian meshes. */
int wt_lap_strong_cons(wt_ctx* ctx, wt_ws* ws, const void* u, void* Lu, double h, double tau);

/* Scalar wave on a prescribed 4-metric, fully second order.
 * wt_curved4_background replaces eval_curved_background!
 * (src/wave_curved_rhs.jl:373-418) for the analytic metrics named by
 * WT_CURVED4_*: fills ginv (10,N,N,N,Ne: tt,tx,ty,tz,xx,xy,xz,yy,yz,zz) and
 * gamma (4,N,N,N,Ne: contracted Christoffels), device arrays in the mesh
 * precision; params = (A, d) of the gauge wave H = A sin(2 pi (x - t)/d).
 * wt_rhs_curved4 replaces wave_curved_rhs_mesh! (conservative = 0,
 * src/wave_curved_rhs.jl:155-187) and wave_curved_rhs_conservative_mesh!
 * (conservative = 1, tau as its keyword, the reference default (N-1)^2;
 * src/wave_curved_rhs.jl:330-362): phiddot = d_tt phi on uniform Cartesian
 * elements of edge h, faces without a neighbour seeing zero traces. */
int wt_curved4_background(wt_ctx* ctx, wt_mesh* mesh, int kind, const double* params, double t, void* ginv,
                          void* gamma);
int wt_rhs_curved4(wt_ctx* ctx, wt_ws* ws, const void* phi, const void* phidot, void* phiddot, const void* ginv,
                   const void* gamma, double h, int conservative, double tau);

/* ---- reductions (FP64 accumulation, synchronous) ----------------------------- */
/* wave3d_energy (src/wave3d_curved.jl:268-287). */
int wt_energy(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, const void* Phi, const void* Pi, int use_metric,
              double* E);
/* The lapse-weighted energy (no counterpart in the reference):
 * E_alpha = sum 1/2 [(alpha/sqrt(gamma)) Pi^2 + alpha sqrt(gamma) gamma^{ij} dPhi_i dPhi_j] H,
 * the reference energy's integrand times the lapse.  wave3d_energy is exactly
 * conserved only for alpha = 1 (src/wave3d_curved.jl:263-266); for a static
 * background with zero shift the split-form semi-discretisation conserves
 * E_alpha instead (its gradient / divergence pair is skew-adjoint in Hd), so it
 * is the drift monitor for alpha != 1.  Same arguments as wt_energy. */
int wt_energy_lapse(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, const void* Phi, const void* Pi, int use_metric,
                    double* E);
/* SIPG Hamiltonian 1/2<ut,ut>_H - 1/2<u, L_SAT u>_H (test/kernels3d_tests.jl:39-47). */
int wt_energy_sipg(wt_ctx* ctx, wt_ws* ws, const void* u, const void* ut, double tau, double* E);
/* sqrt(sum (a-b)^2 H), H = Hphys (use_metric 0) or Hd (1) (src/evolve.jl:1353-1354);
 * b may be NULL (norm of a). */
int wt_l2_diff(wt_ctx* ctx, wt_ws* ws, const void* a, const void* b, int use_metric, double* out);

/* ---- time stepping ----------------------------------------------------------- */
/* nsteps classic RK4 steps (OrdinaryDiffEq RK4(), adaptive=false; in-repo
 * restatement test/wave3d_tests.jl:32-44) of the conservative system, with
 * the stage update fused into the RHS kernels (low-storage form).  Phi, Pi
 * are updated in place.  Sets WT_ENONFINITE if the state became non-finite
 * (checked at the end; the reference asserts isfinite per sample). */
int wt_step_rk4_curved(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, int nsteps,
                       double eps_ko, const wt_bc_desc* bc, int use_metric);
/* One half of RK4 stage `stage` (0..3) of wt_step_rk4_curved (eps_ko = 0),
 * for callers that exchange halos between the halves (a z-slab partition):
 * part 1 evaluates the gradient, the flux and the boundary terms and updates
 * Phi's stage; part 2 the divergence and Pi's stage.  Calling parts 1, 2 of
 * stages 0..3 in order is one wt_step_rk4_curved step, with the same kernels
 * and results.  Time-dependent backgrounds are re-sampled at part 1 and their
 * time advanced after stage 3. */
int wt_rk4_stage_curved(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, int stage,
                        int part, const wt_bc_desc* bc, int use_metric);
/* Halo of a z-slab after part 1 of stage `stage`: the fields other elements read
 * across a face before part 2 and the next stage -- the Phi that the next
 * stage reads (the caller's Phi after stage 3) and the three flux components --
 * restricted to element layer `layer` (M[0] M[1] consecutive elements), copied
 * into buf (pack = 1) or from buf back into the fields (pack = 0), in the
 * mesh's precision, asynchronously on the context stream.  buf holds
 * wt_halo_size values (known once a first stage part has run on ws). */
/* Kreiss-Oliger dissipation on a slab partition: its z passes reach six element
 * layers, so such a partition keeps six ghost layers beyond each cut and
 * refreshes them once per stage.  wt_rk4_stage_curved_ko runs one whole RK4
 * stage of wt_step_rk4_curved with eps_ko != 0 (the RHS with dissipation, then
 * both stage updates: the same kernels as that path).  wt_halo_state_copy then
 * copies `count` element layers from `layer` of the state the next stage reads
 * (the stage outputs; the caller's Phi and Pi after stage 3) into buf (pack = 1,
 * Phi's layers then Pi's) or back (pack = 0), asynchronously on the context
 * stream. */
int wt_rk4_stage_curved_ko(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, int stage,
                           double eps_ko, const wt_bc_desc* bc, int use_metric);
int wt_halo_state_copy(wt_ctx* ctx, wt_ws* ws, void* Phi, void* Pi, int stage, int layer, int count, void* buf,
                       int pack);
int wt_halo_size(const wt_ws* ws, long long* values);
int wt_halo_copy(wt_ctx* ctx, wt_ws* ws, void* Phi, int stage, int layer, void* buf, int pack);
/* The face-plane exchange of a z-slab partition (no counterpart in the
 * reference).  An owned element next to a cut reads, of the ghost element
 * across it, only the face plane they share: the Phi trace its gradient's
 * SAT reads and the flux trace its divergence's SAT reads.  So a partition
 * may run both stage halves on its owned layers only
 * (wt_rk4_stage_curved_layers: the elements of layers layer0 ..
 * layer0 + nlayers - 1; an analytic cube's layer is M[0] M[1] consecutive
 * elements) and exchange just those planes: wt_halo_face_copy packs (pack = 1)
 * or unpacks (pack = 0) face `face` (4: -z, 5: +z) of element layer `layer` --
 * per element the n^2 face values of the Phi the next stage reads (and, for
 * the compensated FP32 form, its small part) and of the three flux
 * components -- wt_halo_face_size values, asynchronously on the context
 * stream.  The sender packs its boundary layer's face toward the cut, the
 * receiver unpacks the same face of its ghost layer (the same element).
 * Ghost layers are then never computed.  A time-dependent background is
 * re-sampled at every part-1 call and its time advanced at the part-2 call of
 * stage 3, so make one such call per step. */
int wt_rk4_stage_curved_layers(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt,
                               int stage, int part, int layer0, int nlayers, const wt_bc_desc* bc, int use_metric);
int wt_halo_face_size(const wt_ws* ws, long long* values);
int wt_halo_face_copy(wt_ctx* ctx, wt_ws* ws, void* Phi, int stage, int layer, int face, void* buf, int pack);
/* Fixed-step explicit Runge-Kutta methods of pick_integrator_first_order
 * (src/evolve.jl:43-48; evolve3d runs them with adaptive = false):
 * WT_ERK_RK4 (the fused low-storage RK4 above) and WT_ERK_TSIT5 (Tsitouras
 * 2011, fifth order).  Time-dependent backgrounds are re-sampled at every
 * stage time.  Vern7 (N >= 7 in the reference) has no built-in tableau: a caller
 * passes its published coefficients to wt_step_erk_curved_tableau. */
enum { WT_ERK_RK4 = 0, WT_ERK_TSIT5 = 1 };
#define WT_ERK_MAX_STAGES 16
int wt_step_erk_curved(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt, int nsteps,
                       int method, double eps_ko, const wt_bc_desc* bc, int use_metric);
/* The same with the caller's explicit Butcher tableau: stages s (1..WT_ERK_MAX_STAGES),
 * c[s], A[s*s] row major with A[i*s + j] = 0 for j >= i, b[s], all finite
 * (WT_EINVAL otherwise).  It runs any explicit method with its published
 * coefficients, e.g. Verner's 7(6) pair, which pick_integrator_first_order
 * chooses for N >= 7 (Vern7, 10 stages; its 7th-order weights).  The workspace
 * holds 2 s state-sized slope buffers.  No counterpart in the reference as an
 * entry point (OrdinaryDiffEq takes the method as a type). */
int wt_step_erk_curved_tableau(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt,
                               int nsteps, int stages, const double* c, const double* A, const double* b,
                               double eps_ko, const wt_bc_desc* bc, int use_metric);
/* The method's Butcher tableau (host only): stages, c[s], A[s*s] (row major), b[s]. */
int wt_erk_tableau(int method, int* stages, double* c, double* A, double* b);
/* RK4 of the SIPG system as first-order (u, ut):
 * u' = ut + eps mu^-5 sum_d D_d^6 u,  ut' = rhs_wave3d!(u, ut) + eps mu^-5 sum_d D_d^6 ut. */
int wt_step_rk4_sipg(wt_ctx* ctx, wt_ws* ws, void* u, void* ut, double dt, int nsteps,
                     const double bdry_values[6], double tau, double sommerfeld_R, double eps_ko);
/* End-to-end evolve with host buffers, the shape of evolve3d(formulation =
 * :conservative) (src/evolve.jl:1149-1366): upload Phi/Pi, then nsamples times
 * run steps_per_sample RK4 steps, copy the state back into Phi_host/Pi_host
 * and the energy into energy[s] (may be NULL).  Phi_host/Pi_host hold the
 * final state on return.  Each sample is copied device to device into a
 * staging pair and from there to the host on two copy streams, so the copy
 * overlaps the next sample's steps (page-locked host buffers make it
 * asynchronous).  The host does not wait inside the loop: energies are
 * collected on the device and summed at the end, and the non-finite check
 * (WT_ENONFINITE) runs every 16 samples and at the end.  The four state-sized
 * device buffers it needs are allocated on the first call and kept by the
 * workspace. */
int wt_evolve_curved_host(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, double* Phi_host, double* Pi_host,
                          double dt, int steps_per_sample, int nsamples, double eps_ko, const wt_bc_desc* bc,
                          int use_metric, double* energy);
/* The same for an FP32 mesh with FP32 host buffers (no reference counterpart:
 * the reference's evolve3d keeps Float64 host arrays). */
int wt_evolve_curved_host_f32(wt_ctx* ctx, wt_ws* ws, const wt_coef* coef, float* Phi_host, float* Pi_host,
                              double dt, int steps_per_sample, int nsamples, double eps_ko, const wt_bc_desc* bc,
                              int use_metric, double* energy);

/* Device-side diagnostics in place of evolve3d's per-sample host copies of the
 * whole state (src/evolve.jl:1339-1358): wt_gather_nodes copies the values of
 * `field` at `count` node indices (e.g. the 1-D slice evolve3d records) to
 * host_out as FP64; L2 norms and energies come from wt_l2_diff / wt_energy.
 * Snapshots: wt_snapshot_save writes Phi and Pi with a 64-byte header (magic
 * "WTB2SNP1", version, N, Ne, precision, field count, t) to a file;
 * wt_snapshot_load reads one back into a mesh of the same N, Ne and precision.
 * No counterpart in the reference for the file format (IDEAS.md:57). */
int wt_gather_nodes(wt_ctx* ctx, wt_mesh* mesh, const void* field, const int64_t* nodes, int count,
                    double* host_out);
int wt_snapshot_save(wt_ctx* ctx, wt_mesh* mesh, const void* Phi, const void* Pi, double t, const char* path);
int wt_snapshot_load(wt_ctx* ctx, wt_mesh* mesh, void* Phi, void* Pi, double* t, const char* path);

/* ---- batches of independent solves ----------------------------------------
 * No counterpart in the reference, which advances one solve per evolve3d
 * call (src/evolve.jl:1149-1358); the batch advances many solves of uneven
 * element counts and orders together.  Members are existing (workspace,
 * coefficients, Phi, Pi) sets on curvilinear meshes, each with its own dt and
 * boundary data; they are grouped by (n, precision, kernel path), each group
 * is one work list of (solve, element) tiles run by one kernel launch per RK4
 * stage, and one RK4 step of all groups is a CUDA graph, captured when the
 * membership changes and replayed by wt_batch_step; the groups' launches are
 * parallel branches of that graph.  The first step after a change also picks
 * the launch variant of the generic (n != 8) kernels, K1 and K2 separately, by
 * timing (autotuner, on by default): 0 the generic kernels at their default
 * elements per CTA, 1 at the alternative count, 2 (n = 4 and 6) the persistent
 * kernels that copy the next group of tiles into shared memory by cp.async
 * while they compute the current one; all three give the same bits
 * (wt_batch_group_info's epb_variant: bits 0-1 K1's variant, bits 2-3 K2's).  A member with a time-dependent background is re-sampled at
 * every stage time inside the graph (its mesh must keep the set-up geometry).
 * Every member advances by the same number of steps per call; results equal
 * wt_step_rk4_curved on each member alone. */
int wt_batch_create(wt_ctx* ctx, wt_batch** out);
int wt_batch_destroy(wt_batch* batch);
int wt_batch_add(wt_batch* batch, wt_ws* ws, const wt_coef* coef, void* Phi, void* Pi, double dt,
                 const wt_bc_desc* bc, int* slot);
int wt_batch_remove(wt_batch* batch, int slot);
int wt_batch_set_autotune(wt_batch* batch, int on);
/* Fix the launch variants of the generic groups' K1 and K2 (0, 1, 2 as above;
 * -1, the default, leaves the choice to the autotuner; 2 falls back to 0 where
 * a group's order has no pipelined kernels).  Takes effect at the next step. */
int wt_batch_set_variant(wt_batch* batch, int k1, int k2);
int wt_batch_step(wt_batch* batch, int nsteps);
int wt_batch_info(wt_batch* batch, int* nsolves, long long* nodes, int* ngroups);
int wt_batch_group_info(wt_batch* batch, int group, int* N, int* precision, int* n8_path, int* epb_variant,
                        long long* tiles);

/* ---- serving a stream of solve requests -------------------------------------
 * No counterpart in the reference (one solve per evolve3d call,
 * src/evolve.jl:1149-1358).  A server owns one batch on a context.  A request
 * names an analytic mesh, a background (static, or time-dependent and then
 * re-sampled at every RK4 stage inside the batch), initial data of Phi (Pi = 0), a
 * CFL number and a step count, and arrives at a time on the server's clock
 * (seconds since wt_serve_create).  Each scheduling round (wt_serve_poll):
 *   1. requests whose arrival time has passed join the wait queue;
 *   2. the queue is ordered (WT_SERVE_HRRN: highest response ratio
 *      (wait + S) / S first, S = 2 nodes steps / rate + 0.05 s the estimated
 *      service time; WT_SERVE_SJF: least nodes x steps first; WT_SERVE_FIFO:
 *      arrival order; ties by arrival, then submission);
 *   3. requests are admitted from the head of the queue while the admitted
 *      ones' estimated device bytes fit hbm_budget, fewer than max_active run
 *      and the running requests hold fewer than fill_nodes nodes; admission
 *      builds the request's mesh, coefficients, workspace and state on the
 *      device and adds it to the batch;
 *   4. the batch advances by min(tick, the fewest steps any running request
 *      has left) RK4 steps and the stream is synchronised; requests with no
 *      steps left leave the batch (their finish time is taken here) and free
 *      their memory (the final state stays while keep_results is set).
 * A request's estimated bytes are nodes x (bytes per node of its running form +
 * 272 for the FP64 set-up geometry held while it is built); the running form
 * holds 520 (FP64, n = 8), 480 (FP64), 300 (FP32, n = 8) or 260 (FP32) bytes
 * per node.  Results equal wt_step_rk4_curved on each request alone. */
typedef struct wt_server wt_server;
enum { WT_SERVE_HRRN = 0, WT_SERVE_SJF = 1, WT_SERVE_FIFO = 2 };
#define WT_SERVE_AUTO (-1)  /* precision per request: FP32 when steps <= auto_fp32_max_steps, else FP64 */
#define WT_SERVE_MAX_IC 128
typedef struct {
  double hbm_budget;         /* bytes the admitted requests may hold (estimate above) */
  int tick;                  /* most RK4 steps per round, >= 1 */
  int max_active;            /* most requests running together; 0 = no limit */
  long long fill_nodes;      /* admit only while running requests hold fewer nodes; 0 = no limit */
  int order;                 /* WT_SERVE_HRRN, WT_SERVE_SJF or WT_SERVE_FIFO */
  int precision;             /* WT_F64, WT_F32 or WT_SERVE_AUTO */
  int fp32_form;             /* wt_mesh_set_fp32_form of FP32 requests */
  int auto_fp32_max_steps;   /* threshold of WT_SERVE_AUTO */
  int keep_results;          /* keep each finished request's final state (wt_serve_result_state) */
  double rate_f64, rate_f32; /* DOF-updates/s of the service estimate; <= 0: 3e9 and 6e9 */
  int preempt;               /* 1: preemptive admission (below); 0: none */
} wt_serve_desc;
/* Preemptive admission (preempt = 1): when the request at the head of the
 * queue cannot start (budget, max_active or fill_nodes), running requests with
 * at least twice its remaining work (nodes x steps left) are preempted
 * (wt_serve_preempt), the one with the most remaining work first, until it
 * can -- but only if preempting the eligible ones makes room at all.  A request
 * is preempted this way at most once, so no two requests trade places forever;
 * a preempted request resumes from its host checkpoint, to the same bits. */
typedef struct {
  double arrival;            /* seconds on the server's clock */
  wt_mesh_desc mesh;         /* analytic mesh; precision is chosen by the server */
  wt_background_desc bg;     /* any kind; a time-dependent one (gauge wave, sine shift) keeps its mesh's set-up geometry and is re-sampled at every RK4 stage */
  int ic_kind, nic;          /* wt_initial_data of Phi at t = 0 */
  double ic[WT_SERVE_MAX_IC];
  double cfl, max_speed;     /* dt = cfl * wt_mesh_min_spacing / max_speed */
  int steps;                 /* RK4 steps, >= 1 */
  wt_bc_desc bc;             /* data pointers must be NULL */
} wt_serve_request;
typedef struct {
  int precision;             /* the form the request ran in */
  long long nodes;
  int steps;
  double dt;
  double arrival, admitted, finished;  /* server clock; latency = finished - arrival */
} wt_serve_result;
int wt_serve_create(wt_ctx* ctx, const wt_serve_desc* desc, wt_server** out);
int wt_serve_destroy(wt_server* server);
/* queue a request (WT_EINVAL when it can never fit the budget); rid numbers
 * requests 0, 1, ... in submission order */
int wt_serve_submit(wt_server* server, const wt_serve_request* req, int* rid);
/* one scheduling round; *finished = requests that finished in it.  With nothing
 * running and nothing arrived it sleeps until the next arrival (at most 10 ms). */
int wt_serve_poll(wt_server* server, int* finished);
/* rounds until every submitted request has finished; WT_ENONFINITE if a state
 * became non-finite */
int wt_serve_run(wt_server* server);
/* WT_EINVAL until request rid has finished */
int wt_serve_get_result(const wt_server* server, int rid, wt_serve_result* out);
/* A request's state: WAITING (submitted, not running; PREEMPTED if it ran and
 * waits with a host checkpoint), RUNNING, FINISHED or CANCELLED, with the steps
 * it has left and how often it was preempted (any pointer may be NULL). */
enum { WT_REQ_WAITING = 0, WT_REQ_RUNNING = 1, WT_REQ_FINISHED = 2, WT_REQ_CANCELLED = 3, WT_REQ_PREEMPTED = 4 };
int wt_serve_status(const wt_server* server, int rid, int* status, int* steps_left, int* preemptions);
/* Cancel a request that has not finished: a waiting one leaves the queue, a
 * running one leaves the batch and its device memory (and its share of the
 * budget) is released at once.  WT_EINVAL if it finished or was cancelled. */
int wt_serve_cancel(wt_server* server, int rid);
/* Preempt a running request: its state is saved to a host checkpoint
 * (wt_state_checkpoint_save), it leaves the batch, its device memory and budget
 * share are released, and it waits again with the steps it has left, in the
 * admission order of those.  When admitted again it is rebuilt and resumes from
 * the checkpoint; with a static background its final state equals the one of
 * an uninterrupted run, bit for bit (a time-dependent background resumes at the
 * time the host recorded, which may differ from the device's in the last bit).
 * WT_EINVAL unless the request is running. */
int wt_serve_preempt(wt_server* server, int rid);
/* copy a finished request's kept final state into device buffers of its
 * precision (nodes values each), on the context stream */
int wt_serve_result_state(wt_server* server, int rid, void* Phi, void* Pi);
int wt_serve_info(const wt_server* server, int* waiting, int* active, int* done, double* used_bytes,
                  double* peak_bytes);
/* the estimated device bytes and precision of a request under desc (host only) */
int wt_serve_cost(const wt_serve_desc* desc, const wt_serve_request* req, double* bytes, int* precision);
/* The admission order of step 2 as a permutation of count waiting requests
 * (host only, no device): arrival times, estimated service seconds and work
 * (nodes x steps) per request, listed in submission order. */
int wt_serve_queue_order(int order, double now, int count, const double* arrival, const double* service,
                         const double* work, int* perm);
/* The requests preemptive admission would preempt for a head request (host only,
 * no device): count running requests (nodes, steps left, estimated bytes, times
 * preempted), the bytes in use and the head's nodes, steps left and bytes.
 * victims (count entries of room) gets their indices in preemption order,
 * *nvictims their number (0: preempt nothing). */
int wt_serve_preempt_choice(const wt_serve_desc* desc, double used, int count, const long long* nodes,
                            const int* steps_left, const double* cost, const int* preemptions, long long head_nodes,
                            int head_steps_left, double head_cost, int* victims, int* nvictims);

/* ---- evolve3d in one call ------------------------------------------------------
 * The keyword set of evolve3d(formulation = :conservative; T, N, M, mesh_kind,
 * background, ic, bc, eps_KO, t0, t1, Nt, cfl) (src/evolve.jl:1149-1166) as one
 * descriptor, over this library's mesh, background and initial-data
 * descriptors.  wt_evolve3d builds the mesh, coefficients and workspace,
 * fills the initial state at t0, and integrates to t1 with the reference's
 * time sampling (src/evolve.jl:1209-1213, 1311-1352):
 *   dt = cfl * (smallest node spacing) / max_speed, and with eps_ko != 0 at
 *   most 1.4 / (eps_ko mu); the samples are range(t0, t1, nt); before sample n
 *   the solve takes RK4 steps of dt while its time is below ts[n], the time
 *   accumulated in the mesh precision, and a step that would pass t1 is
 *   shortened to end on t1 (the integrator's stop at the end of its span).
 * At each sample it records the time reached, the energy (wt_energy) and the
 * L2 distance (Hd-weighted with use_metric, else Hphys) of Phi to the initial
 * data family at that time when ic_exact = 1 (ic = :exact), else the L2 norm
 * of Phi.  The final state goes to Phi_host, Pi_host (nodes values of the mesh
 * precision; wt_solve_nodes gives the count).  A non-finite state ends it with
 * WT_ENONFINITE.  Every device object is released before it returns. */
typedef struct {
  int mesh_kind;              /* 0: analytic hex (mesh); WT_MESH_CUBED_CUBE / _INFLATED_CUBE / _RADIAL_SHELL (patch) */
  wt_mesh_desc mesh;          /* mesh_kind 0 */
  wt_patch_desc patch;        /* mesh_kind > 0 */
  int precision;              /* T: WT_F64 or WT_F32 (overrides the mesh descriptors') */
  wt_background_desc bg;
  int ic_kind, nic;           /* wt_initial_state at t0 */
  double ic[WT_SERVE_MAX_IC];
  int ic_exact;               /* 1: the initial-data family is the exact solution (ic = :exact) */
  wt_bc_desc bc;              /* data pointers must be NULL; all kinds 0: none (bc3d = nothing) */
  int use_metric;             /* 1: curvilinear split form (the reference passes the metric bundle) */
  double eps_ko;
  double t0, t1;
  int nt;                     /* samples, >= 1 */
  double cfl, max_speed;
} wt_solve_desc;
typedef struct {
  double dt;                  /* the step */
  double dx;                  /* the smallest node spacing */
  double mu;                  /* the Kreiss-Oliger spectral radius (0 without dissipation) */
  long long steps;            /* RK4 steps taken, the shortened last one included */
} wt_solve_info;
/* why desc is not a valid solve ("" if it is), written to msg (host only, no device) */
int wt_solve_desc_check(const wt_solve_desc* desc, char* msg, int msglen);
/* nodes of the mesh desc describes (host only) */
int wt_solve_nodes(const wt_solve_desc* desc, long long* nodes);
/* The sampling schedule (host only): steps[n] = RK4 steps before sample n,
 * after steps[n - 1]; the last step taken is shortened to dt_last (dt if no
 * step is shortened); ts_actual[n] = the time at sample n.  precision: the
 * type the time accumulates in.  WT_EINVAL above 1e9 steps. */
int wt_solve_schedule(double t0, double t1, int nt, double dt, int precision, long long* steps, double* dt_last,
                      double* ts_actual);
/* The diagnostic 1-D slice evolve3d records (src/evolve.jl:104-123, 1322-1349):
 * the nodes whose y and z lie strictly within atol of (y, z), in storage order,
 * keeping the first node at each x (within atol), then sorted by x (stable).
 * evolve3d takes atol = sqrt(eps(T)) and (y, z) = the mid-plane (x0 + x1) / 2. */
typedef struct {
  double y, z;          /* the line; NaN: the mid-plane of the mesh's extent */
  long long capacity;   /* room in xs, and per sample in Phi and Pi */
  long long count;      /* out: nodes on the line (nothing is written past capacity) */
  long long* nodes;     /* out: their node indices (capacity; may be NULL) */
  double* xs;           /* out: their x, ascending (capacity) */
  double* Phi;          /* out: [sample][node], nt x capacity values, FP64 */
  double* Pi;
} wt_solve_slice;
/* The slice selection on node-major coordinates xyz[3 * node + c] (host only). */
int wt_slice_select(const double* xyz, long long nodes, double y, double z, double atol, long long capacity,
                    long long* node_out, double* xs_out, long long* count);
/* Any of ts_actual, energy, l2 (nt values each), slice, info may be NULL. */
int wt_evolve3d(wt_ctx* ctx, const wt_solve_desc* desc, void* Phi_host, void* Pi_host, double* ts_actual,
                double* energy, double* l2, wt_solve_slice* slice, wt_solve_info* info);

#ifdef __cplusplus
}
#endif
#endif /* WAVETOY_B200_H */
