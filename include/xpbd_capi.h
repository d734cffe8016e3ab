/*
 * C ABI of the B200 XPBD Gaussian-graph solver (libxpbd_b200.so).
 *
 * The first group is a drop-in for the reference's singleton C ABI: the same 29
 * symbols, argument meanings, clamping and error behaviour as native/xpbd_capi.cu of
 * minn-k/3dgs-isaac-sim-xpbd, so that its src/xpbd_bridge.py loads this library through
 * XPBD_DLL unchanged.  Each declaration names the reference entry point it replaces
 * (file:line in that project).  Conventions, as in the reference:
 *   - all pointers are caller-owned host memory, copied during the call;
 *   - int functions return 0 (or a count) on success and -1 on failure, with the
 *     message in xpbd_last_error() (xpbd_capi.cu:31-43);
 *   - void setters cannot fail and clamp their inputs;
 *   - xpbd_set_attached / positions / shapes / reset / launch / add_rigid_velocity need
 *     one xpbd_step first (the graph is uploaded by the first step, xpbd_capi.cu:169);
 *   - xpbd_step blocks until the GPU has finished the step (xpbd_capi.cu:223).
 *   - Gaussian order is the caller's (PLY/USD) order; positions are float3[n],
 *     quaternions (w, x, y, z).
 *
 * The second group (xpbd_b200_*) has no counterpart in the reference ABI.
 */
#ifndef XPBD_B200_CAPI_H
#define XPBD_B200_CAPI_H

#ifdef __cplusplus
#define XPBD_API extern "C" __attribute__((visibility("default")))
#else
#define XPBD_API __attribute__((visibility("default")))
#endif

/* ---- reference entry points (native/xpbd_capi.cu) ---------------------- */

/* xpbd_capi.cu:66 — message of the last failed call */
XPBD_API const char* xpbd_last_error(void);
/* xpbd_capi.cu:71-102 — n Gaussians (pos[3n], activated scales[3n], normalised
 * rots[4n] w,x,y,z, activated opacity[n]) and e undirected edges (edges[2e], rest[e],
 * stiff[e]).  Frees any previous scene. */
XPBD_API int xpbd_create(int n, const float* pos, const float* scales, const float* rots, const float* opacity,
	int e, const int* edges, const float* rest, const float* stiff);
/* xpbd_capi.cu:104-109 — frees the scene and clears colliders and pins */
XPBD_API void xpbd_destroy(void);
/* xpbd_capi.cu:111 */
XPBD_API int xpbd_count(void);
/* xpbd_capi.cu:113-119 — iterations per step, dt, Jacobi under-relaxation, velocity
 * damping, stiffness / inverse-mass scales, distance / shape compliance, shape blend,
 * angle compliance / blend (angle constraint: accepted, not solved — as in the runtime) */
XPBD_API void xpbd_set_solver(int iters, float dt, float underRelax, float velDamping, float stiffnessScale,
	float invMassScale, float distCompliance, float shapeCompliance, float shapeBlend, float angleCompliance,
	float angleBlend);
/* xpbd_capi.cu:121-127 */
XPBD_API void xpbd_set_constraints(int distance, int shape, int angle, int volume);
/* xpbd_capi.cu:130-137 — volume compliance, cluster ring k, member cap, leader spacing;
 * clusters are rebuilt at the next step */
XPBD_API void xpbd_set_volume(float compliance, int ringK, int maxMembers, int leaderMinHop);
/* xpbd_capi.cu:140-145 — ground plane (point contact) and gravity along -up */
XPBD_API void xpbd_set_ground(int enabled, float ux, float uy, float uz, float height, float friction,
	float restitution, float contactRadius, float contactSlop, float gravity);
/* xpbd_capi.cu:148 — object-level shape keeping: accepted, not implemented (a warning
 * is printed when a positive stiffness is set) */
XPBD_API void xpbd_set_object_shape(float stiffness);
/* xpbd_capi.cu:151 — accepted, no effect */
XPBD_API void xpbd_set_object_shape_gpu(int enabled);
/* xpbd_capi.cu:154-158 — up to 32 kinematic colliders: types (0 sphere, 1 box,
 * 2 capsule), poses[12 count] (row-major local->world R, centre), dims[3 count] */
XPBD_API void xpbd_set_colliders(int count, const int* types, const float* poses, const float* dims, float margin,
	float friction);
/* xpbd_capi.cu:161-164 — per collider of the last step: hits, pushed displacement sum,
 * contact centroid; returns the number filled */
XPBD_API int xpbd_collider_stats(int* hits, float* push, float* centroid, int maxCount);
/* xpbd_capi.cu:167-172 — adds dv + dw x (x - center) to every free Gaussian's velocity */
XPBD_API int xpbd_add_rigid_velocity(const float* dv, const float* dw, const float* center);
/* xpbd_capi.cu:179-191 — ellipsoid contact shapes: bit 1 colliders, bit 2 ground, 0 off.
 * Each Gaussian meets them as its opacity-tau iso-ellipsoid (semi-axes capped at
 * radiusCap when > 0), packed from the created shapes, then re-packed from the deformed
 * shapes by every xpbd_compute_shapes.  Before the first step the pack waits for the
 * scene's upload.  Ends with the scene (create / destroy). */
XPBD_API int xpbd_set_contact_shape(int enabled, float tau, float radiusCap);
/* xpbd_capi.cu:195-200 — pins idx[count] at pos[3 count] (inverse mass 0, velocity 0);
 * count 0 releases; the previous pins' inverse masses are restored first */
XPBD_API int xpbd_set_attached(int count, const int* idx, const float* pos, float weight);
/* xpbd_capi.cu:203-206 — spatial-hash self-collision */
XPBD_API void xpbd_set_self_collision(int enabled, float radiusScale, float excludeScale, int withinBody);
/* xpbd_capi.cu:209-212 — out[0] candidates, out[1] active particles, out[2] over-cap
 * replacements, of the last step */
XPBD_API void xpbd_self_collision_stats(int* out);
/* xpbd_capi.cu:215 — shape-matching rotation: 1 FP64 polar (default), 0 FP32 path */
XPBD_API void xpbd_set_shape_robust(int enabled);
/* xpbd_capi.cu:218-225 — one solver step; blocks until done */
XPBD_API int xpbd_step(void);
/* xpbd_capi.cu:228-232 — device pointer to the committed positions, float3[n], valid
 * until the next create/destroy; 0 before the first step */
XPBD_API unsigned long long xpbd_positions_device(void);
/* xpbd_capi.cu:235-243 */
XPBD_API int xpbd_positions_host(float* out, int n);
/* xpbd_capi.cu:248-260 — deformed Gaussian scales[3n] / quats[4n] (either may be NULL);
 * returns the number of Gaussians whose shape changed, or -1 */
XPBD_API int xpbd_compute_shapes(float deformEps, float* hostScales, float* hostQuats, int n);
/* xpbd_capi.cu:263-269 — back to rest, zero velocity, pins released */
XPBD_API int xpbd_reset(void);
/* xpbd_capi.cu:272-276 — rest pose rotated by tilt (axis * angle) about the centre of
 * mass, velocity lin + ang x (x - com) */
XPBD_API int xpbd_launch(const float* lin, const float* ang, const float* tilt);
/* xpbd_capi.cu:281-288 — press harness: plates at the rest extent of axis 0/1/2, the max
 * (or, fromLo, the min) one closing at rampPerSec up to maxDispPct (0.01..1) of the
 * extent; centres past a plate are projected onto it (no friction).  While it runs the
 * ground, gravity, object shape keeping and self-collision are not applied.  -1 before
 * the first step or when an 8 % end slab is empty. */
XPBD_API int xpbd_press_start(int axis, float rampPerSec, float maxDispPct, int fromLo);
/* xpbd_capi.cu:291 — settle 90 steps at 25/50/75/100 % of the displacement (default on) */
XPBD_API void xpbd_press_autolog(int enabled);
/* xpbd_capi.cu:294 — plates off, every inverse mass back to 1 (positions kept) */
XPBD_API void xpbd_press_stop(void);
/* xpbd_capi.cu:297-303 — plate coordinates lo/hi, displacement, maximum; 1 while a press
 * runs.  xpbd_reset and xpbd_launch end a press. */
XPBD_API int xpbd_press_state(float* lo, float* hi, float* curDisp, float* maxDisp);
/* xpbd_capi.cu:306-310 — enables per-step volume-weighted J statistics and returns
 * the last ones computed (mean, std) */
XPBD_API void xpbd_volume_stats(int enable, float* jvw, float* jvwStd);

/* ---- extensions (no counterpart in the reference ABI) ------------------- */

/* ChainMail displacement propagation (runChainmailGPU, forward.cu:12808-13006; the
 * reference's C ABI cannot reach it because xpbd_create forces XPBD mode,
 * xpbd_capi.cu:98).  Material constants as setChainmailMaterialParams
 * (forward.cu:4844-4858). */
XPBD_API void xpbd_b200_chainmail_set_material(float global_scale, float air, float skin, float bone,
	int use_edge_stiffness, float edge_influence);
/* Seeds start a wave: Gaussian idx[k] moves by delta[3k..3k+2] and its arrival time
 * becomes 0 (applySeedCommandsKernel, forward.cu:5907-5924), in order.  After a step. */
XPBD_API int xpbd_b200_chainmail_seed(int count, const int* idx, const float* delta);
/* prop_iters propagation sweeps, relax_iters relax sweeps and one closing relax sweep on
 * the current positions (the reference's dense path; its defaults 20, 5, 0.5, 0.99, 0.1). */
XPBD_API int xpbd_b200_chainmail_run(int prop_iters, int relax_iters, float prop_strength, float relax_stiffness,
	float relax_damping);
/* Propagation sweeps on work lists of the Gaussians next to the last sweep's changes (1,
 * default) or over every Gaussian (0).  The results are identical. */
XPBD_API void xpbd_b200_chainmail_set_frontier(int enabled);
/* Build the volume clusters' member lists (k-ring BFS and farthest-point subsample,
 * forward.cu:9814-10033) on the GPU (1, default; leader spacing 1 only) or on the host
 * (0).  The lists are identical either way; takes effect at the next upload or rebuild. */
XPBD_API void xpbd_b200_set_gpu_builder(int enabled);
/* The graph as an APGGRPH1 file (exportPhysicsGraph, forward.cu:4612-4663), in the
 * order given to xpbd_create; after the first step.  0 or -1. */
XPBD_API int xpbd_b200_export_graph(const char* path);
/* Arrival times (caller order; 1e9 where the wave has not arrived); returns N or -1. */
XPBD_API int xpbd_b200_chainmail_times(float* out, int n);

/* ---- Splatting of the current Gaussians into a device image (the viewer's 3DGS
 * rasteriser, CudaRasterizer::Rasterizer::forward, rasterizer_impl.cu:201-470, with
 * preprocessCUDA / renderCUDA, forward.cu:1919-2650), no graphics API. ---- */
/* Colours: sh_degree -1 -> RGB per Gaussian (colors_precomp); 0..3 -> (d+1)^2 RGB
 * spherical-harmonic coefficients per Gaussian, [n][coeffs][3] (shs).  After
 * xpbd_create; kept until the next create.  0 or -1. */
XPBD_API int xpbd_b200_render_set_colors(int n, int sh_degree, const float* data);
/* antialiasing (the reference's flag), an optional crop box (boxmin/boxmax; NULL = none)
 * and per-pixel picking of the first Gaussian with alpha > 0.1 (id_buffer). */
XPBD_API void xpbd_b200_render_set_options(int antialiasing, const float* box_min, const float* box_max, int pick);
/* Checker floor in place of the background under the solver's ground plane
 * (setGroundRender, forward.cu:4448-4462). */
XPBD_API void xpbd_b200_render_set_floor(int visible, const float* origin, float checker, float fade_radius);
/* One frame: view / proj column-major 4x4 (world->view, world->clip), camera position,
 * image size, tan of the half fields of view, scale modifier; deform_eps >= 0 renders
 * the deformed shapes of xpbd_compute_shapes(deform_eps), < 0 the created ones; bg
 * RGB (NULL = black); out (3 x H x W floats, channel-major, NULL = keep on the device).
 * Returns the number of (tile, Gaussian) pairs (num_rendered) or -1. */
XPBD_API long long xpbd_b200_render(const float* view, const float* proj, const float* campos, int width, int height,
	float tan_fovx, float tan_fovy, float scale_modifier, float deform_eps, const float* bg, float* out);
/* Device pointer of the last image (float, 3 x H x W). */
XPBD_API unsigned long long xpbd_b200_render_device(void);
/* Last frame's final transmittance, contributor count and picked Gaussian per pixel
 * (-1 none; picking on) and the screen radius per Gaussian (0 culled); NULL skips one. */
XPBD_API int xpbd_b200_render_aux(float* final_T, int* n_contrib, int* pick, long long npix, int* radii, int n);

/* Independent solver instances: a new engine (own scene, settings and stream), its
 * release, and the choice of the engine that the reference entry points above act on
 * from the calling thread (NULL: the process-wide default engine). */
XPBD_API void* xpbd_b200_engine_new(void);
XPBD_API void xpbd_b200_engine_free(void* handle);
XPBD_API void xpbd_b200_engine_select(void* handle);
/* Restrict each collider of the last xpbd_set_colliders call to one object (graph
 * component id, as numbered by first Gaussian; -1 = every Gaussian), so that objects
 * packed into one scene are gripped independently. */
XPBD_API int xpbd_b200_set_collider_objects(int count, const int* obj);
/* Colliders for scenes that pack many objects: any number of colliders (same layout as
 * xpbd_set_colliders), each bound to one object id obj[c]; a Gaussian is tested only
 * against its own object's colliders.  Replaces the xpbd_set_colliders list (and is
 * replaced by the next xpbd_set_colliders call); xpbd_collider_stats does not cover it. */
XPBD_API int xpbd_b200_set_colliders_many(int count, const int* types, const float* poses, const float* dims,
	const int* obj, float margin, float friction);
/* Run the engine on a caller-owned cudaStream_t (NULL: the library's own stream). */
XPBD_API int xpbd_b200_set_stream(void* stream);
/* Enqueue `substeps` steps without waiting for them. */
XPBD_API int xpbd_b200_step_async(int substeps);
/* k substeps in one call, each preceded by its collider poses (poses[s * 12 * ncol ...],
 * types and dims fixed) and, after the first step, its pin targets
 * (targets[s * 3 * npins ...]): xpbd_set_colliders + xpbd_set_attached +
 * xpbd_b200_step_async(1) per substep, without a call per substep. */
XPBD_API int xpbd_b200_step_substeps(int k, int ncol, const int* types, const float* poses, const float* dims,
	float margin, float friction, int npins, const int* idx, const float* targets);
/* Wait for the engine's stream. */
XPBD_API int xpbd_b200_sync(void);
/* Gauss-Seidel colour sweeps for the distance / volume constraints instead of the
 * Jacobi default (the reference's forward.cu:3780-3812 toggles). */
XPBD_API void xpbd_b200_set_gs(int distance, int volume);
/* Volume kernel shape: 0 auto (4 lanes per cluster / node, or xpbd_b200_set_volume_lanes),
 * 1 one thread per cluster (the reference's thread kernels' summation
 * order), 2 one warp per cluster (its warp kernels' order). */
XPBD_API void xpbd_b200_set_volume_warp_mode(int mode);
/* Lanes per cluster for the volume solve (2, 4, 8, 32: the staged and register forms)
 * and per node for the volume gather (4, 8, 32) in automatic mode; 0 restores the
 * automatic choice (solve: the one-pass moment form on 4 lanes; gather: 4 lanes). */
XPBD_API void xpbd_b200_set_volume_lanes(int solve_lanes, int gather_lanes);
/* 1 (default): replay each step from a captured CUDA graph; 0: launch kernel by kernel. */
XPBD_API void xpbd_b200_set_graph(int enabled);
/* Step forms, all with the same results bit for bit: the kernel sequence (form 0); the
 * substep as ONE cooperative launch with grid-wide barriers between its phases (form 1,
 * where the configuration allows it: no self-collision, object mode or Gauss-Seidel
 * forms); the sequence with its distance and volume kernels compiled for 6 or 8
 * resident blocks per SM (forms 2, 3).  Mode 0 (default) runs form 0, 1 runs form 1,
 * 2 lets the autotuner time every form on the first steps after each capture and keep
 * the fastest.  xpbd_b200_tuning fills out[7]: form in use, decided, mean trial ms of
 * forms 0 and 1, launches per step of the form in use, mean trial ms of forms 2 and 3. */
XPBD_API void xpbd_b200_set_fused(int mode);
XPBD_API int xpbd_b200_tuning(float* out);
/* Self-collision candidate lists of a one-object scene: 1 (default) from a grid of the
 * predicted positions with cells of the search radius, re-ordered into the reference's
 * visiting order; 0 from the reference's own 27-cell scan of the start-position hash
 * (selfColBuildKernel).  The lists are identical either way. */
XPBD_API void xpbd_b200_set_selfcol_near(int enabled);
/* 1 (default): keep Gaussians in Morton order inside the engine (caller order at the
 * ABI; results identical); 0: caller order.  Takes effect at the next upload. */
XPBD_API void xpbd_b200_set_reorder(int enabled);
/* Per-kernel CUDA-event timing of subsequent steps (launches then go kernel by kernel). */
XPBD_API int xpbd_b200_set_profiling(int enabled);
/* Accumulated per-stage milliseconds and launch counts; returns the number of stages. */
XPBD_API int xpbd_b200_stage_times(double* ms, long long* counts, int max_stages);
XPBD_API void xpbd_b200_reset_stage_times(void);
XPBD_API const char* xpbd_b200_stage_name(int stage);
/* Kernels launched by the engine since load (graph replays count every kernel node). */
XPBD_API long long xpbd_b200_launch_count(void);
/* Topology sizes after the first step: N, edges, cluster members, reverse entries, GS
 * edges, GS edge colours, GS clusters, GS cluster colours, hash table, candidates. */
XPBD_API int xpbd_b200_sizes(long long* out);
/* Stage buffers by name, for parity checks (count only when out is NULL). */
XPBD_API int xpbd_b200_debug_int(const char* name, int* out, long long cap);
XPBD_API int xpbd_b200_debug_float(const char* name, float* out, long long cap);
/* Serving arena: many sessions resident in one engine's packed buffers, advanced
 * together by one launch sequence (one CUDA-graph replay) per substep.  Capacities in
 * rows (Gaussians), directed edges, cluster members and reverse-list entries, each at
 * most 2^31-1 (32-bit CSR offsets).  A session joins with arena_admit(arena, engine): an
 * engine handle (xpbd_b200_engine_new) that has built its scene and taken at least one
 * step; its state and topology are copied in (the engine may then be freed) and its
 * slot is returned, or -2 when it does not fit even after compaction, or -1 on error.
 * Sessions share the solver settings; self-collision, ground, object shape and contact
 * shapes stay off.  arena_retire frees a slot; arena_step enqueues k substeps of every
 * live session with per-substep collider poses poses[k][ncol][12] acting on the sessions
 * col_slot[ncol] and pins (session pin_slot[p], its Gaussian pin_idx[p] in the session's
 * order) at targets[k][npin][3]; arena_positions copies a session's committed positions
 * (float3[n], its order); usage fills out[10]: rows used / capacity, edges, members,
 * reverse entries (used, capacity), live Gaussians, sessions. */
XPBD_API void* xpbd_b200_arena_new(long long rows, long long edges, long long members, long long rev);
XPBD_API int xpbd_b200_arena_admit(void* arena, void* session);
XPBD_API int xpbd_b200_arena_retire(void* arena, int slot);
XPBD_API int xpbd_b200_arena_step(void* arena, int k, int ncol, const int* types, const float* poses,
	const float* dims, const int* col_slot, float margin, float friction, int npin, const int* pin_slot,
	const int* pin_idx, const float* targets);
XPBD_API int xpbd_b200_arena_positions(void* arena, int slot, float* out, int n);
XPBD_API int xpbd_b200_arena_sync(void* arena);
XPBD_API int xpbd_b200_arena_usage(void* arena, long long* out);
XPBD_API void xpbd_b200_arena_free(void* arena);
/* Current positions from the caller (float3[n], caller order), velocities kept; after
 * the first step.  Lets a caller teleport the state, and a test run the deformed-shape
 * writeback on positions another solver produced. */
XPBD_API int xpbd_b200_set_positions(const float* pos, int n);
/* The once-per-step self-collision build on given start / predicted positions
 * (x[3n], p[3n]); returns the candidate total.  Solver state is left unchanged. */
XPBD_API int xpbd_b200_selfcol_build(const float* x, const float* p);

/* No counterpart in the reference: the once-per-step self-collision candidate build on
 * caller-owned device buffers, for callers that cannot allocate device memory (a host
 * application that owns the device heap and forbids cudaMalloc, whose implicit
 * synchronisation would stall its frame).  All scratch lives in one static device array
 * sized for n <= 65,536 particles (about 5.4 MB, held by every GPU that loads the library
 * until exit); larger n is rejected with -1.  x, p, rest: device float4[n] (start,
 * predicted and rest positions, w ignored); obj_id: device int[n] or NULL (one object);
 * spacing and the scales as for xpbd_set_self_collision; outputs contacts int[32 n],
 * counts int[n] and optionally total int[1], all device memory; runs on `stream`.
 * Calls share the scratch and must not overlap on the GPU; the first call on a device
 * looks up the array's address and should come before any stream capture. */
XPBD_API int xpbd_b200_selfcol_candidates_static(int n, const float* x, const float* p, const float* rest,
	const int* obj_id, float spacing, float radius_scale, float exclude_scale, int within_body, int* contacts,
	int* counts, int* total, void* stream);

#endif
