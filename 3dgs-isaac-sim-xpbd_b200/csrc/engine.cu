// Host engine and C ABI of the B200 XPBD Gaussian-graph solver.
//
// One Engine holds one scene resident in HBM.  A step (runXPBDSimulation,
// forward.cu:12038-12751) is enqueued as a fixed kernel sequence on the engine's stream;
// all step settings live in a device-side StepParams block that is refreshed before each
// step, so the sequence is captured once into a CUDA graph and replayed until its
// topology (iteration count, enabled constraints, colour counts) changes.  The C ABI
// at the bottom exposes the reference's 29 singleton entry points (xpbd_capi.cu) on top
// of a process-global engine, plus this library's extensions (xpbd_b200_*).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "../../include/xpbd_capi.h"
#include "kernels.cuh"
#include "render.cuh"
#include "xpbd_internal.h"

namespace xpbd {

static thread_local std::string g_err;

static int fail(const char* fmt, ...)
{
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	g_err = buf;
	return -1;
}

#define CK(expr)                                                                           \
	do {                                                                                   \
		const cudaError_t e_ = (expr);                                                     \
		if (e_ != cudaSuccess) return fail("%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
			__FILE__, __LINE__);                                                           \
	} while (0)

// fn(begin, end) over [0, n) in chunks on all host threads (upload-time host work)
template <typename F>
void parallel_for(int n, F fn)
{
	const int workers = std::max(1, std::min<int>(std::thread::hardware_concurrency(), 64));
	if (n < 4096 || workers == 1) { fn(0, n); return; }
	std::atomic<int> next{ 0 };
	const int chunk = std::max(1024, n / (workers * 8));
	std::vector<std::thread> pool;
	for (int w = 0; w < workers; ++w)
		pool.emplace_back([&]() {
			for (;;) {
				const int b = next.fetch_add(chunk);
				if (b >= n) break;
				fn(b, std::min(n, b + chunk));
			}
		});
	for (auto& t : pool) t.join();
}

template <typename T>
struct DBuf {
	T* p = nullptr;
	size_t n = 0;
	DBuf() = default;
	DBuf(const DBuf&) = delete;
	DBuf& operator=(const DBuf&) = delete;
	~DBuf() { release(); }
	cudaError_t alloc(size_t count)
	{
		release();
		n = count;
		if (count == 0) return cudaSuccess;
		return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * count);
	}
	void release()
	{
		if (p) cudaFree(p);
		p = nullptr;
		n = 0;
	}
	size_t bytes() const { return sizeof(T) * n; }
};

// Rows [0, n) in chunks of 256, each chunk sorted by row length (longest first): the
// groups of a warp then run rows of similar length, and the chunk keeps them local
static std::vector<int> length_order(int n, const std::vector<int>& off)
{
	std::vector<int> ord(n);
	for (int r = 0; r < n; ++r) ord[r] = r;
	for (int c0 = 0; c0 < n; c0 += 256) {
		const int c1 = std::min(n, c0 + 256);
		std::stable_sort(ord.begin() + c0, ord.begin() + c1,
			[&](int a, int b) { return off[a + 1] - off[a] > off[b + 1] - off[b]; });
	}
	return ord;
}

// Solver settings.  Like the reference's file-static settings (forward.cu:53-92,
// 224-265, 300-361) they outlive create/destroy; defaults are the reference's.
struct Settings {
	int iters = 20;
	float dt = 1.0f / 60.0f, under_relax = 0.6f, vel_damping = 0.59f, stiffness_scale = 1.0f,
		inv_mass_scale = 1.0f, dist_compliance = 1e-3f, shape_compliance = 0.0f, shape_blend = 0.1f,
		angle_compliance = 0.0f, angle_blend = 0.2f;
	bool use_distance = true, use_shape = false, use_angle = false, use_volume = false, shape_robust = true;
	float vol_compliance = 1e-6f, vol_aniso = 0.05f;
	int ring_k = 1, max_members = 64, leader_min_hop = 1;
	bool topo_dirty = false;
	bool dist_gs = false, vol_gs = false;
	int warp_mode = 0;               // 0 auto (warp when mean members >= 40), 1 thread, 2 warp
	bool sc_enabled = false, sc_within = false;
	float sc_radius_scale = 1.5f, sc_exclude_scale = 2.0f, sc_search_scale = 1.5f, sc_fast_rel = 0.0f;
	bool ground_on = false;
	float ground_n[3] = { 0.0f, 0.0f, 1.0f };
	float ground_h = 0.0f, ground_friction = 0.5f, ground_restitution = 0.3f, ground_radius = 0.0f,
		ground_slop = 0.0f, ground_gravity = 0.0f;
	float object_shape = 0.0f;
	bool jstats = true;
	KinCollider kin[kMaxColliders];
	int kin_obj[kMaxColliders];      // object each collider acts on (-1: every Gaussian)
	std::vector<KinCollider> kin_ext; // batched colliders (any number), each bound to one object
	int kin_count = 0;
	float kin_margin = 0.0f, kin_friction = 0.0f;
	bool use_graph = true;
	bool reorder = true;             // Morton order inside the engine (results unchanged)
	int lanes_a = 0, lanes_b = 0;    // volume kernel lanes per cluster / node (0 = automatic)
	dev::CmMaterial cm{ 1.0f, 0.1f, 0.1f, 0.1f, 1.0f, 1 };   // ChainMail material (forward.cu:66-71)
	bool cm_frontier = true;         // ChainMail sweeps on work lists (false: every sweep dense)
	bool obj_gpu = true;             // object mode's weighted device fit (xpbd_set_object_shape_gpu)
	bool gpu_builder = true;         // cluster members (BFS + farthest point) built on the GPU
	bool press_autolog = true;       // press harness: settle at 25/50/75/100 % (forward.cu:565)
	int fused = 0;                   // substep as one cooperative launch: 0 never, 1 always, 2 the faster (timed)
	int sc_near = 1;                 // one-object scenes: candidate lists from the near-pair grid
	Settings()
	{
		for (auto& v : kin_obj) v = -1;
	}
};

enum Stage {
	ST_PREDICT, ST_DISTANCE, ST_VOL_SOLVE, ST_VOL_GATHER, ST_VOL_GS, ST_SHAPE, ST_SC_BUILD, ST_SC_SOLVE,
	ST_PROJECT, ST_VELOCITY, ST_JSTATS, ST_OTHER, ST_RENDER_PREPARE, ST_RENDER_SORT, ST_RENDER_TILES, ST_COUNT
};
static const char* kStageNames[ST_COUNT] = { "predict", "distance", "volume_solve", "volume_gather", "volume_gs",
	"shape", "selfcol_build", "selfcol_solve", "project", "velocity", "jstats", "other", "render_prepare",
	"render_sort", "render_tiles" };

class Engine {
public:
	// solver settings of this instance (the reference keeps one global set)
	Settings S;
	// ---- created inputs (caller order) ----
	int n = 0, n_edges = 0;
	std::vector<float> in_pos, in_scales, in_rots, in_opacity, in_rest, in_stiff;
	std::vector<int> in_edges;
	bool built = false, stepped = false;
	int generation = 0;

	// ---- host topology (caller index space) and the internal order ----
	std::vector<int> perm, inv;
	std::vector<unsigned long long> lcode;   // Morton code in its component's box, per caller index
	HostGraph graph;
	HostClusters clusters;
	HostEdgeColoring coloring;
	bool coloring_built = false;
	std::vector<int> obj_id;
	int num_objects = 0;
	bool single_object = true;
	float spacing = 0.0f;
	int sc_table = 0;

	// ---- device state ----
	DBuf<float4> pos_curr, pos_next, pos_tmp, vel, pos_rest, shape_rest;
	DBuf<float4> shape_q;    // per Gaussian: eigenvector frame of its last FP64 polar decomposition
	// ChainMail: (arrival time, density), sweep flags / marks / work list / scratch, seeds
	DBuf<float2> cm_td;
	DBuf<unsigned char> cm_flag;
	DBuf<unsigned int> cm_mark;
	DBuf<int> cm_work, cm_seed_idx;
	DBuf<float4> cm_spos;
	DBuf<float> cm_stime, cm_seed_delta, cm_time_out;
	DBuf<dev::CmState> cm_state;
	// object mode: rest offsets q (FP64, internal order), per-object rest centroid, sum q,
	// count, previous centroid, fit parameters, centroid move, block partials, fit weights,
	// boxes; self-collision active set, cross-object corrections and their frame sums
	DBuf<double> obj_q, obj_shift, obj_sumq, obj_partial;
	DBuf<float> obj_c0, obj_params, obj_disp, obj_w, obj_boxes, push_partial, push_T;
	DBuf<int> obj_count;
	DBuf<unsigned char> sc_active;
	DBuf<float4> sc_cross, sc_accum;
	// splatting (xpbd_b200_render*): per-Gaussian projection, depth order, tile pairs,
	// tile ranges, the image and its per-pixel extras; colours and options outlive frames
	struct Render {
		DBuf<float4> xy;     // pixel centre and the half widths of the alpha >= 1/255 box
		DBuf<float4> conic, rgb;
		DBuf<int4> rect;
		DBuf<unsigned int> dkey, dkey_s;
		DBuf<unsigned char> tkey, tkey_s;   // tile keys, 16-bit when the tile count allows, else 32-bit
		DBuf<int> iota, order, radii, touched, val, val_s, n_contrib, pick, torder;
		DBuf<int2> ranges;
		DBuf<float> image, final_T, colors, opacity, rest_sc, rest_q;
		DBuf<long long> cnt, offs;
		DBuf<unsigned long long> d_total;
		cudaEvent_t ev_total = nullptr;
		DBuf<unsigned char> temp;
		long long* h_total = nullptr;   // pinned: pair count of the frame
		std::vector<float> h_colors;    // caller order; uploaded on the next frame
		int sh_deg = -1, sh_coeffs = 0;
		bool colors_dirty = false;
		int antialias = 0, pick_on = 0;
		bool box_on = false;
		float box_lo[3] = {}, box_hi[3] = {};
		bool floor_on = false;
		float floor_origin[3] = {}, floor_checker = 1.0f, floor_fade = 10.0f;
		int W = 0, H = 0;
		long long pairs = 0;
		void release()
		{
			xy.release(); conic.release(); rgb.release(); rect.release(); dkey.release(); dkey_s.release();
			tkey.release(); tkey_s.release(); torder.release();
			iota.release(); order.release(); radii.release(); touched.release();
			cnt.release(); offs.release(); val.release(); val_s.release(); n_contrib.release(); pick.release();
			ranges.release(); image.release(); final_T.release(); colors.release(); opacity.release();
			rest_sc.release(); rest_q.release(); temp.release();
			if (h_total) cudaFreeHost(h_total);
			h_total = nullptr;
			d_total.release();
			if (ev_total) cudaEventDestroy(ev_total);
			ev_total = nullptr;
			colors_dirty = !h_colors.empty();
			W = H = 0;
			pairs = 0;
		}
	} rs;
	bool obj_shift_valid = false;    // a previous object step set the centroids (boxes usable)
	bool last_sc_limited = false;    // the last step's self-collision build used the box filter
	// wall-clock milliseconds of the upload phases (debug_float "build_ms"): graph, order,
	// state upload, cluster members, cluster lists, sorted copies, rest state, the rest
	double build_ms[8] = {};
	std::chrono::steady_clock::time_point build_t0;
	void build_mark(int phase)
	{
		const auto t = std::chrono::steady_clock::now();
		build_ms[phase] += std::chrono::duration<double, std::milli>(t - build_t0).count();
		build_t0 = t;
	}
	DBuf<float> pos_out3;
	DBuf<int> off, nbr;
	DBuf<float> ndist, nstiff, lam;
	DBuf<int> vol_off, vol_idx, rev_off, rev_idx, mat_type, vol_gs_order;
	DBuf<int> vol_idx_s, rev_idx_s;  // the same lists, rows sorted along the Morton curve
	DBuf<int> gather_order;          // gather group -> node: nodes of similar reverse-list length side by side
	DBuf<float> det_rest, v_rest, rest_len, sigma_rest, lam_vol;
	DBuf<float4> rec;
	DBuf<int2> gs_edge;
	DBuf<float> gs_rest, gs_stiff, gs_lam;
	DBuf<unsigned int> sc_keys;
	DBuf<int> sc_bucket, sc_start, sc_cursor, sc_idx_sorted, sc_contacts, sc_counts, sc_block_sums, d_obj_id;
	// near-pair grid of one-object scenes: keys, bucket counts / starts, (p, index) by bucket
	DBuf<unsigned int> nf_keys;
	DBuf<int> nf_bucket, nf_start;
	DBuf<float4> nf_p;
	int nf_cap = 0;                  // cells of the near-pair grid at most
	DBuf<float4> sc_dp, sc_sp, sc_sr, sc_sx;
	DBuf<float> d_scales, d_rots, d_out_scales, d_out_quats, inv_mass_saved;
	// ellipsoid contact shapes (xpbd_set_contact_shape; forward.cu:150-160, 6733-6757):
	// bit 1 colliders, bit 2 ground; per Gaussian M = k^2 Sigma (two float4), the longest
	// semi-axis and the per-step support radius along the ground normal.  Like the
	// reference's (xpbd_capi.cu:55-56) the setting ends with the scene.
	int contact_bits = 0;
	float contact_tau = 0.2f, contact_cap = 0.0f;
	bool contact_packed = false;
	DBuf<float> d_opacity, c_rmax, c_rg;
	DBuf<float4> c_shape;
	DBuf<int> d_perm;
	DBuf<KinCollider> d_kin_ext;
	DBuf<int2> d_kin_range;
	std::vector<KinCollider> h_kin_sorted;
	std::vector<int2> h_kin_range;
	DBuf<int> att_idx;
	DBuf<float> att_pos;
	bool att_active = false;
	StepParams* d_params = nullptr;
	StepParams* h_params = nullptr;      // current ring slot
	static constexpr int kParamSlots = 8;
	StepParams* h_param_ring = nullptr;  // pinned; a slot is rewritten only after its copy ran
	cudaEvent_t param_ev[kParamSlots] = {};
	int param_next = 0;
	DevCounters* d_ctr = nullptr;
	DevCounters* h_ctr = nullptr;
	static constexpr int kStagingSlots = 4;
	struct Staging { int* idx = nullptr; float* pos = nullptr; int cap = 0; cudaEvent_t ev = nullptr; };
	Staging staging[kStagingSlots];
	int staging_next = 0;

	// ---- press harness (squashStart / the per-step ramp, forward.cu:4311-4396, 12095-12111):
	// two plates on the load axis at the rest extent; one closes at ramp_per_sec up to
	// max_disp, pausing press_dwell_frames at each quarter when autolog is on.  While it
	// runs the ground, gravity, object shape keeping and self-collision are not applied.
	bool press_active = false, press_from_lo = false;
	int press_axis = 1, press_ckpt = 0, press_dwell = 0;
	float press_lo = 0.0f, press_hi = 0.0f, press_cur = 0.0f, press_max = 0.0f, press_ramp = 0.0f;
	static constexpr int kPressDwellFrames = 90;

	void press_reset()
	{
		press_active = false;
		press_cur = 0.0f;
		press_ckpt = 0;
		press_dwell = 0;
	}

	// squashStart (forward.cu:4311-4396) in press mode
	int press_start(int axis, float ramp, float max_disp_pct, bool from_lo)
	{
		if (axis < 0 || axis > 2) axis = 1;
		const float slab = 0.08f;
		max_disp_pct = fmaxf(0.01f, fminf(1.0f, max_disp_pct));
		float lo = FLT_MAX, hi = -FLT_MAX;
		for (int i = 0; i < n; ++i) {
			const float v = in_pos[3 * (size_t)i + axis];
			lo = fminf(lo, v);
			hi = fmaxf(hi, v);
		}
		const float extent = hi - lo;
		const float top = hi - slab * extent, bot = lo + slab * extent;
		int ntop = 0, nbot = 0;
		for (int i = 0; i < n; ++i) {
			const float v = in_pos[3 * (size_t)i + axis];
			if (v >= top) ++ntop;
			else if (v <= bot) ++nbot;
		}
		if (ntop == 0 || nbot == 0) return fail("xpbd_press_start: squashStart failed (empty %d %% slab on axis %d)", 8, axis);
		press_axis = axis;
		press_ramp = ramp;
		press_lo = lo;
		press_hi = hi;
		press_max = max_disp_pct * extent;
		press_from_lo = from_lo;
		press_cur = 0.0f;
		press_ckpt = 0;
		press_dwell = 0;
		press_active = true;
		return 0;
	}

	// the per-step ramp with its checkpoint dwells (forward.cu:12095-12111)
	void press_advance()
	{
		if (!press_active) return;
		static const float ckpt[4] = { 0.25f, 0.50f, 0.75f, 1.00f };
		if (S.press_autolog && press_dwell > 0) {
			if (--press_dwell == 0) ++press_ckpt;
			return;
		}
		press_cur = fminf(press_cur + press_ramp * S.dt, press_max);
		if (S.press_autolog && press_ckpt < 4) {
			const float target = ckpt[press_ckpt] * press_max;
			if (press_cur >= target) {
				press_cur = target;
				press_dwell = kPressDwellFrames;
			}
		}
	}

	// ---- execution ----
	cudaStream_t stream = nullptr;
	bool own_stream = false;
	cudaGraphExec_t graph_exec = nullptr;
	// the same substep as one cooperative launch, and the autotuner that times both forms
	// on the first steps after a capture (they give identical results) and keeps the faster
	// the step forms the autotuner chooses from, all with the same results: 0 the kernel
	// sequence, 1 the fused launch, 2 and 3 the sequence with its distance and volume
	// kernels compiled for 6 and 8 resident blocks per SM
	static constexpr int kForms = 4;
	static constexpr int kFormOcc[kForms] = { 0, 0, 6, 8 };
	cudaGraphExec_t graph_form[kForms] = {};
	long long form_kernels[kForms] = {};
	cudaGraphExec_t& graph_fused = graph_form[1];
	long long& graph_fused_kernels = form_kernels[1];
	static constexpr int kTuneRounds = 3;
	cudaEvent_t tune_ev[kForms * kTuneRounds][2] = {};
	int tune_forms[kForms] = {}, tune_nforms = 0;
	int tune_n = 0, tune_choice = 0;
	bool tune_done = true;
	float tune_ms[kForms] = {};
	int fused_grid = 0;
	void destroy_forms()
	{
		graph_form[0] = nullptr;   // the sequence's graph is graph_exec, destroyed with it
		for (int f = 1; f < kForms; ++f)
			if (graph_form[f]) { cudaGraphExecDestroy(graph_form[f]); graph_form[f] = nullptr; }
	}
	std::vector<long long> graph_key;
	long long graph_kernels = 0;
	long long launches = 0;
	bool profiling = false;
	struct Rec { int stage; cudaEvent_t a, b; };
	std::vector<Rec> prof_records;
	std::vector<cudaEvent_t> event_pool;
	size_t event_next = 0;
	double prof_ms[ST_COUNT] = {};
	long long prof_count[ST_COUNT] = {};

	~Engine() { release(); }

	void release()
	{
		if (graph_exec) cudaGraphExecDestroy(graph_exec);
		graph_exec = nullptr;
		destroy_forms();
		for (auto& pr : tune_ev)
			for (auto& e : pr)
				if (e) { cudaEventDestroy(e); e = nullptr; }
		graph_key.clear();
		free_device();
		if (d_params) cudaFree(d_params);
		for (auto& e : param_ev) if (e) { cudaEventSynchronize(e); cudaEventDestroy(e); e = nullptr; }
		if (h_param_ring) cudaFreeHost(h_param_ring);
		h_param_ring = nullptr;
		if (d_ctr) cudaFree(d_ctr);
		if (h_ctr) cudaFreeHost(h_ctr);
		for (auto& st : staging) {
			if (st.ev) cudaEventSynchronize(st.ev), cudaEventDestroy(st.ev);
			if (st.idx) cudaFreeHost(st.idx);
			if (st.pos) cudaFreeHost(st.pos);
			st = Staging();
		}
		d_params = nullptr; h_params = nullptr; d_ctr = nullptr; h_ctr = nullptr;
		for (auto& e : event_pool) cudaEventDestroy(e);
		event_pool.clear();
		prof_records.clear();
		if (own_stream && stream) cudaStreamDestroy(stream);
		stream = nullptr;
		own_stream = false;
	}

	void free_device()
	{
		pos_curr.release(); pos_next.release(); pos_tmp.release(); vel.release(); pos_rest.release();
		shape_rest.release(); shape_q.release();
		cm_td.release(); cm_flag.release(); cm_mark.release(); cm_work.release(); cm_seed_idx.release();
		cm_spos.release(); cm_stime.release(); cm_seed_delta.release(); cm_time_out.release(); cm_state.release();
		obj_q.release(); obj_shift.release(); obj_sumq.release(); obj_partial.release(); obj_c0.release();
		obj_params.release(); obj_disp.release(); obj_w.release(); obj_boxes.release(); push_partial.release();
		push_T.release(); obj_count.release(); sc_active.release(); sc_cross.release(); sc_accum.release();
		obj_shift_valid = false;
		pos_out3.release(); off.release(); nbr.release(); ndist.release(); nstiff.release(); lam.release();
		vol_off.release(); vol_idx.release(); rev_off.release(); rev_idx.release(); mat_type.release();
		vol_idx_s.release(); rev_idx_s.release(); gather_order.release();
		vol_gs_order.release(); det_rest.release(); v_rest.release(); rest_len.release(); sigma_rest.release();
		lam_vol.release(); rec.release(); gs_edge.release(); gs_rest.release(); gs_stiff.release(); gs_lam.release();
		sc_keys.release(); sc_bucket.release(); sc_start.release(); sc_cursor.release(); sc_idx_sorted.release();
		sc_contacts.release(); sc_counts.release(); sc_block_sums.release(); d_obj_id.release(); sc_dp.release();
		nf_keys.release(); nf_bucket.release(); nf_start.release(); nf_p.release();
		sc_sp.release(); sc_sr.release(); sc_sx.release();
		d_scales.release(); d_rots.release(); d_out_scales.release(); d_out_quats.release(); inv_mass_saved.release();
		d_opacity.release(); c_rmax.release(); c_rg.release(); c_shape.release();
		contact_packed = false;
		att_idx.release(); att_pos.release(); d_perm.release(); d_kin_ext.release(); d_kin_range.release();
		rs.release();
		att_active = false;
		coloring_built = false;
		sc_table = 0;
		built = false;
	}

	int ensure_stream()
	{
		if (!stream) {
			CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
			own_stream = true;
		}
		if (!d_params) {
			CK(cudaMalloc(&d_params, sizeof(StepParams)));
			CK(cudaMallocHost(&h_param_ring, sizeof(StepParams) * kParamSlots));
			for (auto& e : param_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
			h_params = h_param_ring;
			CK(cudaMalloc(&d_ctr, sizeof(DevCounters)));
			CK(cudaMallocHost(&h_ctr, sizeof(DevCounters)));
			CK(cudaMemsetAsync(d_ctr, 0, sizeof(DevCounters), stream));
			memset(h_ctr, 0, sizeof(DevCounters));
		}
		return 0;
	}

	// ------------------------------------------------------------------ build
	// Internal order: device slot r holds the caller's Gaussian perm[r] (Morton order of the
	// rest positions, so that graph, cluster and hash-cell neighbours sit close in memory);
	// inv[perm[r]] = r.  Every topology is built in the caller's index space — the
	// reference's construction order is index-dependent — and only then relabelled, with
	// every list keeping its order, so the kernels see exactly the reference's sequences.
	// 63-bit Morton code of each Gaussian's rest position within the box `lo`..`hi`
	static unsigned long long morton_code(const float* p, const float* lo, const float* hi)
	{
		auto spread = [](unsigned long long v) {
			v &= 0x1fffffull;
			v = (v | v << 32) & 0x1f00000000ffffull;
			v = (v | v << 16) & 0x1f0000ff0000ffull;
			v = (v | v << 8) & 0x100f00f00f00f00full;
			v = (v | v << 4) & 0x10c30c30c30c30c3ull;
			v = (v | v << 2) & 0x1249249249249249ull;
			return v;
		};
		unsigned long long c = 0;
		for (int a = 0; a < 3; ++a) {
			const float ext = hi[a] > lo[a] ? hi[a] - lo[a] : 1.0f;
			float u = (p[a] - lo[a]) / ext;
			if (!std::isfinite(u)) u = 0.0f;
			u = std::min(std::max(u, 0.0f), 1.0f);
			c |= spread((unsigned long long)(u * 2097151.0f)) << a;
		}
		return c;
	}

	// Internal order: objects (graph components) one after another, in the order of their
	// lowest caller index, each along the Morton curve of its own box; a single object
	// gets the Morton order of the scene's box.  Objects that share space (a packed batch)
	// then keep their rows, and the cache lines they gather, to themselves.
	void compute_order()
	{
		perm.resize(n);
		inv.resize(n);
		std::vector<int> parent(n);
		for (int i = 0; i < n; ++i) parent[i] = i;
		auto root = [&](int x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
		for (int i = 0; i < n; ++i)
			for (int e = graph.off[i]; e < graph.off[i + 1]; ++e) {
				const int j = graph.nbr[e];
				if (j < 0 || j >= n) continue;
				const int ri = root(i), rj = root(j);
				if (ri != rj) parent[ri] = rj;
			}
		std::vector<float> clo(3 * (size_t)n, FLT_MAX), chi(3 * (size_t)n, -FLT_MAX);
		std::vector<int> rank(n, -1), comp(n);
		int comps = 0;
		for (int i = 0; i < n; ++i) {
			const int r = root(i);
			comp[i] = r;
			if (rank[r] < 0) rank[r] = comps++;
			for (int a = 0; a < 3; ++a) {
				const float v = in_pos[3 * i + a];
				if (std::isfinite(v)) { clo[3 * r + a] = std::min(clo[3 * r + a], v); chi[3 * r + a] = std::max(chi[3 * r + a], v); }
			}
		}
		// Morton code within each component's own box: also orders the rows of the 4- and
		// 8-lane volume lists the same way whatever the renumbering and whatever other
		// objects share the scene
		lcode.resize(n);
		for (int i = 0; i < n; ++i) {
			const int r = comp[i];
			lcode[i] = morton_code(&in_pos[3 * i], &clo[3 * r], &chi[3 * r]);
		}
		for (int i = 0; i < n; ++i) perm[i] = i;
		if (S.reorder && n > 1)
			std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) {
				const int ra = rank[comp[a]], rb = rank[comp[b]];
				if (ra != rb) return ra < rb;
				return lcode[a] < lcode[b];
			});
		for (int r = 0; r < n; ++r) inv[perm[r]] = r;
	}

	// caller-order CSR (off[N+1], idx) -> internal order, neighbour order kept
	void relabel_csr(const std::vector<int>& off_o, const std::vector<int>& idx_o, std::vector<int>& off_i,
		std::vector<int>& idx_i, std::vector<int>* src_pos = nullptr) const
	{
		off_i.assign(n + 1, 0);
		for (int r = 0; r < n; ++r) off_i[r + 1] = off_i[r] + (off_o[perm[r] + 1] - off_o[perm[r]]);
		idx_i.resize(std::max(off_i[n], 1));
		if (src_pos) src_pos->resize(std::max(off_i[n], 1));
		parallel_for(n, [&](int r0, int r1) {
			for (int r = r0; r < r1; ++r) {
				const int o = perm[r];
				for (int e = off_o[o], d = off_i[r]; e < off_o[o + 1]; ++e, ++d) {
					const int j = idx_o[e];
					idx_i[d] = (j >= 0 && j < n) ? inv[j] : j;
					if (src_pos) (*src_pos)[d] = e;
				}
			}
		});
	}

	template <typename T>
	std::vector<T> to_internal(const T* src, int width) const
	{
		std::vector<T> out((size_t)n * width);
		for (int r = 0; r < n; ++r)
			for (int a = 0; a < width; ++a) out[(size_t)r * width + a] = src[(size_t)perm[r] * width + a];
		return out;
	}

	int upload_positions(const float* pos3, const float* vel3)
	{
		std::vector<float4> p4(n), v4(n);
		for (int r = 0; r < n; ++r) {
			const int o = perm[r];
			p4[r] = make_float4(pos3[3 * o], pos3[3 * o + 1], pos3[3 * o + 2], 1.0f);
			v4[r] = vel3 ? make_float4(vel3[3 * o], vel3[3 * o + 1], vel3[3 * o + 2], 0.0f) : make_float4(0, 0, 0, 0);
		}
		CK(cudaMemcpyAsync(pos_curr.p, p4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(vel.p, v4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(pos_out3.p, pos3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, stream));
		return sync();
	}

	// ensureChainmailGPU (forward.cu:10519-10845): graph upload, colourings, clusters
	int build()
	{
		for (double& v : build_ms) v = 0.0;
		build_t0 = std::chrono::steady_clock::now();
		free_device();
		if (graph_exec) { cudaGraphExecDestroy(graph_exec); graph_exec = nullptr; }
		destroy_forms();
		graph_key.clear();
		if (ensure_stream()) return -1;
		build_graph(n, n_edges, in_edges.data(), in_rest.data(), in_stiff.data(), graph);
		build_mark(0);
		compute_order();
		build_mark(1);
		const int m = graph.off[n];
		CK(d_perm.alloc(n));
		CK(cudaMemcpyAsync(d_perm.p, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream));
		CK(pos_curr.alloc(n)); CK(pos_next.alloc(n)); CK(pos_tmp.alloc(n)); CK(vel.alloc(n)); CK(pos_rest.alloc(n));
		CK(pos_out3.alloc(3 * (size_t)n));
		{
			std::vector<float4> r4(n);
			for (int r = 0; r < n; ++r) {
				const int o = perm[r];
				r4[r] = make_float4(in_pos[3 * o], in_pos[3 * o + 1], in_pos[3 * o + 2], 0.0f);
			}
			CK(cudaMemcpyAsync(pos_rest.p, r4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, stream));
		}
		if (upload_positions(in_pos.data(), nullptr)) return -1;
		{
			std::vector<int> off_i, nbr_i, src;
			relabel_csr(graph.off, graph.nbr, off_i, nbr_i, &src);
			std::vector<float> nd(std::max(m, 1)), ns(std::max(m, 1));
			for (int e = 0; e < m; ++e) { nd[e] = graph.ndist[src[e]]; ns[e] = graph.nstiff[src[e]]; }
			CK(off.alloc(n + 1)); CK(nbr.alloc(std::max(m, 1))); CK(ndist.alloc(std::max(m, 1)));
			CK(nstiff.alloc(std::max(m, 1))); CK(lam.alloc(std::max(m, 1)));
			CK(cudaMemcpyAsync(off.p, off_i.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, stream));
			if (m > 0) {
				CK(cudaMemcpyAsync(nbr.p, nbr_i.data(), sizeof(int) * m, cudaMemcpyHostToDevice, stream));
				CK(cudaMemcpyAsync(ndist.p, nd.data(), sizeof(float) * m, cudaMemcpyHostToDevice, stream));
				CK(cudaMemcpyAsync(nstiff.p, ns.data(), sizeof(float) * m, cudaMemcpyHostToDevice, stream));
			}
			CK(shape_rest.alloc(n)); CK(shape_q.alloc(n));
			CK(cudaMemsetAsync(shape_q.p, 0, shape_q.bytes(), stream));   // zero = identity start
			dev::k_shape_rest<<<blocks_for(n), kBlock, 0, stream>>>(n, pos_rest.p, off.p, nbr.p, shape_rest.p);
			CK(cudaGetLastError());
			CK(cudaStreamSynchronize(stream));
		}
		CK(d_scales.alloc(3 * (size_t)n)); CK(d_rots.alloc(4 * (size_t)n));
		CK(d_out_scales.alloc(3 * (size_t)n)); CK(d_out_quats.alloc(4 * (size_t)n));
		{
			const auto sc = to_internal(in_scales.data(), 3);
			const auto rt = to_internal(in_rots.data(), 4);
			const auto op = to_internal(in_opacity.data(), 1);
			CK(d_opacity.alloc(n));
			CK(cudaMemcpyAsync(d_scales.p, sc.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice, stream));
			CK(cudaMemcpyAsync(d_rots.p, rt.data(), sizeof(float) * 4 * n, cudaMemcpyHostToDevice, stream));
			CK(cudaMemcpyAsync(d_opacity.p, op.data(), sizeof(float) * n, cudaMemcpyHostToDevice, stream));
			CK(cudaStreamSynchronize(stream));
		}
		if (contact_bits && pack_contact(false)) return -1;   // set before the scene was on the device
		CK(det_rest.alloc(n)); CK(v_rest.alloc(n)); CK(rest_len.alloc(n)); CK(sigma_rest.alloc(6 * (size_t)n));
		CK(mat_type.alloc(n)); CK(lam_vol.alloc(n)); CK(rec.alloc(3 * rec_rows()));
		CK(cudaMemsetAsync(rec.p, 0xff, rec.bytes(), stream));   // every record NaN: no record yet
		CK(cudaMemsetAsync(lam_vol.p, 0, lam_vol.bytes(), stream));
		build_components(graph, 50, obj_id, num_objects);
		single_object = std::all_of(obj_id.begin(), obj_id.end(), [&](int v) { return v == obj_id[0]; });
		{
			const auto oi = to_internal(obj_id.data(), 1);
			CK(d_obj_id.alloc(n));
			CK(cudaMemcpyAsync(d_obj_id.p, oi.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream));
			CK(cudaStreamSynchronize(stream));
		}
		if (build_object_cache()) return -1;
		spacing = graph_spacing(graph);
		S.topo_dirty = false;
		if (rebuild_clusters()) return -1;
		CK(cudaStreamSynchronize(stream));
		++generation;
		built = true;
		build_mark(7);
		return 0;
	}

	// rebuildVolumeClusters (forward.cu:9814-10403): host BFS/FPS, then rest covariance on the GPU
	int rebuild_clusters()
	{
		build_mark(2);
		if (S.gpu_builder && n > 0) {
			if (build_members_gpu()) return -1;
		}
		else
			build_clusters(graph, in_pos.data(), S.ring_k, S.max_members, S.leader_min_hop, clusters);
		build_mark(4);
		std::vector<int> voff_i, vidx_i, roff_i, ridx_i;
		relabel_csr(clusters.vol_off, clusters.vol_idx, voff_i, vidx_i);
		relabel_csr(clusters.rev_off, clusters.rev_idx, roff_i, ridx_i);
		CK(vol_off.alloc(n + 1)); CK(vol_idx.alloc(vidx_i.size())); CK(rev_off.alloc(n + 1)); CK(rev_idx.alloc(ridx_i.size()));
		CK(cudaMemcpyAsync(vol_off.p, voff_i.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(vol_idx.p, vidx_i.data(), sizeof(int) * vidx_i.size(), cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(rev_off.p, roff_i.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(rev_idx.p, ridx_i.data(), sizeof(int) * ridx_i.size(), cudaMemcpyHostToDevice, stream));
		{
			// copies of both lists with every row sorted along the Morton curve of the component
			// (caller index breaking ties), for the 4- and 8-lane kernels: the lanes of a cluster
			// read neighbouring Gaussians (fewer cache lines per warp load)
			std::vector<unsigned long long> kcode(n);
			for (int r = 0; r < n; ++r) kcode[r] = lcode[perm[r]];
			auto sorted_rows = [&](const std::vector<int>& off_i, std::vector<int> idx_i) {
				// (code in the component's box, caller index); invalid entries last
				auto less = [&](int a, int b) {
					const bool va = a >= 0 && a < n, vb = b >= 0 && b < n;
					if (!va || !vb) return va && !vb;
					if (kcode[a] != kcode[b]) return kcode[a] < kcode[b];
					return perm[a] < perm[b];
				};
				parallel_for(n, [&](int r0, int r1) {
					for (int r = r0; r < r1; ++r) std::sort(idx_i.begin() + off_i[r], idx_i.begin() + off_i[r + 1], less);
				});
				return idx_i;
			};
			build_mark(4);
			const auto vs = sorted_rows(voff_i, vidx_i);
			const auto rs = sorted_rows(roff_i, ridx_i);
			CK(vol_idx_s.alloc(vs.size())); CK(rev_idx_s.alloc(rs.size()));
			CK(cudaMemcpyAsync(vol_idx_s.p, vs.data(), sizeof(int) * vs.size(), cudaMemcpyHostToDevice, stream));
			CK(cudaMemcpyAsync(rev_idx_s.p, rs.data(), sizeof(int) * rs.size(), cudaMemcpyHostToDevice, stream));
			{
				const std::vector<int> ord = length_order(n, roff_i);
				CK(gather_order.alloc(n));
				CK(cudaMemcpyAsync(gather_order.p, ord.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream));
				CK(cudaStreamSynchronize(stream));
			}
			CK(cudaStreamSynchronize(stream));
			build_mark(5);
		}
		vol_gs_order.release();
		std::vector<int> order_i(clusters.gs_order.size());
		for (size_t t = 0; t < order_i.size(); ++t) order_i[t] = inv[clusters.gs_order[t]];
		if (!order_i.empty()) {
			CK(vol_gs_order.alloc(order_i.size()));
			CK(cudaMemcpyAsync(vol_gs_order.p, order_i.data(), sizeof(int) * order_i.size(), cudaMemcpyHostToDevice,
				stream));
		}
		const int blocks = (n + kBlock - 1) / kBlock;
		dev::k_volume_rest<<<blocks, kBlock, 0, stream>>>(n, pos_rest.p, vol_off.p, vol_idx.p, off.p, nbr.p,
			S.vol_aniso, sigma_rest.p, det_rest.p, v_rest.p, rest_len.p, mat_type.p);
		CK(cudaGetLastError());
		CK(cudaMemsetAsync(lam_vol.p, 0, lam_vol.bytes(), stream));
		CK(cudaStreamSynchronize(stream));
		if (graph_exec) { cudaGraphExecDestroy(graph_exec); graph_exec = nullptr; }
		destroy_forms();
		graph_key.clear();
		++generation;
		build_mark(6);
		return 0;
	}

	// ------------------------------------------------------------------ object mode
	// objectEnsureRestCache (forward.cu:11376-11440): per object (graph component of at
	// least 50) the rest centroid c0 (FP64 sums in caller order, stored as float), the rest
	// offsets q = rest - c0 (float difference widened to FP64), sum q and the count; the
	// previous centroid starts at c0.
	int build_object_cache()
	{
		const int K = num_objects;
		if (K <= 0) return 0;
		std::vector<double> sum(3 * (size_t)K, 0.0);
		std::vector<int> cnt(K, 0);
		for (int i = 0; i < n; ++i) {
			const int id = obj_id[i];
			if (id < 0) continue;
			for (int a = 0; a < 3; ++a) sum[3 * id + a] += in_pos[3 * i + a];
			++cnt[id];
		}
		std::vector<float> c0(3 * (size_t)K);
		std::vector<double> shift(3 * (size_t)K);
		for (int k = 0; k < K; ++k)
			for (int a = 0; a < 3; ++a) {
				c0[3 * k + a] = (float)(sum[3 * k + a] / std::max(cnt[k], 1));
				shift[3 * k + a] = (double)c0[3 * k + a];
			}
		std::vector<double> q(3 * (size_t)n, 0.0), sumq(3 * (size_t)K, 0.0);
		for (int i = 0; i < n; ++i) {
			const int id = obj_id[i];
			if (id < 0) continue;
			const int r = inv[i];
			for (int a = 0; a < 3; ++a) {
				const double v = (double)(in_pos[3 * i + a] - c0[3 * id + a]);
				q[3 * (size_t)r + a] = v;
				sumq[3 * id + a] += v;
			}
		}
		CK(obj_q.alloc(3 * (size_t)n)); CK(obj_shift.alloc(3 * (size_t)K)); CK(obj_sumq.alloc(3 * (size_t)K));
		CK(obj_c0.alloc(3 * (size_t)K)); CK(obj_count.alloc(K)); CK(obj_params.alloc(16 * (size_t)K));
		CK(obj_disp.alloc(K)); CK(obj_w.alloc(n)); CK(obj_boxes.alloc(6 * (size_t)K)); CK(push_T.alloc(4 * (size_t)K));
		CK(obj_partial.alloc((size_t)blocks_for(n).x * K * 16));
		CK(push_partial.alloc((size_t)blocks_for(n).x * K * 4));
		CK(cudaMemcpyAsync(obj_q.p, q.data(), sizeof(double) * q.size(), cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(obj_shift.p, shift.data(), sizeof(double) * shift.size(), cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(obj_sumq.p, sumq.data(), sizeof(double) * sumq.size(), cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(obj_c0.p, c0.data(), sizeof(float) * c0.size(), cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(obj_count.p, cnt.data(), sizeof(int) * K, cudaMemcpyHostToDevice, stream));
		CK(cudaMemsetAsync(obj_params.p, 0, obj_params.bytes(), stream));
		CK(cudaMemsetAsync(obj_disp.p, 0, obj_disp.bytes(), stream));
		dev::k_fill<<<blocks_for(n), kBlock, 0, stream>>>(n, obj_w.p, 1.0f);
		CK(cudaGetLastError());
		obj_shift_valid = false;
		return sync();
	}

	// updateContactShapes (forward.cu:6739-6757): pack every Gaussian's contact ellipsoid
	// from the created shapes (internal order) or from the last deformed shapes that
	// xpbd_compute_shapes wrote (caller order)
	int pack_contact(bool deformed)
	{
		if (!c_shape.p) { CK(c_shape.alloc(2 * (size_t)n)); CK(c_rmax.alloc(n)); CK(c_rg.alloc(n)); }
		const float cap = (std::isfinite(contact_cap) && contact_cap > 0.0f) ? contact_cap : 0.0f;
		dev::k_contact_pack<<<blocks_for(n), kBlock, 0, stream>>>(n, deformed ? d_out_scales.p : d_scales.p,
			deformed ? d_out_quats.p : d_rots.p, deformed ? d_perm.p : (const int*)nullptr, d_opacity.p, contact_tau,
			cap, c_shape.p, c_rmax.p);
		CK(cudaGetLastError());
		contact_packed = true;
		return 0;
	}
	// runXPBDSimulation's contactOn (forward.cu:12223-12228, 12550)
	bool contact_col() const { return (contact_bits & 1) && contact_packed; }
	bool contact_ground() const { return (contact_bits & 2) && contact_packed && S.ground_on; }

	bool object_on() const { return S.object_shape > 0.0f && num_objects > 0 && !press_active; }
	// the self-collision build keeps only Gaussians near another object (forward.cu:11808-11816)
	bool sc_limited() const
	{
		return selfcol_on() && object_on() && !S.sc_within && obj_shift_valid && num_objects >= 1 &&
			num_objects <= dev::kObjMaxK;
	}
	bool obj_push() const { return selfcol_on() && object_on(); }

	int ensure_sc_object_buffers()
	{
		if (!obj_push()) return 0;
		if (!sc_active.p) CK(sc_active.alloc(n));
		if (!sc_cross.p) CK(sc_cross.alloc(n));
		if (!sc_accum.p) CK(sc_accum.alloc(n));
		return 0;
	}

	// object shape keeping after predict (forward.cu:12141-12166, device path 11671-11702);
	// the weighted fit while Gaussians are pinned, the plain fit otherwise or with more
	// than 64 objects (where the reference fits on the host)
	void enqueue_object_step(dim3 G, dim3 B)
	{
		const int K = num_objects;
		const bool weighted = att_active && S.obj_gpu && K <= dev::kObjMaxK;
		const int stride = weighted ? 16 : 12;
		for (int k0 = 0; k0 < K; k0 += dev::kObjMaxK)
			launch(ST_PREDICT, G, B, dev::k_obj_accum, n, (const float4*)pos_next.p, (const int*)d_obj_id.p,
				(const double*)obj_q.p, (const double*)obj_shift.p, K, k0, std::min(dev::kObjMaxK, K - k0),
				weighted ? (const float*)obj_w.p : (const float*)nullptr, stride, obj_partial.p);
		launch(ST_PREDICT, dim3(K), dim3(256), dev::k_obj_solve, (int)G.x, K, (const double*)obj_partial.p, stride,
			(const int*)obj_count.p, (const double*)obj_sumq.p, (const float*)obj_c0.p, obj_shift.p, obj_params.p,
			obj_disp.p);
		if (selfcol_on() && K <= dev::kObjMaxK) {
			launch(ST_PREDICT, dim3((6 * K + 255) / 256), dim3(256), dev::k_obj_boxes_init, K, obj_boxes.p);
			launch(ST_PREDICT, G, B, dev::k_obj_boxes, n, (const float4*)pos_next.p, (const int*)d_obj_id.p, K,
				obj_boxes.p);
		}
		launch(ST_PREDICT, G, B, dev::k_obj_match, n, pos_next.p, (const float4*)pos_rest.p, (const int*)d_obj_id.p,
			(const float*)obj_params.p, S.object_shape);
	}

	// ------------------------------------------------------------------ ChainMail
	// ensureChainmailGPU's time / density upload (forward.cu:10679-10698, 10826): every
	// arrival time 1e9 (not reached), density = opacity.  Allocated on first use.
	int ensure_chainmail()
	{
		if (cm_td.p) return 0;
		const auto dens = to_internal(in_opacity.data(), 1);
		std::vector<float2> td(n);
		for (int i = 0; i < n; ++i) td[i] = make_float2(1e9f, dens[i]);
		CK(cm_td.alloc(n)); CK(cm_flag.alloc(n)); CK(cm_mark.alloc((n + 31) / 32)); CK(cm_work.alloc(n));
		CK(cm_spos.alloc(n)); CK(cm_stime.alloc(n)); CK(cm_time_out.alloc(n)); CK(cm_state.alloc(1));
		CK(cudaMemcpyAsync(cm_td.p, td.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, stream));
		CK(cudaMemsetAsync(cm_flag.p, 0, cm_flag.bytes(), stream));
		CK(cudaMemsetAsync(cm_mark.p, 0, cm_mark.bytes(), stream));
		CK(cudaMemsetAsync(cm_state.p, 0, cm_state.bytes(), stream));
		return sync();
	}

	int cm_publish(float* time_out)
	{
		dev::k_cm_publish<<<blocks_for(n), kBlock, 0, stream>>>(n, pos_curr.p, cm_td.p, d_perm.p, pos_out3.p, time_out);
		CK(cudaGetLastError());
		return 0;
	}

	int chainmail_seed(int count, const int* idx, const float* delta)
	{
		if (ensure_chainmail()) return -1;
		if (count == 0) return 0;
		std::vector<int> ii(count);
		for (int k = 0; k < count; ++k) ii[k] = inv[idx[k]];
		if ((int)cm_seed_idx.n < count) { CK(cm_seed_idx.alloc(count)); CK(cm_seed_delta.alloc(3 * (size_t)count)); }
		CK(cudaMemcpyAsync(cm_seed_idx.p, ii.data(), sizeof(int) * count, cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(cm_seed_delta.p, delta, sizeof(float) * 3 * count, cudaMemcpyHostToDevice, stream));
		dev::k_cm_seed<<<1, 1, 0, stream>>>(count, cm_seed_idx.p, cm_seed_delta.p, pos_curr.p, cm_td.p, cm_flag.p,
			cm_state.p);
		CK(cudaGetLastError());
		if (cm_publish(nullptr)) return -1;
		return sync();
	}

	// runChainmailGPU, dense path (forward.cu:12901-12999): prop_iters propagation
	// sweeps (frontier form), relax_iters relax sweeps and the closing relax sweep
	int chainmail_run(int prop_iters, int relax_iters, float strength, float stiffness, float damping)
	{
		if (ensure_chainmail()) return -1;
		const dev::CmMaterial M = S.cm;
		const dim3 B(kBlock);
		const dim3 G = blocks_for(n);
		const dim3 GS(std::min<unsigned>(G.x, 148u * 8u));   // grid-stride kernels
		for (int it = 0; it < prop_iters; ++it) {
			dev::k_cm_begin<<<1, 1, 0, stream>>>(n, S.cm_frontier ? n / 4 : -1, cm_state.p);
			dev::k_cm_expand<<<GS, B, 0, stream>>>(n, off.p, nbr.p, cm_flag.p, cm_mark.p, cm_work.p, cm_state.p);
			dev::k_cm_sweep<<<GS, B, 0, stream>>>(n, pos_curr.p, cm_td.p, off.p, nbr.p, ndist.p, nstiff.p, cm_work.p,
				cm_state.p, M, strength, cm_spos.p, cm_stime.p);
			dev::k_cm_commit<<<GS, B, 0, stream>>>(n, pos_curr.p, cm_td.p, cm_work.p, cm_spos.p, cm_stime.p, cm_flag.p,
				cm_mark.p, cm_state.p);
			launches += 4;
		}
		float4* a = pos_curr.p;
		float4* b = pos_tmp.p;
		for (int it = 0; it <= relax_iters; ++it) {
			dev::k_cm_relax<<<G, B, 0, stream>>>(n, a, b, cm_td.p, off.p, nbr.p, ndist.p, nstiff.p, M, stiffness, damping);
			++launches;
			std::swap(a, b);
		}
		if (a != pos_curr.p)
			CK(cudaMemcpyAsync(pos_curr.p, a, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream));
		CK(cudaGetLastError());
		if (cm_publish(cm_time_out.p)) return -1;
		return sync();
	}

	// k-ring BFS + farthest-point member list of every node on the GPU (caller index
	// space), in chunks of nodes, gathered into one host CSR; then leader selection (the
	// greedy cover for leader spacing >= 2), the CSRs and colouring on the host
	// (builder.cpp).  A list longer than the kernel's candidate buffer is built on the host.
	int build_members_gpu()
	{
		const int cap = std::max(1, S.max_members);
		const int width = std::min(cap, dev::kBallCap);    // longer balls are the host's
		const int m = graph.off[n];
		DBuf<int> d_off, d_nbr, d_members, d_counts;
		DBuf<float> d_rest3;
		const int chunk = (int)std::max<long long>(1, std::min<long long>(n, (512ll << 20) / (4ll * width)));
		CK(d_off.alloc(n + 1)); CK(d_nbr.alloc(std::max(m, 1))); CK(d_rest3.alloc(3 * (size_t)n));
		CK(d_members.alloc((size_t)chunk * width)); CK(d_counts.alloc(chunk));
		CK(cudaMemcpyAsync(d_off.p, graph.off.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, stream));
		if (m > 0) CK(cudaMemcpyAsync(d_nbr.p, graph.nbr.data(), sizeof(int) * m, cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(d_rest3.p, in_pos.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice, stream));
		CK(cudaFuncSetAttribute(dev::k_build_members, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dev::kBuildSmem));
		std::vector<int> flat((size_t)chunk * width), counts(n);
		std::vector<long long> loff(n + 1, 0);
		std::vector<int> lidx;
		for (int c0 = 0; c0 < n; c0 += chunk) {
			const int c1 = std::min(n, c0 + chunk), cn = c1 - c0;
			const int blocks = std::min((cn + dev::kBuildWarps - 1) / dev::kBuildWarps, 148 * 16);
			dev::k_build_members<<<blocks, dev::kBuildWarps * 32, dev::kBuildSmem, stream>>>(n, c0, c1, d_off.p, d_nbr.p,
				d_rest3.p, S.ring_k, width, d_members.p, d_counts.p);
			CK(cudaGetLastError());
			CK(cudaMemcpyAsync(counts.data() + c0, d_counts.p, sizeof(int) * cn, cudaMemcpyDeviceToHost, stream));
			CK(cudaMemcpyAsync(flat.data(), d_members.p, sizeof(int) * (size_t)cn * width, cudaMemcpyDeviceToHost, stream));
			CK(cudaStreamSynchronize(stream));
			for (int i = c0; i < c1; ++i) {
				const int k = counts[i];   // -1: the ball outgrew the buffer, the host builds the list
				if (k > 0) lidx.insert(lidx.end(), flat.begin() + (size_t)(i - c0) * width,
					flat.begin() + (size_t)(i - c0) * width + k);
				loff[i + 1] = loff[i] + std::max(k, 0);
			}
		}
		build_mark(3);
		build_clusters_from_lists(graph, in_pos.data(), S.ring_k, cap, S.leader_min_hop, loff, lidx, counts, clusters);
		return 0;
	}

	int ensure_coloring()
	{
		if (coloring_built) return 0;
		build_edge_coloring(graph, coloring);
		const size_t ne = coloring.edge.size();
		std::vector<int2> e_i(std::max<size_t>(ne, 1));
		for (size_t e = 0; e < ne; ++e) e_i[e] = make_int2(inv[coloring.edge[e].x], inv[coloring.edge[e].y]);
		CK(gs_edge.alloc(std::max<size_t>(ne, 1))); CK(gs_rest.alloc(std::max<size_t>(ne, 1)));
		CK(gs_stiff.alloc(std::max<size_t>(ne, 1))); CK(gs_lam.alloc(std::max<size_t>(ne, 1)));
		if (ne) {
			CK(cudaMemcpyAsync(gs_edge.p, e_i.data(), sizeof(int2) * ne, cudaMemcpyHostToDevice, stream));
			CK(cudaMemcpyAsync(gs_rest.p, coloring.rest.data(), sizeof(float) * ne, cudaMemcpyHostToDevice, stream));
			CK(cudaMemcpyAsync(gs_stiff.p, coloring.stiff.data(), sizeof(float) * ne, cudaMemcpyHostToDevice, stream));
		}
		CK(cudaStreamSynchronize(stream));
		coloring_built = true;
		if (graph_exec) { cudaGraphExecDestroy(graph_exec); graph_exec = nullptr; }
		destroy_forms();
		graph_key.clear();
		return 0;
	}

	// selfColEnsureBuffers (forward.cu:11728-11758): table = pow2 >= max(1024, 2N)
	int ensure_selfcol()
	{
		if (sc_table) return 0;
		int table = 1024;
		while (table < 2 * n) table <<= 1;
		sc_table = table;
		const int buckets = table + 1;   // + sentinel bucket
		CK(sc_keys.alloc(n)); CK(sc_bucket.alloc(buckets + 1)); CK(sc_start.alloc(buckets + 1));
		CK(sc_cursor.alloc(buckets)); CK(sc_idx_sorted.alloc(n)); CK(sc_contacts.alloc((size_t)n * kSelfColMax));
		nf_cap = std::max(4096, 2 * n);
		CK(nf_keys.alloc(n)); CK(nf_bucket.alloc(nf_cap + 1)); CK(nf_start.alloc(nf_cap + 2)); CK(nf_p.alloc(n));
		CK(sc_block_sums.alloc((std::max(buckets, nf_cap) + 2 + 1023) / 1024 + 1));
		CK(cudaMemsetAsync(nf_bucket.p, 0, nf_bucket.bytes(), stream));
		CK(sc_counts.alloc(n)); CK(sc_dp.alloc(n)); CK(sc_sp.alloc(n)); CK(sc_sr.alloc(n)); CK(sc_sx.alloc(n));
		CK(cudaMemsetAsync(sc_counts.p, 0, sc_counts.bytes(), stream));
		return 0;
	}

	// ------------------------------------------------------------------ params
	int upload_params()
	{
		CK(cudaEventSynchronize(param_ev[param_next]));
		h_params = h_param_ring + param_next;
		fill_params();
		CK(cudaMemcpyAsync(d_params, h_params, sizeof(StepParams), cudaMemcpyHostToDevice, stream));
		CK(cudaEventRecord(param_ev[param_next], stream));
		param_next = (param_next + 1) % kParamSlots;
		return 0;
	}

	// batched colliders: stable-sorted by object, one [begin, end) range per object id
	int upload_ext_colliders()
	{
		if (S.kin_ext.empty()) return 0;
		const int count = (int)S.kin_ext.size();
		int objects = 0;
		for (const auto& k : S.kin_ext) objects = std::max(objects, k.obj + 1);
		h_kin_sorted.assign(S.kin_ext.begin(), S.kin_ext.end());
		std::stable_sort(h_kin_sorted.begin(), h_kin_sorted.end(),
			[](const KinCollider& a, const KinCollider& b) { return a.obj < b.obj; });
		h_kin_range.assign(std::max(objects, 1), make_int2(0, 0));
		for (int c = 0; c < count; ++c) {
			const int o = h_kin_sorted[c].obj;
			if (o < 0) continue;
			if (h_kin_range[o].y == 0) h_kin_range[o].x = c;
			h_kin_range[o].y = c + 1;
			h_kin_sorted[c].obj = -1;   // selected by range; no per-collider filter on the device
		}
		if ((int)d_kin_ext.n < count || (int)d_kin_range.n < (int)h_kin_range.size()) {
			CK(cudaStreamSynchronize(stream));
			CK(d_kin_ext.alloc(std::max<size_t>(count, 64)));
			CK(d_kin_range.alloc(std::max<size_t>(h_kin_range.size(), 64)));
			if (graph_exec) { cudaGraphExecDestroy(graph_exec); graph_exec = nullptr; }
			destroy_forms();
			graph_key.clear();
		}
		CK(cudaMemcpyAsync(d_kin_ext.p, h_kin_sorted.data(), sizeof(KinCollider) * count, cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(d_kin_range.p, h_kin_range.data(), sizeof(int2) * h_kin_range.size(),
			cudaMemcpyHostToDevice, stream));
		return 0;
	}

	void fill_params()
	{
		StepParams& P = *h_params;
		memset(&P, 0, sizeof(P));
		P.dt = S.dt;
		P.inv_mass_scale = S.inv_mass_scale;
		P.stiffness_scale = S.stiffness_scale;
		P.under_relax = S.under_relax;
		P.dist_compliance = S.dist_compliance;
		P.vol_compliance = S.vol_compliance;
		P.shape_compliance = S.shape_compliance;
		P.shape_blend = S.shape_blend;
		P.vel_damping = S.vel_damping;
		// stepPhysicsOnly gravity: -g * n when g > 0 and no press runs (forward.cu:13257-13259)
		if (S.ground_gravity > 0.0f && !press_active) {
			P.gx = -S.ground_gravity * S.ground_n[0];
			P.gy = -S.ground_gravity * S.ground_n[1];
			P.gz = -S.ground_gravity * S.ground_n[2];
		}
		P.ground_on = (S.ground_on && !press_active) ? 1 : 0;   // groundOn (forward.cu:12140)
		P.press_on = press_active ? 1 : 0;
		P.press_axis = press_axis;
		P.press_lo = press_lo + ((press_active && press_from_lo) ? press_cur : 0.0f);
		P.press_hi = press_hi - ((press_active && !press_from_lo) ? press_cur : 0.0f);
		for (int k = 0; k < 3; ++k) P.gn[k] = S.ground_n[k];
		P.ground_plane = S.ground_h + S.ground_radius;
		P.ground_slop = S.ground_slop;
		P.ground_friction = S.ground_friction;
		P.ground_restitution = S.ground_restitution;
		P.resting_speed = 2.0f * S.ground_gravity * S.dt;
		P.kin_count = S.kin_count;
		P.kin_margin = S.kin_margin;
		P.kin_friction = S.kin_friction;
		memcpy(P.kin, S.kin, sizeof(KinCollider) * S.kin_count);
		P.kin_filtered = 0;
		P.kin_ext_ranges = (int)h_kin_range.size();
		for (int c = 0; c < S.kin_count; ++c) {
			P.kin[c].obj = S.kin_obj[c];
			if (S.kin_obj[c] >= 0) P.kin_filtered = 1;
		}
		// selfColBuild constants (forward.cu:11798-11831), host float arithmetic
		const float dc = S.sc_radius_scale * spacing;
		const float search = S.sc_search_scale * dc;
		const float excl = S.sc_exclude_scale * dc;
		P.sc_dc = dc;
		P.sc_search = search;
		P.sc_excl2 = excl * excl;
		P.sc_cross_excl2 = dc * dc;
		P.sc_fast_rel = S.sc_fast_rel * dc;
		P.sc_search_plus16dc = search + 16.0f * dc;
		P.sc_within = S.sc_within ? 1 : 0;
		P.sc_single_object = single_object ? 1 : 0;
	}

	// the c.z column of the cluster records (after the 2 x rows float4 of M and c.xy; rows =
	// the scene's Gaussians, or an arena's capacity)
	float* recz() const { return reinterpret_cast<float*>(rec.p + 2 * rec_rows()); }
	// record slots: the rows rounded up to a multiple of 8
	size_t rec_rows() const { return ((size_t)(arena ? rows_cap : n) + 7) & ~(size_t)7; }

	bool use_warp() const
	{
		if (S.warp_mode == 2) return true;
		if (S.warp_mode == 1) return false;
		return clusters.avg_members >= 40.0f;
	}
	bool selfcol_on() const
	{
		return S.sc_enabled && spacing > 0.0f && S.sc_radius_scale * spacing > 0.0f && !press_active;
	}
	bool dist_gs_on() const { return S.use_distance && S.dist_gs && coloring_built && !coloring.edge.empty(); }
	bool vol_gs_on() const { return S.use_volume && S.vol_gs && clusters.gs_color_off.size() > 1; }

	std::vector<long long> topology_key() const
	{
		return { (long long)generation, S.iters, S.use_distance, dist_gs_on(), S.use_volume, vol_gs_on(), vol_lanes(), gather_lanes(),
			S.use_shape, S.shape_robust, selfcol_on(), S.kin_count > 0 || S.ground_on || selfcol_on() || press_active, S.jstats,
			(long long)S.kin_ext.empty(), (long long)(size_t)d_kin_ext.p,
			(long long)coloring.color_off.size(), (long long)clusters.gs_color_off.size(), (long long)sc_table,
			object_on(), att_active && S.obj_gpu, sc_limited(), obj_push(), contact_col(), contact_ground(),
			selfcol_on() && sc_near_on() };
	}

	// ------------------------------------------------------------------ launching
	template <typename K, typename... A>
	void launch(int stage, dim3 grid, dim3 block, K kernel, A... args)
	{
		cudaEvent_t a = nullptr, b = nullptr;
		if (profiling) {
			a = next_event();
			b = next_event();
			cudaEventRecord(a, stream);
		}
		kernel<<<grid, block, 0, stream>>>(args...);
		++launches;
		if (profiling) {
			cudaEventRecord(b, stream);
			prof_records.push_back({ stage, a, b });
		}
	}
	cudaEvent_t next_event()
	{
		if (event_next == event_pool.size()) {
			cudaEvent_t e;
			cudaEventCreate(&e);
			event_pool.push_back(e);
		}
		return event_pool[event_next++];
	}
	static dim3 blocks_for(long long items, int per_block = kBlock)
	{
		return dim3((unsigned)((items + per_block - 1) / per_block));
	}

	bool sc_near_on() const { return S.sc_near && single_object; }

	// The once-per-step self-collision build (selfColBuild, forward.cu:11796-11849): cell
	// size from the largest predicted displacement, then the candidate lists.  One-object
	// scenes take the near-pair grid (k_sc_build_near); otherwise the reference's hash of
	// the start positions, its stable counting sort and the 27-cell scan.  ref_structure
	// also builds the hash / sorted order / cell ranges when the near-pair grid is used
	// (the stage check reads them).
	int enqueue_sc_build(const unsigned char* active, bool ref_structure = false)
	{
		const int N = n;
		const dim3 B(kBlock), G = blocks_for(N);
		const int buckets = sc_table + 1, scan_n = buckets + 1, nb = (scan_n + 1023) / 1024;
		const unsigned mask = (unsigned)(sc_table - 1);
		const bool near = sc_near_on();
		// displacement max (and, for the near-pair grid, the box of the predicted positions)
		launch(ST_SC_BUILD, dim3(std::min<unsigned>(G.x, 148u * 8u)), B, dev::k_sc_disp, N, (const float4*)pos_curr.p,
			(const float4*)pos_next.p, d_ctr, active, near ? 1 : 0);
		launch(ST_SC_BUILD, dim3(1), dim3(1), dev::k_sc_setup, (const StepParams*)d_params, d_ctr);
		if (!near || ref_structure) {
			CK(cudaMemsetAsync(sc_bucket.p, 0, sc_bucket.bytes(), stream));
			CK(cudaMemsetAsync(sc_cursor.p, 0, sc_cursor.bytes(), stream));
			launch(ST_SC_BUILD, G, B, dev::k_sc_keys, N, (const float4*)pos_curr.p, (const DevCounters*)d_ctr, mask,
				(unsigned)sc_table, sc_keys.p, sc_bucket.p, active);
			launch(ST_SC_BUILD, dim3(nb), dim3(1024), dev::k_scan_blocks, (const int*)sc_bucket.p, sc_start.p, scan_n,
				sc_block_sums.p);
			launch(ST_SC_BUILD, dim3(1), dim3(1024), dev::k_scan_sums, sc_block_sums.p, nb);
			launch(ST_SC_BUILD, dim3(nb), dim3(1024), dev::k_scan_add, sc_start.p, scan_n, (const int*)sc_block_sums.p);
			launch(ST_SC_BUILD, G, B, dev::k_sc_scatter, N, (const unsigned*)sc_keys.p, (const int*)sc_start.p,
				sc_cursor.p, sc_idx_sorted.p);
			launch(ST_SC_BUILD, blocks_for(buckets), B, dev::k_sc_order, buckets, (const int*)sc_start.p,
				sc_idx_sorted.p, (const int*)d_perm.p);
		}
		if (near) {
			// dense grid of the predicted positions: cell size, counts, starts, scatter
			const int fscan = nf_cap + 1, fnb = (fscan + 1023) / 1024;
			launch(ST_SC_BUILD, dim3(1), dim3(1), dev::k_sc_near_setup, (const StepParams*)d_params, d_ctr, nf_cap);
			CK(cudaMemsetAsync(nf_bucket.p, 0, nf_bucket.bytes(), stream));
			launch(ST_SC_BUILD, G, B, dev::k_sc_near_keys, N, (const float4*)pos_curr.p, (const float4*)pos_next.p,
				active, (const DevCounters*)d_ctr, nf_keys.p, nf_bucket.p);
			launch(ST_SC_BUILD, dim3(fnb), dim3(1024), dev::k_scan_blocks, (const int*)nf_bucket.p, nf_start.p, fscan,
				sc_block_sums.p);
			launch(ST_SC_BUILD, dim3(1), dim3(1024), dev::k_scan_sums, sc_block_sums.p, fnb);
			launch(ST_SC_BUILD, dim3(fnb), dim3(1024), dev::k_scan_add, nf_start.p, fscan, (const int*)sc_block_sums.p);
			launch(ST_SC_BUILD, G, B, dev::k_sc_near_scatter, N, (const unsigned*)nf_keys.p, (const int*)nf_start.p,
				nf_bucket.p, (const float4*)pos_next.p, nf_p.p, sc_counts.p);
			launch(ST_SC_BUILD, G, B, dev::k_sc_build_near, N, (const StepParams*)d_params, (const float4*)pos_curr.p,
				(const float4*)pos_next.p, (const float4*)pos_rest.p, active, (const int*)nf_start.p, mask,
				(const float4*)nf_p.p, (const int*)d_perm.p, d_ctr, sc_contacts.p, sc_counts.p);
			return 0;
		}
		launch(ST_SC_BUILD, G, B, dev::k_sc_pack, N, (const int*)sc_idx_sorted.p, (const float4*)pos_curr.p,
			(const float4*)pos_next.p, (const float4*)pos_rest.p, (const int*)d_obj_id.p, sc_sp.p, sc_sr.p, sc_sx.p);
		launch(ST_SC_BUILD, G, B, dev::k_sc_build_sorted, N, (const StepParams*)d_params, (const float4*)pos_curr.p,
			(const float4*)pos_next.p, (const float4*)pos_rest.p, (const int*)sc_idx_sorted.p, (const int*)sc_start.p,
			mask, (const int*)d_obj_id.p, (const float4*)sc_sp.p, (const float4*)sc_sr.p, (const float4*)sc_sx.p,
			d_ctr, sc_contacts.p, sc_counts.p, active);
		return 0;
	}

	// volume kernel shapes: lanes per cluster (Kernel A) and per node (Kernel B);
	// 0 = one thread per cluster / node
	int vol_lanes() const
	{
		if (S.warp_mode == 2) return 32;
		if (S.warp_mode == 1) return 0;
		if (S.lanes_a > 0) return S.lanes_a;
		return 4;   // measured best on B200 for 10-64 members (sweep of 2/4/8/32)
	}
	int gather_lanes() const
	{
		if (S.warp_mode == 2) return 32;
		if (S.warp_mode == 1) return 0;
		if (S.lanes_b > 0) return S.lanes_b;
		return 4;
	}

	// the substep forms the fused launch covers (dev::k_substep_fused)
	bool fused_eligible() const
	{
		return !selfcol_on() && !object_on() && !dist_gs_on() && !vol_gs_on() &&
			(!S.use_volume || (vol_lanes() == 4 && S.lanes_a == 0 && gather_lanes() == 4)) && !S.use_angle && n > 0;
	}

	// one step as a single cooperative launch (results identical to enqueue_step's sequence)
	int enqueue_step_fused()
	{
		if (!fused_grid) {
			int dev_id = 0, sms = 0, per_sm = 0;
			CK(cudaGetDevice(&dev_id));
			CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id));
			CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_substep_fused, kBlock, 0));
			if (per_sm <= 0) return fail("fused substep: no block of the kernel fits an SM");
			fused_grid = sms * per_sm;
		}
		const int grid = (int)std::max<long long>(1, std::min<long long>(fused_grid, ((long long)n * 4 + kBlock - 1) / kBlock));
		const bool cc = contact_col(), cg = contact_ground();
		dev::SubstepArgs A;
		memset(&A, 0, sizeof(A));
		A.n = n; A.iters = S.iters; A.use_distance = S.use_distance; A.use_volume = S.use_volume;
		A.use_shape = S.use_shape; A.shape_robust = S.shape_robust;
		A.project = S.kin_count > 0 || !S.kin_ext.empty() || S.ground_on || press_active;
		A.P = d_params;
		A.pos_curr = pos_curr.p; A.pos_next = pos_next.p; A.pos_tmp = pos_tmp.p; A.vel = vel.p; A.lam_vol = lam_vol.p;
		A.cshape = (cc || cg) ? c_shape.p : nullptr; A.crmax = cc ? c_rmax.p : nullptr; A.crg = cg ? c_rg.p : nullptr;
		A.off = off.p; A.nbr = nbr.p; A.ndist = ndist.p; A.nstiff = nstiff.p; A.lam = lam.p;
		A.vol_off = vol_off.p; A.vol_idx = vol_idx_s.p; A.mat_type = mat_type.p; A.rev_off = rev_off.p;
		A.rev_idx = rev_idx_s.p; A.det_rest = det_rest.p; A.rest_len = rest_len.p; A.rec = rec.p; A.recz = recz();
		A.pos_rest = pos_rest.p; A.shape_rest = shape_rest.p; A.shape_q = shape_q.p; A.ctr = d_ctr;
		A.obj_id = d_obj_id.p; A.ext_kin = S.kin_ext.empty() ? nullptr : d_kin_ext.p; A.ext_range = d_kin_range.p;
		A.pos_out3 = pos_out3.p; A.perm = d_perm.p;
		CK(cudaMemsetAsync(d_ctr, 0, offsetof(DevCounters, jstats), stream));
		cudaLaunchConfig_t cfg = {};
		cfg.gridDim = dim3(grid);
		cfg.blockDim = dim3(kBlock);
		cfg.stream = stream;
		cudaLaunchAttribute attr[1];
		attr[0].id = cudaLaunchAttributeCooperative;
		attr[0].val.cooperative = 1;
		cfg.attrs = attr;
		cfg.numAttrs = 1;
		CK(cudaLaunchKernelEx(&cfg, dev::k_substep_fused, A));
		++launches;
		if (S.jstats) {
			CK(cudaMemsetAsync(d_ctr->jstats, 0, sizeof(double) * 3, stream));
			launch(ST_JSTATS, blocks_for(n), dim3(kBlock), dev::k_jstats, n, (const float4*)pos_curr.p,
				(const int*)vol_off.p, (const int*)vol_idx.p, (const float*)det_rest.p, (const int*)mat_type.p,
				(const float*)v_rest.p, d_ctr);
		}
		CK(cudaGetLastError());
		return 0;
	}

	// one step's kernel sequence (the body of runXPBDSimulation); occ = 6 or 8 launches the
	// distance and default volume kernels compiled for that many blocks per SM
	int enqueue_step(int occ = 0)
	{
		const int N = n;
		const dim3 B(kBlock), G = blocks_for(N);
		const dim3 GW = blocks_for((long long)N * 32);   // one warp per Gaussian / cluster
		const bool sc = selfcol_on();
		CK(cudaMemsetAsync(d_ctr, 0, offsetof(DevCounters, jstats), stream));
		const bool cc = contact_col(), cg = contact_ground();
		const float4* cshape = (cc || cg) ? (const float4*)c_shape.p : (const float4*)nullptr;
		const float* crmax = cc ? (const float*)c_rmax.p : (const float*)nullptr;
		const float* crg = cg ? (const float*)c_rg.p : (const float*)nullptr;
		launch(ST_PREDICT, G, B, dev::k_predict, N, (const StepParams*)d_params, (const float4*)pos_curr.p, pos_next.p,
			vel.p, S.use_volume ? lam_vol.p : (float*)nullptr, cshape, cg ? c_rg.p : (float*)nullptr);
		if (object_on()) enqueue_object_step(G, B);
		const unsigned char* active = sc_limited() ? (const unsigned char*)sc_active.p : nullptr;
		if (sc) {
			if (active)
				launch(ST_SC_BUILD, G, B, dev::k_sc_active, N, (const StepParams*)d_params, (const float4*)pos_curr.p,
					(const float4*)pos_next.p, (const int*)d_obj_id.p, (const float*)obj_boxes.p,
					(const float*)obj_disp.p, num_objects, sc_active.p, d_ctr);
			if (enqueue_sc_build(active)) return -1;
			if (obj_push()) CK(cudaMemsetAsync(sc_accum.p, 0, sc_accum.bytes(), stream));
		}
		float4* pin = pos_next.p;
		float4* pout = pos_tmp.p;
		const bool dgs = dist_gs_on(), vgs = vol_gs_on();
		const bool project = S.kin_count > 0 || !S.kin_ext.empty() || S.ground_on || sc || press_active;
		for (int it = 0; it < S.iters; ++it) {
			const int first = (it == 0), last = (it == S.iters - 1);
			if (dgs) {
				for (size_t c = 0; c + 1 < coloring.color_off.size(); ++c) {
					const int begin = coloring.color_off[c], count = coloring.color_off[c + 1] - begin;
					if (count <= 0) continue;
					launch(ST_DISTANCE, blocks_for(count), B, dev::k_distance_gs, begin, count, N,
						(const StepParams*)d_params, pin, (const int2*)gs_edge.p, (const float*)gs_rest.p,
						(const float*)gs_stiff.p, gs_lam.p, first ? 0 : 1);
				}
			}
			else if (S.use_distance) {
				auto k = occ == 8 ? dev::k_distance_occ<8> : occ == 6 ? dev::k_distance_occ<6> : dev::k_distance_jacobi;
				launch(ST_DISTANCE, G, B, k, N, (const StepParams*)d_params, (const float4*)pin,
					pout, (const int*)off.p, (const int*)nbr.p, (const float*)ndist.p, (const float*)nstiff.p, lam.p,
					first ? 0 : 1, last ? 0 : 1);
				std::swap(pin, pout);
			}
			if (S.use_volume) {
				if (vgs) {
					for (size_t c = 0; c + 1 < clusters.gs_color_off.size(); ++c) {
						const int begin = clusters.gs_color_off[c], count = clusters.gs_color_off[c + 1] - begin;
						if (count <= 0) continue;
						launch(ST_VOL_GS, blocks_for(count, 64), dim3(64), dev::k_volume_gs, begin, count,
							(const int*)vol_gs_order.p, N, (const StepParams*)d_params, pin, (const int*)vol_off.p,
							(const int*)vol_idx.p, (const float*)det_rest.p, (const int*)mat_type.p, lam_vol.p,
							(const float*)rest_len.p, 1);
					}
				}
				else {
					const int la = vol_lanes(), lb = gather_lanes();
					const int rl = first ? 0 : 1;
					const StepParams* dp = d_params;
					const float4* cpin = pin;
					if (la == 4 && S.lanes_a == 0)
						// automatic: one pass over the members (any count), 4 lanes per cluster
						launch(ST_VOL_SOLVE, blocks_for((long long)N * 4), B,
							occ == 8 ? dev::k_volume_solve_occ<4, 8> : occ == 6 ? dev::k_volume_solve_occ<4, 6>
							: dev::k_volume_solve_onepass<4>, N, dp, cpin,
							(const int*)vol_off.p, (const int*)vol_idx_s.p, (const float*)det_rest.p,
							(const int*)mat_type.p, lam_vol.p, rec.p, recz(), rl);
					else if (la == 32)
						launch(ST_VOL_SOLVE, blocks_for((long long)N * 32), B, dev::k_volume_solve_group<32, 8>, N, dp, cpin,
							(const int*)vol_off.p, (const int*)vol_idx.p, (const float*)det_rest.p, (const int*)mat_type.p,
							lam_vol.p, rec.p, recz(), rl);
					else if (la == 8)
						launch(ST_VOL_SOLVE, blocks_for((long long)N * 8), B, dev::k_volume_solve_slots<8, 8, true>, N, dp,
							cpin, (const int*)vol_off.p, (const int*)vol_idx_s.p, (const float*)det_rest.p,
							(const int*)mat_type.p, lam_vol.p, rec.p, recz(), rl);
					else if (la == 4)   // 4 lanes, members staged in shared memory (two-pass sums)
						launch(ST_VOL_SOLVE, blocks_for((long long)N * 4, dev::kSmemBlock), dim3(dev::kSmemBlock),
							dev::k_volume_solve_smem<4, 16>, N, dp, cpin, (const int*)vol_off.p, (const int*)vol_idx_s.p,
							(const float*)det_rest.p, (const int*)mat_type.p, lam_vol.p, rec.p, recz(), rl);
					else if (la == 3)   // 4 lanes, positions re-read from L1 instead of shared memory
						launch(ST_VOL_SOLVE, blocks_for((long long)N * 4), B, dev::k_volume_solve_slots<4, 16, false>, N, dp,
							cpin, (const int*)vol_off.p, (const int*)vol_idx_s.p, (const float*)det_rest.p,
							(const int*)mat_type.p, lam_vol.p, rec.p, recz(), rl);
					else if (la == 2)
						launch(ST_VOL_SOLVE, blocks_for((long long)N * 2), B, dev::k_volume_solve_slots<2, 32, false>, N, dp,
							cpin, (const int*)vol_off.p, (const int*)vol_idx_s.p, (const float*)det_rest.p,
							(const int*)mat_type.p, lam_vol.p, rec.p, recz(), rl);
					else
						launch(ST_VOL_SOLVE, G, B, dev::k_volume_solve_thread, N, dp, cpin, (const int*)vol_off.p,
							(const int*)vol_idx.p, (const float*)det_rest.p, (const int*)mat_type.p, lam_vol.p, rec.p, recz(), rl);
					if (lb == 32)
						launch(ST_VOL_GATHER, blocks_for((long long)N * 32), B, dev::k_volume_gather_group<32>, N, dp, cpin,
							pout, (const int*)rev_off.p, (const int*)rev_idx.p, (const float4*)rec.p, (const float*)recz(), (const float*)rest_len.p, (const int*)gather_order.p);
					else if (lb == 8)
						launch(ST_VOL_GATHER, blocks_for((long long)N * 8), B, dev::k_volume_gather_group<8>, N, dp, cpin,
							pout, (const int*)rev_off.p, (const int*)rev_idx_s.p, (const float4*)rec.p, (const float*)recz(), (const float*)rest_len.p, (const int*)gather_order.p);
					else if (lb == 4)
						launch(ST_VOL_GATHER, blocks_for((long long)N * 4), B,
							occ == 8 ? dev::k_volume_gather_occ<4, 8> : occ == 6 ? dev::k_volume_gather_occ<4, 6>
							: dev::k_volume_gather_group<4>, N, dp, cpin,
							pout, (const int*)rev_off.p, (const int*)rev_idx_s.p, (const float4*)rec.p, (const float*)recz(), (const float*)rest_len.p, (const int*)gather_order.p);
					else
						launch(ST_VOL_GATHER, G, B, dev::k_volume_gather_thread, N, dp, cpin, pout, (const int*)rev_off.p,
							(const int*)rev_idx.p, (const float4*)rec.p, (const float*)recz(), (const float*)rest_len.p);
					std::swap(pin, pout);
				}
			}
			if (S.use_shape) {
				if (S.shape_robust)
					launch(ST_SHAPE, G, B, dev::k_shape_match<true>, N, (const StepParams*)d_params, (const float4*)pin,
						pout, (const float4*)pos_rest.p, (const int*)off.p, (const int*)nbr.p,
						(const float4*)shape_rest.p, shape_q.p);
				else
					launch(ST_SHAPE, G, B, dev::k_shape_match<false>, N, (const StepParams*)d_params, (const float4*)pin,
						pout, (const float4*)pos_rest.p, (const int*)off.p, (const int*)nbr.p,
						(const float4*)shape_rest.p, shape_q.p);
				std::swap(pin, pout);
			}
			if (sc)
				launch(ST_SC_SOLVE, G, B, dev::k_sc_solve, N, (const StepParams*)d_params, (const float4*)pin,
					(const float4*)pos_curr.p, (const float4*)pos_rest.p, (const int*)sc_contacts.p,
					(const int*)sc_counts.p, (const DevCounters*)d_ctr, sc_dp.p,
					obj_push() ? sc_cross.p : (float4*)nullptr);
			if (project)
				launch(ST_PROJECT, G, B, dev::k_project, N, (const StepParams*)d_params, pin, (const float4*)pos_curr.p,
					sc ? (const int*)sc_counts.p : (const int*)nullptr, (const float4*)sc_dp.p, d_ctr, last ? 1 : 0,
					(const int*)d_obj_id.p, S.kin_ext.empty() ? (const KinCollider*)nullptr : (const KinCollider*)d_kin_ext.p,
					(const int2*)d_kin_range.p, (const float4*)sc_cross.p, obj_push() ? sc_accum.p : (float4*)nullptr,
					cshape, crmax, crg);
		}
		if (obj_push()) {   // contact push (forward.cu:12587-12597)
			const int K = num_objects;
			for (int k0 = 0; k0 < K; k0 += dev::kObjMaxK)
				launch(ST_PROJECT, G, B, dev::k_obj_push_sum, N, (const int*)d_obj_id.p, (const float4*)sc_accum.p, K, k0,
					std::min(dev::kObjMaxK, K - k0), (const DevCounters*)d_ctr, push_partial.p);
			launch(ST_PROJECT, dim3((K + 63) / 64), dim3(64), dev::k_obj_push_solve, (int)G.x, K,
				(const float*)push_partial.p, (const DevCounters*)d_ctr, S.object_shape, push_T.p);
			launch(ST_PROJECT, G, B, dev::k_obj_push_apply, N, (const StepParams*)d_params, (const int*)d_obj_id.p,
				(const float4*)sc_accum.p, (const float*)push_T.p, (const DevCounters*)d_ctr, pin, crg);
		}
		launch(ST_VELOCITY, G, B, dev::k_velocity, N, (const StepParams*)d_params, pos_curr.p, (const float4*)pin,
			vel.p, pos_out3.p, (const int*)d_perm.p, crg);
		if (S.jstats) {
			CK(cudaMemsetAsync(d_ctr->jstats, 0, sizeof(double) * 3, stream));
			launch(ST_JSTATS, G, B, dev::k_jstats, N, (const float4*)pos_curr.p, (const int*)vol_off.p,
				(const int*)vol_idx.p, (const float*)det_rest.p, (const int*)mat_type.p, (const float*)v_rest.p,
				d_ctr);
		}
		CK(cudaGetLastError());
		return 0;
	}

	// ------------------------------------------------------------------ step
	int step_async()
	{
		if (!built) {
			if (build()) return -1;
		}
		else if (S.topo_dirty) {
			S.topo_dirty = false;
			if (rebuild_clusters()) return -1;
		}
		if (S.use_distance && S.dist_gs && ensure_coloring()) return -1;
		if (S.sc_enabled && ensure_selfcol()) return -1;
		if (ensure_sc_object_buffers()) return -1;
		const bool sc_limited_now = sc_limited();
		if (upload_ext_colliders()) return -1;   // sets the object ranges fill_params reads
		press_advance();
		if (upload_params()) return -1;
		if (profiling || !S.use_graph) {
			// eager launches (per-kernel events in profiling mode): the chosen sequence form
			if (enqueue_step(kFormOcc[tune_choice == 1 ? 0 : tune_choice])) return -1;
		}
		else {
			auto key = topology_key();
			key.push_back(S.fused);
			if (!graph_exec || key != graph_key) {
				if (graph_exec) { cudaGraphExecDestroy(graph_exec); graph_exec = nullptr; }
				destroy_forms();
				if (capture(0, &graph_exec, &graph_kernels)) return -1;
				graph_form[0] = graph_exec;
				form_kernels[0] = graph_kernels;
				// the other forms; one that fails to capture is left out (the sequence carries on)
				for (int f = 1; f < kForms; ++f) {
					const bool want = (f == 1) ? (S.fused != 0 && fused_eligible()) : (S.fused == 2);
					if (want && capture(f, &graph_form[f], &form_kernels[f])) {
						cudaGetLastError();
						graph_form[f] = nullptr;
					}
				}
				graph_key = key;
				tune_nforms = 0;
				for (int f = 0; f < kForms; ++f)
					if (graph_form[f] && (S.fused == 2 || f == (S.fused == 1 ? 1 : 0))) tune_forms[tune_nforms++] = f;
				if (tune_nforms == 0) tune_forms[tune_nforms++] = 0;
				tune_done = tune_nforms == 1;
				tune_choice = tune_forms[0];
				tune_n = 0;
				for (float& v : tune_ms) v = 0.0f;
			}
			int variant = tune_choice;
			cudaEvent_t* ev = nullptr;
			if (!tune_done) {
				if (tune_n == tune_nforms * kTuneRounds) {
					// every trial step enqueued: the timings decide (one wait, once per capture)
					float sum[kForms] = {};
					for (int t = 0; t < tune_n; ++t) {
						float ms = 0.0f;
						CK(cudaEventSynchronize(tune_ev[t][1]));
						CK(cudaEventElapsedTime(&ms, tune_ev[t][0], tune_ev[t][1]));
						sum[tune_forms[t % tune_nforms]] += ms;
					}
					int best = tune_forms[0];
					for (int q = 0; q < tune_nforms; ++q) {
						const int f = tune_forms[q];
						tune_ms[f] = sum[f] / kTuneRounds;
						if (tune_ms[f] < tune_ms[best]) best = f;
					}
					tune_choice = best;
					tune_done = true;
					variant = tune_choice;
				}
				else {
					variant = tune_forms[tune_n % tune_nforms];
					ev = tune_ev[tune_n++];
					for (int q = 0; q < 2; ++q)
						if (!ev[q]) CK(cudaEventCreate(&ev[q]));
					CK(cudaEventRecord(ev[0], stream));
				}
			}
			cudaError_t el = cudaGraphLaunch(graph_form[variant], stream);
			if (el != cudaSuccess && variant != 0) {
				// a form that will not launch leaves the candidates; the sequence takes the step
				cudaGetLastError();
				cudaGraphExecDestroy(graph_form[variant]);
				graph_form[variant] = nullptr;
				int k = 0;
				for (int q = 0; q < tune_nforms; ++q)
					if (tune_forms[q] != variant) tune_forms[k++] = tune_forms[q];
				tune_nforms = std::max(k, 1);
				tune_forms[0] = tune_nforms == 1 && k == 0 ? 0 : tune_forms[0];
				tune_done = true;
				tune_choice = 0;
				if (ev) { CK(cudaEventRecord(ev[1], stream)); ev = nullptr; }
				variant = 0;
				el = cudaGraphLaunch(graph_form[0], stream);
			}
			CK(el);
			if (variant == 1) fused_pending = true;
			if (ev) CK(cudaEventRecord(ev[1], stream));
			launches += form_kernels[variant];
		}
		last_sc_limited = sc_limited_now;
		if (object_on()) obj_shift_valid = true;
		stepped = true;
		return 0;
	}

	// one captured step: the kernel sequence or the fused launch
	int capture(int form, cudaGraphExec_t* exec, long long* kernels)
	{
		cudaGraph_t g = nullptr;
		CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
		const long long before = launches;
		const int rc = form == 1 ? enqueue_step_fused() : enqueue_step(kFormOcc[form]);
		const cudaError_t ec = cudaStreamEndCapture(stream, &g);
		if (rc) { if (g) cudaGraphDestroy(g); return -1; }
		CK(ec);
		*kernels = launches - before;
		launches = before;
		const cudaError_t ei = cudaGraphInstantiate(exec, g, 0);
		cudaGraphDestroy(g);
		CK(ei);
		return 0;
	}

	bool fused_pending = false;      // a fused launch ran since the last sync

	int sync()
	{
		if (!stream) return 0;
		CK(cudaStreamSynchronize(stream));
		CK(cudaGetLastError());
		if (fused_pending && d_ctr) {
			fused_pending = false;
			CK(cudaMemcpy(&h_ctr->bar_timeout, &d_ctr->bar_timeout, sizeof(unsigned int), cudaMemcpyDeviceToHost));
			if (h_ctr->bar_timeout) return fail("fused substep: a grid barrier wait ran out (results invalid)");
		}
		return 0;
	}

	int read_counters()
	{
		CK(cudaMemcpyAsync(h_ctr, d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, stream));
		CK(cudaStreamSynchronize(stream));
		return 0;
	}

	void profile_collect()
	{
		if (!prof_records.empty()) cudaStreamSynchronize(stream);
		for (const auto& r : prof_records) {
			float ms = 0.0f;
			if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
				prof_ms[r.stage] += ms;
				prof_count[r.stage] += 1;
			}
		}
		prof_records.clear();
		event_next = 0;
	}

	// ------------------------------------------------------------------ serving arena
	// Many independent sessions resident in one engine's buffers and advanced by one
	// launch sequence (one graph replay) per substep.  A session is a scene built and
	// stepped once by an engine of its own; admission copies its state and topology into
	// the next free rows, edges, members and reverse entries (every array is filled in
	// admission order, so each CSR stays monotone), shifting its indices by the segment's
	// bases.  Retirement freezes the rows in place (inverse mass 0, velocity 0: no kernel
	// moves them and no live row refers to them); trailing retired segments are dropped,
	// and when the tail is full the live segments are moved down (compaction).  Every
	// kernel works per row, per cluster or per edge, and each session's colliders act on
	// its rows only (per-slot ranges of the batched collider list), so a session's
	// trajectory in the arena is the one it has alone, bit for bit.
	struct ArenaSeg {
		int slot = -1, row0 = 0, rows = 0;
		long long e0 = 0, ne = 0, m0 = 0, nm = 0, r0 = 0, nr = 0;
		bool live = false;
		std::vector<int> inv;   // session caller index -> row within the segment
	};
	bool arena = false;
	std::vector<ArenaSeg> segs;
	int rows_cap = 0, rows_used = 0, next_slot = 0;
	long long e_cap = 0, m_cap = 0, r_cap = 0, e_used = 0, m_used = 0, r_used = 0;

	int arena_init(long long rows, long long edges, long long members, long long rev)
	{
		if (rows <= 0 || rows > INT_MAX - 1 || edges <= 0 || members <= 0 || rev <= 0 || edges > INT_MAX ||
			members > INT_MAX || rev > INT_MAX)
			return fail("xpbd_b200_arena_new: invalid capacity (each of rows, edges, members, reverse entries "
				"1..2^31-1: the CSR offsets are 32-bit)");
		if (ensure_stream()) return -1;
		arena = true;
		rows_cap = (int)rows; e_cap = edges; m_cap = members; r_cap = rev;
		const size_t R = (size_t)rows;
		CK(pos_curr.alloc(R)); CK(pos_next.alloc(R)); CK(pos_tmp.alloc(R)); CK(vel.alloc(R)); CK(pos_rest.alloc(R));
		CK(shape_rest.alloc(R)); CK(shape_q.alloc(R)); CK(pos_out3.alloc(3 * R)); CK(d_perm.alloc(R));
		CK(d_obj_id.alloc(R)); CK(lam_vol.alloc(R)); CK(det_rest.alloc(R)); CK(rest_len.alloc(R));
		CK(mat_type.alloc(R)); CK(rec.alloc(3 * rec_rows())); CK(inv_mass_saved.alloc(R));
		CK(off.alloc(R + 1)); CK(vol_off.alloc(R + 1)); CK(rev_off.alloc(R + 1));
		CK(nbr.alloc((size_t)edges)); CK(ndist.alloc((size_t)edges)); CK(nstiff.alloc((size_t)edges));
		CK(lam.alloc((size_t)edges)); CK(vol_idx_s.alloc((size_t)members)); CK(rev_idx_s.alloc((size_t)rev));
		CK(cudaMemsetAsync(off.p, 0, sizeof(int), stream));
		CK(cudaMemsetAsync(vol_off.p, 0, sizeof(int), stream));
		CK(cudaMemsetAsync(rev_off.p, 0, sizeof(int), stream));
		CK(cudaMemsetAsync(rec.p, 0xff, rec.bytes(), stream));
		n = 0;
		built = true;
		stepped = true;
		return sync();
	}

	// the settings every session of an arena must share (the launch sequence is common)
	static bool same_step_settings(const Settings& a, const Settings& b)
	{
		return a.iters == b.iters && a.dt == b.dt && a.under_relax == b.under_relax && a.vel_damping == b.vel_damping &&
			a.stiffness_scale == b.stiffness_scale && a.inv_mass_scale == b.inv_mass_scale &&
			a.dist_compliance == b.dist_compliance && a.shape_compliance == b.shape_compliance &&
			a.shape_blend == b.shape_blend && a.use_distance == b.use_distance && a.use_shape == b.use_shape &&
			a.use_volume == b.use_volume && a.shape_robust == b.shape_robust && a.vol_compliance == b.vol_compliance &&
			a.dist_gs == b.dist_gs && a.vol_gs == b.vol_gs && a.warp_mode == b.warp_mode && a.lanes_a == b.lanes_a &&
			a.lanes_b == b.lanes_b && a.ground_on == b.ground_on && a.object_shape == b.object_shape &&
			a.sc_enabled == b.sc_enabled;
	}

	// copy `count` elements of src into dst + at, adding `delta` to every non-negative entry
	int copy_shift(const int* src, int* dst, long long count, int delta)
	{
		if (count <= 0) return 0;
		dev::k_copy_shift<<<(unsigned)((count + kBlock - 1) / kBlock), kBlock, 0, stream>>>(count, src, dst, delta);
		CK(cudaGetLastError());
		return 0;
	}

	template <typename T>
	int copy_d2d(T* dst, const T* src, size_t count)
	{
		if (count) CK(cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyDeviceToDevice, stream));
		return 0;
	}

	// admits a built and stepped session engine; returns its slot, -2 when it does not fit
	int arena_admit(Engine& src)
	{
		if (!arena) return fail("xpbd_b200_arena_admit: not an arena");
		if (&src == this || src.arena || !src.built || !src.stepped || src.n <= 0)
			return fail("xpbd_b200_arena_admit: the session must be a built and stepped scene");
		const Settings& t = src.S;
		if (t.sc_enabled || t.ground_on || t.object_shape > 0.0f || t.dist_gs || t.vol_gs || t.use_angle ||
			src.contact_bits || (t.use_volume && src.vol_lanes() != 4) || (t.use_volume && src.gather_lanes() != 4))
			return fail("xpbd_b200_arena_admit: sessions step with Jacobi distance and volume (4-lane kernels), "
				"shape matching and colliders; self-collision, ground, object shape and contact shapes stay off");
		bool any_live = false;
		for (const auto& g : segs) any_live = any_live || g.live;
		if (any_live && !same_step_settings(S, t))
			return fail("xpbd_b200_arena_admit: the session's solver settings differ from the arena's");
		const int rows = src.n;
		const long long ne = src.graph.off[rows], nm = src.clusters.vol_off[rows], nr = src.clusters.rev_off[rows];
		auto fits = [&]() {
			return rows_used + (long long)rows <= rows_cap && e_used + ne <= e_cap && m_used + nm <= m_cap &&
				r_used + nr <= r_cap;
		};
		// compaction only helps when retired segments left holes below the tail
		bool holes = false;
		for (const auto& g : segs) holes = holes || !g.live;
		if (!fits() && holes && arena_compact()) return -1;
		if (!fits()) return -2;
		if (!any_live) {
			const auto kin = S.kin_ext;
			S = t;
			S.kin_ext = kin;
			S.kin_count = 0;
			S.jstats = false;
			S.topo_dirty = false;
			S.use_graph = true;
		}
		if (src.sync()) return -1;
		ArenaSeg g;
		g.slot = next_slot++;
		g.row0 = rows_used; g.rows = rows;
		g.e0 = e_used; g.ne = ne; g.m0 = m_used; g.nm = nm; g.r0 = r_used; g.nr = nr;
		g.live = true;
		g.inv = src.inv;
		const size_t r0 = (size_t)g.row0;
		if (copy_d2d(pos_curr.p + r0, src.pos_curr.p, rows) || copy_d2d(vel.p + r0, src.vel.p, rows) ||
			copy_d2d(pos_rest.p + r0, src.pos_rest.p, rows) || copy_d2d(shape_rest.p + r0, src.shape_rest.p, rows) ||
			copy_d2d(shape_q.p + r0, src.shape_q.p, rows) || copy_d2d(pos_out3.p + 3 * r0, src.pos_out3.p, 3 * (size_t)rows) ||
			copy_d2d(det_rest.p + r0, src.det_rest.p, rows) || copy_d2d(rest_len.p + r0, src.rest_len.p, rows) ||
			copy_d2d(mat_type.p + r0, src.mat_type.p, rows) ||
			copy_d2d(ndist.p + g.e0, src.ndist.p, (size_t)ne) || copy_d2d(nstiff.p + g.e0, src.nstiff.p, (size_t)ne))
			return -1;
		if (copy_shift(src.d_perm.p, d_perm.p + r0, rows, g.row0) ||
			copy_shift(src.off.p, off.p + r0, rows + 1, (int)g.e0) || copy_shift(src.nbr.p, nbr.p + g.e0, ne, g.row0) ||
			copy_shift(src.vol_off.p, vol_off.p + r0, rows + 1, (int)g.m0) ||
			copy_shift(src.vol_idx_s.p, vol_idx_s.p + g.m0, nm, g.row0) ||
			copy_shift(src.rev_off.p, rev_off.p + r0, rows + 1, (int)g.r0) ||
			copy_shift(src.rev_idx_s.p, rev_idx_s.p + g.r0, nr, g.row0))
			return -1;
		dev::k_fill_int<<<blocks_for(rows), kBlock, 0, stream>>>(rows, d_obj_id.p + r0, g.slot);
		// the inverse masses a pin release restores: the session's own saved ones while it
		// has pins, else its current ones
		if (src.att_active && src.inv_mass_saved.p) {
			if (copy_d2d(inv_mass_saved.p + r0, src.inv_mass_saved.p, rows)) return -1;
		}
		else
			dev::k_get_w<<<blocks_for(rows), kBlock, 0, stream>>>(rows, pos_curr.p + r0, inv_mass_saved.p + r0);
		CK(cudaGetLastError());
		// the session's colliders of its last step are the previous poses of its slot's
		for (int c = 0; c < t.kin_count; ++c) {
			KinCollider K = t.kin[c];
			K.obj = g.slot;
			col_prev[col_key(g.slot, c)] = K;
		}
		rows_used += rows; e_used += ne; m_used += nm; r_used += nr;
		n = rows_used;
		segs.push_back(std::move(g));
		++generation;
		if (sync()) return -1;
		return segs.back().slot;
	}

	ArenaSeg* arena_seg(int slot)
	{
		for (auto& g : segs)
			if (g.slot == slot && g.live) return &g;
		return nullptr;
	}

	int arena_retire(int slot)
	{
		ArenaSeg* g = arena_seg(slot);
		if (!g) return fail("xpbd_b200_arena_retire: no live session in slot %d", slot);
		dev::k_freeze_rows<<<blocks_for(g->rows), kBlock, 0, stream>>>(g->rows, pos_curr.p + g->row0, vel.p + g->row0,
			inv_mass_saved.p + g->row0);
		CK(cudaGetLastError());
		g->live = false;
		while (!segs.empty() && !segs.back().live) {
			const ArenaSeg& b = segs.back();
			rows_used = b.row0; e_used = b.e0; m_used = b.m0; r_used = b.r0;
			segs.pop_back();
		}
		n = rows_used;
		++generation;
		return 0;
	}

	// moves the live segments down over the retired ones (through a staging buffer, since
	// source and destination may overlap) and shifts their indices
	int arena_compact()
	{
		if (sync()) return -1;
		size_t stage_bytes = 0;
		for (const auto& g : segs)
			if (g.live)
				stage_bytes = std::max(stage_bytes, std::max({ sizeof(float4) * (size_t)g.rows, sizeof(float) * 3 * (size_t)g.rows,
					sizeof(int) * (size_t)(g.rows + 1), sizeof(int) * (size_t)g.ne, sizeof(int) * (size_t)g.nm,
					sizeof(int) * (size_t)g.nr }));
		DBuf<unsigned char> stage;
		if (stage_bytes) CK(stage.alloc(stage_bytes));
		auto move = [&](void* base, size_t elem, long long from, long long to, long long count) -> int {
			if (from == to || count <= 0) return 0;
			unsigned char* b = static_cast<unsigned char*>(base);
			CK(cudaMemcpyAsync(stage.p, b + elem * from, elem * count, cudaMemcpyDeviceToDevice, stream));
			CK(cudaMemcpyAsync(b + elem * to, stage.p, elem * count, cudaMemcpyDeviceToDevice, stream));
			return 0;
		};
		auto move_shift = [&](int* base, long long from, long long to, long long count, int delta) -> int {
			if (count <= 0 || (from == to && delta == 0)) return 0;
			CK(cudaMemcpyAsync(stage.p, base + from, sizeof(int) * count, cudaMemcpyDeviceToDevice, stream));
			return copy_shift(reinterpret_cast<const int*>(stage.p), base + to, count, delta);
		};
		std::vector<ArenaSeg> kept;
		int rows = 0;
		long long e = 0, m = 0, r = 0;
		for (auto& g : segs) {
			if (!g.live) continue;
			const int dr = rows - g.row0;
			const long long de = e - g.e0, dm = m - g.m0, drv = r - g.r0;
			if (dr || de || dm || drv) {
				const long long a = g.row0, b = rows, k = g.rows;
				if (move(pos_curr.p, sizeof(float4), a, b, k) || move(vel.p, sizeof(float4), a, b, k) ||
					move(pos_rest.p, sizeof(float4), a, b, k) || move(shape_rest.p, sizeof(float4), a, b, k) ||
					move(shape_q.p, sizeof(float4), a, b, k) || move(pos_out3.p, 3 * sizeof(float), a, b, k) ||
					move(det_rest.p, sizeof(float), a, b, k) || move(rest_len.p, sizeof(float), a, b, k) ||
					move(inv_mass_saved.p, sizeof(float), a, b, k) || move(mat_type.p, sizeof(int), a, b, k) ||
					move(d_obj_id.p, sizeof(int), a, b, k) || move(ndist.p, sizeof(float), g.e0, e, g.ne) ||
					move(nstiff.p, sizeof(float), g.e0, e, g.ne))
					return -1;
				if (move_shift(d_perm.p, a, b, k, dr) || move_shift(off.p, a, b, k + 1, (int)de) ||
					move_shift(nbr.p, g.e0, e, g.ne, dr) || move_shift(vol_off.p, a, b, k + 1, (int)dm) ||
					move_shift(vol_idx_s.p, g.m0, m, g.nm, dr) || move_shift(rev_off.p, a, b, k + 1, (int)drv) ||
					move_shift(rev_idx_s.p, g.r0, r, g.nr, dr))
					return -1;
				g.row0 = rows; g.e0 = e; g.m0 = m; g.r0 = r;
			}
			rows += g.rows; e += g.ne; m += g.nm; r += g.nr;
			kept.push_back(std::move(g));
		}
		segs.swap(kept);
		rows_used = rows; e_used = e; m_used = m; r_used = r;
		n = rows_used;
		++generation;
		return sync();
	}

	// k substeps of every live session: per substep the colliders (col_slot[c]: the
	// session each acts on) and the pins (session pin_slot[p], its Gaussian pin_idx[p])
	int arena_step(int k, int ncol, const int* types, const float* poses, const float* dims, const int* col_slot,
		float margin, float friction, int npin, const int* pin_slot, const int* pin_idx, const float* targets)
	{
		if (!arena) return fail("xpbd_b200_arena_step: not an arena");
		if (n <= 0) return 0;
		std::vector<int> rowsel(std::max(npin, 1));
		for (int p = 0; p < npin; ++p) {
			ArenaSeg* g = arena_seg(pin_slot[p]);
			if (!g || pin_idx[p] < 0 || pin_idx[p] >= g->rows)
				return fail("xpbd_b200_arena_step: pin %d (slot %d, Gaussian %d) is not in a live session", p, pin_slot[p],
					pin_idx[p]);
			rowsel[p] = g->row0 + g->inv[pin_idx[p]];
		}
		for (int s = 0; s < k; ++s) {
			set_colliders_many(ncol, types, poses + (size_t)s * 12 * ncol, dims, col_slot, margin, friction);
			if (set_attached(npin, rowsel.data(), targets + (size_t)s * 3 * npin, 1.0f, true)) return -1;
			if (step_async()) return -1;
		}
		return 0;
	}

	// batched colliders, each bound to one object; a collider's previous pose (for the
	// friction of the moving surface) is the last pose of the same (object, ordinal within
	// the object), so the list may grow or shrink between calls as objects come and go
	std::map<long long, KinCollider> col_prev;
	static long long col_key(int obj, int ordinal) { return ((long long)obj << 24) | (long long)ordinal; }

	void set_colliders_many(int count, const int* types, const float* poses, const float* dims, const int* obj,
		float margin, float friction)
	{
		std::map<long long, KinCollider> seen;
		std::map<int, int> ordinal;
		std::vector<KinCollider> next(count);
		for (int c = 0; c < count; ++c) {
			KinCollider& K = next[c];
			const long long key = col_key(obj[c] < 0 ? -1 : obj[c], ordinal[obj[c] < 0 ? -1 : obj[c]]++);
			const auto it = col_prev.find(key);
			const KinCollider* prev = it != col_prev.end() ? &it->second : nullptr;
			const bool keep = prev && prev->type == types[c];
			for (int a = 0; a < 9; ++a) K.Rp[a] = keep ? prev->R[a] : poses[12 * c + a];
			for (int a = 0; a < 3; ++a) K.tp[a] = keep ? prev->t[a] : poses[12 * c + 9 + a];
			K.type = types[c];
			for (int a = 0; a < 9; ++a) K.R[a] = poses[12 * c + a];
			for (int a = 0; a < 3; ++a) { K.t[a] = poses[12 * c + 9 + a]; K.h[a] = fmaxf(dims[3 * c + a], 0.0f); }
			K.obj = obj[c] < 0 ? -1 : obj[c];
			seen[key] = K;
		}
		col_prev.swap(seen);
		S.kin_ext.swap(next);
		S.kin_count = 0;
		S.kin_margin = (std::isfinite(margin) && margin > 0.0f) ? margin : 0.0f;
		S.kin_friction = (std::isfinite(friction) && friction > 0.0f) ? friction : 0.0f;
	}

	// ------------------------------------------------------------------ attach
	// setAttachedParticles (forward.cu:6759-6788): restore the saved inverse masses, save
	// them on first use, then pin idx[] at pos[].
	int set_attached(int count, const int* idx, const float* pos, float weight = 1.0f, bool rows = false)
	{
		const int N = n;
		if (att_active)
			dev::k_set_w<<<blocks_for(N), kBlock, 0, stream>>>(N, pos_curr.p, inv_mass_saved.p, 0.0f);
		if (count <= 0 || !idx || !pos) {
			att_active = false;
			CK(cudaGetLastError());
			return 0;
		}
		if (!att_active) {
			if (!inv_mass_saved.p) CK(inv_mass_saved.alloc(N));
			dev::k_get_w<<<blocks_for(N), kBlock, 0, stream>>>(N, pos_curr.p, inv_mass_saved.p);
		}
		// targets go through a small ring of pinned staging slots; a slot is reused only
		// after the event recorded behind its last copy has completed
		if ((int)att_idx.n < count) {
			CK(att_idx.alloc(count));
			CK(att_pos.alloc(3 * (size_t)count));
		}
		Staging& st = staging[staging_next];
		staging_next = (staging_next + 1) % kStagingSlots;
		if (st.ev) CK(cudaEventSynchronize(st.ev));
		else CK(cudaEventCreateWithFlags(&st.ev, cudaEventDisableTiming));
		if (count > st.cap) {
			if (st.idx) cudaFreeHost(st.idx);
			if (st.pos) cudaFreeHost(st.pos);
			st.idx = nullptr;
			st.pos = nullptr;
			st.cap = 0;
			CK(cudaMallocHost(&st.idx, sizeof(int) * count));
			CK(cudaMallocHost(&st.pos, sizeof(float) * 3 * count));
			st.cap = count;
		}
		for (int k = 0; k < count; ++k)
			st.idx[k] = (idx[k] >= 0 && idx[k] < N) ? (rows ? idx[k] : inv[idx[k]]) : -1;
		memcpy(st.pos, pos, sizeof(float) * 3 * count);
		CK(cudaMemcpyAsync(att_idx.p, st.idx, sizeof(int) * count, cudaMemcpyHostToDevice, stream));
		CK(cudaMemcpyAsync(att_pos.p, st.pos, sizeof(float) * 3 * count, cudaMemcpyHostToDevice, stream));
		CK(cudaEventRecord(st.ev, stream));
		float* w = (object_on() && obj_w.p) ? obj_w.p : nullptr;
		if (w) dev::k_fill<<<blocks_for(N), kBlock, 0, stream>>>(N, w, 1.0f);
		dev::k_attach<<<blocks_for(count), kBlock, 0, stream>>>(count, att_idx.p, att_pos.p, N, pos_curr.p, vel.p, w,
			fmaxf(weight, 1.0f));
		CK(cudaGetLastError());
		att_active = true;
		return 0;
	}
};

// The reference ABI addresses one solver instance.  Here it addresses the calling
// thread's current engine: the process-wide default, or one selected with
// xpbd_b200_engine_select (several resident scenes, one per session).
static Engine* g_default_engine = nullptr;
static thread_local Engine* t_current_engine = nullptr;

static Engine* cur_engine()
{
	if (t_current_engine) return t_current_engine;
	if (!g_default_engine) g_default_engine = new Engine();
	return g_default_engine;
}

static Engine& engine() { return *cur_engine(); }

// Tangent basis of the floor: the world axis least parallel to n, made orthogonal to n,
// and n x t1 (the reference viewer's checker axes, forward.cu:284-297).
static void floor_basis(const float n[3], float t1[3], float t2[3])
{
	float a[3] = { 0.0f, 0.0f, 0.0f };
	const float ax = fabsf(n[0]), ay = fabsf(n[1]), az = fabsf(n[2]);
	a[(ax <= ay && ax <= az) ? 0 : (ay <= az ? 1 : 2)] = 1.0f;
	const float d = a[0] * n[0] + a[1] * n[1] + a[2] * n[2];
	float x = a[0] - d * n[0], y = a[1] - d * n[1], z = a[2] - d * n[2];
	const float len = sqrtf(x * x + y * y + z * z);
	if (len > 1e-12f) { x /= len; y /= len; z /= len; }
	t1[0] = x; t1[1] = y; t1[2] = z;
	t2[0] = n[1] * z - n[2] * y;
	t2[1] = n[2] * x - n[0] * z;
	t2[2] = n[0] * y - n[1] * x;
}

// Pairs of the frame (m > 0) in depth order, stable-sorted by tile key (Key: 16 or
// 32 bits), then the tile ranges.
template <typename Key>
static int render_bin(Engine& E, long long m, int tiles_x, int tiles)
{
	auto& R = E.rs;
	cudaStream_t st = E.stream;
	const int n = E.n;
	if (R.tkey.n < sizeof(Key) * (size_t)m || R.val.n < (size_t)m) {
		const size_t cap = (size_t)m + m / 4;
		CK(R.tkey.alloc(cap * sizeof(Key))); CK(R.tkey_s.alloc(cap * sizeof(Key)));
		CK(R.val.alloc(cap)); CK(R.val_s.alloc(cap));
	}
	Key* tk = reinterpret_cast<Key*>(R.tkey.p);
	Key* tks = reinterpret_cast<Key*>(R.tkey_s.p);
	dev::k_splat_pairs<Key><<<Engine::blocks_for(n), kBlock, 0, st>>>(n, R.order.p, R.offs.p, R.rect.p, tiles_x, tk,
		R.val.p);
	CK(cudaGetLastError());
	int bits = 1;
	while ((1LL << bits) < tiles) ++bits;
	size_t t3b = 0;
	CK(cub::DeviceRadixSort::SortPairs(nullptr, t3b, tk, tks, R.val.p, R.val_s.p, (int)m, 0, bits, st));
	if (R.temp.n < t3b) CK(R.temp.alloc(t3b));
	CK(cub::DeviceRadixSort::SortPairs(R.temp.p, t3b, tk, tks, R.val.p, R.val_s.p, (int)m, 0, bits, st));
	dev::k_splat_ranges<Key><<<Engine::blocks_for(tiles), kBlock, 0, st>>>(tiles, (int)m, tks, R.ranges.p);
	CK(cudaGetLastError());
	E.launches += 2;
	return 0;
}

// One splatted frame of the current positions (Rasterizer::forward,
// rasterizer_impl.cu:201-470, without the solver step that the reference runs inside
// its preprocess).  Shapes: the deformed scales / quaternions of xpbd_compute_shapes
// when deform_eps >= 0, the created ones otherwise.  Returns the (tile, Gaussian) pair
// count, the reference's num_rendered.
static long long render_frame(Engine& E, const float* view, const float* proj, const float* campos, int W, int H,
	float tan_fovx, float tan_fovy, float scale_mod, float deform_eps, const float* bg, float* out)
{
	if (!E.stepped) return fail("xpbd_b200_render: no step yet");
	if (!view || !proj || !campos || W <= 0 || H <= 0 || !(tan_fovx > 0.0f) || !(tan_fovy > 0.0f))
		return fail("xpbd_b200_render: invalid camera");
	auto& R = E.rs;
	const int n = E.n;
	if (R.h_colors.empty()) return fail("xpbd_b200_render: no colours (xpbd_b200_render_set_colors)");
	cudaStream_t st = E.stream;
	const int tiles_x = (W + dev::kTile - 1) / dev::kTile, tiles_y = (H + dev::kTile - 1) / dev::kTile;
	const int tiles = tiles_x * tiles_y;
	if ((long long)W * H > (1LL << 30)) return fail("xpbd_b200_render: image too large");
	// per-Gaussian buffers, created shapes and opacity (caller order), colours
	if (R.xy.n != (size_t)n) {
		CK(R.xy.alloc(n)); CK(R.conic.alloc(n)); CK(R.rgb.alloc(n)); CK(R.rect.alloc(n));
		CK(R.dkey.alloc(n)); CK(R.dkey_s.alloc(n)); CK(R.iota.alloc(n)); CK(R.order.alloc(n));
		CK(R.radii.alloc(n)); CK(R.touched.alloc(n)); CK(R.cnt.alloc(n)); CK(R.offs.alloc((size_t)n + 1));
		CK(R.opacity.alloc(n)); CK(R.d_total.alloc(1));
		CK(cudaMemcpyAsync(R.opacity.p, E.in_opacity.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st));
		dev::k_iota<<<Engine::blocks_for(n), kBlock, 0, st>>>(n, R.iota.p);
		CK(cudaGetLastError());
		++E.launches;
	}
	if (!R.h_total) CK(cudaMallocHost(reinterpret_cast<void**>(&R.h_total), sizeof(long long)));
	if (R.colors_dirty || R.colors.n != R.h_colors.size()) {
		CK(R.colors.alloc(R.h_colors.size()));
		CK(cudaMemcpyAsync(R.colors.p, R.h_colors.data(), sizeof(float) * R.h_colors.size(), cudaMemcpyHostToDevice,
			st));
		R.colors_dirty = false;
	}
	// stage timings under xpbd_b200_set_profiling (render_prepare / _sort / _tiles)
	auto seg_begin = [&]() -> cudaEvent_t {
		cudaEvent_t a = nullptr;
		if (E.profiling) {
			a = E.next_event();
			cudaEventRecord(a, st);
		}
		return a;
	};
	auto seg_end = [&](int stage, cudaEvent_t a) {
		if (!E.profiling) return;
		cudaEvent_t b = E.next_event();
		cudaEventRecord(b, st);
		E.prof_records.push_back({ stage, a, b });
	};
	cudaEvent_t seg = seg_begin();
	const float* sc;
	const float* q;
	if (deform_eps >= 0.0f) {
		CK(cudaMemsetAsync(&E.d_ctr->shapes_deformed, 0, sizeof(unsigned int) * 2, st));
		dev::k_deformed_shapes<<<Engine::blocks_for(n), kBlock, 0, st>>>(n, E.pos_rest.p, E.pos_curr.p, E.off.p,
			E.nbr.p, E.d_scales.p, E.d_rots.p, deform_eps, E.d_out_scales.p, E.d_out_quats.p, E.d_ctr, E.d_perm.p);
		CK(cudaGetLastError());
		++E.launches;
		sc = E.d_out_scales.p;
		q = E.d_out_quats.p;
	} else {
		if (R.rest_sc.n != 3 * (size_t)n) {
			CK(R.rest_sc.alloc(3 * (size_t)n)); CK(R.rest_q.alloc(4 * (size_t)n));
			CK(cudaMemcpyAsync(R.rest_sc.p, E.in_scales.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st));
			CK(cudaMemcpyAsync(R.rest_q.p, E.in_rots.data(), sizeof(float) * 4 * n, cudaMemcpyHostToDevice, st));
		}
		sc = R.rest_sc.p;
		q = R.rest_q.p;
	}
	if (R.W != W || R.H != H) {
		CK(R.image.alloc(3 * (size_t)W * H)); CK(R.final_T.alloc((size_t)W * H)); CK(R.n_contrib.alloc((size_t)W * H));
		CK(R.pick.alloc((size_t)W * H)); CK(R.ranges.alloc(tiles));
		CK(R.torder.alloc(tiles));
		R.W = W;
		R.H = H;
	}
	dev::RenderFrame F;
	memset(&F, 0, sizeof(F));
	memcpy(F.view, view, sizeof(F.view));
	memcpy(F.proj, proj, sizeof(F.proj));
	memcpy(F.campos, campos, sizeof(F.campos));
	F.tan_fovx = tan_fovx;
	F.tan_fovy = tan_fovy;
	F.focal_x = W / (2.0f * tan_fovx);
	F.focal_y = H / (2.0f * tan_fovy);
	F.scale_mod = scale_mod;
	for (int k = 0; k < 3; ++k) {
		F.box_lo[k] = R.box_on ? R.box_lo[k] : -FLT_MAX;
		F.box_hi[k] = R.box_on ? R.box_hi[k] : FLT_MAX;
		F.bg[k] = bg ? bg[k] : 0.0f;
	}
	F.W = W; F.H = H; F.tiles_x = tiles_x; F.tiles_y = tiles_y;
	F.sh_deg = R.sh_deg;
	F.sh_coeffs = R.sh_coeffs;
	F.antialias = R.antialias;
	F.pick = R.pick_on;
	if (R.floor_on) {
		// renderCUDA's checker floor under the solver's ground plane (FORWARD::render,
		// forward.cu:2663-2680)
		const float* gn = E.S.ground_n;
		float t1[3], t2[3];
		floor_basis(gn, t1, t2);
		const float inv_checker = 1.0f / fmaxf(R.floor_checker, 1e-8f);
		F.floor_on = 1;
		for (int k = 0; k < 3; ++k) {
			F.fl_cam[k] = campos[k];
			F.fl_rx[k] = view[4 * k] * tan_fovx;
			F.fl_ry[k] = view[4 * k + 1] * tan_fovy;
			F.fl_rz[k] = view[4 * k + 2];
			F.fl_n[k] = gn[k];
			F.fl_t1[k] = t1[k] * inv_checker;
			F.fl_t2[k] = t2[k] * inv_checker;
			F.fl_origin[k] = R.floor_origin[k];
		}
		F.fl_camh = gn[0] * campos[0] + gn[1] * campos[1] + gn[2] * campos[2] - E.S.ground_h;
		F.fl_pix = 2.0f * tan_fovy / (float)H * inv_checker;
		F.fl_inv_fade2 = 1.0f / fmaxf(R.floor_fade * R.floor_fade, 1e-12f);
	}
	// 1. project every Gaussian
	dev::k_splat_prepare<<<Engine::blocks_for(n), kBlock, 0, st>>>(n, F, E.pos_out3.p, sc, q, R.opacity.p,
		R.colors.p, R.xy.p, R.conic.p, R.rgb.p, R.dkey.p, R.radii.p, R.rect.p, R.touched.p);
	CK(cudaGetLastError());
	seg_end(ST_RENDER_PREPARE, seg);
	seg = seg_begin();
	// 2. the pair count goes to the host while the GPU sorts by depth and scans the
	// tile counts in that order; the host waits for it only before the pair stage
	CK(cudaMemsetAsync(R.d_total.p, 0, sizeof(unsigned long long), st));
	dev::k_splat_total<<<Engine::blocks_for(n), kBlock, 0, st>>>(n, R.touched.p, R.d_total.p);
	CK(cudaGetLastError());
	CK(cudaMemcpyAsync(R.h_total, R.d_total.p, sizeof(long long), cudaMemcpyDeviceToHost, st));
	if (!R.ev_total) CK(cudaEventCreateWithFlags(&R.ev_total, cudaEventDisableTiming));
	CK(cudaEventRecord(R.ev_total, st));
	size_t need = 0, t1b = 0, t2b = 0;
	CK(cub::DeviceRadixSort::SortPairs(nullptr, t1b, R.dkey.p, R.dkey_s.p, R.iota.p, R.order.p, n, 0, 32, st));
	CK(cub::DeviceScan::InclusiveSum(nullptr, t2b, R.cnt.p, R.offs.p + 1, n, st));
	need = std::max(t1b, t2b);
	if (R.temp.n < need) CK(R.temp.alloc(need));
	CK(cub::DeviceRadixSort::SortPairs(R.temp.p, t1b, R.dkey.p, R.dkey_s.p, R.iota.p, R.order.p, n, 0, 32, st));
	dev::k_splat_counts<<<Engine::blocks_for(n), kBlock, 0, st>>>(n, R.order.p, R.touched.p, R.cnt.p);
	CK(cudaGetLastError());
	CK(cudaMemsetAsync(R.offs.p, 0, sizeof(long long), st));
	CK(cub::DeviceScan::InclusiveSum(R.temp.p, t2b, R.cnt.p, R.offs.p + 1, n, st));
	E.launches += 3;
	CK(cudaEventSynchronize(R.ev_total));
	const long long m = *R.h_total;
	if (m < 0 || m > INT_MAX) return fail("xpbd_b200_render: %lld tile pairs (limit %d)", m, INT_MAX);
	// 3. (tile, Gaussian) pairs in depth order, stable sort by tile, tile ranges, and
	// the tiles ordered longest list first for the compositing launch
	CK(cudaMemsetAsync(R.ranges.p, 0, sizeof(int2) * tiles, st));
	if (m > 0) {
		const bool narrow = tiles <= 65536;
		if (narrow ? render_bin<unsigned short>(E, m, tiles_x, tiles) : render_bin<unsigned int>(E, m, tiles_x, tiles))
			return -1;
	}
	dev::k_tile_order<<<1, 1024, 0, st>>>(tiles, R.ranges.p, R.torder.p);
	CK(cudaGetLastError());
	++E.launches;
	seg_end(ST_RENDER_SORT, seg);
	seg = seg_begin();
	// 4. composite every tile
	if (R.pick_on) CK(cudaMemsetAsync(R.pick.p, 0xff, sizeof(int) * (size_t)W * H, st));
	dev::k_splat_tiles<<<tiles, dev::kTileThreads, 0, st>>>(F, R.torder.p, R.ranges.p, R.val_s.p, R.xy.p,
		R.conic.p, R.rgb.p, R.image.p, R.final_T.p, R.n_contrib.p, R.pick.p);
	CK(cudaGetLastError());
	++E.launches;
	seg_end(ST_RENDER_TILES, seg);
	R.pairs = m;
	if (out) {
		CK(cudaMemcpyAsync(out, R.image.p, sizeof(float) * 3 * (size_t)W * H, cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
	}
	return m;
}

}  // namespace xpbd

using namespace xpbd;

// ============================================================================
// C ABI: the reference's entry points (xpbd_capi.cu:66-310); XPBD_API carries the
// extern "C" linkage
// ============================================================================

XPBD_API const char* xpbd_last_error(void) { return g_err.c_str(); }

XPBD_API int xpbd_create(int n, const float* pos, const float* scales, const float* rots, const float* opacity, int e,
	const int* edges, const float* rest, const float* stiff)
{
	Engine& E = engine();
	E.sync();
	E.free_device();
	E.n = 0;
	E.stepped = false;
	E.contact_bits = 0;
	if (n <= 0 || !pos || !scales || !rots || !opacity || e < 0 || (e > 0 && (!edges || !rest || !stiff)))
		return fail("xpbd_create: invalid arguments");
	E.n = n;
	E.n_edges = e;
	E.in_pos.assign(pos, pos + 3 * (size_t)n);
	E.in_scales.assign(scales, scales + 3 * (size_t)n);
	E.in_rots.assign(rots, rots + 4 * (size_t)n);
	E.in_opacity.assign(opacity, opacity + n);
	E.rs.h_colors.clear();
	E.rs.colors_dirty = false;
	E.in_edges.assign(edges ? edges : (const int*)nullptr, edges ? edges + 2 * (size_t)e : (const int*)nullptr);
	E.in_rest.assign(rest ? rest : (const float*)nullptr, rest ? rest + e : (const float*)nullptr);
	E.in_stiff.assign(stiff ? stiff : (const float*)nullptr, stiff ? stiff + e : (const float*)nullptr);
	// the scene goes to the device with the first step (Engine::build); create itself makes
	// no CUDA call
	return 0;
}

XPBD_API void xpbd_destroy(void)
{
	engine().S.kin_count = 0;
	{
		cur_engine()->sync();
		cur_engine()->free_device();
		cur_engine()->n = 0;
		cur_engine()->stepped = false;
		cur_engine()->contact_bits = 0;
	}
}

XPBD_API int xpbd_count(void) { return cur_engine()->n; }

XPBD_API void xpbd_set_solver(int iters, float dt, float underRelax, float velDamping, float stiffnessScale,
	float invMassScale, float distCompliance, float shapeCompliance, float shapeBlend, float angleCompliance,
	float angleBlend)
{
	// setXPBDParams (forward.cu:4896-4922)
	engine().S.iters = iters < 1 ? 1 : iters;
	engine().S.dt = fmaxf(1e-5f, dt);
	engine().S.under_relax = fmaxf(0.0f, underRelax);
	engine().S.vel_damping = fmaxf(0.0f, velDamping);
	engine().S.stiffness_scale = fmaxf(0.0f, stiffnessScale);
	engine().S.inv_mass_scale = fmaxf(0.0f, invMassScale);
	engine().S.dist_compliance = fmaxf(0.0f, distCompliance);
	engine().S.shape_compliance = fmaxf(0.0f, shapeCompliance);
	engine().S.shape_blend = fminf(fmaxf(0.0f, shapeBlend), 1.0f);
	engine().S.angle_compliance = fmaxf(0.0f, angleCompliance);
	engine().S.angle_blend = fminf(fmaxf(0.0f, angleBlend), 1.0f);
}

XPBD_API void xpbd_set_constraints(int distance, int shape, int angle, int volume)
{
	engine().S.use_distance = distance != 0;
	engine().S.use_shape = shape != 0;
	engine().S.use_angle = angle != 0;
	engine().S.use_volume = volume != 0;
}

XPBD_API void xpbd_set_volume(float compliance, int ringK, int maxMembers, int leaderMinHop)
{
	// setVolumeParams / setVolumeRingK / setVolumeLeaderParams (forward.cu:3849, 3934-3966)
	engine().S.vol_compliance = compliance;
	engine().S.ring_k = std::max(1, std::min(8, ringK));
	engine().S.max_members = std::max(8, std::min(8192, maxMembers));
	engine().S.leader_min_hop = std::max(1, std::min(8, leaderMinHop));
	engine().S.topo_dirty = true;
}

XPBD_API void xpbd_set_ground(int enabled, float ux, float uy, float uz, float height, float friction,
	float restitution, float contactRadius, float contactSlop, float gravity)
{
	// setGroundParams (forward.cu:4430-4446)
	float nx = ux, ny = uy, nz = uz;
	const float len = sqrtf(nx * nx + ny * ny + nz * nz);
	if (!(len > 1e-8f) || !std::isfinite(len)) { nx = 0.0f; ny = 0.0f; nz = 1.0f; }
	else { nx /= len; ny /= len; nz /= len; }
	engine().S.ground_n[0] = nx; engine().S.ground_n[1] = ny; engine().S.ground_n[2] = nz;
	engine().S.ground_on = enabled != 0;
	engine().S.ground_h = std::isfinite(height) ? height : 0.0f;
	engine().S.ground_friction = fmaxf(0.0f, friction);
	engine().S.ground_restitution = fminf(fmaxf(restitution, 0.0f), 1.0f);
	engine().S.ground_radius = fmaxf(0.0f, contactRadius);
	engine().S.ground_slop = fmaxf(0.0f, contactSlop);
	engine().S.ground_gravity = fmaxf(0.0f, gravity);
}

XPBD_API void xpbd_set_object_shape(float stiffness)
{
	// setObjectModeParams(stiffness, no body contact, components >= 50) (xpbd_capi.cu:148,
	// forward.cu:4464-4477)
	float s = fminf(fmaxf(stiffness, 0.0f), 1.0f);
	if (!std::isfinite(s)) s = 0.0f;
	engine().S.object_shape = s;
}

// setObjectShapeGPU (forward.cu:4521): 1 = the weighted device fit while Gaussians are
// pinned (default); 0 = the plain fit always (the reference's host path)
XPBD_API void xpbd_set_object_shape_gpu(int enabled) { engine().S.obj_gpu = enabled != 0; }

XPBD_API void xpbd_set_colliders(int count, const int* types, const float* poses, const float* dims, float margin,
	float friction)
{
	// setKinematicColliders (forward.cu:4478-4500)
	if (count < 0) count = 0;
	if (count > kMaxColliders) count = kMaxColliders;
	const bool same = (count == engine().S.kin_count);
	for (int c = 0; c < count; ++c) {
		KinCollider& K = engine().S.kin[c];
		const bool keep = same && K.type == types[c];
		for (int a = 0; a < 9; ++a) K.Rp[a] = keep ? K.R[a] : poses[12 * c + a];
		for (int a = 0; a < 3; ++a) K.tp[a] = keep ? K.t[a] : poses[12 * c + 9 + a];
		K.type = types[c];
		for (int a = 0; a < 9; ++a) K.R[a] = poses[12 * c + a];
		for (int a = 0; a < 3; ++a) { K.t[a] = poses[12 * c + 9 + a]; K.h[a] = fmaxf(dims[3 * c + a], 0.0f); }
	}
	for (int c = 0; c < count; ++c) engine().S.kin_obj[c] = -1;
	engine().S.kin_ext.clear();
	engine().S.kin_count = count;
	engine().S.kin_margin = (std::isfinite(margin) && margin > 0.0f) ? margin : 0.0f;
	engine().S.kin_friction = (std::isfinite(friction) && friction > 0.0f) ? friction : 0.0f;
}

XPBD_API int xpbd_collider_stats(int* hits, float* push, float* centroid, int maxCount)
{
	// getKinematicColliderStats (forward.cu:4502-4519)
	const int n = std::min(maxCount, engine().S.kin_count);
	if (n <= 0 || !cur_engine()->stepped) return 0;
	if (cur_engine()->read_counters()) return 0;
	const DevCounters& C = *cur_engine()->h_ctr;
	for (int c = 0; c < n; ++c) {
		if (hits) hits[c] = C.kin_hits[c];
		const float* a = &C.kin_push[kColliderAcc * c];
		for (int k = 0; k < 3; ++k) {
			if (push) push[3 * c + k] = a[k];
			if (centroid) centroid[3 * c + k] = (a[6] > 0.0f) ? a[3 + k] / a[6] : engine().S.kin[c].t[k];
		}
	}
	return n;
}

XPBD_API int xpbd_add_rigid_velocity(const float* dv, const float* dw, const float* center)
{
	if (!cur_engine()->stepped) return fail("xpbd_add_rigid_velocity: no step yet");
	Engine& E = *cur_engine();
	dev::k_add_rigid_velocity<<<Engine::blocks_for(E.n), kBlock, 0, E.stream>>>(E.n, E.pos_curr.p, E.vel.p,
		make_float3(dv[0], dv[1], dv[2]), make_float3(dw[0], dw[1], dw[2]), make_float3(center[0], center[1], center[2]));
	CK(cudaGetLastError());
	return E.sync();
}

XPBD_API int xpbd_set_contact_shape(int enabled, float tau, float radiusCap)
{
	// xpbd_capi.cu:181-191: packs from the created shapes now, or at the scene's upload
	// (the first step) when it is not on the device yet
	Engine& E = *cur_engine();
	if (E.n <= 0) return fail("xpbd_set_contact_shape: call xpbd_create first");
	E.contact_bits = enabled;
	E.contact_tau = tau;
	E.contact_cap = radiusCap;
	if (!enabled) return 0;
	if (E.built) {
		if (E.pack_contact(false)) return fail("xpbd_set_contact_shape: pack failed: %s", g_err.c_str());
		return E.sync();
	}
	return 0;
}

XPBD_API int xpbd_set_attached(int count, const int* idx, const float* pos, float weight)
{
	if (!cur_engine()->stepped) return fail("xpbd_set_attached: no step yet");
	if (cur_engine()->set_attached(count, idx, pos, weight)) return -1;
	return 0;
}

XPBD_API void xpbd_set_self_collision(int enabled, float radiusScale, float excludeScale, int withinBody)
{
	// setSelfCollisionParams (forward.cu:4532-4540)
	engine().S.sc_enabled = enabled != 0;
	engine().S.sc_within = withinBody != 0;
	engine().S.sc_radius_scale = fminf(fmaxf(std::isfinite(radiusScale) ? radiusScale : 1.5f, 0.1f), 10.0f);
	engine().S.sc_exclude_scale = fminf(fmaxf(std::isfinite(excludeScale) ? excludeScale : 2.0f, 1.05f), 20.0f);
}

XPBD_API void xpbd_self_collision_stats(int* out)
{
	out[0] = out[1] = out[2] = 0;
	if (!cur_engine()->stepped || !engine().S.sc_enabled) return;
	if (cur_engine()->read_counters()) return;
	out[0] = (int)cur_engine()->h_ctr->sc_contacts;
	out[1] = cur_engine()->last_sc_limited ? (int)cur_engine()->h_ctr->sc_active : cur_engine()->n;
	out[2] = (int)cur_engine()->h_ctr->sc_overflow;
}

XPBD_API void xpbd_set_shape_robust(int enabled) { engine().S.shape_robust = enabled != 0; }

XPBD_API int xpbd_step(void)
{
	if (cur_engine()->n <= 0) return fail("xpbd_step: call xpbd_create first");
	if (cur_engine()->step_async()) return -1;
	return cur_engine()->sync();
}

XPBD_API unsigned long long xpbd_positions_device(void)
{
	if (!cur_engine()->stepped) return 0ull;
	return reinterpret_cast<unsigned long long>(cur_engine()->pos_out3.p);
}

XPBD_API int xpbd_positions_host(float* out, int n)
{
	if (!cur_engine()->stepped) return fail("xpbd_positions_host: no step yet");
	Engine& E = *cur_engine();
	if (!out || n != E.n) return fail("xpbd_positions_host: size mismatch");
	CK(cudaMemcpyAsync(out, E.pos_out3.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, E.stream));
	return E.sync();
}

XPBD_API int xpbd_compute_shapes(float deformEps, float* hostScales, float* hostQuats, int n)
{
	if (!cur_engine()->stepped) return fail("xpbd_compute_shapes: no step yet");
	Engine& E = *cur_engine();
	if (n != E.n) return fail("xpbd_compute_shapes: size mismatch");
	CK(cudaMemsetAsync(&E.d_ctr->shapes_deformed, 0, sizeof(unsigned int) * 2, E.stream));
	dev::k_deformed_shapes<<<Engine::blocks_for(n), kBlock, 0, E.stream>>>(n, E.pos_rest.p, E.pos_curr.p, E.off.p,
		E.nbr.p, E.d_scales.p, E.d_rots.p, deformEps, E.d_out_scales.p, E.d_out_quats.p, E.d_ctr, E.d_perm.p);
	CK(cudaGetLastError());
	// ellipsoid contacts follow the shapes as drawn, from the next step on (xpbd_capi.cu:255-256)
	if (E.contact_bits && E.pack_contact(true)) return -1;
	if (hostScales)
		CK(cudaMemcpyAsync(hostScales, E.d_out_scales.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, E.stream));
	if (hostQuats)
		CK(cudaMemcpyAsync(hostQuats, E.d_out_quats.p, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost, E.stream));
	if (E.read_counters()) return -1;
	return (int)E.h_ctr->shapes_deformed;
}

XPBD_API int xpbd_reset(void)
{
	// setAttachedParticles(0) then squashReset (forward.cu:4411-4427)
	if (!cur_engine()->stepped) return fail("xpbd_reset: no step yet");
	Engine& E = *cur_engine();
	if (E.set_attached(0, nullptr, nullptr)) return -1;
	E.press_reset();
	CK(cudaMemsetAsync(E.lam_vol.p, 0, E.lam_vol.bytes(), E.stream));
	return E.upload_positions(E.in_pos.data(), nullptr);
}

XPBD_API int xpbd_launch(const float* lin, const float* ang, const float* tilt)
{
	// groundLaunch (forward.cu:4551-4610): rest pose rotated about the centre of mass,
	// rigid velocity field, inverse masses 1
	if (!cur_engine()->stepped) return fail("xpbd_launch: no step yet");
	Engine& E = *cur_engine();
	const int N = E.n;
	double cx = 0.0, cy = 0.0, cz = 0.0;
	for (int i = 0; i < N; ++i) { cx += E.in_pos[3 * i]; cy += E.in_pos[3 * i + 1]; cz += E.in_pos[3 * i + 2]; }
	const float comX = float(cx / N), comY = float(cy / N), comZ = float(cz / N);
	const float ax = tilt ? tilt[0] : 0.0f, ay = tilt ? tilt[1] : 0.0f, az = tilt ? tilt[2] : 0.0f;
	const float th = sqrtf(ax * ax + ay * ay + az * az);
	float R[9] = { 1, 0, 0, 0, 1, 0, 0, 0, 1 };
	if (th > 1e-8f) {
		const float kx = ax / th, ky = ay / th, kz = az / th;
		const float s = sinf(th), c = cosf(th), t = 1.0f - c;
		R[0] = c + t * kx * kx; R[1] = t * kx * ky - s * kz; R[2] = t * kx * kz + s * ky;
		R[3] = t * ky * kx + s * kz; R[4] = c + t * ky * ky; R[5] = t * ky * kz - s * kx;
		R[6] = t * kz * kx - s * ky; R[7] = t * kz * ky + s * kx; R[8] = c + t * kz * kz;
	}
	const float vx = lin ? lin[0] : 0.0f, vy = lin ? lin[1] : 0.0f, vz = lin ? lin[2] : 0.0f;
	const float wx = ang ? ang[0] : 0.0f, wy = ang ? ang[1] : 0.0f, wz = ang ? ang[2] : 0.0f;
	std::vector<float> p3(3 * (size_t)N), v3(3 * (size_t)N);
	for (int i = 0; i < N; ++i) {
		const float px = E.in_pos[3 * i] - comX, py = E.in_pos[3 * i + 1] - comY, pz = E.in_pos[3 * i + 2] - comZ;
		const float rx = R[0] * px + R[1] * py + R[2] * pz;
		const float ry = R[3] * px + R[4] * py + R[5] * pz;
		const float rz = R[6] * px + R[7] * py + R[8] * pz;
		p3[3 * i] = comX + rx; p3[3 * i + 1] = comY + ry; p3[3 * i + 2] = comZ + rz;
		v3[3 * i] = vx + (wy * rz - wz * ry); v3[3 * i + 1] = vy + (wz * rx - wx * rz); v3[3 * i + 2] = vz + (wx * ry - wy * rx);
	}
	CK(cudaMemsetAsync(E.lam_vol.p, 0, E.lam_vol.bytes(), E.stream));
	E.press_reset();   // groundLaunch ends a press (forward.cu:4599-4602)
	return E.upload_positions(p3.data(), v3.data());
}

XPBD_API int xpbd_press_start(int axis, float rampPerSec, float maxDispPct, int fromLo)
{
	// xpbd_capi.cu:281-288: squashSetPress(true), squashSetPressFromLo, squashStart(axis, 0.08, ...)
	Engine& E = *cur_engine();
	if (!E.stepped) return fail("xpbd_press_start: step once first");
	return E.press_start(axis, rampPerSec, maxDispPct, fromLo != 0);
}
XPBD_API void xpbd_press_autolog(int enabled) { engine().S.press_autolog = enabled != 0; }
XPBD_API void xpbd_press_stop(void)
{
	// squashStop (forward.cu:4398-4409): the plates leave, every inverse mass back to 1
	Engine& E = *cur_engine();
	if (!E.press_active) return;
	E.press_active = false;
	if (E.n > 0 && E.pos_curr.p) {
		dev::k_set_w<<<Engine::blocks_for(E.n), kBlock, 0, E.stream>>>(E.n, E.pos_curr.p, nullptr, 1.0f);
		E.sync();
	}
}
XPBD_API int xpbd_press_state(float* lo, float* hi, float* cur, float* mx)
{
	// squashGetProgress + squashGetPlates (forward.cu:4675-4689)
	const Engine& E = *cur_engine();
	if (cur) *cur = E.press_cur;
	if (mx) *mx = E.press_max;
	if (lo) *lo = E.press_lo + ((E.press_active && E.press_from_lo) ? E.press_cur : 0.0f);
	if (hi) *hi = E.press_hi - ((E.press_active && !E.press_from_lo) ? E.press_cur : 0.0f);
	return E.press_active ? 1 : 0;
}

XPBD_API void xpbd_volume_stats(int enable, float* jvw, float* jvwStd)
{
	// setVolumeJStatsEnabled + getVolumeJVolumeWeighted (forward.cu:4081-4099)
	engine().S.jstats = enable != 0;
	float m = 1.0f, s = 0.0f;
	if (cur_engine()->stepped && !cur_engine()->read_counters()) {
		const double* a = cur_engine()->h_ctr->jstats;
		if (a[0] > 0.0) {
			const double mean = a[1] / a[0];
			m = (float)mean;
			s = (float)sqrt(fmax(0.0, a[2] / a[0] - mean * mean));
		}
	}
	if (jvw) *jvw = m;
	if (jvwStd) *jvwStd = s;
}

// ============================================================================
// extensions (no counterpart in the reference ABI)
// ============================================================================
XPBD_API int xpbd_b200_set_collider_objects(int count, const int* obj)
{
	Settings& st = engine().S;
	if (count != st.kin_count || (count > 0 && !obj))
		return fail("xpbd_b200_set_collider_objects: %d filters for %d colliders", count, st.kin_count);
	for (int c = 0; c < count; ++c) st.kin_obj[c] = obj[c] < 0 ? -1 : obj[c];
	return 0;
}

XPBD_API int xpbd_b200_set_colliders_many(int count, const int* types, const float* poses, const float* dims,
	const int* obj, float margin, float friction)
{
	if (count < 0 || (count > 0 && (!types || !poses || !dims || !obj)))
		return fail("xpbd_b200_set_colliders_many: invalid arguments");
	engine().set_colliders_many(count, types, poses, dims, obj, margin, friction);
	return 0;
}

// ChainMail (forward.cu:12808-13006).  The reference's C ABI cannot reach it: xpbd_create
// forces XPBD mode (xpbd_capi.cu:98); these expose its GPU path on the same scene.
XPBD_API void xpbd_b200_chainmail_set_material(float global_scale, float air, float skin, float bone,
	int use_edge_stiffness, float edge_influence)
{
	// setChainmailMaterialParams (forward.cu:4844-4858)
	dev::CmMaterial& M = engine().S.cm;
	M.global = fmaxf(1e-4f, global_scale);
	M.air = fmaxf(1e-4f, air);
	M.skin = fmaxf(1e-4f, skin);
	M.bone = fmaxf(1e-4f, bone);
	M.use_edge = use_edge_stiffness != 0;
	M.influence = fmaxf(0.0f, edge_influence);
}

XPBD_API void xpbd_b200_chainmail_set_frontier(int enabled) { engine().S.cm_frontier = enabled != 0; }

XPBD_API void xpbd_b200_set_gpu_builder(int enabled) { engine().S.gpu_builder = enabled != 0; }

// exportPhysicsGraph (forward.cu:4612-4663): the directed graph and rest positions as an
// APGGRPH1 file, in the order given to xpbd_create (the reference writes its viewer's
// internal order; tools/import_graph.py renumbers either by matching positions)
XPBD_API int xpbd_b200_render_set_colors(int n, int sh_degree, const float* data)
{
	// colours of the splatting pass: RGB per Gaussian (sh_degree -1, the reference's
	// colors_precomp) or (sh_degree + 1)^2 RGB spherical-harmonic coefficients per
	// Gaussian ([n][coeffs][3], the reference's shs) evaluated toward the camera
	Engine& E = *cur_engine();
	if (E.n <= 0 || n != E.n) return fail("xpbd_b200_render_set_colors: size mismatch (create first)");
	if (!data || sh_degree < -1 || sh_degree > 3) return fail("xpbd_b200_render_set_colors: invalid arguments");
	const int coeffs = sh_degree < 0 ? 1 : (sh_degree + 1) * (sh_degree + 1);
	E.rs.h_colors.assign(data, data + (size_t)3 * coeffs * n);
	E.rs.sh_deg = sh_degree;
	E.rs.sh_coeffs = coeffs;
	E.rs.colors_dirty = true;
	return 0;
}

XPBD_API void xpbd_b200_render_set_options(int antialiasing, const float* box_min, const float* box_max, int pick)
{
	auto& R = cur_engine()->rs;
	R.antialias = antialiasing != 0;
	R.pick_on = pick != 0;
	R.box_on = box_min && box_max;
	for (int k = 0; k < 3; ++k) {
		R.box_lo[k] = R.box_on ? box_min[k] : 0.0f;
		R.box_hi[k] = R.box_on ? box_max[k] : 0.0f;
	}
}

XPBD_API void xpbd_b200_render_set_floor(int visible, const float* origin, float checker, float fade_radius)
{
	// setGroundRender (forward.cu:4448-4462); the plane is the solver's ground
	auto& R = cur_engine()->rs;
	R.floor_on = visible != 0 && origin;
	if (!R.floor_on) return;
	for (int k = 0; k < 3; ++k) R.floor_origin[k] = origin[k];
	R.floor_checker = fmaxf(checker, 1e-8f);
	R.floor_fade = fmaxf(fade_radius, 1e-8f);
}

XPBD_API long long xpbd_b200_render(const float* view, const float* proj, const float* campos, int width, int height,
	float tan_fovx, float tan_fovy, float scale_modifier, float deform_eps, const float* bg, float* out)
{
	return render_frame(*cur_engine(), view, proj, campos, width, height, tan_fovx, tan_fovy, scale_modifier,
		deform_eps, bg, out);
}

XPBD_API unsigned long long xpbd_b200_render_device(void)
{
	return reinterpret_cast<unsigned long long>(cur_engine()->rs.image.p);
}

XPBD_API int xpbd_b200_render_aux(float* final_T, int* n_contrib, int* pick, long long npix, int* radii, int n)
{
	Engine& E = *cur_engine();
	auto& R = E.rs;
	if (!R.image.p) return fail("xpbd_b200_render_aux: no frame yet");
	const long long np = (long long)R.W * R.H;
	if ((final_T || n_contrib || pick) && npix != np) return fail("xpbd_b200_render_aux: %lld pixels, not %lld", npix, np);
	if (radii && n != E.n) return fail("xpbd_b200_render_aux: size mismatch");
	if (pick && !R.pick_on) return fail("xpbd_b200_render_aux: picking is off");
	if (final_T) CK(cudaMemcpyAsync(final_T, R.final_T.p, sizeof(float) * np, cudaMemcpyDeviceToHost, E.stream));
	if (n_contrib) CK(cudaMemcpyAsync(n_contrib, R.n_contrib.p, sizeof(int) * np, cudaMemcpyDeviceToHost, E.stream));
	if (pick) CK(cudaMemcpyAsync(pick, R.pick.p, sizeof(int) * np, cudaMemcpyDeviceToHost, E.stream));
	if (radii) CK(cudaMemcpyAsync(radii, R.radii.p, sizeof(int) * E.n, cudaMemcpyDeviceToHost, E.stream));
	return E.sync();
}

XPBD_API int xpbd_b200_export_graph(const char* path)
{
	Engine& E = *cur_engine();
	if (!E.built || !path) return fail("xpbd_b200_export_graph: no graph yet (create and step first)");
	const int N = E.n, M = E.graph.off[N];
	std::vector<int> cnt(N);
	for (int i = 0; i < N; ++i) cnt[i] = E.graph.off[i + 1] - E.graph.off[i];
	FILE* f = fopen(path, "wb");
	if (!f) return fail("xpbd_b200_export_graph: cannot open %s", path);
	bool ok = fwrite("APGGRPH1", 1, 8, f) == 8;
	ok = ok && fwrite(&N, sizeof(int), 1, f) == 1 && fwrite(&M, sizeof(int), 1, f) == 1;
	ok = ok && fwrite(E.in_pos.data(), sizeof(float), 3 * (size_t)N, f) == 3 * (size_t)N;
	ok = ok && fwrite(E.graph.off.data(), sizeof(int), N, f) == (size_t)N;
	ok = ok && fwrite(cnt.data(), sizeof(int), N, f) == (size_t)N;
	ok = ok && fwrite(E.graph.nbr.data(), sizeof(int), M, f) == (size_t)M;
	ok = ok && fwrite(E.graph.ndist.data(), sizeof(float), M, f) == (size_t)M;
	ok = ok && fwrite(E.graph.nstiff.data(), sizeof(float), M, f) == (size_t)M;
	ok = (fclose(f) == 0) && ok;
	return ok ? 0 : fail("xpbd_b200_export_graph: write failed: %s", path);
}

XPBD_API int xpbd_b200_chainmail_seed(int count, const int* idx, const float* delta)
{
	Engine& E = *cur_engine();
	if (!E.stepped) return fail("xpbd_b200_chainmail_seed: no step yet");
	if (count < 0 || (count > 0 && (!idx || !delta))) return fail("xpbd_b200_chainmail_seed: invalid arguments");
	for (int k = 0; k < count; ++k)
		if (idx[k] < 0 || idx[k] >= E.n) return fail("xpbd_b200_chainmail_seed: index %d out of range", idx[k]);
	return E.chainmail_seed(count, idx, delta);
}

XPBD_API int xpbd_b200_chainmail_run(int prop_iters, int relax_iters, float prop_strength, float relax_stiffness,
	float relax_damping)
{
	Engine& E = *cur_engine();
	if (!E.stepped) return fail("xpbd_b200_chainmail_run: no step yet");
	if (prop_iters < 0 || relax_iters < 0) return fail("xpbd_b200_chainmail_run: negative iteration count");
	return E.chainmail_run(prop_iters, relax_iters, prop_strength, relax_stiffness, relax_damping);
}

XPBD_API int xpbd_b200_chainmail_times(float* out, int n)
{
	Engine& E = *cur_engine();
	if (!E.stepped || !out || n < E.n) return fail("xpbd_b200_chainmail_times: invalid arguments");
	if (E.ensure_chainmail()) return -1;
	if (E.cm_publish(E.cm_time_out.p)) return -1;
	CK(cudaMemcpyAsync(out, E.cm_time_out.p, sizeof(float) * E.n, cudaMemcpyDeviceToHost, E.stream));
	if (E.sync()) return -1;
	return E.n;
}

XPBD_API void* xpbd_b200_engine_new(void) { return new (std::nothrow) Engine(); }

XPBD_API void xpbd_b200_engine_free(void* handle)
{
	Engine* e = static_cast<Engine*>(handle);
	if (!e || e == g_default_engine) return;
	if (t_current_engine == e) t_current_engine = nullptr;
	e->sync();
	delete e;
}

XPBD_API void xpbd_b200_engine_select(void* handle) { t_current_engine = static_cast<Engine*>(handle); }

XPBD_API int xpbd_b200_set_stream(void* stream)
{
	Engine& E = engine();
	if (E.own_stream && E.stream) {
		cudaStreamSynchronize(E.stream);
		cudaStreamDestroy(E.stream);
	}
	E.own_stream = false;
	E.stream = static_cast<cudaStream_t>(stream);
	if (E.graph_exec) { cudaGraphExecDestroy(E.graph_exec); E.graph_exec = nullptr; }
	E.destroy_forms();
	E.graph_key.clear();
	if (!E.stream) return E.ensure_stream();
	return 0;
}

XPBD_API int xpbd_b200_step_async(int substeps)
{
	if (cur_engine()->n <= 0) return fail("xpbd_b200_step_async: call xpbd_create first");
	for (int s = 0; s < substeps; ++s)
		if (cur_engine()->step_async()) return -1;
	return 0;
}

// k substeps in one call, each preceded by what a caller sets per substep: the colliders'
// poses (the reference list: types / dims fixed, poses[s * 12 * ncol ...]) and, after the
// first step, the pinned Gaussians' targets (targets[s * 3 * npins ...], weight 1).  The
// same as xpbd_set_colliders + xpbd_set_attached + xpbd_b200_step_async(1) per substep.
XPBD_API int xpbd_b200_step_substeps(int k, int ncol, const int* types, const float* poses, const float* dims,
	float margin, float friction, int npins, const int* idx, const float* targets)
{
	Engine& E = *cur_engine();
	if (E.n <= 0) return fail("xpbd_b200_step_substeps: call xpbd_create first");
	if (k < 0 || ncol < 0 || npins < 0 || (ncol > 0 && (!types || !poses || !dims)) ||
		(npins > 0 && (!idx || !targets)))
		return fail("xpbd_b200_step_substeps: invalid arguments");
	for (int s = 0; s < k; ++s) {
		if (ncol > 0) xpbd_set_colliders(ncol, types, poses + (size_t)s * 12 * ncol, dims, margin, friction);
		if (npins > 0 && E.stepped && E.set_attached(npins, idx, targets + (size_t)s * 3 * npins, 1.0f)) return -1;
		if (E.step_async()) return -1;
	}
	return 0;
}

XPBD_API int xpbd_b200_sync(void) { return cur_engine()->stream ? cur_engine()->sync() : 0; }

// ---- serving arena ----
XPBD_API void* xpbd_b200_arena_new(long long rows, long long edges, long long members, long long rev)
{
	Engine* e = new (std::nothrow) Engine();
	if (!e) { fail("xpbd_b200_arena_new: out of host memory"); return nullptr; }
	if (e->arena_init(rows, edges, members, rev)) { delete e; return nullptr; }
	return e;
}

XPBD_API int xpbd_b200_arena_admit(void* arena, void* session)
{
	if (!arena || !session) return fail("xpbd_b200_arena_admit: null handle");
	return static_cast<Engine*>(arena)->arena_admit(*static_cast<Engine*>(session));
}

XPBD_API int xpbd_b200_arena_retire(void* arena, int slot)
{
	if (!arena) return fail("xpbd_b200_arena_retire: null handle");
	return static_cast<Engine*>(arena)->arena_retire(slot);
}

XPBD_API int xpbd_b200_arena_step(void* arena, int k, int ncol, const int* types, const float* poses, const float* dims,
	const int* col_slot, float margin, float friction, int npin, const int* pin_slot, const int* pin_idx,
	const float* targets)
{
	if (!arena || k < 0 || ncol < 0 || npin < 0 || (ncol > 0 && (!types || !poses || !dims || !col_slot)) ||
		(npin > 0 && (!pin_slot || !pin_idx || !targets)))
		return fail("xpbd_b200_arena_step: invalid arguments");
	return static_cast<Engine*>(arena)->arena_step(k, ncol, types, poses, dims, col_slot, margin, friction, npin,
		pin_slot, pin_idx, targets);
}

XPBD_API int xpbd_b200_arena_positions(void* arena, int slot, float* out, int n)
{
	if (!arena || !out) return fail("xpbd_b200_arena_positions: invalid arguments");
	Engine& A = *static_cast<Engine*>(arena);
	const auto* g = A.arena_seg(slot);
	if (!g || n != g->rows) return fail("xpbd_b200_arena_positions: no live session of %d Gaussians in slot %d", n, slot);
	CK(cudaMemcpyAsync(out, A.pos_out3.p + 3 * (size_t)g->row0, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToHost,
		A.stream));
	return A.sync();
}

XPBD_API int xpbd_b200_arena_sync(void* arena)
{
	if (!arena) return fail("xpbd_b200_arena_sync: null handle");
	return static_cast<Engine*>(arena)->sync();
}

XPBD_API int xpbd_b200_arena_usage(void* arena, long long* out)
{
	if (!arena || !out) return fail("xpbd_b200_arena_usage: invalid arguments");
	const Engine& A = *static_cast<Engine*>(arena);
	long long live = 0, sessions = 0;
	for (const auto& g : A.segs)
		if (g.live) { live += g.rows; ++sessions; }
	out[0] = A.rows_used; out[1] = A.rows_cap; out[2] = A.e_used; out[3] = A.e_cap; out[4] = A.m_used;
	out[5] = A.m_cap; out[6] = A.r_used; out[7] = A.r_cap; out[8] = live; out[9] = sessions;
	return 0;
}

XPBD_API void xpbd_b200_arena_free(void* arena)
{
	Engine* e = static_cast<Engine*>(arena);
	if (!e) return;
	e->sync();
	delete e;
}

XPBD_API void xpbd_b200_set_gs(int distance, int volume)
{
	engine().S.dist_gs = distance != 0;
	engine().S.vol_gs = volume != 0;
}

XPBD_API void xpbd_b200_set_volume_warp_mode(int mode) { engine().S.warp_mode = std::max(0, std::min(2, mode)); }

XPBD_API void xpbd_b200_set_graph(int enabled) { engine().S.use_graph = enabled != 0; }

XPBD_API void xpbd_b200_set_fused(int mode) { engine().S.fused = std::max(0, std::min(2, mode)); }
XPBD_API void xpbd_b200_set_selfcol_near(int enabled) { engine().S.sc_near = enabled ? 1 : 0; }

XPBD_API int xpbd_b200_tuning(float* out)
{
	// [0] form in use (0 kernel sequence, 1 fused launch, 2 / 3 the sequence with 6 / 8
	// blocks per SM for distance and volume), [1] 1 once decided, [2] [3] mean trial-step
	// ms of forms 0 and 1, [4] launches per step of the form in use, [5] [6] of forms 2, 3
	const Engine& E = *cur_engine();
	if (!out) return fail("xpbd_b200_tuning: null output");
	out[0] = (float)E.tune_choice;
	out[1] = E.tune_done ? 1.0f : 0.0f;
	out[2] = E.tune_ms[0];
	out[3] = E.tune_ms[1];
	out[4] = (float)E.form_kernels[E.tune_choice];
	out[5] = E.tune_ms[2];
	out[6] = E.tune_ms[3];
	return 0;
}

XPBD_API void xpbd_b200_set_reorder(int enabled) { engine().S.reorder = enabled != 0; }

XPBD_API void xpbd_b200_set_volume_lanes(int solve_lanes, int gather_lanes)
{
	auto ok = [](int v) { return v == 0 || v == 2 || v == 3 || v == 4 || v == 8 || v == 32; };
	engine().S.lanes_a = ok(solve_lanes) ? solve_lanes : 0;
	engine().S.lanes_b = (ok(gather_lanes) && gather_lanes != 2 && gather_lanes != 3) ? gather_lanes : 0;
}

XPBD_API int xpbd_b200_set_profiling(int enabled)
{
	Engine& E = engine();
	if (E.profiling) E.profile_collect();
	E.profiling = enabled != 0;
	return 0;
}

XPBD_API int xpbd_b200_stage_times(double* ms, long long* counts, int max_stages)
{
	Engine& E = engine();
	E.profile_collect();
	const int k = std::min(max_stages, (int)ST_COUNT);
	for (int s = 0; s < k; ++s) {
		if (ms) ms[s] = E.prof_ms[s];
		if (counts) counts[s] = E.prof_count[s];
	}
	return k;
}

XPBD_API void xpbd_b200_reset_stage_times(void)
{
	Engine& E = engine();
	E.profile_collect();
	for (int s = 0; s < ST_COUNT; ++s) { E.prof_ms[s] = 0.0; E.prof_count[s] = 0; }
}

XPBD_API const char* xpbd_b200_stage_name(int stage)
{
	return (stage >= 0 && stage < ST_COUNT) ? kStageNames[stage] : "";
}

XPBD_API long long xpbd_b200_launch_count(void) { return cur_engine()->launches; }

XPBD_API int xpbd_b200_sizes(long long* out)
{
	// [0] N, [1] directed edges, [2] cluster members, [3] reverse entries, [4] GS edges,
	// [5] GS edge colours, [6] GS clusters, [7] GS cluster colours, [8] hash table, [9] candidates
	for (int k = 0; k < 10; ++k) out[k] = 0;
	if (!cur_engine()->built) return -1;
	Engine& E = *cur_engine();
	out[0] = E.n;
	out[1] = E.graph.off[E.n];
	out[2] = E.clusters.vol_off.empty() ? 0 : E.clusters.vol_off[E.n];
	out[3] = E.clusters.rev_off.empty() ? 0 : E.clusters.rev_off[E.n];
	out[4] = (long long)E.coloring.edge.size();
	out[5] = E.coloring.color_off.empty() ? 0 : (long long)E.coloring.color_off.size() - 1;
	out[6] = (long long)E.clusters.gs_order.size();
	out[7] = E.clusters.gs_color_off.empty() ? 0 : (long long)E.clusters.gs_color_off.size() - 1;
	out[8] = E.sc_table;
	if (E.sc_table && !E.read_counters()) out[9] = E.h_ctr->sc_contacts;
	return 0;
}

namespace {
template <typename T>
int copy_dev(const T* src, long long count, T* out, long long cap, cudaStream_t st)
{
	if (!src || count < 0) return -1;
	if (!out) return (int)count;
	if (cap < count) return -1;
	if (count > 0) {
		if (cudaMemcpyAsync(out, src, sizeof(T) * (size_t)count, cudaMemcpyDeviceToHost, st) != cudaSuccess) return -1;
		if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
	}
	return (int)count;
}
template <typename T>
int copy_host(const std::vector<T>& v, long long count, T* out, long long cap)
{
	if (count < 0 || (long long)v.size() < count) return -1;
	if (!out) return (int)count;
	if (cap < count) return -1;
	std::copy(v.begin(), v.begin() + count, out);
	return (int)count;
}
// device array in internal order -> caller order (rows of `width`)
template <typename T>
int dev_to_caller(const Engine& E, const T* src, int width, T* out, long long cap)
{
	const long long count = (long long)E.n * width;
	if (!src) return -1;
	if (!out) return (int)count;
	if (cap < count) return -1;
	std::vector<T> tmp(count);
	if (copy_dev(src, count, tmp.data(), count, E.stream) < 0) return -1;
	for (int r = 0; r < E.n; ++r)
		for (int a = 0; a < width; ++a) out[(size_t)E.perm[r] * width + a] = tmp[(size_t)r * width + a];
	return (int)count;
}
}  // namespace

// Stage buffers by name, in the reference's layouts (counts per row instead of N+1
// row starts, sorted hash order, candidate lists).  Count only when out == NULL.
XPBD_API int xpbd_b200_debug_int(const char* name, int* out, long long cap)
{
	if (!cur_engine()->built) return -1;
	Engine& E = *cur_engine();
	const int N = E.n;
	const std::string s(name);
	auto counts_of = [&](const std::vector<int>& off) {
		std::vector<int> c(N);
		for (int i = 0; i < N; ++i) c[i] = off[i + 1] - off[i];
		return c;
	};
	if (s == "nbr_offset") return copy_host(E.graph.off, N, out, cap);
	if (s == "nbr_count") return copy_host(counts_of(E.graph.off), N, out, cap);
	if (s == "nbr_idx") return copy_host(E.graph.nbr, E.graph.off[N], out, cap);
	if (s == "vol_offset") return copy_host(E.clusters.vol_off, N, out, cap);
	if (s == "vol_count") return copy_host(counts_of(E.clusters.vol_off), N, out, cap);
	if (s == "vol_idx") return copy_host(E.clusters.vol_idx, E.clusters.vol_off[N], out, cap);
	if (s == "rev_offset") return copy_host(E.clusters.rev_off, N, out, cap);
	if (s == "rev_count") return copy_host(counts_of(E.clusters.rev_off), N, out, cap);
	if (s == "rev_idx") return copy_host(E.clusters.rev_idx, E.clusters.rev_off[N], out, cap);
	if (s == "vol_gs_order") return copy_host(E.clusters.gs_order, (long long)E.clusters.gs_order.size(), out, cap);
	if (s == "vol_gs_color_offset")
		return copy_host(E.clusters.gs_color_off, (long long)E.clusters.gs_color_off.size(), out, cap);
	if (s == "obj_id") return copy_host(E.obj_id, N, out, cap);
	if (s == "mat_type") return dev_to_caller(E, E.mat_type.p, 1, out, cap);
	if (s == "gs_edge" || s == "gs_color_offset") {
		if (E.ensure_coloring()) return -1;
		if (s == "gs_color_offset") return copy_host(E.coloring.color_off, (long long)E.coloring.color_off.size(), out, cap);
		std::vector<int> flat(2 * E.coloring.edge.size());
		for (size_t e = 0; e < E.coloring.edge.size(); ++e) { flat[2 * e] = E.coloring.edge[e].x; flat[2 * e + 1] = E.coloring.edge[e].y; }
		return copy_host(flat, (long long)flat.size(), out, cap);
	}
	if (!E.sc_table) return -1;
	if (s == "sc_keys") return dev_to_caller(E, reinterpret_cast<const int*>(E.sc_keys.p), 1, out, cap);
	if (s == "sc_count") return dev_to_caller(E, E.sc_counts.p, 1, out, cap);
	if (s == "sc_idx_sorted") {
		const int r = copy_dev(E.sc_idx_sorted.p, N, out, cap, E.stream);
		if (r > 0 && out)
			for (int t = 0; t < N; ++t) out[t] = E.perm[out[t]];
		return r;
	}
	if (s == "sc_contact") {
		const int r = dev_to_caller(E, E.sc_contacts.p, kSelfColMax, out, cap);
		if (r > 0 && out)
			for (long long t = 0; t < (long long)N * kSelfColMax; ++t) {
				const int c = out[t];
				if (c >= 0 && c < N) out[t] = E.perm[c];
				else if (c < 0 && -c - 1 < N) out[t] = -(E.perm[-c - 1] + 1);
			}
		return r;
	}
	if (s == "sc_keys_sorted" || s == "sc_cell_start" || s == "sc_cell_end") {
		std::vector<int> start(E.sc_table + 2), keys(N), idx(N);
		if (copy_dev(E.sc_start.p, E.sc_table + 2, start.data(), E.sc_table + 2, E.stream) < 0) return -1;
		if (s == "sc_keys_sorted") {
			if (copy_dev(reinterpret_cast<const int*>(E.sc_keys.p), N, keys.data(), N, E.stream) < 0) return -1;
			if (copy_dev(E.sc_idx_sorted.p, N, idx.data(), N, E.stream) < 0) return -1;
			std::vector<int> ks(N);
			for (int t = 0; t < N; ++t) ks[t] = keys[idx[t]];
			return copy_host(ks, N, out, cap);
		}
		std::vector<int> v(E.sc_table);
		for (int k = 0; k < E.sc_table; ++k) {
			const bool any = start[k + 1] > start[k];
			v[k] = (s == "sc_cell_start") ? (any ? start[k] : -1) : (any ? start[k + 1] : -1);
		}
		return copy_host(v, E.sc_table, out, cap);
	}
	return -1;
}

XPBD_API int xpbd_b200_debug_float(const char* name, float* out, long long cap)
{
	if (!cur_engine()->built) return -1;
	Engine& E = *cur_engine();
	const int N = E.n;
	const std::string s(name);
	if (s == "det_rest") return dev_to_caller(E, E.det_rest.p, 1, out, cap);
	if (s == "sigma_rest") return dev_to_caller(E, E.sigma_rest.p, 6, out, cap);
	if (s == "v_rest") return dev_to_caller(E, E.v_rest.p, 1, out, cap);
	if (s == "rest_len") return dev_to_caller(E, E.rest_len.p, 1, out, cap);
	if (s == "gs_rest" || s == "gs_stiff") {
		if (E.ensure_coloring()) return -1;
		const auto& v = (s == "gs_rest") ? E.coloring.rest : E.coloring.stiff;
		return copy_host(v, (long long)v.size(), out, cap);
	}
	if (s == "vel" || s == "inv_mass") {
		std::vector<float4> tmp(N);
		if (copy_dev(s == "vel" ? E.vel.p : E.pos_curr.p, N, tmp.data(), N, E.stream) < 0) return -1;
		std::vector<float> v(s == "vel" ? 3 * (size_t)N : N);
		for (int r = 0; r < N; ++r) {
			const int i = E.perm[r];
			if (s == "vel") { v[3 * i] = tmp[r].x; v[3 * i + 1] = tmp[r].y; v[3 * i + 2] = tmp[r].z; }
			else v[i] = tmp[r].w;
		}
		return copy_host(v, (long long)v.size(), out, cap);
	}
	if (s == "build_ms") {
		const std::vector<float> v(E.build_ms, E.build_ms + 8);
		return copy_host(v, 8, out, cap);
	}
	if (s == "cluster_active") {   // 1 where the last iteration's cluster gave a record, else 0
		const long long slots = 2LL * (long long)E.rec_rows();
		std::vector<float4> tmp((size_t)slots);
		if (copy_dev(E.rec.p, slots, tmp.data(), slots, E.stream) < 0) return -1;
		std::vector<float> v(N);
		for (int r = 0; r < N; ++r) {
			const size_t b = 2 * (size_t)r + 1;   // the record's second half
			v[E.perm[r]] = std::isfinite(tmp[b].z) ? 1.0f : 0.0f;
		}
		return copy_host(v, (long long)v.size(), out, cap);
	}
	if (s == "self_col") {
		if (!out) return 3;
		if (cap < 3) return -1;
		if (E.read_counters()) return -1;
		out[0] = E.spacing;
		out[1] = engine().S.sc_radius_scale * E.spacing;
		out[2] = E.h_ctr->sc_reach;
		return 3;
	}
	return -1;
}

XPBD_API int xpbd_b200_set_positions(const float* pos, int n)
{
	Engine& E = *cur_engine();
	if (!E.stepped) return fail("xpbd_b200_set_positions: no step yet");
	if (!pos || n != E.n) return fail("xpbd_b200_set_positions: size mismatch");
	DBuf<float> tmp;
	CK(tmp.alloc(3 * (size_t)n));
	CK(cudaMemcpyAsync(tmp.p, pos, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, E.stream));
	dev::k_set_positions<<<Engine::blocks_for(n), kBlock, 0, E.stream>>>(n, tmp.p, E.d_perm.p, E.pos_curr.p,
		E.pos_out3.p);
	CK(cudaGetLastError());
	return E.sync();
}

// The once-per-step self-collision build on caller-given start / predicted positions
// (x[3N], p[3N]); the candidate total, or -1.  Used to check the hash, order and
// candidate lists stage by stage.
XPBD_API int xpbd_b200_selfcol_build(const float* x, const float* p)
{
	if (!cur_engine()->built || !x || !p) return fail("xpbd_b200_selfcol_build: no scene");
	Engine& E = *cur_engine();
	if (E.ensure_selfcol()) return -1;
	if (E.upload_params()) return -1;
	const int N = E.n;
	std::vector<float4> a(N), b(N);
	for (int r = 0; r < N; ++r) {
		const int i = E.perm[r];
		a[r] = make_float4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 1.0f);
		b[r] = make_float4(p[3 * i], p[3 * i + 1], p[3 * i + 2], 1.0f);
	}
	std::vector<float4> keep_curr(N), keep_next(N);
	CK(cudaMemcpyAsync(keep_curr.data(), E.pos_curr.p, sizeof(float4) * N, cudaMemcpyDeviceToHost, E.stream));
	CK(cudaMemcpyAsync(keep_next.data(), E.pos_next.p, sizeof(float4) * N, cudaMemcpyDeviceToHost, E.stream));
	CK(cudaStreamSynchronize(E.stream));
	CK(cudaMemcpyAsync(E.pos_curr.p, a.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, E.stream));
	CK(cudaMemcpyAsync(E.pos_next.p, b.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, E.stream));
	CK(cudaMemsetAsync(E.d_ctr, 0, sizeof(DevCounters), E.stream));
	if (E.enqueue_sc_build(nullptr, true)) return -1;
	CK(cudaGetLastError());
	if (E.read_counters()) return -1;
	// restore the solver state this stage check borrowed
	CK(cudaMemcpyAsync(E.pos_curr.p, keep_curr.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, E.stream));
	CK(cudaMemcpyAsync(E.pos_next.p, keep_next.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, E.stream));
	CK(cudaStreamSynchronize(E.stream));
	return (int)E.h_ctr->sc_contacts;
}

// ============================================================================
// Allocation-free self-collision candidate build
//
// For callers that may not allocate device memory: a host application that owns the
// whole device heap (a simulator that hands plug-ins its buffers and forbids
// cudaMalloc, whose implicit device synchronisation would stall its frame), or code
// running where allocation is not allowed at all.  The caller passes inputs and
// outputs in its own device memory; every scratch buffer of the build (hash keys,
// bucket counts and starts, the ordered index, the cell-ordered copies, counters and
// the step constants) lives in one file-scope __device__ array sized for
// kStaticMaxN particles, which every GPU that loads this library holds until exit.
// ============================================================================
namespace xpbd {
namespace noalloc {

constexpr int kStaticMaxN = 65536;

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
constexpr int table_for(int n)
{
	int t = 1024;
	while (t < 2 * n) t <<= 1;
	return t;
}
constexpr int kTable = table_for(kStaticMaxN);              // 131072
constexpr int kBuckets = kTable + 1;                        // + sentinel bucket
constexpr int kScanN = kBuckets + 1;
constexpr int kScanBlocks = (kScanN + 1023) / 1024;
// byte offsets inside the scratch array
constexpr size_t kOffParams = 0;
constexpr size_t kOffCtr = align256(kOffParams + sizeof(StepParams));
constexpr size_t kOffKeys = align256(kOffCtr + sizeof(DevCounters));
constexpr size_t kOffBucket = align256(kOffKeys + sizeof(unsigned int) * kStaticMaxN);
constexpr size_t kOffStart = align256(kOffBucket + sizeof(int) * kScanN);
constexpr size_t kOffCursor = align256(kOffStart + sizeof(int) * kScanN);
constexpr size_t kOffSorted = align256(kOffCursor + sizeof(int) * kBuckets);
constexpr size_t kOffSums = align256(kOffSorted + sizeof(int) * kStaticMaxN);
constexpr size_t kOffObj = align256(kOffSums + sizeof(int) * (kScanBlocks + 1));
constexpr size_t kOffSp = align256(kOffObj + sizeof(int) * kStaticMaxN);
constexpr size_t kOffSr = align256(kOffSp + sizeof(float4) * kStaticMaxN);
constexpr size_t kOffSx = align256(kOffSr + sizeof(float4) * kStaticMaxN);
constexpr size_t kScratchBytes = align256(kOffSx + sizeof(float4) * kStaticMaxN);   // about 5.4 MB

static __device__ __align__(256) unsigned char g_selfcol_scratch[kScratchBytes];

// Device address of g_selfcol_scratch, looked up once per device with that device
// current (the host-side symbol is only a stand-in, never a device address).
constexpr int kMaxDevices = 64;
static unsigned char* g_scratch_addr[kMaxDevices] = {};
static std::mutex g_scratch_mutex;

static int scratch_for_current_device(unsigned char** out)
{
	int dev = 0;
	CK(cudaGetDevice(&dev));
	if (dev < 0 || dev >= kMaxDevices) return fail("selfcol static: device ordinal %d out of range", dev);
	std::lock_guard<std::mutex> lock(g_scratch_mutex);
	if (!g_scratch_addr[dev]) {
		void* p = nullptr;
		CK(cudaGetSymbolAddress(&p, g_selfcol_scratch));
		g_scratch_addr[dev] = static_cast<unsigned char*>(p);
	}
	*out = g_scratch_addr[dev];
	return 0;
}

// the self-collision constants of one call, passed by value
struct SelfColConsts {
	float dc, search, excl2, cross_excl2, fast_rel, search_plus16dc;
	int within, single_object;
};

// writes the call's constants into the StepParams block of the scratch array (every other
// field zero), so that no host memory is copied to the device
__global__ void __launch_bounds__(256) k_static_params(StepParams* __restrict__ P, SelfColConsts c)
{
	unsigned int* w = reinterpret_cast<unsigned int*>(P);
	for (size_t k = threadIdx.x; k < sizeof(StepParams) / sizeof(unsigned int); k += blockDim.x) w[k] = 0u;
	__syncthreads();
	if (threadIdx.x == 0) {
		P->sc_dc = c.dc;
		P->sc_search = c.search;
		P->sc_excl2 = c.excl2;
		P->sc_cross_excl2 = c.cross_excl2;
		P->sc_fast_rel = c.fast_rel;
		P->sc_search_plus16dc = c.search_plus16dc;
		P->sc_within = c.within;
		P->sc_single_object = c.single_object;
	}
}

}  // namespace noalloc
}  // namespace xpbd

// Self-collision candidate lists (the once-per-step build of the solver step,
// forward.cu:11796-11849) for n <= 65,536 particles, with no device allocation.
//
//   x, p, rest  device float4[n]: start positions, predicted positions, rest positions
//               (w ignored)
//   obj_id      device int[n] object id per particle, or NULL (one object)
//   spacing, radius_scale, exclude_scale, within_body
//               as for xpbd_set_self_collision; spacing is the median shortest graph
//               edge (contact distance = radius_scale * spacing)
//   contacts    device int[32 n] out: candidate codes, j or -(j + 1) for fast
//               cross-object pairs, first counts[i] valid per particle
//   counts      device int[n] out
//   total       device int out (candidate total), or NULL
//   stream      cudaStream_t to run on (NULL: legacy default stream)
//
// Returns 0 once the work is enqueued, -1 with xpbd_last_error() on bad arguments or a
// CUDA error.  Nothing is copied from host memory: the constants travel as a kernel
// argument.  All scratch sits in one static device array per GPU, reused by every call:
// calls that overlap on the GPU (different streams, or several host threads) race on it
// and must be serialised by the caller.  The first call on a device looks up the array's
// device address; make that first call outside any CUDA stream capture.  The count of
// over-cap replacements (xpbd_self_collision_stats' third figure) is not reported here.
XPBD_API int xpbd_b200_selfcol_candidates_static(int n, const float* x, const float* p, const float* rest,
	const int* obj_id, float spacing, float radius_scale, float exclude_scale, int within_body, int* contacts,
	int* counts, int* total, void* stream)
{
	using namespace xpbd::noalloc;
	if (n <= 0 || n > kStaticMaxN)
		return fail("xpbd_b200_selfcol_candidates_static: n = %d outside 1..%d (the static scratch limit)", n,
			kStaticMaxN);
	if (!x || !p || !rest || !contacts || !counts)
		return fail("xpbd_b200_selfcol_candidates_static: null input or output pointer");
	if (!(spacing > 0.0f) || !std::isfinite(spacing))
		return fail("xpbd_b200_selfcol_candidates_static: spacing must be positive");
	unsigned char* base = nullptr;
	if (scratch_for_current_device(&base)) return -1;
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	auto* d_params = reinterpret_cast<StepParams*>(base + kOffParams);
	auto* d_ctr = reinterpret_cast<DevCounters*>(base + kOffCtr);
	auto* keys = reinterpret_cast<unsigned int*>(base + kOffKeys);
	auto* bucket = reinterpret_cast<int*>(base + kOffBucket);
	auto* start = reinterpret_cast<int*>(base + kOffStart);
	auto* cursor = reinterpret_cast<int*>(base + kOffCursor);
	auto* sorted = reinterpret_cast<int*>(base + kOffSorted);
	auto* sums = reinterpret_cast<int*>(base + kOffSums);
	auto* obj0 = reinterpret_cast<int*>(base + kOffObj);
	auto* sp = reinterpret_cast<float4*>(base + kOffSp);
	auto* sr = reinterpret_cast<float4*>(base + kOffSr);
	auto* sx = reinterpret_cast<float4*>(base + kOffSx);
	// step constants as the solver derives them (forward.cu:4532-4540, 11798-11831)
	const float rs = fminf(fmaxf(std::isfinite(radius_scale) ? radius_scale : 1.5f, 0.1f), 10.0f);
	const float es = fminf(fmaxf(std::isfinite(exclude_scale) ? exclude_scale : 2.0f, 1.05f), 20.0f);
	const float dc = rs * spacing;
	const float search = 1.5f * dc;
	const float excl = es * dc;
	SelfColConsts c;
	c.dc = dc;
	c.search = search;
	c.excl2 = excl * excl;
	c.cross_excl2 = dc * dc;
	c.fast_rel = 0.0f * dc;
	c.search_plus16dc = search + 16.0f * dc;
	c.within = within_body ? 1 : 0;
	c.single_object = obj_id ? 0 : 1;
	k_static_params<<<1, 256, 0, st>>>(d_params, c);
	// everything the build accumulates into starts from zero on every call
	CK(cudaMemsetAsync(d_ctr, 0, sizeof(DevCounters), st));
	CK(cudaMemsetAsync(bucket, 0, sizeof(int) * kScanN, st));
	CK(cudaMemsetAsync(cursor, 0, sizeof(int) * kBuckets, st));
	if (!obj_id) {
		CK(cudaMemsetAsync(obj0, 0, sizeof(int) * n, st));
		obj_id = obj0;
	}
	const int table = table_for(n), buckets = table + 1, scan_n = buckets + 1, nb = (scan_n + 1023) / 1024;
	const auto* X = reinterpret_cast<const float4*>(x);
	const auto* Pp = reinterpret_cast<const float4*>(p);
	const auto* R = reinterpret_cast<const float4*>(rest);
	const dim3 B(kBlock), G((n + kBlock - 1) / kBlock);
	dev::k_sc_disp<<<G, B, 0, st>>>(n, X, Pp, d_ctr, nullptr, 0);
	dev::k_sc_setup<<<1, 1, 0, st>>>(d_params, d_ctr);
	dev::k_sc_keys<<<G, B, 0, st>>>(n, X, d_ctr, (unsigned)(table - 1), (unsigned)table, keys, bucket, nullptr);
	dev::k_scan_blocks<<<nb, 1024, 0, st>>>(bucket, start, scan_n, sums);
	dev::k_scan_sums<<<1, 1024, 0, st>>>(sums, nb);
	dev::k_scan_add<<<nb, 1024, 0, st>>>(start, scan_n, sums);
	dev::k_sc_scatter<<<G, B, 0, st>>>(n, keys, start, cursor, sorted);
	dev::k_sc_order<<<(buckets + kBlock - 1) / kBlock, B, 0, st>>>(buckets, start, sorted, (const int*)nullptr);
	dev::k_sc_pack<<<G, B, 0, st>>>(n, sorted, X, Pp, R, obj_id, sp, sr, sx);
	dev::k_sc_build_sorted<<<G, B, 0, st>>>(n, d_params, X, Pp, R, sorted, start, (unsigned)(table - 1), obj_id, sp,
		sr, sx, d_ctr, contacts, counts, nullptr);
	if (total)
		CK(cudaMemcpyAsync(total, &d_ctr->sc_contacts, sizeof(int), cudaMemcpyDeviceToDevice, st));
	CK(cudaGetLastError());
	return 0;
}
